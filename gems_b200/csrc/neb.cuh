// neb.cuh -- nudged elastic band with the images as a batch of systems.
//
// neb (src/NEB.f90:58-220): nimg images of one group, each a system of the
// arena (same atoms, same force field); the first and last never move.
// Images between consecutive fixed ones start on the straight line
// (neb_linin, :331-355).  An iteration is velocity Verlet with unit masses
// (change_atom_mas, :222-234) on the NEB force, with the quick-min velocity
// projection (nebvel, :314-329) before the first and the second half kick;
// the NEB force (nebfce, :236-312) is the improved tangent of Henkelman &
// Jonsson (J. Chem. Phys. 113, 9978, 2000) with a spring force along it.
// Each image's vector work runs in one block with a fixed reduction tree, so
// the result does not depend on how the arena packs the images.
#pragma once
#include "lbfgs.cuh"

namespace gg {

// image k's system id and atom offset, the images' energies (internal units)
struct NebDev {
  const int* sys;     // nimg system ids, in image order
  const int* off;     // nimg atom offsets
  double* e;          // nimg energies; the last image's stays 0 (see gemsgpu_neb)
  double* fsum;       // per image: sum of |F_neb|^2 (for the time step)
  int nimg, n;        // images, atoms per image
  double ks;          // spring constant (internal units)
};

// the straight line between fixed images a < b: p_i = p_{i-1} + (p_b - p_a)/(b - a)
// one thread per atom coordinate, images in order (the reference's running sum)
__global__ void k_neb_interp(Arena A, NebDev N, int a, int b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * N.n) return;
  const int k = t / 3, c = t % 3;
  auto X = [&](int img) -> double* { return reinterpret_cast<double*>(&A.pos[N.off[img] + k]) + c; };
  const double step = (*X(b) - *X(a)) / (double)(b - a);
  for (int i = a + 1; i < b; i++) *X(i) = *X(i - 1) + step;
}

// inq_pot_energy of the images in [i0, i1)
__global__ void __launch_bounds__(LB_THREADS) k_neb_energy(Arena A, NebDev N, int i0) {
  __shared__ double sh[LB_THREADS / 32 + 1];
  const int img = i0 + blockIdx.x;
  const int o = N.off[img];
  double e = 0.0;
  for (int k = threadIdx.x; k < N.n; k += LB_THREADS) e += A.epot[o + k];
  e = lb_bsum(e, sh);
  if (threadIdx.x == 0) N.e[img] = e;
}

// nebfce for interior image 1 + blockIdx.x: the tangent from the energies of
// the image and its neighbours, then F <- F - (F.q)q + q ks(|t+| - |t-|)
__global__ void __launch_bounds__(LB_THREADS) k_neb_force(Arena A, NebDev N) {
  __shared__ double sh[LB_THREADS / 32 + 1];
  const int i = 1 + blockIdx.x;
  const int om = N.off[i - 1], oi = N.off[i], op = N.off[i + 1];
  const double em = N.e[i - 1], ei = N.e[i], ep = N.e[i + 1];
  const double dmin = fabs(ei - em), dplus = fabs(ep - ei);
  const double dmax = fmax(dmin, dplus), dinf = fmin(dmin, dplus);
  // q = wp t+ + wm t-: towards the higher neighbour, or an energy-weighted
  // mix at an extremum.  Exact ties, where the reference keeps whatever
  // tangent it computed last, take the mix with the larger weight on t+.
  double wp, wm;
  if (ep > ei && ei > em) { wp = 1.0; wm = 0.0; }
  else if (!(ep > ei) && !(ei > em)) { wp = 0.0; wm = 1.0; }
  else if (ep < em) { wp = dinf; wm = dmax; }
  else { wp = dmax; wm = dinf; }
  double qq = 0.0, fq = 0.0, tpp = 0.0, tmm = 0.0;
  for (int k = threadIdx.x; k < N.n; k += LB_THREADS) {
    const double4 xm = A.pos[om + k], xi = A.pos[oi + k], xp = A.pos[op + k], F = A.force[oi + k];
    const double tp[3] = {xp.x - xi.x, xp.y - xi.y, xp.z - xi.z};
    const double tm[3] = {xi.x - xm.x, xi.y - xm.y, xi.z - xm.z};
    const double f[3] = {F.x, F.y, F.z};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double q = wp * tp[c] + wm * tm[c];
      qq += q * q;
      fq += f[c] * q;
      tpp += tp[c] * tp[c];
      tmm += tm[c] * tm[c];
    }
  }
  qq = lb_bsum(qq, sh);
  fq = lb_bsum(fq, sh);
  tpp = lb_bsum(tpp, sh);
  tmm = lb_bsum(tmm, sh);
  const double nq = sqrt(qq);
  const double fqn = fq / nq;                       // F . q_hat
  const double fs = N.ks * (sqrt(tpp) - sqrt(tmm));
  double ff = 0.0;
  for (int k = threadIdx.x; k < N.n; k += LB_THREADS) {
    const double4 xm = A.pos[om + k], xi = A.pos[oi + k], xp = A.pos[op + k];
    double4 F = A.force[oi + k];
    const double qx = (wp * (xp.x - xi.x) + wm * (xi.x - xm.x)) / nq;
    const double qy = (wp * (xp.y - xi.y) + wm * (xi.y - xm.y)) / nq;
    const double qz = (wp * (xp.z - xi.z) + wm * (xi.z - xm.z)) / nq;
    F.x = F.x - fqn * qx + qx * fs;
    F.y = F.y - fqn * qy + qy * fs;
    F.z = F.z - fqn * qz + qz * fs;
    A.force[oi + k] = F;
    ff += F.x * F.x + F.y * F.y + F.z * F.z;
  }
  ff = lb_bsum(ff, sh);
  if (threadIdx.x == 0) N.fsum[i] = ff;
}

// nebvel: v <- (v.F / F.F) F when v.F > 0, else 0 (interior images)
__global__ void __launch_bounds__(LB_THREADS) k_neb_vel(Arena A, NebDev N) {
  __shared__ double sh[LB_THREADS / 32 + 1];
  const int o = N.off[1 + blockIdx.x];
  double vf = 0.0, ff = 0.0;
  for (int k = threadIdx.x; k < N.n; k += LB_THREADS) {
    const double4 v = A.vel[o + k], F = A.force[o + k];
    vf += v.x * F.x + v.y * F.y + v.z * F.z;
    ff += F.x * F.x + F.y * F.y + F.z * F.z;
  }
  vf = lb_bsum(vf, sh);
  ff = lb_bsum(ff, sh);
  for (int k = threadIdx.x; k < N.n; k += LB_THREADS) {
    const double4 F = A.force[o + k];
    double4 v = A.vel[o + k];
    if (vf > 0.0) {
      v.x = vf * F.x / ff; v.y = vf * F.y / ff; v.z = vf * F.z / ff;
    } else {
      v.x = 0.0; v.y = 0.0; v.z = 0.0;
    }
    A.vel[o + k] = v;
  }
}

// velocity_verlet_a / _b with one_mass = 1 on the interior images' atoms
// (one thread per atom; blocks tile the interior images' atom ranges)
template <bool FIRST_HALF>
__global__ void k_neb_vv(Arena A, NebDev N, double dt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ni = N.nimg - 2;
  if (t >= ni * N.n) return;
  const int img = 1 + t / N.n, k = t % N.n;
  const int i = N.off[img] + k;
  const double adv = dt * 0.5, adx = adv * dt;
  const double4 F = A.force[i];
  double4 v = A.vel[i];
  if (FIRST_HALF) {
    double4 x = A.pos[i];
    x.x = x.x + dt * v.x + adx * F.x;
    x.y = x.y + dt * v.y + adx * F.y;
    x.z = x.z + dt * v.z + adx * F.z;
    A.pos[i] = x;
    const int s = N.sys[img];
    const SysDev& S = A.sys[s];
    if (S.prec == PREC_MIXED || S.ff == FF_TERSOFF) {
      int bad = 0;
      write_fx(A, S, i, x, A.type[i], bad);
      if (bad) atomicOr(&A.st[s].status, ST_LOST);
    }
    if (!(x.x == x.x && x.y == x.y && x.z == x.z)) atomicOr(&A.st[s].status, ST_NAN);
  }
  v.x = v.x + adv * F.x;
  v.y = v.y + adv * F.y;
  v.z = v.z + adv * F.z;
  A.vel[i] = v;
}

}  // namespace gg
