// lbfgs.cuh -- batched L-BFGS minimisation on the device.
//
// lbfgs_minimizator / lbfgs (src/Quasi_Newton.f90:77-160, 349-663): the
// limited-memory BFGS method of Liu & Nocedal (Math. Prog. B 45, 1989) with
// the line search of More & Thuente (ACM TOMS 20, 1994) in the form of
// mcsrch / mcstep (:703-1096).  The objective is get_fg (:1110-1120):
// f = E_pot in eV and g = -F in eV/A.
//
// Every system runs its own minimisation; the batch advances by function
// evaluations.  Per evaluation round:
//   k_lb_dir   (one block per system) for systems whose line search just
//              succeeded: store the new (s, y) pair, test convergence, build
//              the next direction by the two-loop recursion, start the next
//              line search;
//   k_lb_move  (per atom) x = x0 + stp d for systems that evaluate;
//   skin test, list rebuild if needed, force kernels (the engine's own);
//   k_lb_eval  (one block per system) f and g.d at the trial point, then
//              the line search's tests and, if it continues, its next step.
// The scalar logic of a system runs in thread 0 of its block; vectors are
// per arena atom, so a system's result does not depend on its batch.
#pragma once
#include "kernels.cuh"

namespace gg {

constexpr int LB_MAXM = 8;          // history pairs kept at most
constexpr int LB_THREADS = 512;     // threads of the per-system blocks
constexpr double LB_FTOL = 1e-4;    // sufficient decrease (:467)
constexpr double LB_GTOL = 0.9;     // curvature (module gtol, :20)
constexpr double LB_STPMIN = 1e-20; // (:14)
constexpr double LB_STPMAX = 1e20;
constexpr int LB_MAXFEV = 100;      // evaluations per line search (:469)

enum LbPhase { LB_EVAL = 0, LB_ACCEPT = 1, LB_DONE = 2, LB_FAIL = 3, LB_LIMIT = 4, LB_IDLE = 5 };

struct LbState {
  int phase, iter, itermax, nfun, nfev, point, m, infoc, brackt, stage1, info, pad;
  double eps, xtol, f, finit, dginit, dgtest, stp, stx, fx, dgx, sty, fy, dgy, width, width1, stmin, stmax,
      gnorm;
  double rho[LB_MAXM], alpha[LB_MAXM];
};

struct LbWork {
  double4* x0;    // base point of the line search
  double4* g;     // gradient at the latest evaluation (eV/A)
  double4* gold;  // gradient at the base point
  double4* d;     // search direction (also the two-loop work vector)
  double4* S;     // m planes of cap atoms: steps s_k
  double4* Y;     // m planes: gradient differences y_k
  LbState* st;    // per system id
  int64_t cap;
};

// deterministic sum over the LB_THREADS threads of a block (fixed tree);
// the result is returned to every thread
__device__ __forceinline__ double lb_bsum(double v, double* sh) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
  if (ln == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = ln < LB_THREADS / 32 ? sh[ln] : 0.0;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (ln == 0) sh[LB_THREADS / 32] = v;
  }
  __syncthreads();
  v = sh[LB_THREADS / 32];
  __syncthreads();
  return v;
}

__device__ __forceinline__ double dot4(double4 a, double4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// One safeguarded step of More & Thuente: a cubic or quadratic trial point
// from the interval end stx (fx, dx), the other end sty (fy, dy) and the
// current step stp (fp, dp), by the four cases of their section 4 in the
// order mcstep tests them; then the interval is updated.
__device__ void lb_mt_step(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy, double& stp,
                           double fp, double dp, int& brackt, double stmin, double stmax, int& info) {
  info = 0;
  if ((brackt && (stp <= fmin(stx, sty) || stp >= fmax(stx, sty))) || dx * (stp - stx) >= 0.0 || stmax < stmin)
    return;
  const double sgnd = dp * (dx / fabs(dx));
  double stpf, stpc, stpq;
  bool bound;
  auto gam_of = [](double theta, double a, double b, bool clip) {
    const double sc = fmax(fabs(theta), fmax(fabs(a), fabs(b)));
    double disc = (theta / sc) * (theta / sc) - (a / sc) * (b / sc);
    if (clip) disc = fmax(0.0, disc);
    return sc * sqrt(disc);
  };
  if (fp > fx) {
    info = 1;
    bound = true;
    const double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double gam = gam_of(theta, dx, dp, false);
    if (stp < stx) gam = -gam;
    const double r = ((gam - dx) + theta) / (((gam - dx) + gam) + dp);
    stpc = stx + r * (stp - stx);
    stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx);
    stpf = (fabs(stpc - stx) < fabs(stpq - stx)) ? stpc : stpc + (stpq - stpc) / 2.0;
    brackt = 1;
  } else if (sgnd < 0.0) {
    info = 2;
    bound = false;
    const double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double gam = gam_of(theta, dx, dp, false);
    if (stp > stx) gam = -gam;
    const double r = ((gam - dp) + theta) / (((gam - dp) + gam) + dx);
    stpc = stp + r * (stx - stp);
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    stpf = (fabs(stpc - stp) > fabs(stpq - stp)) ? stpc : stpq;
    brackt = 1;
  } else if (fabs(dp) < fabs(dx)) {
    info = 3;
    bound = true;
    const double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double gam = gam_of(theta, dx, dp, true);
    if (stp > stx) gam = -gam;
    const double r = ((gam - dp) + theta) / ((gam + (dx - dp)) + gam);
    if (r < 0.0 && gam != 0.0) stpc = stp + r * (stx - stp);
    else if (stp > stx) stpc = stmax;
    else stpc = stmin;
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    if (brackt) stpf = (fabs(stp - stpc) < fabs(stp - stpq)) ? stpc : stpq;
    else stpf = (fabs(stp - stpc) > fabs(stp - stpq)) ? stpc : stpq;
  } else {
    info = 4;
    bound = false;
    if (brackt) {
      const double theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp;
      double gam = gam_of(theta, dy, dp, false);
      if (stp > sty) gam = -gam;
      const double r = ((gam - dp) + theta) / (((gam - dp) + gam) + dy);
      stpf = stp + r * (sty - stp);
    } else {
      stpf = (stp > stx) ? stmax : stmin;
    }
  }
  if (fp > fx) {
    sty = stp; fy = fp; dy = dp;
  } else {
    if (sgnd < 0.0) { sty = stx; fy = fx; dy = dx; }
    stx = stp; fx = fp; dx = dp;
  }
  stpf = fmax(stmin, fmin(stmax, stpf));
  stp = stpf;
  if (brackt && bound) {
    const double lim = stx + 0.66 * (sty - stx);
    stp = (sty > stx) ? fmin(lim, stp) : fmax(lim, stp);
  }
}

// top of mcsrch's loop: the interval's bounds and the next trial step
__device__ void lb_next_trial(LbState& L) {
  L.nfev++;
  if (L.brackt) {
    L.stmin = fmin(L.stx, L.sty);
    L.stmax = fmax(L.stx, L.sty);
  } else {
    L.stmin = L.stx;
    L.stmax = L.stp + 4.0 * (L.stp - L.stx);
  }
  L.stp = fmin(fmax(L.stp, LB_STPMIN), LB_STPMAX);
  if ((L.brackt && (L.stp <= L.stmin || L.stp >= L.stmax)) || L.nfev == LB_MAXFEV || L.infoc == 0 ||
      (L.brackt && L.stmax - L.stmin <= L.xtol * L.stmax))
    L.stp = L.stx;
  L.phase = LB_EVAL;
}

// a new line search from the base point (f, dginit = g.d) with step stp
__device__ void lb_start_search(LbState& L, double f, double dginit, double stp) {
  if (!(dginit < 0.0)) {  // not a descent direction
    L.phase = LB_FAIL;
    L.info = 0;
    return;
  }
  L.brackt = 0;
  L.stage1 = 1;
  L.infoc = 1;
  L.nfev = 0;
  L.f = f;
  L.finit = f;
  L.dginit = dginit;
  L.dgtest = LB_FTOL * dginit;
  L.width = LB_STPMAX - LB_STPMIN;
  L.width1 = L.width / 0.5;
  L.stx = 0.0; L.fx = f; L.dgx = dginit;
  L.sty = 0.0; L.fy = f; L.dgy = dginit;
  L.stp = stp;
  lb_next_trial(L);
}

// the tests after an evaluation at stp (f, dg = g.d); the search either
// ends (ACCEPT, or FAIL with mcsrch's info) or takes its next step
__device__ void lb_after_eval(LbState& L, double f, double dg) {
  L.nfun++;
  L.f = f;
  int info = 0;
  const double ftest1 = L.finit + L.stp * L.dgtest;
  if ((L.brackt && (L.stp <= L.stmin || L.stp >= L.stmax)) || L.infoc == 0) info = 6;
  if (L.stp == LB_STPMAX && f <= ftest1 && dg <= L.dgtest) info = 5;
  if (L.stp == LB_STPMIN && (f > ftest1 || dg >= L.dgtest)) info = 4;
  if (L.nfev == LB_MAXFEV) {
    L.phase = LB_FAIL;
    L.info = 3;
    return;
  }
  if (L.brackt && L.stmax - L.stmin <= L.xtol * L.stmax) info = 2;
  if (f <= ftest1 && fabs(dg) <= LB_GTOL * (-L.dginit)) info = 1;
  if (info == 1) {
    L.phase = LB_ACCEPT;
    return;
  }
  if (info != 0) {
    L.phase = LB_FAIL;
    L.info = info;
    return;
  }
  if (L.stage1 && f <= ftest1 && dg >= fmin(LB_FTOL, LB_GTOL) * L.dginit) L.stage1 = 0;
  if (L.stage1 && f <= L.fx && f > ftest1) {
    // first stage: the modified function psi(stp) = f - stp * dgtest
    double fm = f - L.stp * L.dgtest, fxm = L.fx - L.stx * L.dgtest, fym = L.fy - L.sty * L.dgtest;
    double dgm = dg - L.dgtest, dgxm = L.dgx - L.dgtest, dgym = L.dgy - L.dgtest;
    lb_mt_step(L.stx, fxm, dgxm, L.sty, fym, dgym, L.stp, fm, dgm, L.brackt, L.stmin, L.stmax, L.infoc);
    L.fx = fxm + L.stx * L.dgtest;
    L.fy = fym + L.sty * L.dgtest;
    L.dgx = dgxm + L.dgtest;
    L.dgy = dgym + L.dgtest;
  } else {
    lb_mt_step(L.stx, L.fx, L.dgx, L.sty, L.fy, L.dgy, L.stp, f, dg, L.brackt, L.stmin, L.stmax, L.infoc);
  }
  if (L.brackt) {
    if (fabs(L.sty - L.stx) >= 0.66 * L.width1) L.stp = L.stx + 0.5 * (L.sty - L.stx);
    L.width1 = L.width;
    L.width = fabs(L.sty - L.stx);
  }
  lb_next_trial(L);
}

// The first iteration (lbfgs :459-475): g at the start point, d = -g,
// stp = 1/|g|.  With restart=1 only systems still searching start again
// (after the engine had to rebuild its lists mid-round).
__global__ void __launch_bounds__(LB_THREADS) k_lb_init(Arena A, LbWork W, const int* sys, int restart) {
  __shared__ double sh[LB_THREADS / 32 + 1];
  const int s = sys[blockIdx.x];
  LbState& L = W.st[s];
  if (restart && (L.phase == LB_DONE || L.phase == LB_FAIL || L.phase == LB_LIMIT)) return;
  const SysDev& S = A.sys[s];
  const double ui = c_ui_ev();
  double e = 0.0, gg = 0.0;
  for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
    const double4 F = A.force[i];
    const double4 g = make_double4(-F.x * ui, -F.y * ui, -F.z * ui, 0.0);
    W.g[i] = g;
    W.gold[i] = g;
    W.d[i] = make_double4(-g.x, -g.y, -g.z, 0.0);
    W.x0[i] = A.pos[i];
    e += A.epot[i];
    gg += dot4(g, g);
  }
  e = lb_bsum(e, sh);
  gg = lb_bsum(gg, sh);
  if (threadIdx.x == 0) {
    const double f = e * ui;
    if (!restart) L.nfun = 1;
    L.iter = 1;
    L.point = 0;
    L.gnorm = sqrt(gg);
    if (gg == 0.0) {
      L.f = f;
      L.phase = LB_DONE;  // already stationary
    } else {
      lb_start_search(L, f, -gg, 1.0 / L.gnorm);
    }
  }
}

// x = x0 + stp d for the systems that evaluate a trial point
__global__ void __launch_bounds__(BLOCK) k_lb_move(Arena A, LbWork W, BlockMap M) {
  const int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const LbState& L = W.st[s];
  if (L.phase != LB_EVAL) return;  // uniform per block
  const int i = M.first[blockIdx.x] + threadIdx.x;
  if (i >= M.end[blockIdx.x]) return;
  const SysDev& S = A.sys[s];
  const double stp = L.stp;
  const double4 x0 = W.x0[i], d = W.d[i];
  double4 x = A.pos[i];
  x.x = x0.x + stp * d.x;
  x.y = x0.y + stp * d.y;
  x.z = x0.z + stp * d.z;
  A.pos[i] = x;
  if (S.prec == PREC_MIXED || S.ff == FF_TERSOFF) {
    int bad = 0;
    write_fx(A, S, i, x, A.type[i], bad);
    if (bad) atomicOr(&A.st[s].status, ST_LOST);
  }
  if (!(x.x == x.x && x.y == x.y && x.z == x.z)) atomicOr(&A.st[s].status, ST_NAN);
}

// f and g.d at the trial point, then the line search's decision
__global__ void __launch_bounds__(LB_THREADS) k_lb_eval(Arena A, LbWork W, const int* sys) {
  __shared__ double sh[LB_THREADS / 32 + 1];
  const int s = sys[blockIdx.x];
  LbState& L = W.st[s];
  if (L.phase != LB_EVAL) return;
  const SysDev& S = A.sys[s];
  const double ui = c_ui_ev();
  double e = 0.0, dg = 0.0;
  for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
    const double4 F = A.force[i];
    const double4 g = make_double4(-F.x * ui, -F.y * ui, -F.z * ui, 0.0);
    W.g[i] = g;
    e += A.epot[i];
    dg += dot4(g, W.d[i]);
  }
  e = lb_bsum(e, sh);
  dg = lb_bsum(dg, sh);
  if (threadIdx.x == 0) lb_after_eval(L, e * ui, dg);
}

// after an accepted line search (lbfgs :603-640 and, for the next
// iteration, :510-580): the new pair s = stp d, y = g - gold; the
// convergence test |g| / int(max(1, |x|)) <= eps; the two-loop recursion
// d = -H g with H0 = (y.s / y.y) I from the newest pair; the next search
// from x with stp = 1
__global__ void __launch_bounds__(LB_THREADS) k_lb_dir(Arena A, LbWork W, const int* sys) {
  __shared__ double sh[LB_THREADS / 32 + 1];
  __shared__ int go;
  const int s = sys[blockIdx.x];
  LbState& L = W.st[s];
  if (L.phase != LB_ACCEPT) return;
  const SysDev& S = A.sys[s];
  const int m = L.m;
  const int64_t cap = W.cap;
  const int p = L.point;
  const double stp = L.stp;
  double gg = 0.0, xx = 0.0;
  for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
    const double4 d = W.d[i], g = W.g[i], go4 = W.gold[i], x = A.pos[i];
    W.S[p * cap + i] = make_double4(stp * d.x, stp * d.y, stp * d.z, 0.0);
    W.Y[p * cap + i] = make_double4(g.x - go4.x, g.y - go4.y, g.z - go4.z, 0.0);
    gg += dot4(g, g);
    xx += dot4(x, x);
  }
  gg = lb_bsum(gg, sh);
  xx = lb_bsum(xx, sh);
  if (threadIdx.x == 0) {
    L.point = (p + 1) % m;
    L.gnorm = sqrt(gg);
    const double xnorm = (double)(long long)fmax(1.0, sqrt(xx));  // int(max(1, xnorm))
    go = 1;
    if (L.gnorm / xnorm <= L.eps) {
      L.phase = LB_DONE;
      go = 0;
    } else if (L.iter >= L.itermax) {
      L.phase = LB_LIMIT;
      go = 0;
    } else {
      L.iter++;
    }
  }
  __syncthreads();
  if (!go) return;
  const int bound = min(L.iter - 1, m);
  const int np = L.point;
  double ys = 0.0, yy = 0.0;
  for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
    const double4 y = W.Y[p * cap + i], sv = W.S[p * cap + i], g = W.g[i];
    ys += dot4(y, sv);
    yy += dot4(y, y);
    W.d[i] = make_double4(-g.x, -g.y, -g.z, 0.0);  // q = -g
  }
  ys = lb_bsum(ys, sh);
  yy = lb_bsum(yy, sh);
  const double h0 = ys / yy;
  if (threadIdx.x == 0) L.rho[p] = 1.0 / ys;
  __syncthreads();
  double alpha[LB_MAXM];
  int cp = np;
  for (int b = 0; b < bound; b++) {
    cp = (cp + m - 1) % m;
    double sq = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) sq += dot4(W.S[cp * cap + i], W.d[i]);
    sq = lb_bsum(sq, sh);
    const double a = L.rho[cp] * sq;
    alpha[b] = a;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
      const double4 y = W.Y[cp * cap + i];
      double4 q = W.d[i];
      q.x -= a * y.x; q.y -= a * y.y; q.z -= a * y.z;
      W.d[i] = q;
    }
  }
  for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
    double4 q = W.d[i];
    q.x *= h0; q.y *= h0; q.z *= h0;
    W.d[i] = q;
  }
  for (int b = 0; b < bound; b++) {
    double yr = 0.0;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) yr += dot4(W.Y[cp * cap + i], W.d[i]);
    yr = lb_bsum(yr, sh);
    const double beta = alpha[bound - 1 - b] - L.rho[cp] * yr;
    for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
      const double4 sv = W.S[cp * cap + i];
      double4 q = W.d[i];
      q.x += beta * sv.x; q.y += beta * sv.y; q.z += beta * sv.z;
      W.d[i] = q;
    }
    cp = (cp + 1) % m;
  }
  double dg = 0.0;
  for (int i = S.off + threadIdx.x; i < S.off + S.n; i += LB_THREADS) {
    const double4 g = W.g[i];
    W.gold[i] = g;
    W.x0[i] = A.pos[i];
    dg += dot4(g, W.d[i]);
  }
  dg = lb_bsum(dg, sh);
  if (threadIdx.x == 0) lb_start_search(L, L.f, dg, 1.0);
}

}  // namespace gg
