// gems_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the GEMS force/neighbour hot path (alexispaz/GEMS,
// Fortran 2003).  The tests compare the CUDA path against it; it is the timed CPU
// baseline ("port"): only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference legs may load it.  The product library
// (gems_b200/libgemsgpu.so) never links or calls it.
//
// Parity status of this restatement:
//   * pinned against the reference's golden files examples/XYZ (LJ, PBC,
//     O(N^2) list), examples/LJ (dimer scan + velocity Verlet),
//     examples/SMA-TB/bulk (linked cells, SMA-TB, Ermak, LCG stream),
//     examples/NVE (plj, fill, tempgdist, VV) and examples/NVT (plj, Ermak);
//     see tests/test_oracle_golden.py.
//   * Tersoff and FIRE: parity UNPINNED (the reference ships no test for
//     either, its Tersoff.f90 is internally inconsistent and FIRE.f90 does
//     not compile).  They are restated from the published methods and
//     checked by finite differences / energy conservation instead.
//
// Every routine cites the reference file:line it restates.  Arithmetic is
// written in the reference's evaluation order and compiled with
// -ffp-contract=off so that the neighbour predicate is bit-identical to a
// gfortran -O2 build on x86-64 (no FMA contraction).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- units
// Constants.F90:101-175.  Internal units: Angstrom, uma, ps.
const double axps_mxs = 1.0e2;
const double uma_kg = 1.6605402e-27;
const double qe_si = 1.60219e-19;
const double joule_ev = 1.0 / qe_si;
const double ui_ev = axps_mxs * axps_mxs * uma_kg * joule_ev;
const double ev_ui = 1.0 / ui_ev;
const double kB_ev = 8.617385e-05;
const double kB_ui = kB_ev * ev_ui;
const double pi = 3.14159265358979323846264338327950288;
const double pio2 = pi / 2.0;

// ---------------------------------------------------------------- RNG
// Random.F90:145-171 (lcg_ranu, lcg_init_ran) and :213-250 (rang, gasdev).
struct Lcg {
  int32_t idum = -12345789;
  int32_t ix = -1, iy = -1;
  bool gaus_stored = false;
  double g = 0.0;
};

// am = nearest(1.0,-1.0)/im is evaluated in single precision
// (Random.F90:148): (1 - 2^-24) / float(2147483647) = (1 - 2^-24) * 2^-31.
const double lcg_am = (double)((1.0f - 5.9604644775390625e-8f) / 2147483648.0f);

double lcg_ranu(Lcg& s) {
  const int32_t ia = 16807, im = 2147483647, iq = 127773, ir = 2836;
  if (s.idum <= 0 || s.iy < 0) {
    int32_t a = s.idum < 0 ? -s.idum : s.idum;
    s.iy = ((int32_t)(888889999 ^ a)) | 1;
    s.ix = (int32_t)(777755555 ^ a);
    s.idum = a + 1;
  }
  uint32_t x = (uint32_t)s.ix;
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  s.ix = (int32_t)x;
  int32_t k = s.iy / iq;
  s.iy = ia * (s.iy - k * iq) - ir * k;
  if (s.iy < 0) s.iy += im;
  return lcg_am * (double)((im & (s.ix ^ s.iy)) | 1);
}

void lcg_seed(Lcg& s, int seed) {  // lcg_init_ran(lseed): idum=-abs(seed)
  s.idum = -std::abs(seed);
}

double gasdev(Lcg& s) {
  if (s.gaus_stored) {
    s.gaus_stored = false;
    return s.g;
  }
  double v1, v2, rsq;
  for (;;) {
    v1 = 2.0 * lcg_ranu(s) - 1.0;
    v2 = 2.0 * lcg_ranu(s) - 1.0;
    rsq = v1 * v1 + v2 * v2;
    if (rsq > 0.0 && rsq < 1.0) break;
  }
  rsq = std::sqrt(-2.0 * std::log(rsq) / rsq);
  s.g = v2 * rsq;
  s.gaus_stored = true;
  return v1 * rsq;
}

void rang(Lcg& s, double* r1, double* r2) {  // always draws a pair
  *r1 = gasdev(s);
  double aux = gasdev(s);
  if (r2) *r2 = aux;
}

// ---------------------------------------------------------------- system
enum FF { FF_NONE = 0, FF_LJ = 1, FF_SMATB = 2, FF_TERSOFF = 3, FF_SLJ = 4 };
enum INTEG { IT_NONE = 0, IT_VV = 1, IT_ERMAK = 2, IT_FIRE = 3, IT_LGF = 4, IT_AXES = 5, IT_LKD = 6, IT_NORD = 7,
             IT_BROWN = 8 };

// One integrator acting on one coordinate of every atom (integrate objects
// set by `evolve piston_lgf x|y|z` and `evolve ermak_x|y|z`,
// Integration.F90:157-186): a G-JF piston on that box length
// (set_lgf_flex, :652-696) or Ermak Langevin dynamics (set_ermak with a
// coordinate, :909-961).  The reference runs a system's integrators in
// the order they were added.
enum AXMODE { AX_FLEX = 1, AX_ERMAK = 2 };
struct AxisInt {
  int mode = 0, d = 0;
  double fac0 = 0, facg0 = 0, kin = 0, press = 0, ipm = 0, bv = 0, facv = 0, av = 0;  // piston
  double pf = 0, pvel = 0, rangv = 0;
  bool first = true;
  double cc0 = 0, cc1 = 0, cc2 = 0, sdr = 0, sdv = 0, crv1 = 0, crv2 = 0, skt = 0;  // Ermak
};
const int MAXT = 8;

// 27-cell stencil in the reference's order (Neighbour.F90:75-83): 0 is the
// centre, 1..13 the upper half, 14..26 the lower half.
const int cmap[27][3] = {
    {0, 0, 0},   {1, 0, 0},   {1, 1, 0},  {0, 1, 0},   {-1, 1, 0},
    {1, 0, -1},  {1, 1, -1},  {0, 1, -1}, {-1, 1, -1}, {1, 0, 1},
    {1, 1, 1},   {0, 1, 1},   {-1, 1, 1}, {0, 0, 1},   {-1, 0, 0},
    {-1, -1, 0}, {0, -1, 0},  {1, -1, 0}, {-1, 0, 1},  {-1, -1, 1},
    {0, -1, 1},  {1, -1, 1},  {-1, 0, -1}, {-1, -1, -1}, {0, -1, -1},
    {1, -1, -1}, {0, 0, -1}};

struct LJp {
  bool on = false;
  double e = 0, s = 0, rc = 0, rc2 = 0;
  bool shifted_force = false;  // plj (Pairs.F90:282-370)
  double prc = 0, frc = 0;
  double eshift = 0;           // constant energy shift per pair (eV)
  bool sm1 = false;            // sm1 (Pairs.F90:916-1011): smooth step from r1 to rc
  double r1 = 0;
};

struct SLJp {  // slj (Pairs.F90:374-401): LJ with a splined tail from rs to rc
  bool on = false;
  double e = 0, s = 0, rs = 0, rc = 0, rc2 = 0, sa4 = 0, sa8 = 0;
};

struct SMp {  // TB.F90:66-102 per type pair
  bool on = false;
  double ca = 0, eps = 0, p = 0, q = 0, r0 = 0, rci = 0, rce = 0;
  double b1 = 0, b2 = 0, b3 = 0, r1 = 0, r2 = 0, r3 = 0;
};

struct TSp {  // Tersoff 1988 parameter set (single species)
  double A = 0, B = 0, l1 = 0, l2 = 0, beta = 0, n = 1, c = 0, d = 1, h = 0,
         R = 0, D = 0, chi = 1.0;
};

struct Sys {
  int n = 0;
  std::vector<double> pos, vel, acel, force, pos_old, pos_v, vel_v;
  std::vector<double> acel2, acel3, acel4;  // Nordsieck derivatives (Atoms.F90:77-79)
  std::vector<double> epot, mass, one_mass, one_sqrt_mass;
  std::vector<int> type;
  bool boxed = false;
  double box[3] = {0, 0, 0}, one_box[3] = {0, 0, 0};
  int pbc[3] = {0, 0, 0};
  bool mic = true;  // Program_Types.F90:98
  double skin = 1.0;  // nb_dcut, Neighbour.F90:237
  // skin test on minimum-image displacements (the device library's default):
  // an atom wrapped by do_pbc then does not count as having moved a box
  // length.  Forces are unchanged; the list is rebuilt less often.
  bool skin_mic = false;
  bool half = false;  // OpenMP default: full lists (Neighbour.F90:160-171)
  // neighbour list, column-major like list(n1+100,mnb)
  int cap = 0;
  std::vector<int> nn, list;
  bool first = true;
  long nupd = 0;
  bool use_cells = false;
  int ncells[3] = {1, 1, 1};
  double cell[3] = {0, 0, 0};
  std::vector<int> head, clist;
  int overflow = 0, lost = 0;
  // force field
  int ff = FF_NONE;
  int ntypes = 1;
  LJp lj[MAXT][MAXT];
  SLJp slj[MAXT][MAXT];
  SMp sm[MAXT][MAXT];
  double virial[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // pair virial of the last interact (internal units)
  TSp ts;
  double rcut = 0;  // intergroup rcut (max over pairs)
  std::vector<double> band, eband;
  // integrator
  int integ = IT_NONE;
  double dt = 0.002;
  double cc0 = 0, cc1 = 0, cc2 = 0, sdr = 0, sdv = 0, crv1 = 0, crv2 = 0,
         skt = 0, gama = 0, temp = 0;
  Lcg* rng = nullptr;
  double bd_fac1 = 0, bd_fac2 = 0;  // set_cbrownian (Integration.F90:834-853)
  // thermostat run after the integrator's step b (integration_stepb runs
  // every integrator's stepb in the order the deck adds them)
  int thermo = 0;  // 0 none, 1 scalvel, 2 scalvel_after, 3 andersen
  double th_temp = 0, th_soft = 0, th_upto = 0, th_factor = 0, th_nu = 0;
  const double* ext_normals = nullptr;  // optional external normal stream
  // G-JF constant-pressure state (set_lgf, Integration.F90:486-525)
  double lgf_fac0 = 0, lgf_facg0 = 0, lgf_kinetic = 0, lgf_press = 0, lgf_inv_pmass = 0, lgf_bv = 0,
         lgf_facv = 0, lgf_av = 0, lgf_rangv = 0, pvel = 0, pistonf = 0;
  bool lgf_first = true;
  std::vector<AxisInt> axes;  // IT_AXES: the per-coordinate integrators in order
  // LKD piston (set_lkd, Integration.F90:329-355): noise amplitudes, target
  // pressure (internal units), frictions and piston mass
  double lkd_fac0 = 0, lkd_facv = 0, lkd_press = 0, lkd_g0 = 0, lkd_gv = 0, lkd_pmass = 0;
  int ext_used = 0;  // normals of the external stream used this step
  // FIRE state
  double fire_dt = 0, fire_dtmax = 0, fire_alpha = 0.1;
  int fire_np = 0;
  double last_epot = 0;
};

inline double idnint(double x) { return std::round(x); }  // half away from 0

// vdistance(i,j) = pos_i - pos_j with minimum image (Inq_Properties.F90:137-157)
inline void vdist(const Sys& s, int i, int j, double vd[3]) {
  for (int l = 0; l < 3; l++) vd[l] = s.pos[3 * i + l] - s.pos[3 * j + l];
  if (!s.mic) return;
  for (int l = 0; l < 3; l++)
    if (s.pbc[l]) vd[l] = vd[l] - s.box[l] * idnint(vd[l] * s.one_box[l]);
}

inline double dot3(const double v[3]) {  // dot_product(vd,vd), left to right
  return v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
}

void ensure_cap(Sys& s, int cap) {
  if (cap <= s.cap && (int)s.nn.size() == s.n) return;
  s.cap = std::max(cap, s.cap);
  s.nn.assign(s.n, 0);
  s.list.assign((size_t)s.n * s.cap, 0);
}

inline void add_nb(Sys& s, int i, int j) {
  int m = s.nn[i];
  if (m >= s.cap) {
    s.overflow = 1;
    return;
  }
  s.list[(size_t)m * s.n + i] = j;
  s.nn[i] = m + 1;
}

// verlet_self / verlet_selfhalf (Neighbour.F90:676-811): keeps rd <= rlist^2
void verlet_build(Sys& s) {
  double rcut = s.rcut + s.skin;
  rcut = rcut * rcut;
  std::fill(s.nn.begin(), s.nn.end(), 0);
  const int n = s.n;
  if (!s.half) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; i++) {
      double vd[3];
      for (int j = 0; j < n; j++) {
        if (i == j) continue;
        vdist(s, i, j, vd);
        double rd = dot3(vd);
        if (rd > rcut) continue;
        add_nb(s, i, j);
      }
    }
  } else {
    for (int i = 0; i < n; i++) {
      double vd[3];
      for (int j = i + 1; j < n; j++) {
        vdist(s, i, j, vd);
        double rd = dot3(vd);
        if (rd > rcut) continue;
        add_nb(s, i, j);
      }
    }
  }
}

// cell_pbc (Neighbour.F90:1350-1376), 0-based cells
inline bool cell_pbc(const Sys& s, int r[3]) {
  if (s.mic) {
    for (int l = 0; l < 3; l++) r[l] = ((r[l] + s.ncells[l]) % s.ncells[l]);
    return true;
  }
  for (int l = 0; l < 3; l++)
    if (r[l] < 0 || r[l] >= s.ncells[l]) return false;
  return true;
}

// sort_in_cells (Neighbour.F90:927-989): head/next chain, reversed insertion
bool sort_in_cells(Sys& s) {
  int nc = s.ncells[0] * s.ncells[1] * s.ncells[2];
  s.head.assign(nc, -1);
  s.clist.assign(s.n, -1);
  double one_cell[3];
  for (int l = 0; l < 3; l++) one_cell[l] = 1.0 / s.cell[l];
  for (int i = 0; i < s.n; i++) {
    int c[3];
    for (int l = 0; l < 3; l++) {
      double v = s.pos[3 * i + l] * one_cell[l];
      c[l] = (int)v;  // int() truncates toward zero
      if (c[l] < 0 || c[l] >= s.ncells[l]) {
        // Out-of-grid atoms are undefined behaviour in the reference; the
        // restatement clamps them into the grid and records the event.
        s.lost = 1;
        c[l] = c[l] < 0 ? 0 : s.ncells[l] - 1;
      }
    }
    int id = c[0] + s.ncells[0] * (c[1] + s.ncells[1] * c[2]);
    s.clist[i] = s.head[id];
    s.head[id] = i;
  }
  return true;
}

// linkedcell_self / linkedcell_selfhalf (Neighbour.F90:991-1161): strict <
void linkedcell_build(Sys& s) {
  double rcut = s.rcut + s.skin;
  rcut = rcut * rcut;
  std::fill(s.nn.begin(), s.nn.end(), 0);
  sort_in_cells(s);
  const int nc = s.ncells[0] * s.ncells[1] * s.ncells[2];
  const int nstencil = s.half ? 14 : 27;
#pragma omp parallel for schedule(dynamic, 4) if (!s.half)
  for (int ic = 0; ic < nc; ic++) {
    int rc[3] = {ic % s.ncells[0], (ic / s.ncells[0]) % s.ncells[1],
                 ic / (s.ncells[0] * s.ncells[1])};
    for (int nb = 0; nb < nstencil; nb++) {
      int c[3] = {rc[0] + cmap[nb][0], rc[1] + cmap[nb][1], rc[2] + cmap[nb][2]};
      if (!cell_pbc(s, c)) continue;
      int nid = c[0] + s.ncells[0] * (c[1] + s.ncells[1] * c[2]);
      for (int i = s.head[ic]; i >= 0; i = s.clist[i]) {
        int j;
        if (s.half && nb == 0)
          j = s.clist[i];
        else
          j = s.head[nid];
        for (; j >= 0; j = s.clist[j]) {
          if (!s.half && i == j) continue;
          double vd[3];
          vdist(s, j, i, vd);  // respetar el orden
          double rd = dot3(vd);
          if (rd < rcut) add_nb(s, i, j);
        }
      }
    }
  }
}

// intergroup_setcells (Neighbour.F90:587-664) + update (:1242-1299)
void update(Sys& s) {
  s.nupd++;
  s.pos_old = s.pos;
  s.use_cells = false;
  if (s.boxed) {
    double rc = s.rcut + s.skin;
    bool any4 = false;
    for (int l = 0; l < 3; l++) {
      s.ncells[l] = (int)(s.box[l] / rc);
      if (s.ncells[l] >= 4) any4 = true;
    }
    if (any4) {
      s.use_cells = true;
      for (int l = 0; l < 3; l++) s.cell[l] = s.box[l] / s.ncells[l];
    }
  }
  if (s.use_cells)
    linkedcell_build(s);
  else
    verlet_build(s);
}

// test_update (Neighbour.F90:1305-1346)
bool test_update(Sys& s) {
  double d1 = 1.e-16, d2 = 1.e-16;
  for (int i = 0; i < s.n; i++) {
    double vd[3];
    for (int l = 0; l < 3; l++) {
      vd[l] = s.pos[3 * i + l] - s.pos_old[3 * i + l];
      if (s.skin_mic && s.boxed && s.pbc[l]) vd[l] = vd[l] - s.box[l] * idnint(vd[l] * s.one_box[l]);
    }
    double rd = dot3(vd);
    if (rd > d1) {
      d2 = d1;
      d1 = rd;
    } else if (rd > d2) {
      d2 = rd;
    }
  }
  if (std::sqrt(d1) + std::sqrt(d2) > s.skin) {
    update(s);
    return true;
  }
  return false;
}

// x**6 the way gfortran expands it (x3 = x2*x, x6 = x3*x3)
inline double pow6(double x) {
  double x3 = x * x * x;
  return x3 * x3;
}

// lj_interact / plj_interact (Pairs.F90:207-370), full list, newton off
double lj_interact(Sys& s) {
  double etot = 0.0;
  const int n = s.n;
  // the total is summed from the per-atom sums in atom order: the same
  // bits for any thread count (an OpenMP reduction combines the threads'
  // partial sums in an unspecified order)
  std::vector<double> ea(n, 0.0);
  // pair virial W = 1/2 sum over the full list of vd (x) f vd / r (complete;
  // the reference's lj, Pairs.F90:254-272, omits the i-side term)
  std::vector<double> wa(9 * (size_t)n, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int ti = s.type[i];
    double fx = 0, fy = 0, fz = 0, ep = 0;
    double* W = &wa[9 * (size_t)i];
    for (int l = 0; l < s.nn[i]; l++) {
      int j = s.list[(size_t)l * n + i];
      const LJp& P = s.lj[ti][s.type[j]];
      if (!P.on) continue;
      double vd[3];
      vdist(s, j, i, vd);
      double dr = dot3(vd);
      if (dr > P.rc2) continue;
      dr = std::sqrt(dr);
      double s_dr = pow6(P.s / dr);
      double p, f;
      if (P.sm1) {
        // sm1_interact (Pairs.F90:925-1011): p = e (1/2 + 1/2 sin(aux)) - e
        // beyond r1, -e inside; the reference's force carries a factor dr
        // (Pairs.F90:957), kept; the sign flips into this loop's convention
        // (F_i -= f vd / r, the reference's sm1 adds f vd / r)
        if (dr > P.r1) {
          const double aux = pi * (dr - (P.r1 + P.rc) * 0.5) / (P.rc - P.r1);
          p = 0.5 + 0.5 * std::sin(aux);
          f = std::cos(aux) * pio2 * dr / (P.rc - P.r1);
          p = p * P.e - P.e;
          f = -(f * P.e);
        } else {
          p = -P.e;
          f = 0.0;
        }
      } else if (P.shifted_force) {
        p = 4.0 * P.e * (s_dr * s_dr - s_dr) - P.prc - P.frc * (dr - P.rc);
        f = P.e * (48.0 * s_dr - 24.0) * s_dr / dr + P.frc;
      } else {
        p = 4.0 * P.e * (s_dr * s_dr - s_dr) - P.eshift;
        f = P.e * (48.0 * s_dr - 24.0) * s_dr / dr;
      }
      p = p * ev_ui;
      f = f * ev_ui;
      ep = ep + p * 0.5;
      // f == 0 (sm1 inside r1) adds nothing, also at dr == 0 where the
      // reference's -0 vd / dr is not a number
      if (f == 0.0) continue;
      const double f2[3] = {f * vd[0] / dr, f * vd[1] / dr, f * vd[2] / dr};
      fx = fx - f2[0];
      fy = fy - f2[1];
      fz = fz - f2[2];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) W[3 * a + b] += 0.5 * vd[a] * f2[b];
    }
    s.force[3 * i] += fx;
    s.force[3 * i + 1] += fy;
    s.force[3 * i + 2] += fz;
    s.epot[i] += ep;
    ea[i] = ep;
  }
  for (int i = 0; i < n; i++) etot += ea[i];
  for (int k = 0; k < 9; k++) s.virial[k] = 0.0;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 9; k++) s.virial[k] += wa[9 * (size_t)i + k];
  return etot;
}

// slj_set (Pairs.F90:374-401): cut-off and spline coefficients
void slj_set(SLJp& P, double e, double sg, double rs) {
  P.on = true;
  P.e = e;
  P.s = sg;
  P.rs = rs;
  const double s_dr = pow6(sg / rs);
  const double urs = 4.0 * e * (s_dr * s_dr - s_dr);
  const double dudrs = -e * (48.0 * s_dr - 24.0) * s_dr / rs;
  P.rc = rs - 32.0 * urs / (11.0 * dudrs);
  P.rc2 = P.rc * P.rc;
  const double d = P.rc - rs;
  P.sa4 = (8.0 * urs + d * dudrs) / (4 * (d * d * d * d));
  P.sa8 = -(4.0 * urs + d * dudrs) / (4 * (d * d * d * d * d * d * d * d));
}

// slj_interact (Pairs.F90:403-470) over the full list, with the pair virial
// W = sum_i r_i (x) F_i, which with minimum image is 1/2 sum over the
// ordered pairs of vd (x) factor2 (vd = r_j - r_i): the virial the reference
// builds from local and ghost atoms (inq_virial, Inq_Properties.F90:439-527)
double slj_interact(Sys& s) {
  double etot = 0.0;
  const int n = s.n;
  double W[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < n; i++) {
    int ti = s.type[i];
    double fx = 0, fy = 0, fz = 0, ep = 0;
    for (int l = 0; l < s.nn[i]; l++) {
      int j = s.list[(size_t)l * n + i];
      const SLJp& P = s.slj[ti][s.type[j]];
      if (!P.on) continue;
      double vd[3];
      vdist(s, j, i, vd);
      double dr = dot3(vd);
      if (dr > P.rc2) continue;
      dr = std::sqrt(dr);
      double p, f;
      if (dr < P.rs) {
        const double s_dr = pow6(P.s / dr);
        p = 4.0 * P.e * (s_dr - 1.0) * s_dr;
        f = P.e * (48.0 * s_dr - 24.0) * s_dr / dr;
      } else {
        const double s4 = (dr - P.rc) * (dr - P.rc) * (dr - P.rc) * (dr - P.rc);
        p = P.sa4 * s4 + P.sa8 * s4 * s4;
        f = -(4.0 * P.sa4 * s4 + 8.0 * P.sa8 * s4 * s4) / (dr - P.rc);
      }
      p = p * ev_ui;
      f = f * ev_ui;
      ep = ep + p * 0.5;
      etot = etot + p * 0.5;
      const double f2[3] = {f * vd[0] / dr, f * vd[1] / dr, f * vd[2] / dr};
      fx = fx - f2[0];
      fy = fy - f2[1];
      fz = fz - f2[2];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) W[3 * a + b] += 0.5 * vd[a] * f2[b];
    }
    s.force[3 * i] += fx;
    s.force[3 * i + 1] += fy;
    s.force[3 * i + 2] += fz;
    s.epot[i] += ep;
  }
  for (int k = 0; k < 9; k++) s.virial[k] = W[k];
  return etot;
}

// smatb_set (TB.F90:106-170): tail polynomial coefficients (Logsdail 2012)
void smatb_set(SMp& P, double a, double eps, double p, double q, double r0,
               double rci, double rce) {
  P.on = true;
  P.ca = a; P.eps = eps; P.p = p; P.q = q; P.r0 = r0; P.rci = rci; P.rce = rce;
  double dcut = rce - rci;
  double ab = -1.0 / (dcut * dcut * dcut);
  double bb = -(q / r0) / (dcut * dcut);
  double cb = -((q / r0) * (q / r0)) / dcut;
  double aux = eps * std::exp(-q * (rci / r0 - 1.0));
  P.b1 = aux * (12.0 * ab - 6.0 * bb + cb) / (2.0 * (dcut * dcut));
  P.b2 = aux * (15.0 * ab - 7.0 * bb + cb) / dcut;
  P.b3 = aux * (20.0 * ab - 8.0 * bb + cb) / 2.0;
  aux = a * std::exp(-p * (rci / r0 - 1.0));
  bb = -(p / r0) / (dcut * dcut);
  cb = -((p / r0) * (p / r0)) / dcut;
  P.r1 = aux * (12.0 * ab - 6.0 * bb + cb) / (2.0 * (dcut * dcut));
  P.r2 = aux * (15.0 * ab - 7.0 * bb + cb) / dcut;
  P.r3 = aux * (20.0 * ab - 8.0 * bb + cb) / 2.0;
}

// smatb_preinteraction (TB.F90:367-455) + smatb_interact (TB.F90:457-586)
double smatb_interact(Sys& s) {
  const int n = s.n;
  s.band.assign(n, 0.0);
  s.eband.assign(n, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int z1 = s.type[i];
    double band = 0.0;
    for (int l = 0; l < s.nn[i]; l++) {
      int j = s.list[(size_t)l * n + i];
      const SMp& P = s.sm[z1][s.type[j]];
      double vd[3];
      vdist(s, j, i, vd);
      double dr = std::sqrt(dot3(vd));
      if (dr > P.rce) continue;
      double banda;
      if (dr < P.rci) {
        double r0 = P.r0;
        banda = P.eps * P.eps * std::exp(-2.0 * P.q * (dr / r0 - 1.0));
      } else {
        double drm = dr - P.rce;
        double drm2 = drm * drm, drm3 = drm2 * drm, drm4 = drm3 * drm,
               drm5 = drm4 * drm;
        banda = P.b1 * drm5 + P.b2 * drm4 + P.b3 * drm3;
        banda = banda * banda;
      }
      band = band + banda;
    }
    s.band[i] = band;
  }
  for (int i = 0; i < n; i++) s.eband[i] = 1.0 / std::sqrt(s.band[i]);

  const double lev_ui = ev_ui;
  double epot = 0.0;
  std::vector<double> ea(n, 0.0);  // per-atom sums, added in atom order below
  // pair virial W = 1/2 sum over the full list of vd (x) factor vd / r: the
  // SMA-TB forces are central pair forces (the reference's TB.F90:548-564
  // omits the i-side term; this is the complete sum)
  std::vector<double> wa(9 * (size_t)n, 0.0);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    int z1 = s.type[i];
    double f[3] = {0, 0, 0}, ep = 0.0;
    double* W = &wa[9 * (size_t)i];
    for (int l = 0; l < s.nn[i]; l++) {
      int j = s.list[(size_t)l * n + i];
      const SMp& P = s.sm[z1][s.type[j]];
      double vd[3];
      vdist(s, j, i, vd);
      double dr = std::sqrt(dot3(vd));
      double factor = 0.0, repul = 0.0;
      if (dr > P.rce) continue;
      if (dr <= P.rci) {
        double r0 = P.r0;
        repul = P.ca * std::exp(-P.p * (dr / r0 - 1.0));
        factor = 2.0 * repul * (P.p / r0) -
                 P.eps * P.eps * 1.0 / 2.0 *
                     std::exp(-2.0 * P.q * (dr / r0 - 1.0)) *
                     (2.0 * P.q / r0) * (s.eband[i] + s.eband[j]);
      } else {
        double drm = dr - P.rce;
        double drm2 = drm * drm, drm3 = drm2 * drm, drm4 = drm3 * drm,
               drm5 = drm4 * drm;
        factor = (P.b1 * drm5 + P.b2 * drm4 + P.b3 * drm3) *
                 (5.0 * P.b1 * drm4 + 4.0 * P.b2 * drm3 + 3.0 * P.b3 * drm2) *
                 (s.eband[i] + s.eband[j]);
        factor = factor -
                 2.0 * (5.0 * P.r1 * drm4 + 4.0 * P.r2 * drm3 + 3.0 * P.r3 * drm2);
        repul = P.r1 * drm5 + P.r2 * drm4 + P.r3 * drm3;
      }
      double f2[3];
      for (int k = 0; k < 3; k++) {
        f2[k] = factor * lev_ui * vd[k] / dr;
        f[k] = f[k] - f2[k];
      }
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) W[3 * a + b] += 0.5 * vd[a] * f2[b];
      ep = ep + repul * lev_ui;
    }
    double aux2 = std::sqrt(s.band[i]) * lev_ui;
    ep = ep - aux2;
    for (int k = 0; k < 3; k++) s.force[3 * i + k] += f[k];
    s.epot[i] += ep;
    ea[i] = ep;
  }
  for (int i = 0; i < n; i++) epot += ea[i];
  for (int k = 0; k < 9; k++) s.virial[k] = 0.0;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 9; k++) s.virial[k] += wa[9 * (size_t)i + k];
  return epot;
}

// fcut_dfcut (Algebra.F90:391-409)
inline double fcut_dfcut(double r, double r1, double r2, double* dfc) {
  if (r < r1) {
    *dfc = 0.0;
    return 1.0;
  } else if (r > r2) {
    *dfc = 0.0;
    return 0.0;
  }
  double aux = pi * (r - (r1 + r2) * 0.5) / (r2 - r1);
  *dfc = -std::cos(aux) * pio2 / (r2 - r1);
  return 0.5 - 0.5 * std::sin(aux);
}

// Tersoff 1988 (PRB 37, 6991), restated with forces that are the exact
// gradient of E = sum_i sum_{j!=i} 1/2 fc(r_ij) [VR(r_ij) + b_ij VA(r_ij)].
// Same functional form and cutoff as Tersoff.f90:131-341 + Algebra.F90:
// 391-409 (no lambda3 term, chi prefactor); the reference's missing radial
// force on j and its unallocated gradb_k are NOT reproduced.
double tersoff_interact(Sys& s) {
  const TSp& T = s.ts;
  const int n = s.n;
  const double r1 = T.R - T.D, r2 = T.R + T.D;
  const double c2 = T.c * T.c, d2 = T.d * T.d;
  const double btnp = std::pow(T.beta, T.n);
  const double A = T.A * ev_ui, B = T.B * ev_ui;
  double etot = 0.0;
  // Per-atom forces are gathered into a private buffer per thread and
  // reduced in a fixed order afterwards (deterministic).
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  std::vector<double> fbuf((size_t)nth * 3 * n, 0.0);
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* F = &fbuf[(size_t)tid * 3 * n];
    std::vector<int> kk;
    std::vector<double> kv, kr;
#pragma omp for schedule(static)
    for (int i = 0; i < n; i++) {
      // gather bonded neighbours of i (r <= r2)
      kk.clear(); kv.clear(); kr.clear();
      for (int m = 0; m < s.nn[i]; m++) {
        int j = s.list[(size_t)m * n + i];
        double vd[3];
        vdist(s, j, i, vd);  // r_j - r_i
        double rd = std::sqrt(dot3(vd));
        if (rd > r2) continue;
        kk.push_back(j);
        kr.push_back(rd);
        kv.push_back(vd[0] / rd); kv.push_back(vd[1] / rd); kv.push_back(vd[2] / rd);
      }
      const int nb = (int)kk.size();
      for (int a = 0; a < nb; a++) {
        int j = kk[a];
        double rij = kr[a];
        const double* u = &kv[3 * a];
        double dfc;
        double fc = fcut_dfcut(rij, r1, r2, &dfc);
        double vr = A * std::exp(-T.l1 * rij), dvr = -T.l1 * vr;
        double va = -B * std::exp(-T.l2 * rij), dva = -T.l2 * va;
        // zeta_ij and its pieces
        double zij = 0.0;
        for (int b = 0; b < nb; b++) {
          if (b == a) continue;
          double dfk;
          double fk = fcut_dfcut(kr[b], r1, r2, &dfk);
          const double* w = &kv[3 * b];
          double ct = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
          double hc = T.h - ct;
          double g = 1.0 + c2 / d2 - c2 / (d2 + hc * hc);
          zij += fk * g;
        }
        double bij, dbdz;
        if (zij > 1.0e-15) {
          double zn = std::pow(zij, T.n);
          double aux = 1.0 / (1.0 + btnp * zn);
          bij = T.chi * std::pow(aux, 0.5 / T.n);
          dbdz = -0.5 * bij * aux * btnp * std::pow(zij, T.n - 1.0);
        } else {
          bij = T.chi;
          dbdz = 0.0;
        }
        double e = 0.5 * fc * (vr + bij * va);
        s.epot[i] += e;
        // radial part: dE/dr_ij along u (u points i->j)
        double dV = 0.5 * (dfc * (vr + bij * va) + fc * (dvr + bij * dva));
        for (int k = 0; k < 3; k++) {
          F[3 * i + k] += dV * u[k];
          F[3 * j + k] -= dV * u[k];
        }
        if (dbdz == 0.0) continue;
        double pre = 0.5 * fc * va * dbdz;  // dE/dzeta
        for (int b = 0; b < nb; b++) {
          if (b == a) continue;
          int k = kk[b];
          double rik = kr[b];
          const double* w = &kv[3 * b];
          double dfk;
          double fk = fcut_dfcut(rik, r1, r2, &dfk);
          double ct = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
          double hc = T.h - ct;
          double den = d2 + hc * hc;
          double g = 1.0 + c2 / d2 - c2 / den;
          double dg = -2.0 * c2 * hc / (den * den);  // dg/dcos
          // d cos / d r_j = (w - ct u)/rij ; d cos / d r_k = (u - ct w)/rik
          for (int q = 0; q < 3; q++) {
            double dcj = (w[q] - ct * u[q]) / rij;
            double dck = (u[q] - ct * w[q]) / rik;
            double gj = fk * dg * dcj;                      // dzeta/dr_j
            double gk = dfk * g * w[q] + fk * dg * dck;     // dzeta/dr_k
            F[3 * j + q] -= pre * gj;
            F[3 * k + q] -= pre * gk;
            F[3 * i + q] += pre * (gj + gk);
          }
        }
      }
    }
  }
  for (int t = 0; t < nth; t++)
    for (size_t q = 0; q < (size_t)3 * n; q++) s.force[q] += fbuf[(size_t)t * 3 * n + q];
  for (int i = 0; i < n; i++) etot += s.epot[i];  // atom order: the same bits for any thread count
  return etot;
}

// interact (Interaction.f90:135-241): list test/update, zero, force field
double interact(Sys& s, bool* rebuilt) {
  bool rb;
  if (s.first) {
    s.first = false;
    update(s);
    rb = true;
  } else {
    rb = test_update(s);
  }
  if (rebuilt) *rebuilt = rb;
  std::fill(s.force.begin(), s.force.end(), 0.0);
  std::fill(s.epot.begin(), s.epot.end(), 0.0);
  double e = 0.0;
  if (s.ff == FF_LJ) e = lj_interact(s);
  else if (s.ff == FF_SMATB) e = smatb_interact(s);
  else if (s.ff == FF_TERSOFF) e = tersoff_interact(s);
  else if (s.ff == FF_SLJ) e = slj_interact(s);
  s.last_epot = e;
  return e;
}

// do_pbc_1 (Set_Properties.f90:444-470)
void do_pbc(Sys& s) {
  if (!s.boxed) return;
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++)
      if (s.pbc[k]) {
        if (s.pos[3 * i + k] >= s.box[k])
          s.pos[3 * i + k] = s.pos[3 * i + k] - s.box[k];
        else if (s.pos[3 * i + k] < 0.0)
          s.pos[3 * i + k] = s.pos[3 * i + k] + s.box[k];
      }
}

// set_ermak (Integration.F90:909-961)
void set_ermak(Sys& s, double dt, double gama, double temp) {
  s.integ = IT_ERMAK;
  s.dt = dt;
  s.gama = gama;
  s.temp = temp;
  s.cc0 = std::exp(-dt * gama);
  s.cc1 = (1.0 - s.cc0) / gama;
  s.cc2 = (1.0 - s.cc1 / dt) / gama;
  s.sdr = std::sqrt(dt / gama * (2.0 - (3.0 - 4.0 * s.cc0 + s.cc0 * s.cc0) / (dt * gama)));
  s.sdv = std::sqrt(1.0 - s.cc0 * s.cc0);
  s.crv1 = (1.0 - s.cc0) * (1.0 - s.cc0) / (gama * s.sdr * s.sdv);
  s.crv2 = std::sqrt(1.0 - (s.crv1 * s.crv1));
  s.skt = std::sqrt(kB_ui * temp);
}

// velocity_verlet_a (Integration.F90:1150-1168)
void vv_a(Sys& s) {
  double acel_dv = s.dt * 0.5, acel_dx = acel_dv * s.dt;
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++) {
      int q = 3 * i + k;
      s.acel[q] = s.force[q] * s.one_mass[i];
      s.pos[q] = s.pos[q] + s.dt * s.vel[q] + acel_dx * s.acel[q];
      s.vel[q] = s.vel[q] + acel_dv * s.acel[q];
    }
}

// velocity_verlet_b (Integration.F90:1171-1186)
void vv_b(Sys& s) {
  double acel_dv = s.dt * 0.5;
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++) {
      int q = 3 * i + k;
      s.acel[q] = s.force[q] * s.one_mass[i];
      s.vel[q] = s.vel[q] + acel_dv * s.acel[q];
    }
}

// nordsieck_predictor (Integration.F90:1192-1228): the fifth-order Gear
// predictor on the scaled derivatives (vel dt, acel = dt^2/2 F/m after a
// correction, acel2..4 the higher ones); sums left to right as written
void nord_a(Sys& s) {
  for (int q = 0; q < 3 * s.n; q++) {
    s.vel[q] = s.vel[q] * s.dt;
    const double p1 = s.acel[q], p2 = s.acel2[q], p4 = s.acel3[q], p7 = s.acel4[q];
    const double p3 = 3 * p2, p5 = 2 * p4, p6 = 2 * p5, p8 = 5 * p7, p9 = 2 * p8;
    s.pos[q] = p7 + p4 + p2 + p1 + s.vel[q] + s.pos[q];
    s.vel[q] = p8 + p6 + p3 + p1 + p1 + s.vel[q];
    s.acel[q] = p9 + p6 + p5 + p3 + p1;
    s.acel2[q] = p9 + p6 + p2;
    s.acel3[q] = p8 + p4;
  }
}

// nordsieck_corrector (Integration.F90:1230-1268): Allen & Tildesley's
// coefficients for second-order equations (c0 = 3/20)
void nord_b(Sys& s) {
  const double c0 = 3.0 / 20.0, c1 = 251.0 / 360.0, c3 = 11.0 / 18.0, c4 = 1.0 / 6.0, c5 = 1.0 / 60.0;
  const double dt2_2 = s.dt * s.dt / 2.0;
  for (int i = 0; i < s.n; i++) {
    const double half_mass = dt2_2 * s.one_mass[i];
    for (int k = 0; k < 3; k++) {
      const int q = 3 * i + k;
      const double p = half_mass * s.force[q] - s.acel[q];
      s.pos[q] = s.pos[q] + p * c0;
      s.vel[q] = s.vel[q] + p * c1;
      s.acel[q] = s.acel[q] + p;
      s.acel2[q] = s.acel2[q] + p * c3;
      s.acel3[q] = s.acel3[q] + p * c4;
      s.acel4[q] = s.acel4[q] + p * c5;
      s.vel[q] = s.vel[q] / s.dt;
    }
  }
}

// cbrownian (Integration.F90:855-882), the step b of `evolve brownian`
// (step a does nothing): x += F/m dt/gamma + r sqrt(2 kT dt/gamma / m) with
// r the first normal of a rang pair per coordinate; v = (x - x_old) / dt
void brownian_b(Sys& s) {
  for (int i = 0; i < s.n; i++)
    for (int j = 0; j < 3; j++) {
      double r1, r2;
      if (s.ext_normals) {
        r1 = s.ext_normals[6 * i + 2 * j];
      } else {
        rang(*s.rng, &r1, &r2);
      }
      const int q = 3 * i + j;
      const double posold = s.pos[q];
      s.pos[q] = posold + s.one_mass[i] * s.bd_fac1 * s.force[q] + s.one_sqrt_mass[i] * r1 * s.bd_fac2;
      s.vel[q] = (s.pos[q] - posold) / s.dt;
    }
}

void kin(const Sys& s, double* ekin, double* temp);

// scalvel / scalvel_after (Integration.F90:1300-1340): v *= (T0/T)^soft
// with T from the centre-of-mass-free kinetic energy (inq_temperature,
// Inq_Properties.F90:424-434); scalvel_after only when |T - T0| > upto T0
void scalvel(Sys& s) {
  double ek, t;
  kin(s, &ek, &t);
  if (s.thermo == 2 && !(std::fabs(t - s.th_temp) > s.th_upto * s.th_temp)) return;
  if (t == 0.0) return;
  const double factor = std::pow(s.th_temp / t, s.th_soft);
  for (int q = 0; q < 3 * s.n; q++) s.vel[q] = s.vel[q] * factor;
}

// andersen (Integration.F90:1366-1395): each atom collides with
// probability nu dt (one ranu per atom) and takes v = factor / sqrt(m) r
// per coordinate (r the first normal of a rang pair), with the reference's
// factor = sqrt(kB T / (3N)^2) (set_andersen, :1343-1364)
void andersen(Sys& s) {
  const double nudt = s.th_nu * s.dt;
  for (int i = 0; i < s.n; i++) {
    const double r = lcg_ranu(*s.rng);
    if (r > nudt) continue;
    const double vel_med = s.th_factor * s.one_sqrt_mass[i];
    for (int j = 0; j < 3; j++) {
      double r1, r2;
      rang(*s.rng, &r1, &r2);
      s.vel[3 * i + j] = vel_med * r1;
    }
  }
}

// ermak_a (Integration.F90:963-1011).  Normals come from the LCG stream
// (rang, one pair per dimension) or from an external stream of 6 per atom.
void ermak_a(Sys& s) {
  for (int i = 0; i < s.n; i++) {
    double f_lan = s.skt * s.one_sqrt_mass[i];
    for (int j = 0; j < 3; j++) {
      double r1, r2;
      if (s.ext_normals) {
        r1 = s.ext_normals[6 * i + 2 * j];
        r2 = s.ext_normals[6 * i + 2 * j + 1];
      } else {
        rang(*s.rng, &r1, &r2);
      }
      s.pos_v[3 * i + j] = f_lan * s.sdr * r1;
      s.vel_v[3 * i + j] = f_lan * s.sdv * (s.crv1 * r1 + s.crv2 * r2);
    }
    for (int k = 0; k < 3; k++) {
      int q = 3 * i + k;
      s.pos[q] = s.pos[q] + s.cc1 * s.vel[q] + s.cc2 * s.dt * s.acel[q] + s.pos_v[q];
    }
  }
}

// ermak_b (Integration.F90:1013-1031)
void ermak_b(Sys& s) {
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++) {
      int q = 3 * i + k;
      s.vel[q] = s.cc0 * s.vel[q] + (s.cc1 - s.cc2) * s.acel[q] +
                 s.cc2 * s.force[q] * s.one_mass[i] + s.vel_v[q];
      s.acel[q] = s.force[q] * s.one_mass[i];
    }
}

// inq_cm_vel / inq_kin_energy / inq_temperature (Inq_Properties.F90:399-437,
// 669-698): Ekin with the centre-of-mass velocity removed.
void kin(const Sys& s, double* ekin, double* temp) {
  double cm[3] = {0, 0, 0}, mt = 0.0;
  for (int i = 0; i < s.n; i++) mt = mt + s.mass[i];
  if (s.n == 1) {
    for (int k = 0; k < 3; k++) cm[k] = s.vel[k];
  } else {
    for (int i = 0; i < s.n; i++)
      for (int k = 0; k < 3; k++) cm[k] = cm[k] + s.mass[i] * s.vel[3 * i + k];
    for (int k = 0; k < 3; k++) cm[k] = cm[k] / mt;
  }
  double ek = 0.0;
  for (int i = 0; i < s.n; i++) {
    double v[3];
    for (int k = 0; k < 3; k++) v[k] = s.vel[3 * i + k] - cm[k];
    ek = ek + dot3(v) * s.mass[i];
  }
  ek = ek * 0.5;
  *ekin = ek;
  *temp = 2.0 * ek / (kB_ui * (3 * s.n));
}

void cm_vel(const Sys& s, double cm[3]) {
  double mt = 0.0;
  for (int i = 0; i < s.n; i++) mt = mt + s.mass[i];
  cm[0] = cm[1] = cm[2] = 0.0;
  if (s.n == 1) {
    for (int k = 0; k < 3; k++) cm[k] = s.vel[k];
    return;
  }
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++) cm[k] = cm[k] + s.mass[i] * s.vel[3 * i + k];
  for (int k = 0; k < 3; k++) cm[k] = cm[k] / mt;
}

// FIRE (Bitzek et al., PRL 97, 170201 (2006)), following the intent of
// FIRE.f90:40-141 with its three defects fixed: |v| (not v.v) in the mixing,
// f_dec applied on P<=0, and every velocity reset.  Parity unpinned.
const double fire_alpha0 = 0.1, fire_finc = 1.1, fire_fdec = 0.5,
             fire_falpha = 0.99;
const int fire_nmin = 5;

void fire_init(Sys& s, double dt0, double dtmax) {
  s.integ = IT_FIRE;
  s.dt = dt0;
  s.fire_dt = dt0;
  s.fire_dtmax = dtmax;
  s.fire_alpha = fire_alpha0;
  s.fire_np = 0;
  std::fill(s.vel.begin(), s.vel.end(), 0.0);
}

// one FIRE iteration given current forces: MD half steps use velocity Verlet
// with the current fire_dt; returns max |F| (eV/A) after the force call.
void fire_mix(Sys& s) {
  // P = sum_atoms v.F (FIRE.f90:99-105)
  double P = 0.0;
  for (int q = 0; q < 3 * s.n; q++) P = P + s.vel[q] * s.force[q];
  // per-atom mixing v = (1-a) v + a |v| F/|F| (FIRE.f90:107-114, with |v|)
  for (int i = 0; i < s.n; i++) {
    double* v = &s.vel[3 * i];
    const double* f = &s.force[3 * i];
    double vn = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double fn = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    double mixf = fn > 0.0 ? s.fire_alpha * vn / fn : 0.0;
    for (int k = 0; k < 3; k++) v[k] = v[k] * (1.0 - s.fire_alpha) + mixf * f[k];
  }
  if (P > 0.0) {
    s.fire_np++;
    if (s.fire_np > fire_nmin) {
      s.fire_dt = std::min(s.fire_dt * fire_finc, s.fire_dtmax);
      s.fire_alpha = s.fire_alpha * fire_falpha;
    }
  } else {
    s.fire_np = 0;
    s.fire_dt = s.fire_dt * fire_fdec;
    s.fire_alpha = fire_alpha0;
    std::fill(s.vel.begin(), s.vel.end(), 0.0);
  }
  s.dt = s.fire_dt;
}

double fmax_ev(const Sys& s) {
  double m = 0.0;
  for (int i = 0; i < s.n; i++) {
    double v[3] = {s.force[3 * i], s.force[3 * i + 1], s.force[3 * i + 2]};
    m = std::max(m, std::sqrt(dot3(v)));
  }
  return m * ui_ev;
}

// ------------------------------------------------------------------ G-JF NPT
// Constant pressure and temperature Langevin dynamics of Gronbech-Jensen &
// Farago (J. Chem. Phys. 141, 194108, 2014) as set_lgf / lgf_stepa /
// lgf_stepb state it (Integration.F90:486-650): an isotropic piston on the
// box volume with friction pgamav and mass pmass, particles with friction
// pgama0, target pressure press (internal units) and temperature temp.
// Noise: one rang pair for the piston, then one per atom and coordinate, of
// which the first value is used (rang, Random.F90:213-226).
const double atm_ui = 1.01325 * 1.e5 * ((1.0 / (ui_ev * 1.60219e-19)) * 1e-30);  // Constants.F90:186-193

void set_lgf(Sys& s, double dt, double temp, double press, double pgama0, double pgamav, double pmass) {
  s.integ = IT_LGF;
  s.dt = dt;
  s.temp = temp;
  s.lgf_fac0 = std::sqrt(2.0 * pgama0 * kB_ui * temp * dt);
  s.lgf_facg0 = 0.5 * dt * pgama0;
  s.lgf_kinetic = s.n * temp * kB_ui;
  s.lgf_press = press;
  s.lgf_inv_pmass = 1.0 / pmass;
  s.lgf_bv = 1.0 / (1.0 + 0.5 * dt * s.lgf_inv_pmass * pgamav);
  s.lgf_facv = std::sqrt(2.0 * pgamav * kB_ui * temp * dt);
  s.lgf_av = (1.0 - 0.5 * dt * s.lgf_inv_pmass * pgamav) * s.lgf_bv;
  s.lgf_first = true;
  s.pvel = 0.0;
  s.pistonf = 0.0;
  if ((int)s.pos_v.size() < 3 * s.n) s.pos_v.assign(3 * s.n, 0.0);
}

double lgf_normal(Sys& s, int q) {  // q: 0 = piston, 1 + 3i + k = atom i, coordinate k
  if (s.ext_normals) return s.ext_normals[2 * q];
  double r1, r2;
  rang(*s.rng, &r1, &r2);
  return r1;
}

void lgf_a(Sys& s) {
  const double dt = s.dt;
  const double vol0 = s.box[0] * s.box[1] * s.box[2];
  if (s.lgf_first) {
    s.lgf_first = false;
    const double sv = (s.virial[0] + s.virial[4] + s.virial[8]) / 3;
    s.pistonf = (sv + s.lgf_kinetic) / vol0 - s.lgf_press;
  }
  // the box volume, then the lengths: L (V/V_old)^(1/3) with the exponent
  // the single-precision 1./dd of the reference
  const double rangv = lgf_normal(s, 0) * s.lgf_facv;
  double vol = vol0 + s.lgf_bv * dt * (s.pvel + 0.5 * s.lgf_inv_pmass * (dt * s.pistonf + rangv));
  s.lgf_rangv = rangv;
  double box_old[3];
  const double expo = (double)(1.0f / 3.0f);
  for (int k = 0; k < 3; k++) {
    box_old[k] = s.box[k];
    s.box[k] = box_old[k] * std::pow(vol / vol0, expo);
    s.one_box[k] = 1.0 / s.box[k];
  }
  for (int i = 0; i < s.n; i++) {
    const double b0 = 1.0 / (1.0 + s.lgf_facg0 * s.one_mass[i]);
    for (int k = 0; k < 3; k++) {
      const int q = 3 * i + k;
      const double r1 = lgf_normal(s, 1 + q);
      s.pos_v[q] = s.one_mass[i] * s.lgf_fac0 * r1;
      s.acel[q] = s.force[q] * s.one_mass[i];
      s.pos[q] = s.box[k] / box_old[k] * s.pos[q] +
                 2.0 * s.box[k] / (box_old[k] + s.box[k]) * b0 * dt * (s.vel[q] + 0.5 * dt * s.acel[q] + 0.5 * s.pos_v[q]);
    }
  }
}

void lgf_b(Sys& s) {
  const double dt = s.dt;
  const double vol = s.box[0] * s.box[1] * s.box[2];
  const double sv = (s.virial[0] + s.virial[4] + s.virial[8]) / 3;
  const double pf_old = s.pistonf;
  s.pistonf = (sv + s.lgf_kinetic) / vol - s.lgf_press;
  s.pvel = s.lgf_av * s.pvel + 0.5 * s.lgf_inv_pmass * dt * (s.lgf_av * pf_old + s.pistonf) +
           s.lgf_bv * s.lgf_inv_pmass * s.lgf_rangv;
  for (int i = 0; i < s.n; i++) {
    const double b0 = 1.0 / (1.0 + s.lgf_facg0 * s.one_mass[i]);
    const double a0 = (1.0 - s.lgf_facg0 * s.one_mass[i]) * b0;
    for (int k = 0; k < 3; k++) {
      const int q = 3 * i + k;
      s.vel[q] = a0 * s.vel[q] + 0.5 * dt * (a0 * s.acel[q] + s.one_mass[i] * s.force[q]) + b0 * s.pos_v[q];
      s.acel[q] = s.force[q] * s.one_mass[i];
    }
  }
}

// lgf_flex_stepa (Integration.F90:698-776) and ermak_a_x (:1033-1082) for
// each coordinate integrator in turn; every piston sees the volume of the
// step's start (box_setvars runs once all have moved their lengths,
// integration_stepa :243-264).  A piston draws its pair, then one pair per
// atom; an Ermak coordinate one pair per atom.
void axes_a(Sys& s) {
  const double dt = s.dt;
  const double vol0 = s.box[0] * s.box[1] * s.box[2];
  for (AxisInt& a : s.axes) {
    const int d = a.d;
    if (a.mode == AX_FLEX) {
      if (a.first) {
        a.first = false;
        a.pf = (s.virial[4 * d] + a.kin) / vol0 - a.press;
      }
      double r1, r2;
      rang(*s.rng, &r1, &r2);
      const double rangv = r1 * a.facv;
      const double Lo = s.box[d];
      s.box[d] = Lo + a.bv * dt * (a.pvel + 0.5 * a.ipm * (dt * a.pf * vol0 / Lo + rangv));
      a.rangv = rangv;
      for (int i = 0; i < s.n; i++) {
        const double b0 = 1.0 / (1.0 + a.facg0 * s.one_mass[i]);
        rang(*s.rng, &r1, &r2);
        const int q = 3 * i + d;
        s.pos_v[q] = s.one_mass[i] * a.fac0 * r1;
        s.acel[q] = s.force[q] * s.one_mass[i];
        s.pos[q] = s.box[d] / Lo * s.pos[q] +
                   2.0 * s.box[d] / (Lo + s.box[d]) * b0 * dt * (s.vel[q] + 0.5 * dt * s.acel[q] + 0.5 * s.pos_v[q]);
      }
    } else {
      for (int i = 0; i < s.n; i++) {
        const double f_lan = a.skt * s.one_sqrt_mass[i];
        double r1, r2;
        rang(*s.rng, &r1, &r2);
        const int q = 3 * i + d;
        s.pos_v[q] = f_lan * a.sdr * r1;
        s.vel_v[q] = f_lan * a.sdv * (a.crv1 * r1 + a.crv2 * r2);
        s.pos[q] = s.pos[q] + a.cc1 * s.vel[q] + a.cc2 * dt * s.acel[q] + s.pos_v[q];
      }
    }
  }
  for (int k = 0; k < 3; k++) s.one_box[k] = 1.0 / s.box[k];
}

// lgf_flex_stepb (Integration.F90:778-830) and ermak_b_x (:1084-1105)
void axes_b(Sys& s) {
  const double dt = s.dt;
  const double vol = s.box[0] * s.box[1] * s.box[2];
  for (AxisInt& a : s.axes) {
    const int d = a.d;
    if (a.mode == AX_FLEX) {
      const double pf_old = a.pf;
      a.pf = (s.virial[4 * d] + a.kin) / vol - a.press;
      a.pvel = a.av * a.pvel + 0.5 * a.ipm * dt * (a.av * pf_old + a.pf) * vol / s.box[d] + a.bv * a.ipm * a.rangv;
      for (int i = 0; i < s.n; i++) {
        const double b0 = 1.0 / (1.0 + a.facg0 * s.one_mass[i]);
        const double a0 = (1.0 - a.facg0 * s.one_mass[i]) * b0;
        const int q = 3 * i + d;
        s.vel[q] = a0 * s.vel[q] + 0.5 * dt * (a0 * s.acel[q] + s.one_mass[i] * s.force[q]) + b0 * s.pos_v[q];
        s.acel[q] = s.force[q] * s.one_mass[i];
      }
    } else {
      for (int i = 0; i < s.n; i++) {
        const int q = 3 * i + d;
        s.vel[q] = a.cc0 * s.vel[q] + (a.cc1 - a.cc2) * s.acel[q] + a.cc2 * s.force[q] * s.one_mass[i] + s.vel_v[q];
        s.acel[q] = s.force[q] * s.one_mass[i];
      }
    }
  }
}

// ------------------------------------------------------------------ LKD NPT
// Langevin piston of Kolb & Dunweg (J. Chem. Phys. 111, 4453, 1999) as
// lkd_stepa / lkd_stepb state it (Integration.F90:357-484): a half kick of
// the velocities with friction and noise, the piston momentum from the
// instantaneous pressure, the box moved in two half advances with the
// positions drifted in between, then positions and velocities rescaled to
// the final box.  Noise: stepa draws a pair per atom coordinate then the
// piston's, stepb the piston's then a pair per atom coordinate.
void set_lkd(Sys& s, double dt, double temp, double press, double pgama0, double pgamav, double pmass) {
  s.integ = IT_LKD;
  s.dt = dt;
  s.temp = temp;
  s.lkd_fac0 = std::sqrt(kB_ui * temp * dt * pgama0);
  s.lkd_facv = std::sqrt(kB_ui * temp * dt * pgamav);
  s.lkd_press = press;
  s.lkd_g0 = pgama0;
  s.lkd_gv = pgamav;
  s.lkd_pmass = pmass;
  s.pvel = 0.0;
}

// the mean of the pressure tensor's diagonal (inq_pressure,
// Inq_Properties.F90:529-573), internal units, with the virial of the last
// force evaluation
double pressure_trace(const Sys& s) {
  double K[3] = {0, 0, 0};
  for (int i = 0; i < s.n; i++)
    for (int a = 0; a < 3; a++) K[a] += s.vel[3 * i + a] * s.vel[3 * i + a] * s.mass[i];
  const double vol = s.box[0] * s.box[1] * s.box[2];
  return ((K[0] + s.virial[0]) / vol + (K[1] + s.virial[4]) / vol + (K[2] + s.virial[8]) / vol) / 3;
}

void lkd_kick(Sys& s) {
  const double dt = s.dt;
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++) {
      const int q = 3 * i + k;
      double r1, r2;
      rang(*s.rng, &r1, &r2);
      s.acel[q] = s.force[q] * s.one_mass[i];
      s.vel[q] = s.vel[q] + 0.5 * dt * s.acel[q] - 0.5 * dt * s.lkd_g0 * s.one_mass[i] * s.vel[q] +
                 s.one_mass[i] * s.lkd_fac0 * r1;
    }
}

void lkd_piston(Sys& s) {
  const double dt = s.dt;
  const double press = pressure_trace(s);
  double r1, r2;
  rang(*s.rng, &r1, &r2);
  s.pvel = s.pvel + 0.5 * dt * (press - s.lkd_press) - s.lkd_gv * 0.5 * dt * s.pvel / s.lkd_pmass + s.lkd_facv * r1;
}

void lkd_a(Sys& s) {
  const double dt = s.dt;
  const double expo = (double)(1.0f / 3.0f);
  double bo[3];
  for (int k = 0; k < 3; k++) bo[k] = s.box[k];
  lkd_kick(s);
  lkd_piston(s);
  double vol = s.box[0] * s.box[1] * s.box[2];
  for (int k = 0; k < 3; k++) s.box[k] = s.box[k] * std::pow(1.0 + 0.5 * dt * s.pvel / s.lkd_pmass / vol, expo);
  vol = s.box[0] * s.box[1] * s.box[2];
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++) {
      const int q = 3 * i + k;
      s.pos[q] = s.pos[q] + s.vel[q] * dt * bo[k] * bo[k] / (s.box[k] * s.box[k]);
    }
  for (int k = 0; k < 3; k++) {
    s.box[k] = s.box[k] * std::pow(1.0 + 0.5 * dt * s.pvel / s.lkd_pmass / vol, expo);
    s.one_box[k] = 1.0 / s.box[k];
  }
  for (int i = 0; i < s.n; i++)
    for (int k = 0; k < 3; k++) {
      const int q = 3 * i + k;
      s.pos[q] = s.pos[q] * s.box[k] / bo[k];
      s.vel[q] = s.vel[q] * bo[k] / s.box[k];
    }
}

void lkd_b(Sys& s) {
  lkd_piston(s);
  lkd_kick(s);
}

void add_axis(Sys& s, const AxisInt& a) {
  if (s.integ != IT_AXES) s.axes.clear();
  s.integ = IT_AXES;
  if ((int)s.pos_v.size() < 3 * s.n) s.pos_v.assign(3 * s.n, 0.0);
  if ((int)s.vel_v.size() < 3 * s.n) s.vel_v.assign(3 * s.n, 0.0);
  s.axes.push_back(a);
}

void stepa(Sys& s) {
  if (s.integ == IT_VV || s.integ == IT_FIRE) vv_a(s);
  else if (s.integ == IT_ERMAK) ermak_a(s);
  else if (s.integ == IT_LGF) lgf_a(s);
  else if (s.integ == IT_AXES) axes_a(s);
  else if (s.integ == IT_LKD) lkd_a(s);
  else if (s.integ == IT_NORD) nord_a(s);
  do_pbc(s);
}

void stepb(Sys& s) {
  if (s.integ == IT_VV || s.integ == IT_FIRE) vv_b(s);
  else if (s.integ == IT_ERMAK) ermak_b(s);
  else if (s.integ == IT_LGF) lgf_b(s);
  else if (s.integ == IT_AXES) axes_b(s);
  else if (s.integ == IT_LKD) lkd_b(s);
  else if (s.integ == IT_NORD) nord_b(s);
  else if (s.integ == IT_BROWN) brownian_b(s);
  if (s.thermo == 1 || s.thermo == 2) scalvel(s);
  else if (s.thermo == 3) andersen(s);
  do_pbc(s);
  if (s.integ == IT_FIRE) fire_mix(s);
}

// pressure tensor (inq_pressure, Inq_Properties.F90:529-573) in atm: the
// kinetic tensor sum m v v plus the virial, over the volume
void pressure_atm(const Sys& s, double out[9]) {
  double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < s.n; i++)
    for (int a = 0; a < 3; a++)
      for (int b = a; b < 3; b++) K[3 * a + b] += s.vel[3 * i + a] * s.vel[3 * i + b] * s.mass[i];
  for (int a = 1; a < 3; a++)
    for (int b = 0; b < a; b++) K[3 * a + b] = K[3 * b + a];
  const double vol = s.box[0] * s.box[1] * s.box[2];
  const double ui_pa = 1.0 / ((1.0 / (ui_ev * 1.60219e-19)) * 1e-30);
  const double ui_atm_out = ui_pa * 1e-5 * (1.0 / 1.01325);  // write_pressure (Output.F90:767-770)
  for (int k = 0; k < 9; k++) out[k] = (K[k] + s.virial[k]) / vol * ui_atm_out;
}

// ------------------------------------------------------------------ L-BFGS
// lbfgs (Quasi_Newton.f90:349-663): limited-memory BFGS of Liu & Nocedal
// (Math. Prog. B 45, 1989) with the line search of More & Thuente (ACM TOMS
// 20, 1994) as mcsrch (:703-901) / mcstep (:903-1096) state it.  The
// objective is get_fg (:1110-1120): f = interact * ui_ev (eV) and g = -F * ui_ev
// (eV/A).  Constants: lbfgs_minimizator's m = 5, eps = 1e-8, xtol = 1e-15
// (:77-110); gtol = 0.9, stpmin = 1e-20, stpmax = 1e20 (module :14-20);
// ftol = 1e-4, maxfev = 100 (:467-469); itermax = 1000 (:391).

void get_fg(Sys& s, double& f, std::vector<double>& g) {
  f = interact(s, nullptr) * ui_ev;
  for (int q = 0; q < 3 * s.n; q++) g[q] = -s.force[q] * ui_ev;
}

double dotv(const std::vector<double>& a, const std::vector<double>& b, int n) {
  double d = 0.0;
  for (int q = 0; q < n; q++) d += a[q] * b[q];
  return d;
}

// one safeguarded cubic/quadratic step of the interval of uncertainty
// [stx, sty] towards a point satisfying the strong Wolfe conditions (the
// four cases of More & Thuente section 4, as mcstep orders them)
void mt_step(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy, double& stp, double fp,
             double dp, bool& brackt, double stmin, double stmax, int& info) {
  info = 0;
  if ((brackt && (stp <= std::min(stx, sty) || stp >= std::max(stx, sty))) || dx * (stp - stx) >= 0.0 ||
      stmax < stmin)
    return;
  const double sgnd = dp * (dx / std::fabs(dx));
  double stpf, stpc, stpq;
  bool bound;
  auto gamma_of = [](double theta, double a, double b, bool clip) {
    const double sc = std::max(std::fabs(theta), std::max(std::fabs(a), std::fabs(b)));
    double disc = (theta / sc) * (theta / sc) - (a / sc) * (b / sc);
    if (clip) disc = std::max(0.0, disc);
    return sc * std::sqrt(disc);
  };
  if (fp > fx) {
    // case 1: higher function value; the minimum is bracketed
    info = 1;
    bound = true;
    const double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double gam = gamma_of(theta, dx, dp, false);
    if (stp < stx) gam = -gam;
    const double r = ((gam - dx) + theta) / (((gam - dx) + gam) + dp);
    stpc = stx + r * (stp - stx);
    stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx);
    stpf = (std::fabs(stpc - stx) < std::fabs(stpq - stx)) ? stpc : stpc + (stpq - stpc) / 2.0;
    brackt = true;
  } else if (sgnd < 0.0) {
    // case 2: lower value, derivatives of opposite sign; bracketed
    info = 2;
    bound = false;
    const double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double gam = gamma_of(theta, dx, dp, false);
    if (stp > stx) gam = -gam;
    const double r = ((gam - dp) + theta) / (((gam - dp) + gam) + dx);
    stpc = stp + r * (stx - stp);
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    stpf = (std::fabs(stpc - stp) > std::fabs(stpq - stp)) ? stpc : stpq;
    brackt = true;
  } else if (std::fabs(dp) < std::fabs(dx)) {
    // case 3: lower value, same sign, derivative magnitude decreases
    info = 3;
    bound = true;
    const double theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    double gam = gamma_of(theta, dx, dp, true);
    if (stp > stx) gam = -gam;
    const double r = ((gam - dp) + theta) / ((gam + (dx - dp)) + gam);
    if (r < 0.0 && gam != 0.0) stpc = stp + r * (stx - stp);
    else if (stp > stx) stpc = stmax;
    else stpc = stmin;
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    if (brackt) stpf = (std::fabs(stp - stpc) < std::fabs(stp - stpq)) ? stpc : stpq;
    else stpf = (std::fabs(stp - stpc) > std::fabs(stp - stpq)) ? stpc : stpq;
  } else {
    // case 4: lower value, same sign, derivative does not decrease
    info = 4;
    bound = false;
    if (brackt) {
      const double theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp;
      double gam = gamma_of(theta, dy, dp, false);
      if (stp > sty) gam = -gam;
      const double r = ((gam - dp) + theta) / (((gam - dp) + gam) + dy);
      stpf = stp + r * (sty - stp);
    } else {
      stpf = (stp > stx) ? stmax : stmin;
    }
  }
  // update the interval
  if (fp > fx) {
    sty = stp; fy = fp; dy = dp;
  } else {
    if (sgnd < 0.0) { sty = stx; fy = fx; dy = dx; }
    stx = stp; fx = fp; dx = dp;
  }
  stpf = std::max(stmin, std::min(stmax, stpf));
  stp = stpf;
  if (brackt && bound) {
    const double lim = stx + 0.66 * (sty - stx);
    stp = (sty > stx) ? std::min(lim, stp) : std::max(lim, stp);
  }
}

// mcsrch: from x (f, g at x) along s; on return x = x0 + stp s with f, g
// there; info 1 = strong Wolfe conditions met, other values = failure kinds
int mt_search(Sys& s, std::vector<double>& x, double& f, std::vector<double>& g, const std::vector<double>& dir,
              double& stp, double ftol, double gtol, double xtol, double stpmin, double stpmax, int maxfev,
              int& nfev) {
  const int n = 3 * s.n;
  const double dginit = dotv(g, dir, n);
  nfev = 0;
  if (dginit >= 0.0) return 0;  // not a descent direction
  bool brackt = false, stage1 = true;
  int infoc = 1;
  const double finit = f, dgtest = ftol * dginit;
  double width = stpmax - stpmin, width1 = width / 0.5;
  const std::vector<double> x0 = x;
  double stx = 0.0, fx = finit, dgx = dginit;
  double sty = 0.0, fy = finit, dgy = dginit;
  for (nfev = 1; nfev <= maxfev; nfev++) {
    double stmin, stmax;
    if (brackt) {
      stmin = std::min(stx, sty);
      stmax = std::max(stx, sty);
    } else {
      stmin = stx;
      stmax = stp + 4.0 * (stp - stx);
    }
    stp = std::min(std::max(stp, stpmin), stpmax);
    if ((brackt && (stp <= stmin || stp >= stmax)) || nfev == maxfev || infoc == 0 ||
        (brackt && stmax - stmin <= xtol * stmax))
      stp = stx;
    for (int q = 0; q < n; q++) x[q] = x0[q] + stp * dir[q];
    s.pos = x;
    get_fg(s, f, g);
    int info = 0;
    const double dg = dotv(g, dir, n);
    const double ftest1 = finit + stp * dgtest;
    if ((brackt && (stp <= stmin || stp >= stmax)) || infoc == 0) info = 6;
    if (stp == stpmax && f <= ftest1 && dg <= dgtest) info = 5;
    if (stp == stpmin && (f > ftest1 || dg >= dgtest)) info = 4;
    if (nfev == maxfev) return 3;
    if (brackt && stmax - stmin <= xtol * stmax) info = 2;
    if (f <= ftest1 && std::fabs(dg) <= gtol * (-dginit)) info = 1;
    if (info != 0) return info;
    if (stage1 && f <= ftest1 && dg >= std::min(ftol, gtol) * dginit) stage1 = false;
    if (stage1 && f <= fx && f > ftest1) {
      // modified function psi(stp) = f - stp * dgtest while in the first stage
      double fm = f - stp * dgtest, fxm = fx - stx * dgtest, fym = fy - sty * dgtest;
      double dgm = dg - dgtest, dgxm = dgx - dgtest, dgym = dgy - dgtest;
      mt_step(stx, fxm, dgxm, sty, fym, dgym, stp, fm, dgm, brackt, stmin, stmax, infoc);
      fx = fxm + stx * dgtest;
      fy = fym + sty * dgtest;
      dgx = dgxm + dgtest;
      dgy = dgym + dgtest;
    } else {
      mt_step(stx, fx, dgx, sty, fy, dgy, stp, f, dg, brackt, stmin, stmax, infoc);
    }
    if (brackt) {
      if (std::fabs(sty - stx) >= 0.66 * width1) stp = stx + 0.5 * (sty - stx);
      width1 = width;
      width = std::fabs(sty - stx);
    }
  }
  return 3;
}

// returns iflag: 0 converged, -1 line search failed, 1 iteration limit;
// *iters = L-BFGS iterations, *nfun = function evaluations, *fmin = f (eV)
int lbfgs_min(Sys& s, int m, double eps, double xtol, int itermax, int* iters, int* nfun, double* fmin) {
  const int n = 3 * s.n;
  const double ftol = 1e-4, gtol = 0.9, stpmin = 1e-20, stpmax = 1e20;
  const int maxfev = 100;
  std::vector<double> x = s.pos, g(n), gold(n), d(n), q(n);
  std::vector<std::vector<double>> S(m, std::vector<double>(n)), Y(m, std::vector<double>(n));
  std::vector<double> rho(m), alpha(m);
  double f;
  get_fg(s, f, g);
  int nf = 1, point = 0, flag = 1, it = 0;
  for (int k = 0; k < n; k++) d[k] = -g[k];
  double gnorm = std::sqrt(dotv(g, g, n));
  for (it = 1; it <= itermax; it++) {
    double stp = 1.0;
    if (it == 1) {
      stp = 1.0 / gnorm;
    } else {
      // two-loop recursion over the last min(it-1, m) pairs, newest first;
      // H0 = (y.s / y.y) I with the newest pair
      const int bound = std::min(it - 1, m);
      const int newest = (point + m - 1) % m;
      const double ys = dotv(Y[newest], S[newest], n);
      const double yy = dotv(Y[newest], Y[newest], n);
      const double h0 = ys / yy;
      rho[newest] = 1.0 / ys;
      for (int k = 0; k < n; k++) q[k] = -g[k];
      int cp = point;
      for (int b = 0; b < bound; b++) {
        cp = (cp + m - 1) % m;
        alpha[cp] = rho[cp] * dotv(S[cp], q, n);
        for (int k = 0; k < n; k++) q[k] -= alpha[cp] * Y[cp][k];
      }
      for (int k = 0; k < n; k++) q[k] *= h0;
      for (int b = 0; b < bound; b++) {
        const double beta = alpha[cp] - rho[cp] * dotv(Y[cp], q, n);
        for (int k = 0; k < n; k++) q[k] += beta * S[cp][k];
        cp = (cp + 1) % m;
      }
      d = q;
    }
    gold = g;
    int nfev = 0;
    const int info = mt_search(s, x, f, g, d, stp, ftol, gtol, xtol, stpmin, stpmax, maxfev, nfev);
    nf += nfev;
    if (info != 1) {
      flag = -1;
      break;
    }
    for (int k = 0; k < n; k++) {
      S[point][k] = stp * d[k];
      Y[point][k] = g[k] - gold[k];
    }
    point = (point + 1) % m;
    gnorm = std::sqrt(dotv(g, g, n));
    double xnorm = std::sqrt(dotv(x, x, n));
    xnorm = (double)(long)std::max(1.0, xnorm);  // int(max(1, xnorm)), :633
    if (gnorm / xnorm <= eps) {
      flag = 0;
      break;
    }
  }
  if (iters) *iters = std::min(it, itermax);
  if (nfun) *nfun = nf;
  if (fmin) *fmin = f;
  return flag;
}

// ------------------------------------------------------------------ NEB
// neb (NEB.f90:58-220): nimg images of one group, the end points fixed;
// neb_linin (:331-355) fills the images between consecutive fixed ones
// linearly; each iteration is velocity Verlet with unit masses
// (change_atom_mas, :222-234) on the NEB force, with the quick-min velocity
// projection nebvel (:314-329) before stepa and before stepb.  nebfce
// (:236-312) is the improved tangent of Henkelman & Jonsson (J. Chem. Phys.
// 113, 9978, 2000) with a spring force along it.  Kept as the reference has
// them: the last image's energy is never evaluated (the first loop runs to
// nimg-1, :110) and so stays 0 in the tangent choice, and the tangent vector
// keeps its last value when no branch of the choice applies.  The time step
// is set once from the initial RMS NEB force, dt = sqrt(2 m 5e-5 / F_rms)
// (:133).  pneb: nimg x 3n positions, updated in place.
struct Neb {
  int nimg = 0, dim = 0;
  std::vector<double> p, f, v, e, q;
  double ks = 0.0;
};

void neb_load_eval(Sys& s, Neb& N, int i) {
  std::copy(N.p.begin() + (size_t)i * N.dim, N.p.begin() + (size_t)(i + 1) * N.dim, s.pos.begin());
  N.e[i] = interact(s, nullptr);
  std::copy(s.force.begin(), s.force.end(), N.f.begin() + (size_t)i * N.dim);
}

void neb_forces(Neb& N) {
  const int d = N.dim;
  std::vector<double> tp(d), tm(d);
  for (int i = 1; i < N.nimg - 1; i++) {
    const double* pm = &N.p[(size_t)(i - 1) * d];
    const double* pi = &N.p[(size_t)i * d];
    const double* pp = &N.p[(size_t)(i + 1) * d];
    for (int k = 0; k < d; k++) {
      tp[k] = pp[k] - pi[k];
      tm[k] = pi[k] - pm[k];
    }
    const double em = N.e[i - 1], ei = N.e[i], ep = N.e[i + 1];
    const double dmin = std::fabs(ei - em), dplus = std::fabs(ep - ei);
    const double dmax = std::max(dmin, dplus), dinf = std::min(dmin, dplus);
    // the tangent: towards the higher neighbour, or an energy-weighted mix at an extremum
    int kind = -1;  // 0: t+, 1: t-, 2: dmax t+ + dinf t-, 3: dinf t+ + dmax t-
    if (ep > ei) {
      if (ei > em) kind = 0;
      else if (ep > em) kind = 2;
      else if (ep < em) kind = 3;
    } else {
      if (ei > em) {
        if (ep > em) kind = 2;
        else if (ep < em) kind = 3;
      } else {
        kind = 1;
      }
    }
    for (int k = 0; k < d; k++) {
      if (kind == 0) N.q[k] = tp[k];
      else if (kind == 1) N.q[k] = tm[k];
      else if (kind == 2) N.q[k] = dmax * tp[k] + dinf * tm[k];
      else if (kind == 3) N.q[k] = dinf * tp[k] + dmax * tm[k];
    }
    double nq = 0.0;
    for (int k = 0; k < d; k++) nq += N.q[k] * N.q[k];
    const double inv = std::sqrt(nq);
    for (int k = 0; k < d; k++) N.q[k] = N.q[k] / inv;
    double* fi = &N.f[(size_t)i * d];
    double fq = 0.0, tpp = 0.0, tmm = 0.0;
    for (int k = 0; k < d; k++) {
      fq += fi[k] * N.q[k];
      tpp += tp[k] * tp[k];
      tmm += tm[k] * tm[k];
    }
    const double fs = N.ks * (std::sqrt(tpp) - std::sqrt(tmm));
    for (int k = 0; k < d; k++) fi[k] = fi[k] - fq * N.q[k] + N.q[k] * fs;
  }
}

void neb_velocities(Neb& N) {
  const int d = N.dim;
  for (int i = 1; i < N.nimg - 1; i++) {
    double* vi = &N.v[(size_t)i * d];
    const double* fi = &N.f[(size_t)i * d];
    double vf = 0.0, ff = 0.0;
    for (int k = 0; k < d; k++) vf += vi[k] * fi[k];
    if (vf > 0.0) {
      for (int k = 0; k < d; k++) ff += fi[k] * fi[k];
      for (int k = 0; k < d; k++) vi[k] = vf * fi[k] / ff;
    } else {
      for (int k = 0; k < d; k++) vi[k] = 0.0;
    }
  }
}

// returns dt; images between fixed ones are interpolated first
double neb_run(Sys& s, int nimg, double* pneb, const int* fixed, int nfixed, double k_ev, int iter) {
  Neb N;
  N.nimg = nimg;
  N.dim = 3 * s.n;
  const int d = N.dim;
  N.p.assign(pneb, pneb + (size_t)nimg * d);
  std::vector<int> fx(fixed, fixed + nfixed);
  std::sort(fx.begin(), fx.end());
  for (int j = 0; j + 1 < nfixed; j++) {
    const int a = fx[j], b = fx[j + 1];
    for (int i = a + 1; i < b; i++)
      for (int k = 0; k < d; k++)
        N.p[(size_t)i * d + k] = N.p[(size_t)(i - 1) * d + k] + (N.p[(size_t)b * d + k] - N.p[(size_t)a * d + k]) / (double)(b - a);
  }
  N.f.assign((size_t)nimg * d, 0.0);
  N.v.assign((size_t)nimg * d, 0.0);
  N.e.assign(nimg, 0.0);
  N.q.assign(d, 0.0);
  N.ks = k_ev * ev_ui;
  for (int i = 0; i < nimg - 1; i++) neb_load_eval(s, N, i);
  neb_forces(N);
  double fprom = 0.0;
  for (int i = 1; i < nimg - 1; i++)
    for (int k = 0; k < d; k++) fprom += N.f[(size_t)i * d + k] * N.f[(size_t)i * d + k];
  fprom = std::sqrt(fprom / ((double)(nimg - 2) * (double)d));
  const double mass = 1.0;
  const double dt = std::sqrt(2.0 * mass * 5e-5 / fprom);
  const double adv = dt * 0.5, adx = adv * dt;
  for (int ns = 1; ns <= iter; ns++) {
    neb_velocities(N);
    for (int i = 1; i < nimg - 1; i++) {
      double* pi = &N.p[(size_t)i * d];
      double* vi = &N.v[(size_t)i * d];
      const double* fi = &N.f[(size_t)i * d];
      for (int k = 0; k < d; k++) {  // velocity_verlet_a with one_mass = 1
        const double a = fi[k] * 1.0;
        pi[k] = pi[k] + dt * vi[k] + adx * a;
        vi[k] = vi[k] + adv * a;
      }
      neb_load_eval(s, N, i);
    }
    neb_forces(N);
    neb_velocities(N);
    for (int i = 1; i < nimg - 1; i++) {
      double* vi = &N.v[(size_t)i * d];
      const double* fi = &N.f[(size_t)i * d];
      for (int k = 0; k < d; k++) vi[k] = vi[k] + adv * (fi[k] * 1.0);  // velocity_verlet_b
    }
  }
  std::copy(N.p.begin(), N.p.end(), pneb);
  return dt;
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

double orc_ev_ui() { return ev_ui; }
double orc_kB_ui() { return kB_ui; }
int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// ---- RNG objects
void* orc_rng_new(int seed) {
  Lcg* r = new Lcg();
  lcg_seed(*r, seed);
  return r;
}
void orc_rng_free(void* r) { delete (Lcg*)r; }
double orc_ranu(void* r) { return lcg_ranu(*(Lcg*)r); }
void orc_rang(void* r, double* r1, double* r2) { rang(*(Lcg*)r, r1, r2); }
// n pairs from rang, stored r1,r2,r1,r2,... (the Ermak parity stream)
void orc_rang_stream(void* r, long npairs, double* out) {
  for (long k = 0; k < npairs; k++) rang(*(Lcg*)r, &out[2 * k], &out[2 * k + 1]);
}
void orc_rng_state(void* r, int* st) {
  Lcg* l = (Lcg*)r;
  st[0] = l->idum; st[1] = l->ix; st[2] = l->iy; st[3] = l->gaus_stored;
}
// lcg_read_chpseed (Random.F90:186-190): the state a checkpoint holds, in
// its record order idum, iy, ix (no Gaussian is cached between rang pairs)
void orc_rng_set_state(void* r, int idum, int iy, int ix) {
  Lcg* l = (Lcg*)r;
  l->idum = idum;
  l->iy = iy;
  l->ix = ix;
  l->gaus_stored = false;
}

// create_fill (Select_Create.F90:64-135): random sequential addition in
// [origin, origin+frame) with the reference's overlap rule rd < (s_a+s_b)^2.
// `pos` holds n_old existing atoms (with radii sig_old) followed by room for
// `num` new ones.  No minimum image (the created atom has pbc off).
int orc_fill(void* rng, int n_old, double* pos, const double* sig_old,
             int num, double sigma, const double frame[3],
             const double origin[3]) {
  Lcg& r = *(Lcg*)rng;
  const int nmax = 1000;
  std::vector<double> sig(sig_old, sig_old + n_old);
  int n = n_old;
  for (int i = 0; i < num; i++) {
    double a[3];
    int it;
    for (it = 1; it <= nmax; it++) {
      for (int j = 0; j < 3; j++) a[j] = lcg_ranu(r) * frame[j] + origin[j];
      bool ok = true;
      for (int k = 0; k < n; k++) {
        double vd[3] = {a[0] - pos[3 * k], a[1] - pos[3 * k + 1], a[2] - pos[3 * k + 2]};
        double rd = dot3(vd);
        double cut = sigma + sig[k];
        cut = cut * cut;
        if (rd < cut) { ok = false; break; }
      }
      if (ok) break;
    }
    if (it > nmax) return -1;
    for (int j = 0; j < 3; j++) pos[3 * n + j] = a[j];
    sig.push_back(sigma);
    n++;
  }
  return n;
}

// ---- systems
void* orc_sys_new(int n) {
  Sys* s = new Sys();
  s->n = n;
  s->pos.assign(3 * n, 0.0);
  s->vel.assign(3 * n, 0.0);
  s->acel.assign(3 * n, 0.0);
  s->force.assign(3 * n, 0.0);
  s->pos_v.assign(3 * n, 0.0);
  s->vel_v.assign(3 * n, 0.0);
  s->acel2.assign(3 * n, 0.0);
  s->acel3.assign(3 * n, 0.0);
  s->acel4.assign(3 * n, 0.0);
  s->pos_old.assign(3 * n, 0.0);
  s->epot.assign(n, 0.0);
  s->mass.assign(n, 1.0);
  s->one_mass.assign(n, 1.0);
  s->one_sqrt_mass.assign(n, 1.0);
  s->type.assign(n, 0);
  ensure_cap(*s, 256);
  return s;
}
void orc_sys_free(void* p) { delete (Sys*)p; }

void orc_set_pos(void* p, const double* x) { Sys* s = (Sys*)p; std::memcpy(s->pos.data(), x, sizeof(double) * 3 * s->n); }
void orc_get_pos(void* p, double* x) { Sys* s = (Sys*)p; std::memcpy(x, s->pos.data(), sizeof(double) * 3 * s->n); }
void orc_set_vel(void* p, const double* x) { Sys* s = (Sys*)p; std::memcpy(s->vel.data(), x, sizeof(double) * 3 * s->n); }
void orc_get_vel(void* p, double* x) { Sys* s = (Sys*)p; std::memcpy(x, s->vel.data(), sizeof(double) * 3 * s->n); }
void orc_set_acel(void* p, const double* x) { Sys* s = (Sys*)p; std::memcpy(s->acel.data(), x, sizeof(double) * 3 * s->n); }
void orc_get_acel(void* p, double* x) { Sys* s = (Sys*)p; std::memcpy(x, s->acel.data(), sizeof(double) * 3 * s->n); }
void orc_get_force(void* p, double* x) { Sys* s = (Sys*)p; std::memcpy(x, s->force.data(), sizeof(double) * 3 * s->n); }
void orc_get_epot_atoms(void* p, double* x) { Sys* s = (Sys*)p; std::memcpy(x, s->epot.data(), sizeof(double) * s->n); }
void orc_get_band(void* p, double* x) { Sys* s = (Sys*)p; std::memcpy(x, s->band.data(), sizeof(double) * s->n); }

// set_mass (Set_Properties.f90:168-191)
void orc_set_mass(void* p, const double* m) {
  Sys* s = (Sys*)p;
  for (int i = 0; i < s->n; i++) {
    s->mass[i] = m[i];
    if (m[i] == 0.0) {
      s->one_mass[i] = 0.0;
      s->one_sqrt_mass[i] = 0.0;
    } else {
      s->one_mass[i] = 1.0 / m[i];
      s->one_sqrt_mass[i] = std::sqrt(s->one_mass[i]);
    }
  }
}
void orc_set_types(void* p, const int* t, int ntypes) {
  Sys* s = (Sys*)p;
  for (int i = 0; i < s->n; i++) s->type[i] = t[i];
  s->ntypes = ntypes;
}
// box_setvars (Program_Types.F90:126-141); boxed=0 means no box
void orc_set_box(void* p, int boxed, const double* L, const int* pbc) {
  Sys* s = (Sys*)p;
  s->boxed = boxed != 0;
  for (int k = 0; k < 3; k++) {
    s->box[k] = boxed ? L[k] : 0.0;
    s->one_box[k] = boxed ? 1.0 / L[k] : 0.0;
    s->pbc[k] = pbc ? pbc[k] : 0;
  }
}
void orc_set_mic(void* p, int mic) { ((Sys*)p)->mic = mic != 0; }
void orc_set_skin(void* p, double skin) { ((Sys*)p)->skin = skin; }
void orc_set_skin_mode(void* p, int mic) { ((Sys*)p)->skin_mic = mic != 0; }
void orc_set_half(void* p, int half) { ((Sys*)p)->half = half != 0; }
void orc_set_capacity(void* p, int cap) { ensure_cap(*(Sys*)p, cap); }

static void recompute_rcut(Sys* s) {
  double rc = 0.0;
  for (int a = 0; a < MAXT; a++)
    for (int b = 0; b < MAXT; b++) {
      if (s->ff == FF_LJ && s->lj[a][b].on) rc = std::max(rc, s->lj[a][b].rc);
      if (s->ff == FF_SMATB && s->sm[a][b].on) rc = std::max(rc, s->sm[a][b].rce);
    }
  if (s->ff == FF_TERSOFF) rc = s->ts.R + s->ts.D;
  s->rcut = rc;
}

// lj_set / plj_set (Pairs.F90:198-205, 282-291); eshift is an optional
// constant energy shift per pair (eV), 0 for the reference's `lj`.
void orc_set_lj(void* p, int ti, int tj, double e, double sg, double rc,
                int shifted_force, double eshift) {
  Sys* s = (Sys*)p;
  s->ff = FF_LJ;
  LJp P;
  P.on = true; P.e = e; P.s = sg; P.rc = rc; P.rc2 = rc * rc;
  P.shifted_force = shifted_force != 0;
  P.eshift = eshift;
  if (P.shifted_force) {
    double x = sg / rc;
    double x6 = pow6(x);
    P.prc = 4.0 * e * (x6 * x6 - x6);
    double s6 = pow6(sg), s12 = s6 * s6;
    double rc6 = pow6(rc), rc7 = rc6 * rc, rc13 = rc6 * rc6 * rc;
    P.frc = 24.0 * e * (2.0 * (s12 / rc13) - (s6 / rc7));
  }
  s->lj[ti][tj] = P;
  s->lj[tj][ti] = P;
  recompute_rcut(s);
}

// wca_set (Pairs.F90:495-506): LJ cut at 2**(1./6.) sigma, where 1./6. is a
// single-precision literal, and shifted up by e (wca_interact, :508-589)
void orc_set_wca(void* p, int ti, int tj, double e, double sg) {
  orc_set_lj(p, ti, tj, e, sg, std::pow(2.0, (double)(1.0f / 6.0f)) * sg, 0, -e);
}

// sm1_set (Pairs.F90:916-923): r1, r2 (A), e (eV; pair_cli reads it with
// ev_ui, Pairs.F90:183-187)
void orc_set_sm1(void* p, int ti, int tj, double r1, double r2, double e) {
  Sys* s = (Sys*)p;
  s->ff = FF_LJ;
  LJp P;
  P.on = true; P.sm1 = true; P.e = e; P.r1 = r1; P.rc = r2; P.rc2 = r2 * r2;
  s->lj[ti][tj] = P;
  s->lj[tj][ti] = P;
  recompute_rcut(s);
}

// `interact g1 feels g2` (Interaction.f90:69-76, 128-131): half and newton
// off, so only the atoms of g1 feel the pair.  With one type per group the
// pair (ti, tj) then acts on the atoms of type ti only.
void orc_set_feels(void* p, int ti, int tj) {
  Sys* s = (Sys*)p;
  if (ti == tj) return;
  s->lj[tj][ti] = LJp();
  s->slj[tj][ti] = SLJp();
}

void orc_set_smatb(void* p, int ti, int tj, double a, double eps, double pp,
                   double q, double r0, double rci, double rce) {
  Sys* s = (Sys*)p;
  s->ff = FF_SMATB;
  SMp P;
  smatb_set(P, a, eps, pp, q, r0, rci, rce);
  s->sm[ti][tj] = P;
  s->sm[tj][ti] = P;
  recompute_rcut(s);
}
// prm: A, B (eV), lambda1, lambda2, beta, n, c, d, h, R, D, chi
void orc_set_tersoff(void* p, const double* prm) {
  Sys* s = (Sys*)p;
  s->ff = FF_TERSOFF;
  TSp& T = s->ts;
  T.A = prm[0]; T.B = prm[1]; T.l1 = prm[2]; T.l2 = prm[3]; T.beta = prm[4];
  T.n = prm[5]; T.c = prm[6]; T.d = prm[7]; T.h = prm[8]; T.R = prm[9];
  T.D = prm[10]; T.chi = prm[11];
  recompute_rcut(s);
}
void orc_smatb_coeffs(void* p, int ti, int tj, double* out6) {
  const SMp& P = ((Sys*)p)->sm[ti][tj];
  out6[0] = P.b1; out6[1] = P.b2; out6[2] = P.b3;
  out6[3] = P.r1; out6[4] = P.r2; out6[5] = P.r3;
}

// first call builds the list (update), later calls run test_update
double orc_interact(void* p, int* rebuilt) {
  bool rb;
  double e = interact(*(Sys*)p, &rb);
  if (rebuilt) *rebuilt = rb;
  return e;
}
void orc_update(void* p) { Sys* s = (Sys*)p; s->first = false; update(*s); }
long orc_nupd(void* p) { return ((Sys*)p)->nupd; }
int orc_status(void* p) { Sys* s = (Sys*)p; return (s->overflow ? 1 : 0) | (s->lost ? 2 : 0); }
int orc_list_cap(void* p) { return ((Sys*)p)->cap; }
int orc_uses_cells(void* p, int* nc) {
  Sys* s = (Sys*)p;
  for (int k = 0; k < 3; k++) nc[k] = s->ncells[k];
  return s->use_cells;
}
// copy out nn(n) and the column-major list (cap x n)
void orc_get_list(void* p, int* nn, int* list) {
  Sys* s = (Sys*)p;
  std::memcpy(nn, s->nn.data(), sizeof(int) * s->n);
  std::memcpy(list, s->list.data(), sizeof(int) * (size_t)s->n * s->cap);
}

void orc_set_vv(void* p, double dt) { Sys* s = (Sys*)p; s->integ = IT_VV; s->dt = dt; }
// `evolve pred_corr_5` (Integration.F90:143-145)
void orc_set_pred_corr(void* p, double dt) { Sys* s = (Sys*)p; s->integ = IT_NORD; s->dt = dt; }
// acel, acel2, acel3, acel4 (3n each, atom-major) out of or into the system
void orc_get_derivs(void* p, double* out) {
  Sys* s = (Sys*)p;
  const std::vector<double>* v[4] = {&s->acel, &s->acel2, &s->acel3, &s->acel4};
  for (int k = 0; k < 4; k++) std::copy(v[k]->begin(), v[k]->end(), out + (size_t)k * 3 * s->n);
}
void orc_set_derivs(void* p, const double* in) {
  Sys* s = (Sys*)p;
  std::vector<double>* v[4] = {&s->acel, &s->acel2, &s->acel3, &s->acel4};
  for (int k = 0; k < 4; k++) std::copy(in + (size_t)k * 3 * s->n, in + (size_t)(k + 1) * 3 * s->n, v[k]->begin());
}
void orc_set_ermak(void* p, double dt, double gama, double temp, void* rng) {
  Sys* s = (Sys*)p;
  set_ermak(*s, dt, gama, temp);
  s->rng = (Lcg*)rng;
}
void orc_ermak_consts(void* p, double* out8) {
  Sys* s = (Sys*)p;
  out8[0] = s->cc0; out8[1] = s->cc1; out8[2] = s->cc2; out8[3] = s->sdr;
  out8[4] = s->sdv; out8[5] = s->crv1; out8[6] = s->crv2; out8[7] = s->skt;
}
void orc_set_ext_normals(void* p, const double* nrm) { ((Sys*)p)->ext_normals = nrm; }
// `evolve scalvel temp steps` / `evolve scalvel_after temp steps upto`
// (set_scalvel, Integration.F90:1271-1298); upto < 0 selects scalvel
void orc_set_scalvel(void* p, double temp, int steps, double upto) {
  Sys* s = (Sys*)p;
  s->thermo = upto < 0.0 ? 1 : 2;
  s->th_temp = temp;
  s->th_soft = 0.5 / steps;
  s->th_upto = upto;
}
// `evolve andersen temp [nu]` (set_andersen, Integration.F90:1343-1364)
void orc_set_andersen(void* p, double temp, double nu, void* rng) {
  Sys* s = (Sys*)p;
  s->thermo = 3;
  s->th_factor = std::sqrt(kB_ui * temp / ((s->n * 3.0) * (s->n * 3.0)));
  s->th_nu = nu;
  s->rng = (Lcg*)rng;
}
void orc_clear_thermostat(void* p) { ((Sys*)p)->thermo = 0; }

// set_cbrownian (Integration.F90:834-853): `evolve brownian temp gama`
void orc_set_brownian(void* p, double dt, double temp, double gama, void* rng) {
  Sys* s = (Sys*)p;
  s->integ = IT_BROWN;
  s->dt = dt;
  s->bd_fac1 = dt / gama;
  s->bd_fac2 = std::sqrt(2.0 * kB_ui * temp * s->bd_fac1);
  s->rng = (Lcg*)rng;
}
void orc_set_fire(void* p, double dt0, double dtmax) { fire_init(*(Sys*)p, dt0, dtmax); }
double orc_fire_dt(void* p) { return ((Sys*)p)->fire_dt; }
double orc_fmax(void* p) { return fmax_ev(*(Sys*)p); }

void orc_stepa(void* p) { stepa(*(Sys*)p); }
void orc_stepb(void* p) { stepb(*(Sys*)p); }
void orc_do_pbc(void* p) { do_pbc(*(Sys*)p); }

// kinetic energy (CM removed) and temperature
void orc_kin(void* p, double* ekin, double* temp) { kin(*(Sys*)p, ekin, temp); }
double orc_epot_sum(void* p) {  // inq_pot_energy (Inq_Properties.F90:358-375)
  Sys* s = (Sys*)p;
  double e = 0.0;
  for (int i = 0; i < s->n; i++) e = e + s->epot[i];
  return e;
}

// set_gdist (Set_Properties.f90:301-349) over the whole system, in atom order
void orc_gdist(void* p, void* rng, double newtemp) {
  Sys* s = (Sys*)p;
  Lcg& r = *(Lcg*)rng;
  double cm[3];
  cm_vel(*s, cm);
  double factor = kB_ui * newtemp;
  for (int i = 0; i < s->n; i++) {
    double vel_med = std::sqrt(factor * s->one_mass[i]);
    for (int j = 0; j < 3; j++) {
      double r1;
      rang(r, &r1, nullptr);
      s->vel[3 * i + j] = vel_med * r1 + cm[j];
    }
  }
  // set_scal_vel (Set_Properties.f90:351-377)
  double ek, t;
  kin(*s, &ek, &t);
  if (t != 0.0) {
    double f = std::sqrt(newtemp / t);
    for (int q = 0; q < 3 * s->n; q++) s->vel[q] = s->vel[q] * f;
  }
  // remove the centre-of-mass drift (set_add_cmvel)
  cm_vel(*s, cm);
  for (int i = 0; i < s->n; i++)
    for (int k = 0; k < 3; k++) s->vel[3 * i + k] = s->vel[3 * i + k] + (-cm[k]);
}
// `box move` (CLInterpreter.F90:1692-1695): subtract the CM velocity
void orc_remove_cm(void* p) {
  Sys* s = (Sys*)p;
  double cm[3];
  cm_vel(*s, cm);
  for (int i = 0; i < s->n; i++)
    for (int k = 0; k < 3; k++) s->vel[3 * i + k] = s->vel[3 * i + k] + (-cm[k]);
}

// dinamic (Programs.f90:114-167): interact once, then nsteps of
// stepa / interact / stepb; every `each` steps append (Epot, Ekin, Etot, T)
// in eV/K to rows.  Returns the number of rows written.
int orc_dinamica(void* p, int nsteps, int each, double* rows) {
  Sys* s = (Sys*)p;
  interact(*s, nullptr);
  int nr = 0;
  for (int ns = 1; ns <= nsteps; ns++) {
    stepa(*s);
    interact(*s, nullptr);
    stepb(*s);
    if (each > 0 && ns % each == 0 && rows) {
      double ek, t;
      kin(*s, &ek, &t);
      double ep = 0.0;
      for (int i = 0; i < s->n; i++) ep = ep + s->epot[i];
      rows[4 * nr + 0] = ep * ui_ev;
      rows[4 * nr + 1] = ek * ui_ev;
      rows[4 * nr + 2] = rows[4 * nr + 0] + rows[4 * nr + 1];
      rows[4 * nr + 3] = t;
      nr++;
    }
  }
  return nr;
}

// FIRE relaxation to max|F| < fmax_tol (eV/A) or maxit iterations.  Returns
// the number of iterations; *fmax_out the final max|F| in eV/A.
int orc_lbfgs(void* p, int m, double eps, double xtol, int itermax, int* iters, int* nfun, double* fmin) {
  return lbfgs_min(*(Sys*)p, m, eps, xtol, itermax, iters, nfun, fmin);
}

void orc_set_slj(void* p, int ti, int tj, double e, double sg, double rs) {
  Sys* s = (Sys*)p;
  s->ff = FF_SLJ;
  SLJp P;
  slj_set(P, e, sg, rs);
  s->slj[ti][tj] = P;
  s->slj[tj][ti] = P;
  s->rcut = std::max(s->rcut, P.rc);
}

// press in atm (the reference reads it with atm_ui, Integration.F90:157-172)
void orc_set_lgf(void* p, double dt, double temp, double press_atm, double pgama0, double pgamav, double pmass,
                 void* rng) {
  Sys* s = (Sys*)p;
  s->rng = (Lcg*)rng;
  set_lgf(*s, dt, temp, press_atm * atm_ui, pgama0, pgamav, pmass);
}

// `evolve piston_lgf x|y|z T gamma0 P gammav pmass` (Integration.F90:157-172;
// set_lgf_flex :652-696), press in atm; the system's dt is dt
void orc_add_lgf_axis(void* p, int d, double dt, double temp, double press_atm, double pgama0, double pgamav,
                      double pmass, void* rng) {
  Sys* s = (Sys*)p;
  s->rng = (Lcg*)rng;
  s->dt = dt;
  AxisInt a;
  a.mode = AX_FLEX;
  a.d = d;
  a.fac0 = std::sqrt(2.0 * pgama0 * kB_ui * temp * dt);
  a.facg0 = 0.5 * dt * pgama0;
  a.kin = s->n * temp * kB_ui;
  a.press = press_atm * atm_ui;
  a.ipm = 1.0 / pmass;
  a.bv = 1.0 / (1.0 + 0.5 * dt * a.ipm * pgamav);
  a.facv = std::sqrt(2.0 * pgamav * kB_ui * temp * dt);
  a.av = (1.0 - 0.5 * dt * a.ipm * pgamav) * a.bv;
  add_axis(*s, a);
}

// `evolve piston_lkd T gamma0 P gammav pmass` (Integration.F90:150-156),
// press in atm
void orc_set_lkd(void* p, double dt, double temp, double press_atm, double pgama0, double pgamav, double pmass,
                 void* rng) {
  Sys* s = (Sys*)p;
  s->rng = (Lcg*)rng;
  set_lkd(*s, dt, temp, press_atm * atm_ui, pgama0, pgamav, pmass);
}

// `evolve ermak_x|y|z T gamma` (Integration.F90:179-186; set_ermak with a
// coordinate, :909-961)
void orc_add_ermak_axis(void* p, int d, double dt, double gama, double temp, void* rng) {
  Sys* s = (Sys*)p;
  s->rng = (Lcg*)rng;
  s->dt = dt;
  AxisInt a;
  a.mode = AX_ERMAK;
  a.d = d;
  a.cc0 = std::exp(-dt * gama);
  a.cc1 = (1.0 - a.cc0) / gama;
  a.cc2 = (1.0 - a.cc1 / dt) / gama;
  a.sdr = std::sqrt(dt / gama * (2.0 - (3.0 - 4.0 * a.cc0 + a.cc0 * a.cc0) / (dt * gama)));
  a.sdv = std::sqrt(1.0 - a.cc0 * a.cc0);
  a.crv1 = (1.0 - a.cc0) * (1.0 - a.cc0) / (gama * a.sdr * a.sdv);
  a.crv2 = std::sqrt(1.0 - (a.crv1 * a.crv1));
  a.skt = std::sqrt(kB_ui * temp);
  add_axis(*s, a);
}

// pistonf(3), pvel(3) as the reference holds them after a step
// (Integration.F90:66): the isotropic and LKD pistons use index 0
void orc_piston_state(void* p, double* pf3, double* pvel3) {
  Sys* s = (Sys*)p;
  for (int k = 0; k < 3; k++) pf3[k] = pvel3[k] = 0.0;
  if (s->integ == IT_LGF || s->integ == IT_LKD) {
    pf3[0] = s->pistonf;
    pvel3[0] = s->pvel;
  } else if (s->integ == IT_AXES) {
    for (const AxisInt& a : s->axes)
      if (a.mode == AX_FLEX) {
        pf3[a.d] = a.pf;
        pvel3[a.d] = a.pvel;
      }
  }
}

void orc_virial_ev(void* p, double* out9) {
  Sys* s = (Sys*)p;
  for (int k = 0; k < 9; k++) out9[k] = s->virial[k] * ui_ev;
}
void orc_pressure_atm(void* p, double* out9) { pressure_atm(*(Sys*)p, out9); }
void orc_get_box(void* p, double* out3) {
  Sys* s = (Sys*)p;
  for (int k = 0; k < 3; k++) out3[k] = s->box[k];
}
double orc_atm_ui() { return atm_ui; }

double orc_neb(void* p, int nimg, double* pneb, const int* fixed, int nfixed, double k_ev, int iter) {
  return neb_run(*(Sys*)p, nimg, pneb, fixed, nfixed, k_ev, iter);
}

int orc_fire_relax(void* p, double fmax_tol, int maxit, double* fmax_out) {
  Sys* s = (Sys*)p;
  interact(*s, nullptr);
  int it = 0;
  double fm = fmax_ev(*s);
  while (fm >= fmax_tol && it < maxit) {
    stepa(*s);
    interact(*s, nullptr);
    stepb(*s);
    fm = fmax_ev(*s);
    it++;
  }
  if (fmax_out) *fmax_out = fm;
  return it;
}

}  // extern "C"
