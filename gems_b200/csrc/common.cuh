// common.cuh -- data layout shared by the host runtime and the sm_100a kernels.
//
// All systems of a context live in one HBM arena (structure of arrays, one
// slot per atom).  A system owns a contiguous atom range [off, off+n) and a
// contiguous cell range; single systems and batches use the same kernels,
// which walk a block map (block -> system, atom range) so that uneven systems
// pack into one launch without any block straddling two systems.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gg {

// GEMS unit conversion (src/Constants.F90:101-127), fixed at compile time
// in the same operation order as the reference.
__host__ __device__ constexpr double c_ui_ev() {
  return 1.0e2 * 1.0e2 * 1.6605402e-27 * (1.0 / 1.60219e-19);
}
#define EV_UI (1.0 / gg::c_ui_ev())

constexpr int MAXT = 4;            // species per system
constexpr int BLOCK = 256;         // threads per block of every kernel
constexpr int NSTENCIL = 27;

// 27-cell stencil in the reference's order (src/Neighbour.F90:75-83):
// 0 centre, 1..13 the upper half, 14..26 the lower half.  Kept in constant
// memory: a function-local table would be rebuilt in local memory per call.
__constant__ signed char c_stencil[27][3] = {
    {0, 0, 0},   {1, 0, 0},   {1, 1, 0},   {0, 1, 0},   {-1, 1, 0},
    {1, 0, -1},  {1, 1, -1},  {0, 1, -1},  {-1, 1, -1}, {1, 0, 1},
    {1, 1, 1},   {0, 1, 1},   {-1, 1, 1},  {0, 0, 1},   {-1, 0, 0},
    {-1, -1, 0}, {0, -1, 0},  {1, -1, 0},  {-1, 0, 1},  {-1, -1, 1},
    {0, -1, 1},  {1, -1, 1},  {-1, 0, -1}, {-1, -1, -1}, {0, -1, -1},
    {1, -1, -1}, {0, 0, -1}};

__device__ __forceinline__ void stencil(int k, int& dx, int& dy, int& dz) {
  dx = c_stencil[k][0];
  dy = c_stencil[k][1];
  dz = c_stencil[k][2];
}

enum FF : int { FF_NONE = 0, FF_LJ = 1, FF_SMATB = 2, FF_TERSOFF = 3 };
// thermostats run after the integrator's step b (`evolve scalvel`,
// `scalvel_after`, `andersen`)
enum TH : int { TH_NONE = 0, TH_SCALVEL = 1, TH_SCALVEL_AFTER = 2, TH_ANDERSEN = 3 };

enum IT : int { IT_NONE = 0, IT_VV = 1, IT_ERMAK = 2, IT_FIRE = 3, IT_LGF = 4, IT_AXES = 5, IT_LKD = 6, IT_NORD = 7,
                IT_BROWN = 8 };
// IT_AXES: one integrator per coordinate -- a G-JF piston on that box length
// (AX_FLEX) or Ermak dynamics of that coordinate (AX_ERMAK)
enum AX : int { AX_NONE = 0, AX_FLEX = 1, AX_ERMAK = 2 };
enum PREC : int { PREC_FP64 = 0, PREC_MIXED = 1 };

// status bits of a system (SysState::status)
// ST_BOX: a constant-pressure box shrank below three list cut-offs in a
// dimension, or its volume collapsed
// ST_BONDS: a Tersoff atom has more than TS_MAXB bonds, a bond beyond list
// slot 63, or a bond its partner's list does not hold
enum ST : int { ST_OVERFLOW = 1, ST_LOST = 2, ST_NAN = 4, ST_BOX = 8, ST_BONDS = 16 };
// status bits that end a run with an error (an overflow is healed instead)
constexpr int ST_FATAL = ST_NAN | ST_LOST | ST_BOX | ST_BONDS;

// Tersoff gather formulation: bonds per atom, threads per atom of the bond
// kernel (the system's "lanes"), atoms per block
constexpr int TS_MAXB = 12;
constexpr int TS_TPA = 4;

// Parameters of one species pair.  LJ (Pairs.F90:198-291):
//   v[0]=e v[1]=s v[2]=rc v[3]=rc2 v[4]=prc v[5]=frc v[6]=eshift
//   v[7]=shifted_force (0/1)
// slj, LJ with a splined tail (Pairs.F90:374-470), in the same slots:
//   v[0]=e v[1]=s v[2]=rc v[3]=rc2 v[8]=1 (slj form) v[9]=sa4 v[10]=sa8
//   v[11]=rs
// SMA-TB (TB.F90:106-170):
//   v[0]=A v[1]=xi v[2]=p v[3]=q v[4]=r0 v[5]=rci v[6]=rce
//   v[7..9]=b1,b2,b3 v[10..12]=r1,r2,r3 v[13]=on
struct PairP {
  double v[16];
};

// Tersoff 1988: A B l1 l2 beta n c d h R D chi  (A, B in eV)
struct TersoffP {
  double A, B, l1, l2, beta, n, c, d, h, R, D, chi;
};

// Static configuration of a system, written by the host.
struct SysDev {
  int off, n;          // atom range in the arena
  int ff, integ, prec, half;
  int ntypes, param_off;
  int boxed, use_cells;
  int pbc[3];
  int nc[3];
  int cell_off, ncell;
  int use_ext_normals;
  int fx_per[3];       // fixed-point dim is periodic
  double L[3], invL[3];
  double cell[3], inv_cell[3];
  double rlist2, skin, rcut;
  double fx_scale[3], fx_origin[3];
  float fx_inv[3];     // fixed-point unit (A), rounded to float ...
  float fx_inv_lo[3];  // ... and its rounding remainder (hi + lo = unit)
  int skin_mic;        // skin test on minimum-image displacements
  int list_warp;       // list kernel: 0 one CTA per cell, 1 / 2 one warp per cell (128 / 512-candidate tile)
  int list_img;        // list build in the image frame (every periodic dim has >= 3 cells)
  int pad_list;
  // integrator
  double dt;
  double cc0, cc1, cc2, sdr, sdv, crv1, crv2, skt;
  double bd_fac1, bd_fac2;  // set_cbrownian (Integration.F90:834-853): dt/gamma, sqrt(2 kB T dt/gamma)
  // thermostat: scalvel T0, soft = 0.5/steps, upto (scalvel_after), kB_ui;
  // andersen sqrt(kB T)/(3N), nu
  int thermo, pad_th;
  double th[4];
  uint64_t th_seed;
  uint64_t seed;
  double fire_dtmax, fire_fmax;
  int fire_maxit, pad1;
  TersoffP ts;
  // pair virial (pressure) and the G-JF constant-pressure piston
  // (set_lgf, Integration.F90:486-525): particle noise amplitude fac0 and
  // friction half-step facg0, kinetic term N kB T, target pressure,
  // 1/piston mass, piston b, noise amplitude and a
  int virial;          // force kernels accumulate the pair virial
  int cell_cap;        // cells allocated (a moving box may re-grid within them)
  double rlist;        // rcut + skin
  float ncut_r2[8];    // the list's skip-count thresholds (rcut + 1e-4 + k skin/7)^2, k = 0..7
  float nsplit_r2;     // force-order split below ncut_r2[0]: the inner regime (SMA-TB rci^2, Tersoff (R-D)^2)
  double lgf_fac0, lgf_facg0, lgf_kin, lgf_press, lgf_ipm, lgf_bv, lgf_facv, lgf_av;
  // IT_AXES, per coordinate: the mode and its constants --
  // AX_FLEX (set_lgf_flex, Integration.F90:652-696):
  //   fac0 facg0 kin press 1/pmass bv facv av
  // AX_ERMAK (set_ermak, :909-961): cc0 cc1 cc2 sdr sdv crv1 crv2 sqrt(kB T)
  int ax_mode[3];
  int pad3;
  double ax_p[3][8];
  // IT_LKD (set_lkd, Integration.F90:329-355): fac0, facv, target pressure,
  // particle and piston frictions, piston mass
  double lkd[6];
};

// Dynamic state of a system, written only by kernels (and reset by host).
struct SysState {
  int rebuild;      // list must be rebuilt this step
  int status;       // ST_* bits
  int ticket;       // last-block counters
  int ticket2;
  uint64_t step;    // Ermak / Philox counter
  int64_t nupd;     // rebuild count
  double fire_dt, fire_alpha, fire_P;
  int fire_np, fire_done;
  int fire_iter, fire_zero;
  double fmax2;     // max |F|^2 (internal units), FIRE convergence
  unsigned long long fmax2_bits;
  int maxnn, pad;
  // the skin test's bound on how much closer any pair came since the list
  // was built: the two largest displacements (+ the box's change of length
  // for a moving box); 0 right after a build
  double dmax;
  // pair virial W = sum_i r_i (x) F_i of the last force evaluation
  // (internal units; xx yy zz xy xz yz), kinetic tensor sum m v (x) v
  double vir[6], ktens[6];
  // G-JF piston: force (pistonf), velocity, this step's noise, the box
  // ratio and the drift factor 2 L / (L_old + L) of the last box move
  double lgf_pf, lgf_pvel, lgf_rangv, ext_piston;
  double lgf_sc[3], lgf_f2[3];
  double box_b[3];   // box at the last rebuild (list skin vs box motion)
  int lgf_phase;     // 0 until the first piston step (pistonf from the virial)
  int pad2;
  // IT_AXES pistons, per coordinate: force, velocity, last noise, fed
  // normal, phase
  double ax_pf[3], ax_pvel[3], ax_rangv[3], ax_ext[3];
  int ax_phase[3];
  int pad4;
  // IT_LKD: the box at the step's start, after the half advance and final
  // (the piston velocity is lgf_pvel; the fed piston normals of stepa and
  // stepb are ax_ext[0] and ax_ext[1])
  double lkd_bo[3], lkd_bh[3], lkd_bf[3];
  double th_factor;  // scalvel: this step's velocity factor
  double th_vcm[3];  // scalvel: this step's centre-of-mass velocity
};

// Block map: block b covers atoms [first[b], end[b]) of system sys[b];
// sys_blk0[s] / sys_nblk[s] give each system's block range (for last-block
// merges) -- arrays indexed by system id.
struct BlockMap {
  int nblk;
  int apb;             // atoms per block
  int base;            // index of block 0 in the per-block scratch (blk_top2, blk_red): a
                       // system's blocks of a batch's map, launched on their own, keep
                       // the batch's slots, so that concurrent launches do not share them
  const int* sys;
  const int* first;
  const int* end;
  const int* sys_blk0;
  const int* sys_nblk;
};

// Device arena (passed by value to kernels).
struct Arena {
  int64_t cap;          // atom capacity (leading dimension of the list)
  int lcap;             // neighbour capacity per atom
  double4* pos;         // x, y, z, -
  double4* pos_old;     // positions at the last rebuild (test_update)
  double4* vel;
  double4* acel;
  double4* force;
  double4* vel_v;       // Ermak random velocity kick (ermak_a -> ermak_b)
  double4* acel2;       // Nordsieck scaled derivatives (Atoms.F90:77-79); allocated
  double4* acel3;       //   when a system first integrates with the predictor-corrector
  double4* acel4;
  double* epot;         // per atom (internal units)
  double* band;         // SMA-TB density rho_i
  double* eband;        // 1/sqrt(rho_i)
  float* ebandf;        // FP32 copy for the mixed kernels
  int4* fxp;            // fixed-point positions (x, y, z, type) for mixed
  double4* pose;        // FP64 force pass: (x, y, z, 1/sqrt(rho)) from the density pass
  int4* fxe;            // mixed force pass: (fixed-point x, y, z, bits of float 1/sqrt(rho))
  double2* minv;        // (1/m, 1/sqrt(m))
  double* mass;
  int* type;
  int* nn;              // neighbours per atom (flist entries: the full list)
  int* hnn;             // half-list systems: entries of `list` (the half list)
  int* list;            // column-major: list[m * cap + i], the reference's order
  int* flist;           // the same pairs in the force order: the potential's inner
                        // regime, the rest of the cut-off, then the skin bands (list
                        // order within each), so a warp's atoms take the same branch
                        // at the same slot and the skip counts cut a prefix
  uint4* ncut;          // per atom, eight 16-bit counts: flist entries built closer than
                        // rcut + 1e-4 + k skin/7 (k = 0..7; see live_entries)
  int* cell_of;
  int* slot;
  int* cell_count;      // per cell, zero between rebuilds
  int* cell_n;
  int* cell_loc;        // exclusive prefix within a 256-cell chunk
  int* cell_start;      // absolute start in cell_atoms
  int* chunk_sum;       // per 256-cell chunk
  int* cell_atoms;      // atom ids sorted by cell (descending within a cell)
  double4* cell_pos;    // their positions, in the same order (written with it at a rebuild)
  // Tersoff: rslot[m * cap + i] = the slot of i in the flist of its m-th
  // neighbour (255: none), built with the list; per step, tsmask[i] marks
  // the flist slots of i that are bonds and tsfb[a * cap + i] holds the force
  // that centre i's energy puts on the partner of its a-th bond (tsfb32 in
  // mixed precision)
  unsigned char* rslot;
  unsigned char* tidx;  // [m cap + l]: the index of the record l's m-th partner wrote for l
  unsigned long long* tsmask;
  double4* tsfb;        // FP64 systems
  float4* tsfb32;       // mixed systems
  double* ext_normals;  // parity-mode Ermak normals (6 per atom)
  double2* blk_top2;    // per-block top-2 displacement^2
  double* blk_red;      // per-block partial sums
  SysDev* sys;
  SysState* st;
  PairP* prm;
  int* any_rebuild;     // OR over the systems of the last step
  unsigned long long* body_runs;  // executions of graph-captured rebuild chains
};

}  // namespace gg
