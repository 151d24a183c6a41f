// kernels.cuh -- sm_100a kernels of the force/neighbour path.
//
// Conventions
//  * every kernel runs BLOCK threads and walks a BlockMap: block b belongs to
//    one system, so per-system branches never diverge inside a block;
//  * neighbour lists are column-major, list[m * cap + i] (the reference's
//    list(i,m), src/Neighbour.F90:116-117), which makes the m-th neighbour of
//    consecutive atoms a coalesced 128-byte row;
//  * force kernels split an atom's list over K lanes and combine the lanes
//    with a fixed xor-shuffle tree, so results do not depend on scheduling;
//  * the list predicate and the skin test use explicitly rounded FP64
//    operations (no FMA contraction) so they decide exactly as the reference.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>
#include "common.cuh"

namespace gg {

// pi = 4 atan(1) (src/Constants.F90:71)
#define PI_D 3.141592653589793

__device__ __forceinline__ int blk_sys(const BlockMap& M) { return M.sys[blockIdx.x]; }

// ------------------------------------------------------------------ Philox
// Counter-based generator Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11).
__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

__host__ __device__ __forceinline__ uint4 philox10(uint4 c, uint2 k) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = mulhi32(M0, c.x), lo0 = M0 * c.x;
    uint32_t hi1 = mulhi32(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

// Box-Muller on two 32-bit uniforms: u1 in (0,1], u2 in [0,1).  The kick
// needs normal variates, not correctly rounded ones, so the FP32 hardware
// approximations serve (log2, sin, cos on the multi-function unit; the angle
// 2 pi u2 - pi stays in [-pi, pi), where they are accurate, and the shift by
// pi only flips both signs of a symmetric pair).  The kick is applied in FP64.
__device__ __forceinline__ void bm_pair(uint32_t a, uint32_t b, double& n1, double& n2) {
  float u1 = ((float)(a >> 8) + 1.0f) * 5.9604644775390625e-8f;  // (0, 1]
  float u2 = (float)(b >> 8) * 5.9604644775390625e-8f;            // [0, 1)
  float rr = sqrtf(-2.0f * __logf(u1));
  float sn, cs;
  __sincosf(fmaf(6.2831853071795865f, u2, -3.14159265358979f), &sn, &cs);
  n1 = (double)(rr * cs);
  n2 = (double)(rr * sn);
}

// six standard normals for (atom, step) from two Philox blocks
__device__ __forceinline__ void normals6(uint32_t atom, uint64_t step, uint64_t seed, double r[6]) {
  const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  uint4 a = philox10(make_uint4(atom, (uint32_t)step, (uint32_t)(step >> 32), 0u), key);
  uint4 b = philox10(make_uint4(atom, (uint32_t)step, (uint32_t)(step >> 32), 1u), key);
  bm_pair(a.x, a.y, r[0], r[1]);
  bm_pair(a.z, a.w, r[2], r[3]);
  bm_pair(b.x, b.y, r[4], r[5]);
}

// ------------------------------------------------------------------ helpers
// top-2 of squared displacements (test_update, src/Neighbour.F90:1305-1346)
__device__ __forceinline__ double2 top2_merge(double2 a, double2 b) {
  double hi = fmax(a.x, b.x);
  double lo = fmax(fmin(a.x, b.x), fmax(a.y, b.y));
  return make_double2(hi, lo);
}

__device__ __forceinline__ double2 block_top2(double2 v) {
  __shared__ double2 sh[BLOCK / 32];
  for (int o = 16; o; o >>= 1) {
    double2 w;
    w.x = __shfl_xor_sync(0xffffffffu, v.x, o);
    w.y = __shfl_xor_sync(0xffffffffu, v.y, o);
    v = top2_merge(v, w);
  }
  int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
  if (ln == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = ln < BLOCK / 32 ? sh[ln] : make_double2(1.e-16, 1.e-16);
    for (int o = 16; o; o >>= 1) {
      double2 w;
      w.x = __shfl_xor_sync(0xffffffffu, v.x, o);
      w.y = __shfl_xor_sync(0xffffffffu, v.y, o);
      v = top2_merge(v, w);
    }
  }
  __syncthreads();
  return v;  // valid in thread 0
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[BLOCK / 32];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
  if (ln == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = ln < BLOCK / 32 ? sh[ln] : 0.0;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;  // valid in thread 0
}

__device__ __forceinline__ double block_max(double v) {
  __shared__ double sh[BLOCK / 32];
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
  if (ln == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = ln < BLOCK / 32 ? sh[ln] : 0.0;
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  __syncthreads();
  return v;
}

// exact reference predicate: vd = pos_j - pos_i with minimum image
// (vdistance, src/Inq_Properties.F90:137-157), rd = dot_product(vd, vd)
__device__ __forceinline__ double rd_exact(const SysDev& S, double4 xi, double4 xj) {
  double v0 = __dsub_rn(xj.x, xi.x);
  double v1 = __dsub_rn(xj.y, xi.y);
  double v2 = __dsub_rn(xj.z, xi.z);
  if (S.pbc[0]) v0 = __dsub_rn(v0, __dmul_rn(S.L[0], round(__dmul_rn(v0, S.invL[0]))));
  if (S.pbc[1]) v1 = __dsub_rn(v1, __dmul_rn(S.L[1], round(__dmul_rn(v1, S.invL[1]))));
  if (S.pbc[2]) v2 = __dsub_rn(v2, __dmul_rn(S.L[2], round(__dmul_rn(v2, S.invL[2]))));
  return __dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2));
}

// minimum-image pair vector in FP64 for the FP64 force kernels
__device__ __forceinline__ void vd_fp64(const SysDev& S, double4 xi, double4 xj,
                                        double& v0, double& v1, double& v2) {
  v0 = xj.x - xi.x;
  v1 = xj.y - xi.y;
  v2 = xj.z - xi.z;
  if (S.pbc[0]) v0 = v0 - S.L[0] * round(v0 * S.invL[0]);
  if (S.pbc[1]) v1 = v1 - S.L[1] * round(v1 * S.invL[1]);
  if (S.pbc[2]) v2 = v2 - S.L[2] * round(v2 * S.invL[2]);
}

// fixed-point coordinates for the mixed kernels.  Periodic dims map [0,L)
// onto the full 32-bit ring (the int32 difference is the minimum image);
// open dims use 2^22 units per Angstrom around fx_origin (+-512 A).
__device__ __forceinline__ int fx_coord(const SysDev& S, int d, double x, int& bad) {
  if (S.fx_per[d]) {
    double t = floor(x * S.fx_scale[d]);
    long long q = (long long)t;
    return (int)(unsigned int)(unsigned long long)q;
  }
  double t = rint((x - S.fx_origin[d]) * S.fx_scale[d]);
  if (!(fabs(t) < 2147483000.0)) {
    bad = 1;
    t = 0.0;
  }
  return (int)t;
}

__device__ __forceinline__ void write_fx(const Arena& A, const SysDev& S, int i,
                                         double4 p, int ti, int& bad) {
  int4 q;
  q.x = fx_coord(S, 0, p.x, bad);
  q.y = fx_coord(S, 1, p.y, bad);
  q.z = fx_coord(S, 2, p.z, bad);
  q.w = ti;
  A.fxp[i] = q;
}

// squared displacement since the last rebuild.  Reference mode (skin_mic=0)
// takes the raw difference of test_update (src/Neighbour.F90:1320), so an atom
// wrapped by do_pbc counts as having moved a box length and forces a rebuild;
// skin_mic=1 takes the minimum image, which moves no list decision for atoms
// that did not move, only skips those spurious rebuilds.
__device__ __forceinline__ double disp2(const SysDev& S, double4 x, double4 q) {
  double v0 = __dsub_rn(x.x, q.x), v1 = __dsub_rn(x.y, q.y), v2 = __dsub_rn(x.z, q.z);
  if (S.skin_mic) {
    if (S.pbc[0]) v0 = __dsub_rn(v0, __dmul_rn(S.L[0], round(__dmul_rn(v0, S.invL[0]))));
    if (S.pbc[1]) v1 = __dsub_rn(v1, __dmul_rn(S.L[1], round(__dmul_rn(v1, S.invL[1]))));
    if (S.pbc[2]) v2 = __dsub_rn(v2, __dmul_rn(S.L[2], round(__dmul_rn(v2, S.invL[2]))));
  }
  return __dadd_rn(__dadd_rn(__dmul_rn(v0, v0), __dmul_rn(v1, v1)), __dmul_rn(v2, v2));
}

// last block of a system in a launch (the value is the same in every thread
// of the block).  Thread 0 has written the block's partial result; its fence
// orders that write before the ticket, so the last block sees every partial.
__device__ __forceinline__ bool last_block(const BlockMap& M, SysState* st, int s,
                                           int* counter) {
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    int t = atomicAdd(counter, 1);
    last = (t == M.sys_nblk[s] - 1);
    if (last) *counter = 0;
  }
  __syncthreads();
  return last;
}

// warp 0 of a system's last block: top-2 over that system's block results
// The system's top-2 over its blocks' partial results, called by the whole
// last block.  Up to 128 partials one warp merges them; more (a 1M-atom
// system has about 4000 blocks) the whole block does, each thread taking
// every BLOCK-th partial with four loads in flight, then the block's tree.
// The top-2 of a set does not depend on the merge order.  Valid in thread 0.
__device__ __forceinline__ double2 sys_top2(const Arena& A, const BlockMap& M, int s) {
  double2 w = make_double2(1.e-16, 1.e-16);
  const int b0 = M.sys_blk0[s], nb = M.sys_nblk[s];
  if (nb <= 128) {  // uniform across the block
    if (threadIdx.x < 32) {
      for (int b = threadIdx.x; b < nb; b += 32) w = top2_merge(w, __ldcg(&A.blk_top2[b0 + b]));
      for (int o = 16; o; o >>= 1) {
        double2 q;
        q.x = __shfl_xor_sync(0xffffffffu, w.x, o);
        q.y = __shfl_xor_sync(0xffffffffu, w.y, o);
        w = top2_merge(w, q);
      }
    }
    return w;
  }
  int b = threadIdx.x;
  for (; b + 3 * BLOCK < nb; b += 4 * BLOCK) {
    double2 q[4];
#pragma unroll
    for (int u = 0; u < 4; u++) q[u] = __ldcg(&A.blk_top2[b0 + b + u * BLOCK]);
#pragma unroll
    for (int u = 0; u < 4; u++) w = top2_merge(w, q[u]);
  }
  for (; b < nb; b += BLOCK) w = top2_merge(w, __ldcg(&A.blk_top2[b0 + b]));
  return block_top2(w);
}

// ------------------------------------------------------------------ skin test
// Per-block top-2 of |pos - pos_old|^2; the last block of each system
// decides rebuild = sqrt(d1) + sqrt(d2) > nb_dcut (test_update).
__device__ __forceinline__ void skin_finish(const Arena& A, const BlockMap& M, int s,
                                           double2 t) {
  if (threadIdx.x == 0) A.blk_top2[M.base + blockIdx.x] = t;
  if (last_block(M, A.st, s, &A.st[s].ticket)) {
    double2 v = sys_top2(A, M, s);
    if (threadIdx.x == 0) {
      const SysDev& S = A.sys[s];
      SysState& st = A.st[s];
      double box = 0.0;
      if (S.integ == IT_LGF || S.integ == IT_AXES || S.integ == IT_LKD)
        box = fabs(S.L[0] - st.box_b[0]) + fabs(S.L[1] - st.box_b[1]) + fabs(S.L[2] - st.box_b[2]);
      const double D = __dadd_rn(__dadd_rn(__dsqrt_rn(v.x), __dsqrt_rn(v.y)), box);
      int rb = D > S.skin;
      st.dmax = D;
      st.rebuild = rb;
      if (rb) atomicOr(A.any_rebuild, 1);
    }
  }
}

__global__ void k_skin(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  int i = M.first[blockIdx.x] + threadIdx.x;
  double2 t = make_double2(1.e-16, 1.e-16);
  if (i < M.end[blockIdx.x]) t.x = disp2(A.sys[s], A.pos[i], A.pos_old[i]);
  t = block_top2(t);
  skin_finish(A, M, s, t);
}

// mark systems for rebuild (first interact: update(), Interaction.f90:174)
__global__ void k_force_rebuild(Arena A, const int* sys, int nsys) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nsys && sys[k] >= 0) {
    A.st[sys[k]].rebuild = 1;
    atomicOr(A.any_rebuild, 1);
  }
}

// clear the per-chunk status words of a set of systems
__global__ void k_clear_status(Arena A, const int* sys, int nsys) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nsys && sys[k] >= 0) {
    A.st[sys[k]].status = 0;
    A.st[sys[k]].maxnn = 0;
  }
}

// refresh fixed-point positions (after an upload or set_positions)
__global__ void k_refresh_fx(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  int i = M.first[blockIdx.x] + threadIdx.x;
  if (i >= M.end[blockIdx.x]) return;
  const SysDev& S = A.sys[s];
  int bad = 0;
  write_fx(A, S, i, A.pos[i], A.type[i], bad);
  if (bad) atomicOr(&A.st[s].status, ST_LOST);
}

// ------------------------------------------------------------------ binning
// sort_in_cells (src/Neighbour.F90:927-989) as a counting sort:
// k_bin (histogram) -> k_scan1/k_scan2 (prefix) -> k_scatter -> k_sort_cells
__global__ void k_bin(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  if (!A.st[s].rebuild || !S.use_cells) return;
  int i = M.first[blockIdx.x] + threadIdx.x;
  if (i >= M.end[blockIdx.x]) return;
  double4 p = A.pos[i];
  int c0 = (int)__dmul_rn(p.x, S.inv_cell[0]);
  int c1 = (int)__dmul_rn(p.y, S.inv_cell[1]);
  int c2 = (int)__dmul_rn(p.z, S.inv_cell[2]);
  bool lost = false;
  // out-of-grid atoms are undefined behaviour in the reference; here they
  // are clamped into the grid and the system is flagged ST_LOST.
  if (c0 < 0 || c0 >= S.nc[0]) { lost = true; c0 = c0 < 0 ? 0 : S.nc[0] - 1; }
  if (c1 < 0 || c1 >= S.nc[1]) { lost = true; c1 = c1 < 0 ? 0 : S.nc[1] - 1; }
  if (c2 < 0 || c2 >= S.nc[2]) { lost = true; c2 = c2 < 0 ? 0 : S.nc[2] - 1; }
  if (lost || !(p.x == p.x && p.y == p.y && p.z == p.z)) atomicOr(&A.st[s].status, ST_LOST);
  int cid = S.cell_off + c0 + S.nc[0] * (c1 + S.nc[1] * c2);
  A.cell_of[i] = cid;
  A.slot[i] = atomicAdd(&A.cell_count[cid], 1);
}

// per 256-cell chunk: local exclusive prefix, chunk total; resets counts
__global__ void k_scan1(Arena A, BlockMap C) {
  int s = blk_sys(C);
  if (s < 0) return;  // padding block of a fixed-capacity map
  if (!A.st[s].rebuild || !A.sys[s].use_cells) return;
  int c = C.first[blockIdx.x] + threadIdx.x;
  bool act = c < C.end[blockIdx.x];
  int v = act ? A.cell_count[c] : 0;
  if (act) {
    A.cell_n[c] = v;
    A.cell_count[c] = 0;
  }
  __shared__ int sh[BLOCK];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < BLOCK; o <<= 1) {
    int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (act) A.cell_loc[c] = sh[threadIdx.x] - v;
  if (threadIdx.x == BLOCK - 1) A.chunk_sum[C.first[blockIdx.x] >> 8] = sh[BLOCK - 1];
}

// one block per system: exclusive prefix of its chunk totals
__global__ void k_scan2(Arena A, const int* sys, int nsys) {
  int s = sys[blockIdx.x];
  if (s < 0) return;
  const SysDev& S = A.sys[s];
  if (!A.st[s].rebuild || !S.use_cells) return;
  int k0 = S.cell_off >> 8;
  int nk = (S.ncell + BLOCK - 1) / BLOCK;
  __shared__ int sh[BLOCK];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = S.off;
  __syncthreads();
  for (int base = 0; base < nk; base += BLOCK) {
    int k = base + threadIdx.x;
    int v = k < nk ? A.chunk_sum[k0 + k] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < BLOCK; o <<= 1) {
      int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    int excl = carry + sh[threadIdx.x] - v;
    int tot = sh[BLOCK - 1];
    __syncthreads();
    if (k < nk) A.chunk_sum[k0 + k] = excl;
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
}

__global__ void k_scatter(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  if (!A.st[s].rebuild || !A.sys[s].use_cells) return;
  int i = M.first[blockIdx.x] + threadIdx.x;
  if (i >= M.end[blockIdx.x]) return;
  int c = A.cell_of[i];
  int start = A.chunk_sum[c >> 8] + A.cell_loc[c];
  A.cell_atoms[start + A.slot[i]] = i;
}

// one warp per cell: absolute start, then order the cell's atoms by
// descending index -- the order of the reference's head/next chain, which
// is built by inserting atoms in increasing index order.  Each lane ranks
// its atom(s) against the whole cell (cells of up to 64 atoms); larger cells
// fall back to an insertion sort by one lane.
// The rebuild kernels run on a fixed grid.  CTA x owns work items x, x + G,
// x + 2G, ... (G = gridDim.x, so live items spread evenly over the CTAs); it
// tests BLOCK of them at once, one per thread, keeps the live ones in shared
// memory and works through those.  A rebuild of a few systems in a large
// batch, or of a system with many cells, thus costs its work plus one
// parallel test per BLOCK items, not a launch or a serial test per item.
// Items are independent, so the order in which a CTA takes them is free.
template <class Check, class Body>
__device__ __forceinline__ void rebuild_items(int nitems, Check live, Body body) {
  __shared__ int items[BLOCK];
  __shared__ int nlive;
  const int G = gridDim.x;
  for (int base = 0; (int64_t)blockIdx.x + (int64_t)base * G < nitems; base += BLOCK) {
    const int64_t w = (int64_t)blockIdx.x + (int64_t)(base + threadIdx.x) * G;
    if (threadIdx.x == 0) nlive = 0;
    __syncthreads();
    if (w < nitems && live((int)w)) items[atomicAdd(&nlive, 1)] = (int)w;
    __syncthreads();
    const int n = nlive;
    for (int k = 0; k < n; k++) body(items[k]);
    __syncthreads();
  }
}

// map block b of a system flagged for a rebuild (cells or O(N^2) lists)
__device__ __forceinline__ bool rebuild_block(const Arena& A, const BlockMap& M, int b, bool cells) {
  const int s = M.sys[b];
  return s >= 0 && A.st[s].rebuild && (A.sys[s].use_cells != 0) == cells;
}

__global__ void k_sort_cells(Arena A, BlockMap C) {
  rebuild_items(C.nblk, [&](int b) { return rebuild_block(A, C, b, true); }, [&](int b) {
    const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
    const int first = C.first[b], end = C.end[b];
    for (int c = first + warp; c < end; c += BLOCK / 32) {  // C: 8 cells per block
      int start = A.chunk_sum[c >> 8] + A.cell_loc[c];
      int n = A.cell_n[c];
      if (ln == 0) A.cell_start[c] = start;
      int* a = A.cell_atoms + start;
      if (n <= 64) {
        int v0 = ln < n ? a[ln] : -1;
        int v1 = ln + 32 < n ? a[ln + 32] : -1;
        int r0 = 0, r1 = 0;
        // rank = entries greater than mine; empty slots (-1) are greater than none
        for (int k = 0; k < min(n, 32); k++) {
          const int w0 = __shfl_sync(0xffffffffu, v0, k);
          r0 += w0 > v0;
          r1 += w0 > v1;
        }
        for (int k = 0; k < n - 32; k++) {
          const int w1 = __shfl_sync(0xffffffffu, v1, k);
          r0 += w1 > v0;
          r1 += w1 > v1;
        }
        __syncwarp();
        // each lane places its own atoms (id and position) at their ranks
        if (ln < n) {
          a[r0] = v0;
          A.cell_pos[start + r0] = A.pos[v0];
        }
        if (ln + 32 < n) {
          a[r1] = v1;
          A.cell_pos[start + r1] = A.pos[v1];
        }
      } else if (ln == 0) {
        for (int x = 1; x < n; x++) {
          int v = a[x];
          int y = x - 1;
          while (y >= 0 && a[y] < v) {
            a[y + 1] = a[y];
            y--;
          }
          a[y + 1] = v;
        }
        for (int x = 0; x < n; x++) A.cell_pos[start + x] = A.pos[a[x]];  // the lane's own writes
      }
    }
    });
}

// ------------------------------------------------------------------ lists
// Every system's force kernels read `flist`, a full list (each pair from
// both sides), with nn[i] entries.  `list` holds the reference's list, the
// one gemsgpu_get_list returns: the same full list, or for a half-list
// system (Newton on, src/Neighbour.F90:160-171) the half list with hnn[i]
// entries.  A half list with the reaction added to j gives every atom the
// same force, density and energy as the full list (src/TB.F90:432-441,
// 542-552; src/Pairs.F90:248-252), so the force kernels need no half form.
// (the cell-list kernels store pos_old while they stage the home cell's
// atoms, whose positions they load anyway; the O(N^2) kernel here)
__device__ __forceinline__ void list_done(const Arena& A, int s, int i, int m, int mh, bool pos_old) {
  A.nn[i] = m;
  A.hnn[i] = mh;
  if (pos_old) A.pos_old[i] = A.pos[i];
  if (m > A.lcap) atomicOr(&A.st[s].status, ST_OVERFLOW);
  atomicMax(&A.st[s].maxnn, m);
}

// The force order: an atom's entries grouped by distance band at the build,
// slot order within a band.  Band 0 holds the inner regime of the pair
// potential (staged r^2 below nsplit_r2: SMA-TB r <= rci, Tersoff r <= R-D),
// so the lanes of a warp, one atom each, take the same branch at the same
// slot; band 1 the rest below T_0; band b >= 2 the entries that reach b - 1
// of the skip thresholds T_k = (rcut + 1e-4 + k skin/7)^2, k = 0..7.  The
// first ncut[k] entries are then exactly those with staged r^2 below T_k.
//
// Between builds no pair has come closer by more than the skin test's bound
// D (SysState::dmax), so the entries built at r >= rcut + 1e-4 + k skin/7
// with k skin/7 >= D lie beyond every cut-off of the system now and add
// nothing: the force kernels stop before them.  The staged r^2 is within
// err of the exact one (err: the list build's FP32 error bound), so the
// thresholds are raised by err: an entry counts above T_k only if its exact
// r^2 is; the float roundings of r^2 and of the thresholds move a distance
// by under 1e-6 A, inside the 1e-4 A margin.
//
// A warp writes the row of atom i: the first pass counts the entries below
// each threshold (one ballot per threshold and 32 entries), the second
// places each entry at its band's next free position (a match over the
// lanes' bands ranks lanes of one band, and the band's first lane advances
// the band's offset in boff, a 10-entry per-warp scratch).
__device__ __forceinline__ void list_force_order(const Arena& A, const SysDev& S, int i, int n, const int* row,
                                                 const float* rrow, float err, int* boff, int ln) {
  const unsigned FULL = 0xffffffffu, lt = (1u << ln) - 1u;
  float T[8];
#pragma unroll
  for (int k = 0; k < 8; k++) T[k] = __fadd_ru(S.ncut_r2[k], err);
  const float Ts = S.nsplit_r2;  // <= ncut_r2[0]
  int c[8], cs = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) c[k] = 0;
  for (int e0 = 0; e0 < n; e0 += 32) {
    const int e = e0 + ln;
    const float r = e < n ? rrow[e] : __int_as_float(0x7f800000);  // +inf is below no threshold
    cs += __popc(__ballot_sync(FULL, r < Ts));
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] += __popc(__ballot_sync(FULL, r < T[k]));
  }
  if (ln == 0) {
    unsigned short h[8];
#pragma unroll
    for (int k = 0; k < 8; k++) h[k] = (unsigned short)min(c[k], 65535);
    A.ncut[i] = make_uint4(h[0] | (unsigned)h[1] << 16, h[2] | (unsigned)h[3] << 16, h[4] | (unsigned)h[5] << 16,
                           h[6] | (unsigned)h[7] << 16);
  }
  if (ln < 10) {  // band b starts after the entries of the bands below it
    int v = ln == 1 ? cs : 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
      if (ln == k + 2) v = c[k];
    boff[ln] = v;
  }
  __syncwarp();
  for (int e0 = 0; e0 < n; e0 += 32) {
    const int e = e0 + ln;
    const bool v = e < n;
    int b = 10;  // lanes past the row share a band of their own
    if (v) {
      const float r = rrow[e];
      b = r >= Ts;
#pragma unroll
      for (int k = 0; k < 8; k++) b += r >= T[k];
    }
    const unsigned M = __match_any_sync(FULL, b);
    if (v) A.flist[(size_t)(boff[b] + __popc(M & lt)) * A.cap + i] = row[e] & 0x7fffffff;
    __syncwarp();
    if (v && (M & lt) == 0) boff[b] += __popc(M);
    __syncwarp();
  }
}

// the flist entries an atom's force loop must visit this step
__device__ __forceinline__ int live_entries(const Arena& A, const SysDev& S, const SysState& st, int i, int nn) {
  if (!(S.skin > 0.0) || !S.use_cells) return nn;  // O(N^2) lists are not grouped by band
  const double q = st.dmax * 7.0 / S.skin;
  if (!(q <= 7.0)) return nn;
  const int k = (int)ceil(q);
  const unsigned w = __ldg(reinterpret_cast<const unsigned*>(A.ncut + i) + (k >> 1));
  return min(nn, (int)((k & 1) ? (w >> 16) : (w & 0xffffu)));
}

// A warp's staged row of atom i (m accepted candidates in the reference's
// order: ids, bit 31 set on the entries a half list leaves out, and r^2 as
// float, within err of the exact r^2) out to the arena: `list` in the
// reference's order, `flist` in the force order, the skip counts and nn / hnn.
__device__ __forceinline__ void list_row_out(const Arena& A, const SysDev& S, int s, int i, int m,
                                             const int* row, const float* rrow, float err, int* boff, int ln) {
  const int n = min(m, A.lcap);
  // the reference's list: the whole row, or its half-list entries in order
  int mh = 0;
  for (int e0 = 0; e0 < n; e0 += 32) {
    const int e = e0 + ln;
    const bool h = e < n && row[e] >= 0;
    const unsigned hb = __ballot_sync(0xffffffffu, h);
    if (h) A.list[(size_t)(mh + __popc(hb & ((1u << ln) - 1u))) * A.cap + i] = row[e];
    mh += __popc(hb);
  }
  list_force_order(A, S, i, n, row, rrow, err, boff, ln);
  if (ln == 0) list_done(A, s, i, m, mh, false);
}

// ---- the candidate test of the cell-list builds
// A candidate's r^2 is first computed in FP32 from a 16-byte record staged
// per candidate (float4: three coordinates and the atom id as int bits), in
// one of two frames:
//  * image frame (every periodic dim has >= 3 cells, SysDev::list_img):
//    coordinates relative to the cell's origin, each candidate shifted by
//    its stencil cell's periodic image.  With >= 3 cells a periodic dim's
//    three stencil cells are distinct, so an atom appears once in the
//    stencil, at the one image within a cell of the home cell; an image
//    within rlist (<= a cell) of the atom must be that one, so this r^2 is
//    the minimum-image one for every pair within rlist.  Open dims use the
//    plain difference, as rd_exact does.  Components are within 2^-24 of
//    3 cells + rlist (open dims: of L + 3 cells + rlist, atoms lie in the
//    box) per rounding.
//  * integer frame (a periodic dim has fewer cells): integer coordinates, a
//    periodic dim mapping [0, L) onto the 32-bit ring (the wrapped int32
//    difference is the minimum image), an open dim 2^30 units per
//    max(L, rlist) (a difference that wraps is one of more than 2 rlist).
//    The difference shifted right by 10 bits (|v| < 2^21) converts to float
//    exactly through the 1.5 * 2^23 bias, so a component is off by under
//    1025 units plus two float roundings.
// err bounds |r2f - r^2| for pairs near rlist.  r2f < lo (rlist^2 - err)
// is inside the exact test's strict rlist^2 and r2f >= hi (rlist^2 + err)
// outside it; only candidates between take the exact FP64 test (rd_exact,
// the reference's arithmetic).  The lists are therefore the ones the exact
// test over every candidate gives.
struct ListFrame {
  double ls[3];   // integer frame: integer units per Angstrom
  float unit[3];  // integer frame: Angstrom per filter unit (1024 integer units)
  float lo, hi;   // r2f < lo: inside rlist; r2f >= hi: outside
  float err;      // bound on |r2f - r^2| for r^2 < hi
  int img;        // 1: image frame, 0: integer frame
};

__device__ __forceinline__ ListFrame list_frame(const SysDev& S) {
  ListFrame f;
  f.img = S.list_img;
  double sd = 0.0, sd2 = 0.0, dm = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double dk;
    if (f.img) {
      const double span = (S.pbc[k] ? 3.0 * S.cell[k] : S.L[k] + 3.0 * S.cell[k]) + S.rlist;
      dk = 4.0 * 5.9604644775390625e-8 * span;
      f.ls[k] = 0.0;
      f.unit[k] = 0.0f;
    } else {
      const double M = S.pbc[k] ? S.L[k] : 4.0 * fmax(S.L[k], S.rlist);  // Angstrom per 2^32 units
      f.ls[k] = 4294967296.0 / M;
      f.unit[k] = (float)(M * 2.384185791015625e-07);  // M / 2^22
      dk = 1025.0 * M * 2.3283064365386963e-10 + 2.4e-7 * S.rlist;
    }
    sd += dk;
    sd2 += dk * dk;
    dm = fmax(dm, dk);
  }
  const double err = 2.0 * (S.rlist + dm) * sd + sd2 + 1e-6 * S.rlist2;
  f.err = __double2float_ru(err);
  f.lo = __double2float_rd(S.rlist2 - err);
  f.hi = __double2float_ru(S.rlist2 + err);
  return f;
}

// integer-frame record of a position (atom id in w)
__device__ __forceinline__ float4 list_coords(const ListFrame& f, double4 p, int id) {
  return make_float4(__int_as_float((int)(unsigned)(unsigned long long)__double2ll_rn(p.x * f.ls[0])),
                     __int_as_float((int)(unsigned)(unsigned long long)__double2ll_rn(p.y * f.ls[1])),
                     __int_as_float((int)(unsigned)(unsigned long long)__double2ll_rn(p.z * f.ls[2])),
                     __int_as_float(id));
}

// one integer-frame component in Angstrom
__device__ __forceinline__ float list_comp(float a, float b, float unit) {
  const int v = (int)((unsigned)__float_as_int(b) - (unsigned)__float_as_int(a)) >> 10;
  return (__int_as_float(0x4B400000 + v) - 12582912.0f) * unit;
}

template <bool IMG>
__device__ __forceinline__ float list_r2(const ListFrame& f, float4 a, float4 b) {
  float x, y, z;
  if (IMG) {
    x = b.x - a.x;
    y = b.y - a.y;
    z = b.z - a.z;
  } else {
    x = list_comp(a.x, b.x, f.unit[0]);
    y = list_comp(a.y, b.y, f.unit[1]);
    z = list_comp(a.z, b.z, f.unit[2]);
  }
  return fmaf(z, z, fmaf(y, y, x * x));
}

// the staged record of candidate p (id j) of a stencil cell with periodic
// shift sh, for a home cell with origin o
template <bool IMG>
__device__ __forceinline__ float4 list_record(const ListFrame& f, double4 p, int j, double3 sh, double3 o) {
  if (IMG)
    return make_float4((float)(p.x + sh.x - o.x), (float)(p.y + sh.y - o.y), (float)(p.z + sh.z - o.z),
                       __int_as_float(j));
  return list_coords(f, p, j);
}

// a / b for 0 <= a < 2^31, b >= 1 by a double reciprocal and one
// correction (the estimate is off by one at most)
__device__ __forceinline__ int div_small(int a, int b) {
  int q = (int)((double)a * __drcp_rn((double)b));
  const int r = a - q * b;
  q += (r >= b) - (r < 0);
  return q;
}

// the grid coordinates of a system's cell cl (x fastest)
__device__ __forceinline__ void cell_xyz(const SysDev& S, int cl, int& cx, int& cy, int& cz) {
  const int yz = div_small(cl, S.nc[0]);
  cx = cl - yz * S.nc[0];
  cz = div_small(yz, S.nc[1]);
  cy = yz - cz * S.nc[1];
}

// stencil cell k of home cell (cx, cy, cz): its id and the periodic shift
// that takes its atoms to the image next to the home cell (open dims: none)
__device__ __forceinline__ int stencil_cell(const SysDev& S, int k, int cx, int cy, int cz, double3& sh) {
  int dx, dy, dz;
  stencil(k, dx, dy, dz);
  const int ux = cx + dx, uy = cy + dy, uz = cz + dz;
  // ux is in [-1, nc]: one wrap at most
  const int x = ux < 0 ? ux + S.nc[0] : ux >= S.nc[0] ? ux - S.nc[0] : ux;
  const int y = uy < 0 ? uy + S.nc[1] : uy >= S.nc[1] ? uy - S.nc[1] : uy;
  const int z = uz < 0 ? uz + S.nc[2] : uz >= S.nc[2] ? uz - S.nc[2] : uz;
  sh = make_double3(S.pbc[0] ? (ux - x) * S.cell[0] : 0.0, S.pbc[1] ? (uy - y) * S.cell[1] : 0.0,
                    S.pbc[2] ? (uz - z) * S.cell[2] : 0.0);
  return S.cell_off + x + S.nc[0] * (y + S.nc[1] * z);
}

// One warp tests atom i (chain position a of its cell, staged record ri)
// against the staged candidates t0 .. t0 + tn - 1 (records cf[0 .. tn-1]),
// 32 at a time, and appends the accepted ones to the row in candidate
// order: ids (bit 31 on those a half list leaves out) and r^2 as float.
// m counts the accepted candidates, lcap or more.
template <bool IMG>
__device__ __forceinline__ void list_scan_tile(const Arena& A, const SysDev& S, const ListFrame& f, const float4* cf,
                                               int t0, int tn, int i, int a, float4 ri, bool half, int own, int hend,
                                               int* row, float* rrow, int lcap, int& m, int ln) {
  const unsigned FULL = 0xffffffffu, lt = (1u << ln) - 1u;
  for (int q0 = 0; q0 < tn; q0 += 32) {
    const int q = q0 + ln;
    bool in = false, maybe = false;
    int j = -1;
    float r2 = 0.0f;
    if (q < tn) {
      const float4 c = cf[q];
      j = __float_as_int(c.w);
      r2 = list_r2<IMG>(f, ri, c);
      in = r2 < f.lo && j != i;
      maybe = r2 >= f.lo && r2 < f.hi && j != i;
    }
    if (__any_sync(FULL, maybe) && maybe) {  // within the error bound of rlist: the exact test
      const double rd = rd_exact(S, A.pos[i], A.pos[j]);
      in = rd < S.rlist2;
      r2 = (float)rd;
    }
    const unsigned bal = __ballot_sync(FULL, in);
    if (in) {
      const int mm = m + __popc(bal & lt);
      if (mm < lcap) {
        // the half list (linkedcell_selfhalf): the atoms after i in its own
        // cell's chain, then the other 13 cells of the half stencil
        const int g = t0 + q;
        const bool in_half = !half || (g < own ? g > a : g < hend);
        row[mm] = in_half ? j : (int)((unsigned)j | 0x80000000u);  // bit 31: full list only
        rrow[mm] = r2;
      }
    }
    m += __popc(bal);
  }
}

// linkedcell_self / linkedcell_selfhalf (src/Neighbour.F90:991-1161): the
// 27 (or 14) stencil cells in the reference's order with periodic cell
// wrap (cell_pbc, :1350-1376); keep j if rd < (rcut+nb_dcut)^2 (strict).
// For every atom of a cell the candidates are the same sequence: the
// stencil cells of that cell in stencil order, each in its chain order.  So
// one CTA takes one cell: warp 0 scans the stencil cells' counts, the CTA
// stages that sequence's records in shared memory (LIST_TILE candidates at
// a time) and its warps test the cell's atoms against it, one atom per warp
// (list_scan_tile), so each list comes out in the reference's order.  The
// home cell's atoms are the sequence's first candidates, so an atom's own
// record comes from the tile.  A warp stages its atom's row (ids and
// distances), then writes it to `list` as it is and to `flist` in the force
// order.
constexpr int LIST_ATOMS = BLOCK / 32;  // atoms per pass: one per warp
constexpr int LIST_TILE = 512;          // candidates staged at a time
constexpr int LIST_SPLIT = 4;           // CTAs that may share one cell's atoms
__host__ __device__ constexpr size_t list_smem(int lcap) {
  return (size_t)LIST_TILE * sizeof(float4) + (size_t)LIST_ATOMS * lcap * (sizeof(int) + sizeof(float));
}

template <bool IMG>
__device__ __forceinline__ void list_cells_item(const Arena& A, const BlockMap& C, int b, int part, float4* cf,
                                                int* stage, float* stage_rd, int* nb_start, int* nb_pref,
                                                double3* nb_sh, int* boff) {
  const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  const int s = C.sys[b];
  const SysDev& S = A.sys[s];
  const ListFrame f = list_frame(S);
  const bool half = S.half != 0;
  for (int c = C.first[b]; c < C.end[b]; c++) {
    const int cnt0 = A.cell_n[c];
    const int a_first = part * LIST_ATOMS;
    if (a_first >= cnt0) continue;  // uniform per CTA
    const int cl = c - S.cell_off;
    int cx, cy, cz;
    cell_xyz(S, cl, cx, cy, cz);
    const double3 o = make_double3(cx * S.cell[0], cy * S.cell[1], cz * S.cell[2]);
    if (warp == 0) {  // the stencil cells' starts, shifts and first candidates (a warp scan)
      int cn = 0, cs = 0;
      double3 sh = make_double3(0, 0, 0);
      if (ln < NSTENCIL) {
        const int cid = stencil_cell(S, ln, cx, cy, cz, sh);
        cs = A.cell_start[cid];
        cn = A.cell_n[cid];
      }
      int inc = cn;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(FULL, inc, d);
        if (ln >= d) inc += t;
      }
      if (ln < NSTENCIL) {
        nb_start[ln] = cs;
        nb_pref[ln] = inc - cn;
        nb_sh[ln] = sh;
      }
      if (ln == NSTENCIL - 1) nb_pref[NSTENCIL] = inc;
    }
    __syncthreads();
    const int T = nb_pref[NSTENCIL];  // candidates of every atom of the cell
    const int own = nb_pref[1];       // the first cell of the stencil is the cell itself
    const int hend = nb_pref[14];     // end of the half stencil's candidates
    auto stage_tile = [&](int t0, int tn) {
      for (int q = threadIdx.x; q < tn; q += BLOCK) {
        const int g = t0 + q;
        int k = 0;  // the last stencil cell whose first candidate is <= g
#pragma unroll
        for (int step = 16; step; step >>= 1)
          if (k + step < NSTENCIL && nb_pref[k + step] <= g) k += step;
        const int idx = nb_start[k] + (g - nb_pref[k]);
        const int j = A.cell_atoms[idx];
        const double4 p = A.cell_pos[idx];
        cf[q] = list_record<IMG>(f, p, j, nb_sh[k], o);
        if (g < own) A.pos_old[j] = p;  // the home cell's atoms: the list's reference positions
      }
    };
    const bool one = T <= LIST_TILE;  // one tile stays staged for all this CTA's passes
    if (one) {
      stage_tile(0, T);
      __syncthreads();
    }
    for (int a0 = a_first; a0 < cnt0; a0 += LIST_ATOMS * LIST_SPLIT) {
      const int a = a0 + warp;  // this warp's atom: chain position a of the cell
      const bool act = a < cnt0;
      int i = -1;
      float4 ri = make_float4(0, 0, 0, 0);
      if (act) {
        if (one) {
          ri = cf[a];  // the home cell's atoms come first, with no shift
          i = __float_as_int(ri.w);
        } else {
          i = A.cell_atoms[nb_start[0] + a];
          ri = list_record<IMG>(f, A.cell_pos[nb_start[0] + a], i, make_double3(0, 0, 0), o);
        }
      }
      int* row = stage + warp * A.lcap;
      float* rrow = stage_rd + warp * A.lcap;
      int m = 0;
      for (int t0 = 0; t0 < T; t0 += LIST_TILE) {
        const int tn = min(LIST_TILE, T - t0);
        if (!one) {
          __syncthreads();
          stage_tile(t0, tn);
          __syncthreads();
        }
        if (act) list_scan_tile<IMG>(A, S, f, cf, t0, tn, i, a, ri, half, own, hend, row, rrow, A.lcap, m, ln);
      }
      __syncwarp();
      if (act) list_row_out(A, S, s, i, m, row, rrow, f.err, boff, ln);
      __syncwarp();
    }
    __syncthreads();  // nb_* and the tile are rewritten for the next cell
  }
}

__global__ void __launch_bounds__(BLOCK) k_list_cells(Arena A, BlockMap C) {
  extern __shared__ __align__(16) unsigned char list_sh[];
  float4* cf = reinterpret_cast<float4*>(list_sh);                          // LIST_TILE records
  int* stage = reinterpret_cast<int*>(cf + LIST_TILE);                      // LIST_ATOMS x lcap ids
  float* stage_rd = reinterpret_cast<float*>(stage + LIST_ATOMS * A.lcap);  // and their r^2
  __shared__ int nb_start[NSTENCIL], nb_pref[NSTENCIL + 1];
  __shared__ double3 nb_sh[NSTENCIL];
  __shared__ int boff_sh[LIST_ATOMS][16];
  const int warp = threadIdx.x >> 5;
  // work item w = (map block w % nblk, part w / nblk): the part
  // takes atom passes part, part + LIST_SPLIT, ... of each of the block's
  // cells, so a cell of many atoms is shared by up to LIST_SPLIT CTAs
  // part-major numbering: the live items of sparse cells (part 0) spread
  // over every CTA whatever the grid size
  auto live = [&](int w) {
    const int b = w % C.nblk, part = w / C.nblk;
    if (!rebuild_block(A, C, b, true) || A.sys[C.sys[b]].list_warp) return false;
    // one-cell blocks: is there an atom pass for this part?
    return C.end[b] - C.first[b] != 1 || part * LIST_ATOMS < A.cell_n[C.first[b]];
  };
  rebuild_items(C.nblk * LIST_SPLIT, live, [&](int w) {
    const int b = w % C.nblk, part = w / C.nblk;
    if (A.sys[C.sys[b]].list_img)
      list_cells_item<true>(A, C, b, part, cf, stage, stage_rd, nb_start, nb_pref, nb_sh, boff_sh[warp]);
    else
      list_cells_item<false>(A, C, b, part, cf, stage, stage_rd, nb_start, nb_pref, nb_sh, boff_sh[warp]);
  });
}

// The same lists one warp per cell, so no warp idles on cells of few atoms
// and each SM keeps many cells' memory chains in flight (the CTA kernel
// above keeps one per CTA).  Lanes 0..26 read the stencil cells' starts,
// counts and shifts and a warp scan gives each cell's first candidate; the
// warp stages the candidates' records in its shared tile (ids and positions
// from the cell-ordered arrays, two rounds in flight per lane), finding a candidate's
// stencil cell by a binary search over the scan (shuffles); the cell's
// atoms are then tested one after another exactly as in k_list_cells.
// TILE = 128 for cells of about three atoms (Tersoff's 4 A cells), 512 for
// cells of up to about sixteen (a cell with more candidates than TILE is
// staged again for each atom).  Map: 8 cells per block (one per warp).
template <int TILE>
__host__ __device__ constexpr size_t listw_warp_bytes(int lcap) {
  return (size_t)TILE * sizeof(float4) + (size_t)lcap * (sizeof(int) + sizeof(float)) + 16 * sizeof(int);
}
template <int TILE>
__host__ __device__ constexpr size_t listw_smem(int lcap) {
  return (size_t)(BLOCK / 32) * listw_warp_bytes<TILE>(lcap);
}

template <bool IMG, int TILE>
__device__ __forceinline__ void list_cells_w_item(const Arena& A, const BlockMap& C, int b, float4* cf, int* boff,
                                                  int* row, float* rrow) {
  constexpr int U = 2;  // loads in flight per lane while staging
  const int warp = threadIdx.x >> 5, ln = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  const int c = C.first[b] + warp;
  if (c >= C.end[b]) return;  // warp-uniform
  const int s = C.sys[b];
  const SysDev& S = A.sys[s];
  const ListFrame f = list_frame(S);
  const bool half = S.half != 0;
  const int cl = c - S.cell_off;
  int cx, cy, cz;
  cell_xyz(S, cl, cx, cy, cz);
  const double3 o = make_double3(cx * S.cell[0], cy * S.cell[1], cz * S.cell[2]);
  int cs = 0, cn = 0;
  double3 sh = make_double3(0, 0, 0);
  if (ln < NSTENCIL) {
    const int cid = stencil_cell(S, ln, cx, cy, cz, sh);
    cs = A.cell_start[cid];
    cn = A.cell_n[cid];
  }
  int inc = cn;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int t = __shfl_up_sync(FULL, inc, d);
    if (ln >= d) inc += t;
  }
  const int ex = inc - cn;                             // first candidate of stencil cell ln
  const int T = __shfl_sync(FULL, inc, NSTENCIL - 1);  // candidates of every atom of the cell
  const int own = __shfl_sync(FULL, inc, 0);           // the cell itself: its atoms come first
  const int hend = __shfl_sync(FULL, inc, 13);         // end of the half stencil's candidates
  const int beg0 = __shfl_sync(FULL, cs, 0);
  const bool one = T <= TILE;  // one tile stays staged for all the cell's atoms
  auto stage_tile = [&](int t0, int tn) {
    __syncwarp();
    // the records: ids and positions from the cell-ordered arrays (one
    // index, two independent loads), U rounds of candidates in flight
    for (int q0 = 0; q0 < tn; q0 += 32 * U) {
      double4 p[U];
      int jv[U], kv[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int q = q0 + 32 * u + ln;
        const int g = t0 + q;
        // the last stencil cell whose first candidate is <= g (an empty
        // cell shares its first candidate with the next, non-empty one)
        int k = 0;
#pragma unroll
        for (int step = 16; step; step >>= 1) {
          const int kk = min(k + step, NSTENCIL - 1);
          const int e = __shfl_sync(FULL, ex, kk);
          if (k + step < NSTENCIL && e <= g) k = kk;
        }
        const int st = __shfl_sync(FULL, cs, k), ek = __shfl_sync(FULL, ex, k);
        kv[u] = k;
        jv[u] = -1;
        if (q < tn) {
          jv[u] = A.cell_atoms[st + (g - ek)];
          p[u] = A.cell_pos[st + (g - ek)];
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int q = q0 + 32 * u + ln;
        double3 shk = make_double3(0, 0, 0);
        if (IMG)
          shk = make_double3(__shfl_sync(FULL, sh.x, kv[u]), __shfl_sync(FULL, sh.y, kv[u]),
                             __shfl_sync(FULL, sh.z, kv[u]));
        if (q < tn) {
          cf[q] = list_record<IMG>(f, p[u], jv[u], shk, o);
          if (t0 + q < own) A.pos_old[jv[u]] = p[u];  // the home cell's atoms: the list's reference positions
        }
      }
    }
    __syncwarp();
  };
  if (one) stage_tile(0, T);
  for (int a = 0; a < own; a++) {
    int m = 0, i;
    float4 ri;
    if (one) {
      ri = cf[a];  // the home cell's atoms come first, with no shift
      i = __float_as_int(ri.w);
    } else {
      i = A.cell_atoms[beg0 + a];
      ri = list_record<IMG>(f, A.cell_pos[beg0 + a], i, make_double3(0, 0, 0), o);
    }
    for (int t0 = 0; t0 < T; t0 += TILE) {
      const int tn = min(TILE, T - t0);
      if (!one) stage_tile(t0, tn);
      list_scan_tile<IMG>(A, S, f, cf, t0, tn, i, a, ri, half, own, hend, row, rrow, A.lcap, m, ln);
    }
    __syncwarp();
    list_row_out(A, S, s, i, m, row, rrow, f.err, boff, ln);
    __syncwarp();
  }
}

// register bounds measured best: two blocks per SM for both tiles (three
// blocks of the 128 tile spill the staging's positions; the 512 tile's
// 72 KB of tiles fit three, but more registers win)
template <int TILE, bool IMG>
__global__ void __launch_bounds__(BLOCK, 2) k_list_cells_w(Arena A, BlockMap C) {
  extern __shared__ __align__(16) unsigned char listw_sh[];
  const int warp = threadIdx.x >> 5;
  unsigned char* mine = listw_sh + (size_t)warp * listw_warp_bytes<TILE>(A.lcap);
  float4* cf = reinterpret_cast<float4*>(mine);
  int* boff = reinterpret_cast<int*>(cf + TILE);
  int* row = boff + 16;
  float* rrow = reinterpret_cast<float*>(row + A.lcap);
  constexpr int KIND = TILE == 128 ? 1 : 2;  // SysDev::list_warp of the systems this kernel builds
  rebuild_items(C.nblk, [&](int b) {
      if (!rebuild_block(A, C, b, true)) return false;
      const SysDev& S = A.sys[C.sys[b]];
      return S.list_warp == KIND && (S.list_img != 0) == IMG;
    }, [&](int b) { list_cells_w_item<IMG, TILE>(A, C, b, cf, boff, row, rrow); });
}

// verlet_self / verlet_selfhalf (src/Neighbour.F90:676-811): O(N^2) over the
// system in increasing index, keep j if rd <= (rcut+nb_dcut)^2.  Candidate
// positions are staged through shared memory one BLOCK-wide tile at a time.
__global__ void k_list_n2(Arena A, BlockMap M) {
  __shared__ double4 tile[BLOCK];
  rebuild_items(M.nblk, [&](int b) { return rebuild_block(A, M, b, false); }, [&](int b) {
    const int s = M.sys[b];
    const SysDev& S = A.sys[s];
    int i = M.first[b] + threadIdx.x;
    bool act = i < M.end[b];
    double4 xi = act ? A.pos[i] : make_double4(0, 0, 0, 0);
    int m = 0, mh = 0;
    const int j0 = S.off, j1 = S.off + S.n;
    for (int base = j0; base < j1; base += BLOCK) {
      int j = base + threadIdx.x;
      __syncthreads();
      if (j < j1) tile[threadIdx.x] = A.pos[j];
      __syncthreads();
      int nt = min(BLOCK, j1 - base);
      if (act) {
        for (int t = 0; t < nt; t++) {
          int jj = base + t;
          if (jj == i) continue;
          double rd = rd_exact(S, xi, tile[t]);
          if (rd > S.rlist2) continue;
          // flist: every pair in index order (O(N^2) lists are not
          // grouped by band); list: a half list keeps j > i only
          if (m < A.lcap) A.flist[(size_t)m * A.cap + i] = jj;
          m++;
          if (!S.half || jj > i) {
            if (mh < A.lcap) A.list[(size_t)mh * A.cap + i] = jj;
            mh++;
          }
        }
      }
    }
    if (act) list_done(A, s, i, m, mh, true);
    __syncthreads();  // the tile is reused by the next block
  });
}

// rebuild counters; in_graph marks the copy captured inside a conditional
// node, whose executions are counted for the launch statistics
__global__ void k_count_rebuild(Arena A, const int* sys, int nsys, int in_graph) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nsys && sys[k] >= 0 && A.st[sys[k]].rebuild) {
    SysState& st = A.st[sys[k]];
    st.nupd++;
    st.dmax = 0.0;
    for (int d = 0; d < 3; d++) st.box_b[d] = A.sys[sys[k]].L[d];
  }
  if (in_graph && k == 0) atomicAdd(A.body_runs, 1ull);
}

// ------------------------------------------------------------------ reductions
// Six per-system sums (xx yy zz xy xz yz of a tensor): each block sums its
// threads' values; the system's last block adds the block partials in
// block order, so the result is the same bits on every run.
__device__ __forceinline__ void sys6_close(Arena& A, const BlockMap& M, int s, const double w[6], double* dst) {
  double b[6];
#pragma unroll
  for (int k = 0; k < 6; k++) b[k] = block_sum(w[k]);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; k++) A.blk_red[8 * (M.base + blockIdx.x) + k] = b[k];
  if (last_block(M, A.st, s, &A.st[s].ticket2) && threadIdx.x < 32) {
    const int b0 = M.sys_blk0[s], nb = M.sys_nblk[s];
    double t[6] = {0, 0, 0, 0, 0, 0};
    for (int q = threadIdx.x; q < nb; q += 32)
#pragma unroll
      for (int k = 0; k < 6; k++) t[k] += __ldcg(&A.blk_red[8 * (b0 + q) + k]);
#pragma unroll
    for (int k = 0; k < 6; k++)
      for (int o = 16; o; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
    if (threadIdx.x == 0)
      for (int k = 0; k < 6; k++) dst[k] = t[k];
  }
}

// Pair virial W = sum_i r_i (x) F_i.  With minimum-image pairs it is half
// the sum over the full list of vd (x) f vd / r (vd = r_j - r_i), the
// virial inq_virial (Inq_Properties.F90:439-527) builds from local and
// ghost atoms.
__device__ __forceinline__ void virial_close(Arena& A, const BlockMap& M, int s, const double w[6]) {
  sys6_close(A, M, s, w, A.st[s].vir);
}

// Thermostats after step b (integration_stepb runs every integrator's stepb
// in the order the deck adds them, src/Integration.F90:264-275).
// scalvel / scalvel_after (:1300-1340) need the system's kinetic energy
// about its centre of mass (inq_kin_energy / inq_temperature,
// Inq_Properties.F90:399-434), summed as the reference sums it, over
// m |v - v_cm|^2, in two passes: PASS 0 the centre-of-mass velocity, PASS 1
// the sum, T and the factor (T0/T)^soft, applied by k_thermo_apply.  (The
// one-pass form sum m v^2 - M |v_cm|^2 cancels digits when the centre of
// mass drifts fast.)  One atom alone has no kinetic energy about its centre
// of mass and is not scaled.
template <int PASS>
__global__ void k_thermo_sum(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  if (S.thermo != TH_SCALVEL && S.thermo != TH_SCALVEL_AFTER) return;  // the whole system's blocks
  constexpr int NW = PASS == 0 ? 4 : 1;
  int i = M.first[blockIdx.x] + threadIdx.x;
  double w[NW];
#pragma unroll
  for (int k = 0; k < NW; k++) w[k] = 0.0;
  if (i < M.end[blockIdx.x]) {
    const double4 v = A.vel[i];
    const double m = A.mass[i];
    if constexpr (PASS == 0) {
      w[0] = m;
      w[1] = m * v.x;
      w[2] = m * v.y;
      w[3] = m * v.z;
    } else {
      const double* c = A.st[s].th_vcm;
      const double d0 = v.x - c[0], d1 = v.y - c[1], d2 = v.z - c[2];
      w[0] = m * (d0 * d0 + d1 * d1 + d2 * d2);
    }
  }
  double b[NW];
#pragma unroll
  for (int k = 0; k < NW; k++) b[k] = block_sum(w[k]);
  if (threadIdx.x == 0)
    for (int k = 0; k < NW; k++) A.blk_red[8 * (M.base + blockIdx.x) + k] = b[k];
  if (last_block(M, A.st, s, &A.st[s].ticket2) && threadIdx.x < 32) {
    const int b0 = M.sys_blk0[s], nb = M.sys_nblk[s];
    double t[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) t[k] = 0.0;
    for (int q = threadIdx.x; q < nb; q += 32)
#pragma unroll
      for (int k = 0; k < NW; k++) t[k] += __ldcg(&A.blk_red[8 * (b0 + q) + k]);
#pragma unroll
    for (int k = 0; k < NW; k++)
      for (int o = 16; o; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
    if (threadIdx.x == 0) {
      if constexpr (PASS == 0) {
        for (int k = 0; k < 3; k++) A.st[s].th_vcm[k] = t[0] > 0.0 ? t[1 + k] / t[0] : 0.0;
      } else {
        const double ek = S.n > 1 ? 0.5 * t[0] : 0.0;
        const double T = 2.0 * ek / (S.th[3] * (3 * S.n));
        const double T0 = S.th[0];
        double f = 1.0;
        if (T != 0.0 && (S.thermo == TH_SCALVEL || fabs(T - T0) > S.th[2] * T0)) f = pow(T0 / T, S.th[1]);
        A.st[s].th_factor = f;
      }
    }
  }
}

// scalvel: v *= factor.  andersen (:1366-1395): each atom collides with
// probability nu dt and takes v = th[0] / sqrt(m) r per coordinate, th[0]
// the reference's sqrt(kB T / (3N)^2) (set_andersen, :1343-1364); the
// uniform and the normals come from the thermostat's own Philox stream.
__global__ void k_thermo_apply(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  int i = M.first[blockIdx.x] + threadIdx.x;
  if (S.thermo == TH_NONE || i >= M.end[blockIdx.x]) return;
  if (S.thermo == TH_ANDERSEN) {
    const uint64_t step = A.st[s].step;
    const uint2 key = make_uint2((uint32_t)S.th_seed, (uint32_t)(S.th_seed >> 32));
    const uint4 c = philox10(make_uint4((uint32_t)(i - S.off), (uint32_t)step, (uint32_t)(step >> 32), 7u), key);
    const double u = ((double)(c.x >> 8) + 0.5) * 5.9604644775390625e-8;  // (0, 1)
    if (u > S.th[1] * S.dt) return;
    double r[6];
    normals6((uint32_t)(i - S.off), step, S.th_seed, r);
    const double vm = S.th[0] * A.minv[i].y;
    A.vel[i] = make_double4(vm * r[0], vm * r[2], vm * r[4], 0.0);
  } else {
    const double f = A.st[s].th_factor;
    if (f != 1.0) {
      double4 v = A.vel[i];
      v.x = v.x * f;
      v.y = v.y * f;
      v.z = v.z * f;
      A.vel[i] = v;
    }
  }
}

// kinetic tensor sum_i m v (x) v of each system (inq_pressure,
// Inq_Properties.F90:529-573), into SysState::ktens
__global__ void k_kin_tensor(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  int i = M.first[blockIdx.x] + threadIdx.x;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (i < M.end[blockIdx.x]) {
    const double4 v = A.vel[i];
    const double m = A.mass[i];
    w[0] = v.x * v.x * m;
    w[1] = v.y * v.y * m;
    w[2] = v.z * v.z * m;
    w[3] = v.x * v.y * m;
    w[4] = v.x * v.z * m;
    w[5] = v.y * v.z * m;
  }
  sys6_close(A, M, s, w, A.st[s].ktens);
}

// ------------------------------------------------------------------ SMA-TB
// Per species-pair constants of the FP64 kernels.
struct SmFP64 {
  double A, eps2, p, q, r0, rci, rce, b1, b2, b3, r1, r2, r3, pr0, q2r0;
};
__device__ __forceinline__ SmFP64 sm_load(const PairP& P) {
  SmFP64 c;
  c.A = P.v[0];
  c.eps2 = P.v[1] * P.v[1];
  c.p = P.v[2];
  c.q = P.v[3];
  c.r0 = P.v[4];
  c.rci = P.v[5];
  c.rce = P.v[6];
  c.b1 = P.v[7]; c.b2 = P.v[8]; c.b3 = P.v[9];
  c.r1 = P.v[10]; c.r2 = P.v[11]; c.r3 = P.v[12];
  c.pr0 = P.v[2] / P.v[4];
  c.q2r0 = 2.0 * P.v[3] / P.v[4];
  return c;
}

template <int K>
__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
  for (int o = K / 2; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int K>
__device__ __forceinline__ float lane_sumf(float v) {
#pragma unroll
  for (int o = K / 2; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Pair loops of the force kernels: lane `lane` of an atom takes list slots
// lane, lane+K, ...; UNR slots are loaded, then gathered, then computed, so a
// lane keeps UNR independent gathers in flight (the kernels are bound by
// gather latency, not arithmetic).
constexpr int UNR = 4;

// list slots m0, m0+K, ... (UNR of them) of atom i; slots past nn, and ids
// outside the arena (never gather outside it), read as -1
template <int K, int N>
__device__ __forceinline__ void list_group(const Arena& A, int i, int nn, int m0, int (&jj)[N]) {
#pragma unroll
  for (int u = 0; u < N; u++) {
    int m = m0 + u * K;
    int j = m < nn ? __ldg(&A.flist[(size_t)m * A.cap + i]) : -1;
    jj[u] = (unsigned)j < (unsigned)A.cap ? j : -1;
  }
}

// The indices of the next group are loaded while the current group is
// gathered and computed, so a lane waits on one memory latency per group
// instead of two (list load, then the gathers it feeds).
#define PAIR_LOOP_BEGIN(GATHER_T, GATHER)                                      \
  int jn_[UNR];                                                               \
  list_group<K>(A, i, nn, lane, jn_);                                         \
  for (int m0 = lane; m0 < nn; m0 += UNR * K) {                               \
    int jj[UNR];                                                              \
    _Pragma("unroll") for (int u = 0; u < UNR; u++) jj[u] = jn_[u];           \
    GATHER_T gj[UNR];                                                         \
    _Pragma("unroll") for (int u = 0; u < UNR; u++) if (jj[u] >= 0) gj[u] = GATHER(jj[u]); \
    list_group<K>(A, i, nn, m0 + UNR * K, jn_);                               \
    _Pragma("unroll") for (int u = 0; u < UNR; u++) {                         \
      if (jj[u] < 0) continue;                                                \
      const int j = jj[u];                                                    \
      (void)j;
#define PAIR_LOOP_END \
    }                 \
  }


// smatb_preinteraction (src/TB.F90:367-455), FP64: rho_i = sum_j
//   xi^2 exp(-2q(r/r0-1))            r <  rci
//   (b1 d^5 + b2 d^4 + b3 d^3)^2     rci <= r <= rce, d = r - rce
__device__ __forceinline__ const SmFP64* sm_table(const Arena& A, const SysDev& S, SmFP64* sh) {
  const int np = S.ntypes * S.ntypes;
  for (int t = threadIdx.x; t < np; t += BLOCK) sh[t] = sm_load(A.prm[S.param_off + t]);
  __syncthreads();
  return sh;
}

template <int K>
__global__ void __launch_bounds__(BLOCK) k_smatb_rho_fp64(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  __shared__ SmFP64 tab_sh[MAXT * MAXT];
  const SmFP64* tab = sm_table(A, S, tab_sh);
  int i = M.first[blockIdx.x] + threadIdx.x / K;
  int lane = threadIdx.x % K;
  bool act = i < M.end[blockIdx.x];
  double band = 0.0;
  if (act) {
    const double4 xi = A.pos[i];
    const int ti = A.type[i];
    const int nn = live_entries(A, S, A.st[s], i, min(A.nn[i], A.lcap));
    const bool one = S.ntypes == 1;
    auto gat = [&](int j) { return A.pos[j]; };
    PAIR_LOOP_BEGIN(double4, gat)
      const SmFP64& c = tab[one ? 0 : ti * S.ntypes + A.type[j]];
      double v0, v1, v2;
      vd_fp64(S, xi, gj[u], v0, v1, v2);
      double dr = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
      if (dr > c.rce) continue;
      double banda;
      if (dr < c.rci) {
        banda = c.eps2 * exp(-2.0 * c.q * (dr / c.r0 - 1.0));
      } else {
        double d = dr - c.rce, d2 = d * d, d3 = d2 * d;
        banda = (c.b1 * d2 + c.b2 * d + c.b3) * d3;
        banda = banda * banda;
      }
      band += banda;
    PAIR_LOOP_END
  }
  band = lane_sum<K>(band);
  if (act && lane == 0) {
    A.band[i] = band;
    double eb = 1.0 / sqrt(band);
    A.eband[i] = eb;
    A.ebandf[i] = (float)eb;
    const double4 xi = A.pos[i];
    A.pose[i] = make_double4(xi.x, xi.y, xi.z, eb);  // one gather per neighbour in the force pass
  }
}

// smatb_interact (src/TB.F90:457-586), FP64, full list (newton off):
//   r <= rci : factor = 2 A e^{-p(r/r0-1)} p/r0
//                       - xi^2/2 e^{-2q(r/r0-1)} (2q/r0)(eb_i + eb_j)
//   tail     : factor = P P' (eb_i + eb_j) - 2 R'
//   F_i -= factor * ev_ui * vd / r ;  e_i += repul ; e_i -= sqrt(rho_i)
// The FP64 force pass for one thread's lane of atom i; lane 0 stores the
// force and energy and returns the force in F (STORE=false: stores
// nothing and returns the energy in F.w, for the caller to store).
// VIR: also the pair virial of the system (virial_close); SMA-TB forces are
// central pair forces, F_i = -sum_j factor_ij vd / r, so W is the pair sum
// (complete: the reference's TB.F90:548-564 omits the i-side term).
template <int K, bool VIR, bool STORE = true>
__device__ __forceinline__ void force_fp64_body(Arena& A, const BlockMap& M, int s, const SysDev& S,
                                                const SmFP64* tab, int i, int lane, bool act, double4& F) {
  double f0 = 0, f1 = 0, f2 = 0, ep = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (act) {
    const double4 xi = A.pos[i];
    const int ti = A.type[i];
    const double ebi = A.eband[i];
    const int nn = live_entries(A, S, A.st[s], i, min(A.nn[i], A.lcap));
    const bool one = S.ntypes == 1;
    auto gat = [&](int j) { return A.pose[j]; };
    PAIR_LOOP_BEGIN(double4, gat)
      const SmFP64& c = tab[one ? 0 : ti * S.ntypes + A.type[j]];
      double v0, v1, v2;
      vd_fp64(S, xi, gj[u], v0, v1, v2);
      double dr = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
      if (dr > c.rce) continue;
      double factor, repul;
      double ebs = ebi + gj[u].w;
      if (dr <= c.rci) {
        double x = dr / c.r0 - 1.0;
        repul = c.A * exp(-c.p * x);
        factor = 2.0 * repul * c.pr0 - c.eps2 * 0.5 * exp(-2.0 * c.q * x) * c.q2r0 * ebs;
      } else {
        double d = dr - c.rce, d2 = d * d, d3 = d2 * d, d4 = d3 * d;
        double P = (c.b1 * d2 + c.b2 * d + c.b3) * d3;
        double dP = 5.0 * c.b1 * d4 + 4.0 * c.b2 * d3 + 3.0 * c.b3 * d2;
        double dR = 5.0 * c.r1 * d4 + 4.0 * c.r2 * d3 + 3.0 * c.r3 * d2;
        factor = P * dP * ebs - 2.0 * dR;
        repul = (c.r1 * d2 + c.r2 * d + c.r3) * d3;
      }
      double fr = factor * EV_UI / dr;
      f0 -= fr * v0;
      f1 -= fr * v1;
      f2 -= fr * v2;
      ep += repul;
      if constexpr (VIR) {
        const double h = 0.5 * fr;
        w[0] += h * v0 * v0;
        w[1] += h * v1 * v1;
        w[2] += h * v2 * v2;
        w[3] += h * v0 * v1;
        w[4] += h * v0 * v2;
        w[5] += h * v1 * v2;
      }
    PAIR_LOOP_END
  }
  f0 = lane_sum<K>(f0);
  f1 = lane_sum<K>(f1);
  f2 = lane_sum<K>(f2);
  ep = lane_sum<K>(ep);
  if (act && lane == 0) {
    const double e = (ep - sqrt(A.band[i])) * EV_UI;
    if constexpr (STORE) {
      F = make_double4(f0, f1, f2, 0.0);
      A.force[i] = F;
      A.epot[i] = e;
    } else {
      F = make_double4(f0, f1, f2, e);
    }
  }
  if constexpr (VIR) virial_close(A, M, s, w);
}

template <int K, bool VIR>
__global__ void __launch_bounds__(BLOCK) k_smatb_force_fp64(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  __shared__ SmFP64 tab_sh[MAXT * MAXT];
  const SmFP64* tab = sm_table(A, S, tab_sh);
  const int i = M.first[blockIdx.x] + threadIdx.x / K;
  double4 F;
  force_fp64_body<K, VIR>(A, M, s, S, tab, i, threadIdx.x % K, i < M.end[blockIdx.x], F);
}

// ---- mixed precision: FP32 pair math, FP64 accumulation.
// Pair vectors come from fixed-point coordinates, so the subtraction is
// exact and the minimum image is the int32 wrap of periodic dims.
struct SmF32 {
  float kp, kq, r0;    // e1 = 2^(kp (r0 - r)) = exp(-p(r/r0-1)),
                       // e2 = 2^(kq (r0 - r)) = exp(-2q(r/r0-1)); r0 - r is exact
  float A, eps2, c1, c2;
  float rci, rce, rci2, rce2;
  float b1, b2, b3, r1, r2, r3;
  // the force pass's constants with the unit ev_ui folded in: c1, c2; the
  // tail derivatives' coefficients 5 b1, 4 b2, 3 b3 and 2 (5 r1, 4 r2, 3 r3)
  float c1e, c2e, dp5, dp4, dp3, dr5, dr4, dr3;
};
__device__ __forceinline__ SmF32 smf_load(const PairP& P) {
  const double log2e = 1.4426950408889634;
  SmF32 c;
  double A = P.v[0], xi = P.v[1], p = P.v[2], q = P.v[3], r0 = P.v[4];
  c.kp = (float)(p / r0 * log2e);
  c.kq = (float)(2.0 * q / r0 * log2e);
  c.r0 = (float)r0;
  c.A = (float)A;
  c.eps2 = (float)(xi * xi);
  c.c1 = (float)(2.0 * A * p / r0);          // 2 A p/r0 (times e1)
  c.c2 = (float)(xi * xi * q / r0);          // xi^2/2 * 2q/r0 (times e2 * ebs)
  c.rci = (float)P.v[5];
  c.rce = (float)P.v[6];
  c.rci2 = (float)(P.v[5] * P.v[5]);
  c.rce2 = (float)(P.v[6] * P.v[6]);
  c.b1 = (float)P.v[7]; c.b2 = (float)P.v[8]; c.b3 = (float)P.v[9];
  c.r1 = (float)P.v[10]; c.r2 = (float)P.v[11]; c.r3 = (float)P.v[12];
  const double e = EV_UI;
  c.c1e = (float)(2.0 * A * p / r0 * e);
  c.c2e = (float)(xi * xi * q / r0 * e);
  c.dp5 = (float)(5.0 * P.v[7] * e); c.dp4 = (float)(4.0 * P.v[8] * e); c.dp3 = (float)(3.0 * P.v[9] * e);
  c.dr5 = (float)(10.0 * P.v[10] * e); c.dr4 = (float)(8.0 * P.v[11] * e); c.dr3 = (float)(6.0 * P.v[12] * e);
  return c;
}

// exact integer difference, one rounding in the conversion; the unit is
// applied as hi + lo so its float rounding adds no systematic scale error
__device__ __forceinline__ void vd_fx(const SysDev& S, int4 a, int4 b, float& x, float& y,
                                      float& z) {
  float fx = (float)(b.x - a.x), fy = (float)(b.y - a.y), fz = (float)(b.z - a.z);
  x = fmaf(fx, S.fx_inv[0], fx * S.fx_inv_lo[0]);
  y = fmaf(fy, S.fx_inv[1], fy * S.fx_inv_lo[1]);
  z = fmaf(fz, S.fx_inv[2], fz * S.fx_inv_lo[2]);
}

__device__ __forceinline__ float ex2f(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// r = sqrt(r2) and 1/r from one MUFU rsqrt plus a Newton step on r
// (accurate to ~1 ulp without the IEEE sqrt / rcp instruction sequences)
__device__ __forceinline__ float sqrt_nr(float r2, float& rinv) {
  rinv = rsqrtf(r2);
  float r = r2 * rinv;
  return fmaf(0.5f * rinv, fmaf(-r, r, r2), r);
}

// Mixed kernels sum the FP32 pair terms of one group (UNR_R pairs in the
// density pass, UNR_F in the force pass, whose pairs hold more registers)
// in FP32 and add the group sums to FP64 per-atom accumulators (one
// conversion per group).
constexpr int UNR_R = 4;
constexpr int UNR_F = 2;
// ONE: single-species system, constants held in registers; otherwise the
// species-pair table sits in shared memory and is read per pair.
template <bool ONE>
__device__ __forceinline__ const SmF32* smf_table(const Arena& A, const SysDev& S, SmF32* sh) {
  if (ONE) return nullptr;
  const int np = S.ntypes * S.ntypes;
  for (int t = threadIdx.x; t < np; t += BLOCK) sh[t] = smf_load(A.prm[S.param_off + t]);
  __syncthreads();
  return sh;
}

// MINB > 1 asks the compiler to fit MINB blocks per SM (fewer registers,
// more warps to hide gather latency); the autotuner tries both.
template <int K, bool ONE, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_smatb_rho_mixed(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  __shared__ SmF32 tab_sh[ONE ? 1 : MAXT * MAXT];
  const SmF32* tab = smf_table<ONE>(A, S, tab_sh);
  int i = M.first[blockIdx.x] + threadIdx.x / K;
  int lane = threadIdx.x % K;
  bool act = i < M.end[blockIdx.x];
  double band = 0.0;
  if (act) {
    const int4 xi = A.fxp[i];
    const int nn = live_entries(A, S, A.st[s], i, min(A.nn[i], A.lcap));
    const SmF32 c1 = ONE ? smf_load(A.prm[S.param_off]) : SmF32{};
    int jn[UNR_R];
    list_group<K>(A, i, nn, lane, jn);
    for (int m0 = lane; m0 < nn; m0 += UNR_R * K) {
      int jj[UNR_R];
#pragma unroll
      for (int u = 0; u < UNR_R; u++) jj[u] = jn[u];
      int4 gj[UNR_R];
#pragma unroll
      for (int u = 0; u < UNR_R; u++) {
        gj[u] = xi;  // an empty slot: a zero pair vector, masked below
        if (jj[u] >= 0) gj[u] = A.fxp[jj[u]];
      }
      list_group<K>(A, i, nn, m0 + UNR_R * K, jn);  // next group's ids, in flight meanwhile
      float grp = 0.0f;
      // branch-free: both regimes are evaluated and selected, so the
      // group's pairs interleave (a warp's lanes would run both anyway)
#pragma unroll
      for (int u = 0; u < UNR_R; u++) {
        const int4 xj = gj[u];
        const SmF32& c = ONE ? c1 : tab[xi.w * S.ntypes + xj.w];
        float v0, v1, v2;
        vd_fx(S, xi, xj, v0, v1, v2);
        const float r2 = v0 * v0 + v1 * v1 + v2 * v2;
        const bool ok = jj[u] >= 0 && !(r2 > c.rce2);
        float rinv;
        const float dr = sqrt_nr(ok ? r2 : c.rce2, rinv);
        const float bin = c.eps2 * ex2f(c.kq * (c.r0 - dr));
        const float d = dr - c.rce, d3 = d * d * d;
        float bt = fmaf(fmaf(c.b1, d, c.b2), d, c.b3) * d3;
        bt = bt * bt;
        const float banda = dr < c.rci ? bin : bt;
        grp += ok ? banda : 0.0f;
      }
      band += (double)grp;
    }
  }
  band = lane_sum<K>(band);
  if (act && lane == 0) {
    A.band[i] = band;
    double eb = 1.0 / sqrt(band);
    A.eband[i] = eb;
    const float ebf = (float)eb;
    A.ebandf[i] = ebf;
    const int4 xi = A.fxp[i];
    A.fxe[i] = make_int4(xi.x, xi.y, xi.z, __float_as_int(ebf));  // one gather per neighbour
  }
}

// The force pass for one thread's lane of atom i (K lanes per atom); lane 0
// stores the force and energy and returns the force in F (STORE=false:
// stores nothing and returns the energy in F.w, for the caller to store).
// VIR: also the pair virial, FP32 per pair and group, FP64 per atom and system.
template <int K, bool ONE, bool VIR, bool STORE = true>
__device__ __forceinline__ void force_mixed_body(Arena& A, const BlockMap& M, int s, const SysDev& S,
                                                 const SmF32* tab, int i, int lane, bool act, double4& F) {
  double f0 = 0, f1 = 0, f2 = 0, ep = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (act) {
    const int4 xi = A.fxp[i];
    const float ebi = A.ebandf[i];
    const int nn = live_entries(A, S, A.st[s], i, min(A.nn[i], A.lcap));
    const SmF32 c1 = ONE ? smf_load(A.prm[S.param_off]) : SmF32{};
    const int ti = xi.w;
    int jn[UNR_F];
    list_group<K>(A, i, nn, lane, jn);
    for (int m0 = lane; m0 < nn; m0 += UNR_F * K) {
      int jj[UNR_F];
#pragma unroll
      for (int u = 0; u < UNR_F; u++) jj[u] = jn[u];
      int4 gj[UNR_F];
      int tj[UNR_F];
#pragma unroll
      for (int u = 0; u < UNR_F; u++) {
        gj[u] = make_int4(xi.x, xi.y, xi.z, 0);  // an empty slot: a zero pair vector, masked below
        tj[u] = 0;
        if (jj[u] >= 0) {
          gj[u] = A.fxe[jj[u]];
          if (!ONE) tj[u] = A.type[jj[u]];
        }
      }
      list_group<K>(A, i, nn, m0 + UNR_F * K, jn);  // next group's ids, in flight meanwhile
      float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f, ge = 0.0f;
      float gw[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
      // branch-free: both regimes are evaluated and selected, so the
      // group's pairs interleave (a warp's lanes would run both anyway)
#pragma unroll
      for (int u = 0; u < UNR_F; u++) {
        const int4 xj = gj[u];
        const SmF32& c = ONE ? c1 : tab[ti * S.ntypes + tj[u]];
        float v0, v1, v2;
        vd_fx(S, xi, xj, v0, v1, v2);
        const float r2 = v0 * v0 + v1 * v1 + v2 * v2;
        const bool ok = jj[u] >= 0 && !(r2 > c.rce2);
        float rinv;
        const float dr = sqrt_nr(ok ? r2 : c.rce2, rinv);
        const float ebs = ebi + __int_as_float(xj.w);
        const float x = c.r0 - dr;
        const float e1 = ex2f(c.kp * x);
        const float e2 = ex2f(c.kq * x);
        // the tail polynomials in Horner form; factor carries ev_ui
        const float d = dr - c.rce, d2 = d * d, d3 = d2 * d;
        const float P = fmaf(fmaf(c.b1, d, c.b2), d, c.b3) * d3;
        const float dPe = fmaf(fmaf(c.dp5, d, c.dp4), d, c.dp3) * d2;  // ev_ui P'
        const float dRe = fmaf(fmaf(c.dr5, d, c.dr4), d, c.dr3) * d2;  // 2 ev_ui R'
        const bool inner = dr <= c.rci;
        const float factor = inner ? c.c1e * e1 - c.c2e * e2 * ebs : P * dPe * ebs - dRe;
        const float repul = ok ? (inner ? c.A * e1 : fmaf(fmaf(c.r1, d, c.r2), d, c.r3) * d3) : 0.0f;
        const float fr = ok ? factor * rinv : 0.0f;
        g0 = fmaf(fr, v0, g0);
        g1 = fmaf(fr, v1, g1);
        g2 = fmaf(fr, v2, g2);
        ge += repul;
        if constexpr (VIR) {
          const float h = 0.5f * fr;
          gw[0] += h * v0 * v0;
          gw[1] += h * v1 * v1;
          gw[2] += h * v2 * v2;
          gw[3] += h * v0 * v1;
          gw[4] += h * v0 * v2;
          gw[5] += h * v1 * v2;
        }
      }
      f0 -= (double)g0;
      f1 -= (double)g1;
      f2 -= (double)g2;
      ep += (double)ge;
      if constexpr (VIR)
        for (int k = 0; k < 6; k++) w[k] += (double)gw[k];
    }
  }
  f0 = lane_sum<K>(f0);
  f1 = lane_sum<K>(f1);
  f2 = lane_sum<K>(f2);
  ep = lane_sum<K>(ep);
  if (act && lane == 0) {
    const double e = (ep - sqrt(A.band[i])) * EV_UI;
    if constexpr (STORE) {
      F = make_double4(f0, f1, f2, 0.0);
      A.force[i] = F;
      A.epot[i] = e;
    } else {
      F = make_double4(f0, f1, f2, e);
    }
  }
  if constexpr (VIR) virial_close(A, M, s, w);
}

template <int K, bool ONE, int MINB, bool VIR = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_smatb_force_mixed(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  __shared__ SmF32 tab_sh[ONE ? 1 : MAXT * MAXT];
  const SmF32* tab = smf_table<ONE>(A, S, tab_sh);
  const int i = M.first[blockIdx.x] + threadIdx.x / K;
  double4 F;
  force_mixed_body<K, ONE, VIR>(A, M, s, S, tab, i, threadIdx.x % K, i < M.end[blockIdx.x], F);
}

// ------------------------------------------------------------------ LJ
// lj_interact / plj_interact (src/Pairs.F90:207-370), full list:
//   s6 = (s/r)^6 ; p = 4e(s6^2 - s6) [- prc - frc (r - rc)] [- eshift]
//   f = e(48 s6 - 24) s6 / r [+ frc] ; F_i -= f vd / r ; e_i += p/2
// slj_interact (src/Pairs.F90:403-470) for pairs of the slj form:
//   r < rs: p = 4e (s6 - 1) s6, f as LJ;  rs <= r <= rc, d = r - rc:
//   p = sa4 d^4 + sa8 d^8, f = -(4 sa4 d^4 + 8 sa8 d^8) / d
// sm1_interact (src/Pairs.F90:925-1011) for pairs of the sm1 form:
//   r > r1: aux = pi (r - (r1 + rc)/2) / (rc - r1), p = e (1/2 + sin(aux)/2) - e,
//   f = -e cos(aux) (pi/2) r / (rc - r1);  r <= r1: p = -e, f = 0
// wca_interact (src/Pairs.F90:508-589) is LJ with eshift = -e
// VIR: also the pair virial of the system (virial_close).
template <int K, bool VIR>
__global__ void __launch_bounds__(BLOCK) k_lj_fp64(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  int i = M.first[blockIdx.x] + threadIdx.x / K;
  int lane = threadIdx.x % K;
  bool act = i < M.end[blockIdx.x];
  double f0 = 0, f1 = 0, f2 = 0, ep = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (act) {
    const double4 xi = A.pos[i];
    const int ti = A.type[i];
    const int nn = live_entries(A, S, A.st[s], i, min(A.nn[i], A.lcap));
    auto gat = [&](int j) { return A.pos[j]; };
    PAIR_LOOP_BEGIN(double4, gat)
      const PairP& P = A.prm[S.param_off + ti * S.ntypes + A.type[j]];
      double e = P.v[0];
      if (e == 0.0 && P.v[1] == 0.0) continue;
      double v0, v1, v2;
      vd_fp64(S, xi, gj[u], v0, v1, v2);
      double dr = v0 * v0 + v1 * v1 + v2 * v2;
      if (dr > P.v[3]) continue;
      dr = sqrt(dr);
      double p, f;
      if (P.v[8] == 2.0) {
        // sm1: the reference's force carries a factor dr (Pairs.F90:957)
        const double w = P.v[2] - P.v[11];
        if (dr > P.v[11]) {
          const double aux = PI_D * (dr - (P.v[11] + P.v[2]) * 0.5) / w;
          double sn, cs;
          sincos(aux, &sn, &cs);
          p = (0.5 + 0.5 * sn) * e - e;
          f = -(cs * (0.5 * PI_D) * dr / w) * e;
        } else {
          p = -e;
          f = 0.0;
        }
      } else if (P.v[8] != 0.0 && dr >= P.v[11]) {
        const double d = dr - P.v[2];
        const double s4 = d * d * d * d;
        p = P.v[9] * s4 + P.v[10] * s4 * s4;
        f = -(4.0 * P.v[9] * s4 + 8.0 * P.v[10] * s4 * s4) / d;
      } else {
        double t = P.v[1] / dr;
        double t3 = t * t * t;
        double s6 = t3 * t3;
        p = P.v[8] != 0.0 ? 4.0 * e * (s6 - 1.0) * s6 : 4.0 * e * (s6 * s6 - s6);
        f = e * (48.0 * s6 - 24.0) * s6 / dr;
        if (P.v[7] != 0.0) {
          p = p - P.v[4] - P.v[5] * (dr - P.v[2]);
          f = f + P.v[5];
        } else {
          p = p - P.v[6];
        }
      }
      // f == 0 (sm1 inside r1) adds nothing, also for coincident atoms
      double fr = f != 0.0 ? f * EV_UI / dr : 0.0;
      f0 -= fr * v0;
      f1 -= fr * v1;
      f2 -= fr * v2;
      ep += p;
      if constexpr (VIR) {
        const double h = 0.5 * fr;
        w[0] += h * v0 * v0;
        w[1] += h * v1 * v1;
        w[2] += h * v2 * v2;
        w[3] += h * v0 * v1;
        w[4] += h * v0 * v2;
        w[5] += h * v1 * v2;
      }
    PAIR_LOOP_END
  }
  f0 = lane_sum<K>(f0);
  f1 = lane_sum<K>(f1);
  f2 = lane_sum<K>(f2);
  ep = lane_sum<K>(ep);
  if (act && lane == 0) {
    A.force[i] = make_double4(f0, f1, f2, 0.0);
    A.epot[i] = ep * 0.5 * EV_UI;
  }
  if constexpr (VIR) virial_close(A, M, s, w);
}

// The float constants of one LJ species pair, in a per-block table: 4e,
// 48e, 24e, sigma^2, rc^2, and by form -- 0: truncated and shifted (the
// shift), 1: shifted force (prc, frc, rc), 2: slj (rs^2, sa4, sa8, rc).
struct LjF32 {
  float e4, e48, e24, sg2, rc2, sh, frc, rc, rs2, sa4, sa8;
  int form, on;
};
__device__ __forceinline__ LjF32 ljf_load(const PairP& P) {
  LjF32 c;
  const double e = P.v[0], sg = P.v[1];
  c.e4 = (float)(4.0 * e);
  c.e48 = (float)(48.0 * e);
  c.e24 = (float)(24.0 * e);
  c.sg2 = (float)(sg * sg);
  c.rc2 = (float)P.v[3];
  c.rc = (float)P.v[2];
  c.form = P.v[8] != 0.0 ? 2 : P.v[7] != 0.0 ? 1 : 0;
  c.sh = (float)(c.form == 1 ? P.v[4] : P.v[6]);
  c.frc = (float)P.v[5];
  c.rs2 = (float)(P.v[11] * P.v[11]);
  c.sa4 = (float)P.v[9];
  c.sa8 = (float)P.v[10];
  c.on = (float)e != 0.0f;
  return c;
}

// Mixed LJ: FP32 pair math from the fixed-point geometry, the species
// table in shared memory, the FP32 terms of each group of UNR pairs summed
// and the group sums accumulated per atom in FP64.
template <int K, bool VIR = false>
__global__ void __launch_bounds__(BLOCK) k_lj_mixed(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  __shared__ LjF32 tab[MAXT * MAXT];
  for (int t = threadIdx.x; t < S.ntypes * S.ntypes; t += BLOCK) tab[t] = ljf_load(A.prm[S.param_off + t]);
  __syncthreads();
  int i = M.first[blockIdx.x] + threadIdx.x / K;
  int lane = threadIdx.x % K;
  bool act = i < M.end[blockIdx.x];
  double f0 = 0, f1 = 0, f2 = 0, ep = 0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (act) {
    const int4 xi = A.fxp[i];
    const int nn = live_entries(A, S, A.st[s], i, min(A.nn[i], A.lcap));
    const float evui = (float)EV_UI;
    const LjF32* row = tab + xi.w * S.ntypes;
    int jn[UNR];
    list_group<K>(A, i, nn, lane, jn);
    for (int m0 = lane; m0 < nn; m0 += UNR * K) {
      int jj[UNR];
#pragma unroll
      for (int u = 0; u < UNR; u++) jj[u] = jn[u];
      int4 gj[UNR];
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        gj[u] = xi;  // an empty slot: a zero pair vector, masked below
        if (jj[u] >= 0) gj[u] = A.fxp[jj[u]];
      }
      list_group<K>(A, i, nn, m0 + UNR * K, jn);  // next group's ids, in flight meanwhile
      float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f, ge = 0.0f;
      float gw[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        const int4 xj = gj[u];
        const LjF32& c = row[xj.w];
        float v0, v1, v2;
        vd_fx(S, xi, xj, v0, v1, v2);
        const float r2 = v0 * v0 + v1 * v1 + v2 * v2;
        const bool ok = jj[u] >= 0 && !(r2 > c.rc2) && c.on;
        const float ir2 = __frcp_rn(ok ? r2 : c.rc2);
        const float t2 = c.sg2 * ir2;
        const float s6 = t2 * t2 * t2;
        float p = c.e4 * (s6 * s6 - s6);
        float fr = (c.e48 * s6 - c.e24) * s6 * ir2;  // f / r
        if (c.form == 2) {
          // slj (Pairs.F90:403-470): plain LJ inside rs, the quartic-octic
          // spline sa4 d^4 + sa8 d^8 (d = r - rc) from rs to rc
          if (ok && r2 >= c.rs2) {
            const float dr = sqrtf(r2), d = dr - c.rc;
            const float s4 = d * d * d * d;
            p = c.sa4 * s4 + c.sa8 * s4 * s4;
            fr = -(4.0f * c.sa4 * s4 + 8.0f * c.sa8 * s4 * s4) / (d * dr);
          }
        } else if (c.form == 1) {  // shifted force (plj, Pairs.F90:282-370)
          const float dr = sqrtf(ok ? r2 : c.rc2);
          p = p - c.sh - c.frc * (dr - c.rc);
          fr = fr + c.frc / dr;
        } else {
          p = p - c.sh;
        }
        fr = ok ? fr * evui : 0.0f;
        g0 = fmaf(fr, v0, g0);
        g1 = fmaf(fr, v1, g1);
        g2 = fmaf(fr, v2, g2);
        ge += ok ? p : 0.0f;
        if constexpr (VIR) {
          const float h = 0.5f * fr;
          gw[0] += h * v0 * v0;
          gw[1] += h * v1 * v1;
          gw[2] += h * v2 * v2;
          gw[3] += h * v0 * v1;
          gw[4] += h * v0 * v2;
          gw[5] += h * v1 * v2;
        }
      }
      f0 -= (double)g0;
      f1 -= (double)g1;
      f2 -= (double)g2;
      ep += (double)ge;
      if constexpr (VIR)
        for (int k = 0; k < 6; k++) w[k] += (double)gw[k];
    }
  }
  f0 = lane_sum<K>(f0);
  f1 = lane_sum<K>(f1);
  f2 = lane_sum<K>(f2);
  ep = lane_sum<K>(ep);
  if (act && lane == 0) {
    A.force[i] = make_double4(f0, f1, f2, 0.0);
    A.epot[i] = ep * 0.5 * EV_UI;
  }
  if constexpr (VIR) virial_close(A, M, s, w);
}

// ------------------------------------------------------------------ Tersoff
// Tersoff 1988 with the functional form of src/Tersoff.f90:131-341 (chi
// prefactor, no lambda3 term) and the cut-off fcut_dfcut of
// src/Algebra.F90:391-409:
//   E = sum_i E_i,  E_i = sum_{j bonded to i} 1/2 fc(r_ij) [VR(r_ij) + b_ij VA(r_ij)],
//   VR = A e^{-l1 r},  VA = -B e^{-l2 r},  b_ij = chi (1 + (beta zeta_ij)^n)^{-1/2n},
//   zeta_ij = sum_{k != j} fc(r_ik) g(cos theta_ijk),
//   g = 1 + c^2/d^2 - c^2/(d^2 + (h - cos)^2),
// with forces that are the exact gradient of E (the reference's missing
// radial force on j and its unallocated gradb_k are not reproduced).
//
// Gather formulation: no atomics, so the forces are the same bits on every
// run and in every batch.
//  * k_tsf_bonds, per centre atom i (2 or 4 threads): i's bonds (r <= R+D)
//    in flist order; per bond a = (i, j): zeta, b and the force that E_i puts
//    on j, F_j(i) = -dE_i/dx_j, stored in the bond record tsfb[a cap + i].
//    E_i is translation invariant, so the force it puts on i itself is
//    -sum_a F_j(a).  tsmask[i] marks the flist slots that are bonds.
//  * k_tsf_gather, per atom l: F_l = F_l(l) + the records its bond partners
//    wrote for their bonds to l, in l's slot order.  rslot (built with the
//    list) is l's slot in the partner's flist: centre j writes the index of
//    its record for l to tidx at that slot of l, so l reads it from its own
//    row.
// Bond decisions are symmetric (the pair vector seen from j is the exact
// negative of the one seen from i), so every record a gather looks for exists.
//
// R = double: the plain FP64 kernel.  R = float (mixed): geometry from the
// fixed-point copies; the angular sums zeta, their gradients and the bond
// order in FP32; VR, VA, fc and the energy in FP64.  b VA is formed as
// chi VA - chi VA y with y = 1 - (1+x)^{-1/2n}, x = (beta zeta)^n, from log1p
// and expm1, so the FP32 rounding of y costs y's relative error (y ~ 0.04 in
// silicon), not b's.  A bond's triplet force terms are summed in FP32, the
// bond records and the per-atom sums in FP64.

template <typename R>
__device__ __forceinline__ R ts_fc(R r, R r1, R r2, R& dfc) {
  if (r < r1) { dfc = R(0); return R(1); }
  if (r > r2) { dfc = R(0); return R(0); }
  const R pi = R(3.14159265358979323846);
  const R aux = pi * (r - (r1 + r2) * R(0.5)) / (r2 - r1);
  R sn, cs;
  if constexpr (sizeof(R) == 8) sincos(aux, &sn, &cs);
  else sincosf(aux, &sn, &cs);
  dfc = -cs * (pi * R(0.5)) / (r2 - r1);
  return R(0.5) - R(0.5) * sn;
}

// bond order of one bond: b, b VA (FP64) and db/dzeta
__device__ __forceinline__ void ts_border(const TersoffP& T, double z, double va, double& b, double& bva,
                                          double& dbdz) {
  if (z > 1.0e-15) {
    const double zn = pow(z, T.n);
    const double x = pow(T.beta, T.n) * zn;
    const double aux = 1.0 / (1.0 + x);
    b = T.chi * pow(aux, 0.5 / T.n);
    dbdz = -0.5 * b * aux * x / z;
  } else {
    b = T.chi;
    dbdz = 0.0;
  }
  bva = b * va;
}
__device__ __forceinline__ void ts_border(const TersoffP& T, float z, double va, double& b, double& bva,
                                          float& dbdz) {
  if (z > 1.0e-15f) {
    // x = (beta zeta)^n from the MUFU log2 / exp2: b's relative change per
    // relative change of x is (1/2n) x/(1+x) (0.04 in silicon), so their
    // ~2^-22 errors stay below 1e-8 in b; y needs log1p / expm1
    const float x = ex2f((float)T.n * __log2f((float)T.beta * z));
    const float y = -expm1f((float)(-0.5 / T.n) * log1pf(x));
    const double cva = T.chi * va;
    b = T.chi - T.chi * (double)y;
    bva = cva - cva * (double)y;
    dbdz = -0.5f * (float)b * x / ((1.0f + x) * z);
  } else {
    b = T.chi;
    bva = T.chi * va;
    dbdz = 0.0f;
  }
}

// MINB > 1 asks for MINB blocks per SM (fewer registers, more warps to hide
// the gathers).  TPA threads per atom (4 or 2; BLOCK / TPA atoms per block):
// each thread carries the atom's bonds q, q + TPA, ... two at a time, so with
// TPA = 2 a crystal's four bonds give every thread two independent chains.
// The autotuner picks MINB and TPA.
template <typename R, int TPA>
__host__ __device__ constexpr size_t tsf_smem() {
  return (size_t)8 * (BLOCK / TPA) * TS_MAXB * sizeof(R);  // eight per-bond arrays
}

template <typename R, int MINB, int TPA>
__global__ void __launch_bounds__(BLOCK, MINB) k_tsf_bonds(Arena A, BlockMap M) {
  constexpr int APB = BLOCK / TPA;
  constexpr int NB = APB * TS_MAXB;
  constexpr bool MIXED = sizeof(R) == 4;
  constexpr int PER = TS_MAXB / TPA;  // bonds per thread at most
  constexpr int CH = TPA == 2 ? 2 : 1;  // bonds a thread carries at once
  extern __shared__ __align__(16) unsigned char tsf_sh[];
  R* sux = reinterpret_cast<R*>(tsf_sh);
  R* suy = sux + NB;
  R* suz = suy + NB;
  R* sr = suz + NB;
  R* sfc = sr + NB;
  R* sdfc = sfc + NB;
  R* spre = sdfc + NB;
  R* sdv = spre + NB;  // the radial pair derivative dV of each bond (its owner's)
  const int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  const TersoffP& T = S.ts;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, q = threadIdx.x & (TPA - 1), la = threadIdx.x / TPA;
  const int i = M.first[blockIdx.x] + la;
  const bool act = i < M.end[blockIdx.x];
  const int base = la * TS_MAXB;
  const double r1 = T.R - T.D, r2 = T.R + T.D;
  const int nl = act ? live_entries(A, S, A.st[s], i, min(A.nn[i], A.lcap)) : 0;

  // ---- bonds in flist order: the atom's TPA threads test TPA slots at a
  // time and a ballot ranks the bonds they found
  double4 xi = make_double4(0, 0, 0, 0);
  int4 qi = make_int4(0, 0, 0, 0);
  if (act) {
    if constexpr (MIXED) qi = A.fxp[i];
    else xi = A.pos[i];
  }
  int cnt = 0, err = 0;
  unsigned long long mask = 0ull;
  const int tmax = __reduce_max_sync(FULL, (nl + TPA - 1) / TPA);
  constexpr int TB = MIXED ? 4 : 2;  // slot rounds whose loads are issued together
  using P = typename std::conditional<MIXED, int4, double4>::type;
  for (int t0 = 0; t0 < tmax; t0 += TB) {
    int jj[TB], rs[TB];
    P xj[TB];
#pragma unroll
    for (int u = 0; u < TB; u++) {
      const int m = (t0 + u) * TPA + q;
      jj[u] = m < nl ? A.flist[(size_t)m * A.cap + i] : -1;
      rs[u] = m < nl ? A.rslot[(size_t)m * A.cap + i] : 255;
    }
#pragma unroll
    for (int u = 0; u < TB; u++) {
      if ((unsigned)jj[u] < (unsigned)A.cap) {
        if constexpr (MIXED) xj[u] = A.fxp[jj[u]];
        else xj[u] = A.pos[jj[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < TB; u++) {
      if (t0 + u < tmax) {  // uniform across the warp
        const int m = (t0 + u) * TPA + q;
        bool bond = false;
        R u0 = R(0), u1 = R(0), u2 = R(0), rr = R(0);
        if ((unsigned)jj[u] < (unsigned)A.cap) {
          if constexpr (MIXED) {
            float v0, v1, v2, ir;
            vd_fx(S, qi, xj[u], v0, v1, v2);
            rr = sqrt_nr(v0 * v0 + v1 * v1 + v2 * v2, ir);
            u0 = v0 * ir; u1 = v1 * ir; u2 = v2 * ir;
            bond = rr <= (float)r2;
          } else {
            double v0, v1, v2;
            vd_fp64(S, xi, xj[u], v0, v1, v2);
            rr = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
            u0 = v0 / rr; u1 = v1 / rr; u2 = v2 / rr;
            bond = !(rr > r2);
          }
        }
        const unsigned grp = (__ballot_sync(FULL, bond) >> (lane & ~(TPA - 1))) & ((1u << TPA) - 1u);
        if (bond) {
          const int idx = cnt + __popc(grp & ((1u << q) - 1u));
          if (idx < TS_MAXB && m < 64 && rs[u] < 64) {
            const int k = base + idx;
            sux[k] = u0; suy[k] = u1; suz[k] = u2; sr[k] = rr;
            R dfc;
            sfc[k] = ts_fc<R>(rr, R(r1), R(r2), dfc);
            sdfc[k] = dfc;
            mask |= 1ull << m;
            A.tidx[(size_t)rs[u] * A.cap + jj[u]] = (unsigned char)idx;  // where j finds this record
          } else {
            err = 1;
          }
        }
        cnt += __popc(grp);
      }
    }
  }
#pragma unroll
  for (int o = 1; o < TPA; o <<= 1) mask |= __shfl_xor_sync(FULL, mask, o);
  const int nb = min(cnt, TS_MAXB);
  __syncthreads();

  // ---- per bond: zeta, bond order, the pair part (FP64) and dE_i/dzeta.
  // Two of the thread's bonds at a time, each partner bond b read once for both.
  const R h = R(T.h), c2 = R(T.c * T.c), d2 = R(T.d * T.d), c2d2 = R(T.c * T.c / (T.d * T.d));
  const double Aa = T.A * EV_UI, Bb = T.B * EV_UI;
  double ei = 0.0;
#pragma unroll
  for (int c = 0; c < PER; c += CH) {
    const int a0 = q + c * TPA, a1 = q + (c + 1) * TPA;
    const bool h0 = a0 < nb, h1 = CH == 2 && c + 1 < PER && a1 < nb;
    if (!h0) continue;
    const int k1 = h1 ? a1 : a0;
    R ax[CH], ay[CH], az[CH], z[CH];
#pragma unroll
    for (int e = 0; e < CH; e++) {
      const int a = e ? k1 : a0;
      ax[e] = sux[base + a]; ay[e] = suy[base + a]; az[e] = suz[base + a];
      z[e] = R(0);
    }
    for (int b = 0; b < nb; b++) {
      const R bx = sux[base + b], by = suy[base + b], bz = suz[base + b], fcb = sfc[base + b];
#pragma unroll
      for (int e = 0; e < CH; e++) {
        if (b == (e ? a1 : a0) || (e == 1 && !h1)) continue;
        const R ct = ax[e] * bx + ay[e] * by + az[e] * bz;
        const R hc = h - ct, hq = hc * hc;
        z[e] += fcb * (R(1) + c2d2 * hq / (d2 + hq));  // 1 + c2/d2 - c2/(d2+hc2), no cancellation
      }
    }
#pragma unroll
    for (int e = 0; e < CH; e++) {
      if (e == 1 && !h1) break;
      const int a = e ? a1 : a0;
      const double rd = (double)sr[base + a];
      double dfc;
      const double fc = ts_fc<double>(rd, r1, r2, dfc);
      const double vr = Aa * exp(-T.l1 * rd), va = -Bb * exp(-T.l2 * rd);
      double bo, bva;
      R dbdz;
      ts_border(T, z[e], va, bo, bva, dbdz);
      ei += 0.5 * fc * (vr + bva);
      // in mixed precision dV travels in FP32 like the record it ends in
      sdv[base + a] = R(0.5 * (dfc * (vr + bva) + fc * (-T.l1 * vr - T.l2 * bva)));
      spre[base + a] = R(0.5 * fc * va) * dbdz;  // dE_i / dzeta_a
    }
  }
  __syncthreads();

  // ---- per bond a: F_j(i) = -dV_a u_a - sum_{b != a} [(pre_a fc_b + pre_b fc_a) g'(cos_ab)
  //      (u_b - cos_ab u_a)/r_a + pre_b dfc_a g(cos_ab) u_a]; the triplet (a, b) enters
  //      zeta_a through k = j_b and zeta_b through k = j_a with the same angle
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
#pragma unroll
  for (int c = 0; c < PER; c += CH) {
    const int a0 = q + c * TPA, a1 = q + (c + 1) * TPA;
    const bool h0 = a0 < nb, h1 = CH == 2 && c + 1 < PER && a1 < nb;
    if (!h0) continue;
    const int k1 = h1 ? a1 : a0;
    R ax[CH], ay[CH], az[CH], fca[CH], dfca[CH], pa[CH], ira[CH], tx[CH], ty[CH], tz[CH];
#pragma unroll
    for (int e = 0; e < CH; e++) {
      const int a = e ? k1 : a0;
      ax[e] = sux[base + a]; ay[e] = suy[base + a]; az[e] = suz[base + a];
      fca[e] = sfc[base + a]; dfca[e] = sdfc[base + a]; pa[e] = spre[base + a];
      ira[e] = R(1) / sr[base + a];
      tx[e] = ty[e] = tz[e] = R(0);
    }
    for (int b = 0; b < nb; b++) {
      const R bx = sux[base + b], by = suy[base + b], bz = suz[base + b];
      const R fcb = sfc[base + b], pb = spre[base + b];
#pragma unroll
      for (int e = 0; e < CH; e++) {
        if (b == (e ? a1 : a0) || (e == 1 && !h1)) continue;
        const R ct = ax[e] * bx + ay[e] * by + az[e] * bz;
        const R hc = h - ct, iden = R(1) / (d2 + hc * hc);
        const R g = R(1) + c2d2 * (hc * hc) * iden;
        const R dg = R(-2) * c2 * hc * iden * iden;  // dg / dcos
        const R coef = (pa[e] * fcb + pb * fca[e]) * dg * ira[e];
        const R kc = pb * dfca[e] * g;
        tx[e] += coef * (bx - ct * ax[e]) + kc * ax[e];
        ty[e] += coef * (by - ct * ay[e]) + kc * ay[e];
        tz[e] += coef * (bz - ct * az[e]) + kc * az[e];
      }
    }
#pragma unroll
    for (int e = 0; e < CH; e++) {
      if (e == 1 && !h1) break;
      const int a = e ? a1 : a0;
      const double dv = (double)sdv[base + a];
      const double4 fj = make_double4(-(dv * (double)ax[e] + (double)tx[e]), -(dv * (double)ay[e] + (double)ty[e]),
                                      -(dv * (double)az[e] + (double)tz[e]), 0.0);
      if constexpr (MIXED) {
        // the record travels in FP32 (7 digits of one bond's force); the
        // partner adds it to its FP64 sum, and the centre subtracts the
        // same rounded value, so the forces still sum to zero
        const float4 f4 = make_float4((float)fj.x, (float)fj.y, (float)fj.z, 0.0f);
        A.tsfb32[(size_t)a * A.cap + i] = f4;
        f0 -= (double)f4.x;
        f1 -= (double)f4.y;
        f2 -= (double)f4.z;
      } else {
        A.tsfb[(size_t)a * A.cap + i] = fj;
        f0 -= fj.x;
        f1 -= fj.y;
        f2 -= fj.z;
      }
    }
  }
  // the atom's threads combine by a fixed xor tree (same bits in each)
#pragma unroll
  for (int o = 1; o < TPA; o <<= 1) {
    f0 += __shfl_xor_sync(FULL, f0, o);
    f1 += __shfl_xor_sync(FULL, f1, o);
    f2 += __shfl_xor_sync(FULL, f2, o);
    ei += __shfl_xor_sync(FULL, ei, o);
  }
  if (act && q == 0) {
    A.force[i] = make_double4(f0, f1, f2, 0.0);
    A.epot[i] = ei;
    A.tsmask[i] = mask;
  }
  if (act && err) atomicOr(&A.st[s].status, ST_BONDS);
}

// F_l += the bond records of l's partners for their bonds to l (slot order)
template <typename R>
__global__ void __launch_bounds__(BLOCK / 2) k_tsf_gather(Arena A, BlockMap M) {
  const int s = blk_sys(M);
  if (s < 0) return;
  const int i = M.first[blockIdx.x] + threadIdx.x;
  if (i >= M.end[blockIdx.x]) return;
  unsigned long long mk = A.tsmask[i];
  double4 f = A.force[i];
  bool bad = false;
  while (mk) {
    const int m = __ffsll((long long)mk) - 1;
    mk &= mk - 1ull;
    const size_t e = (size_t)m * A.cap + i;
    const int j = A.flist[e];
    const int a = A.tidx[e];
    if ((unsigned)j >= (unsigned)A.cap || a >= TS_MAXB) {
      bad = true;
      continue;
    }
    if constexpr (sizeof(R) == 4) {
      const float4 b = A.tsfb32[(size_t)a * A.cap + j];
      f.x += (double)b.x;
      f.y += (double)b.y;
      f.z += (double)b.z;
    } else {
      const double4 b = A.tsfb[(size_t)a * A.cap + j];
      f.x += b.x;
      f.y += b.y;
      f.z += b.z;
    }
  }
  A.force[i] = f;
  if (bad) atomicOr(&A.st[s].status, ST_BONDS);
}

// reverse slots of the Tersoff systems flagged for a rebuild: for each list
// entry (i, m) with partner j, the slot of i in j's flist (255: none)
__global__ void k_tsf_rslot(Arena A, BlockMap M) {
  rebuild_items(M.nblk, [&](int b) {
      const int s = M.sys[b];
      return s >= 0 && A.st[s].rebuild && A.sys[s].ff == FF_TERSOFF;
    }, [&](int b) {
      const int i = M.first[b] + threadIdx.x;
      if (i >= M.end[b]) return;
      const int n = min(A.nn[i], A.lcap);
      for (int m = 0; m < n; m++) {
        const size_t e = (size_t)m * A.cap + i;
        const int j = A.flist[e];
        int r = 255;
        if ((unsigned)j < (unsigned)A.cap) {
          const int nj = min(min(A.nn[j], A.lcap), 255);
          // the first slot of j's list that holds i, four loads in flight at a time
          for (int k0 = 0; k0 < nj && r == 255; k0 += 4) {
            int v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) v[u] = k0 + u < nj ? A.flist[(size_t)(k0 + u) * A.cap + j] : -1;
#pragma unroll
            for (int u = 3; u >= 0; u--)
              if (v[u] == i) r = k0 + u;
          }
        }
        A.rslot[e] = (unsigned char)r;
      }
    });
}

// interleaved [x1,y1,z1,...] staging <-> double4 arena slots
__global__ void k_unpack3(const double* __restrict__ src, double4* __restrict__ dst, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = make_double4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0);
}
__global__ void k_pack3(const double4* __restrict__ src, double* __restrict__ dst, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double4 v = src[i];
    dst[3 * i] = v.x;
    dst[3 * i + 1] = v.y;
    dst[3 * i + 2] = v.z;
  }
}

// velocity rescale of whole systems (replica exchange): v *= f[k]
__global__ void k_scale_vel(Arena A, BlockMap M, const double* fac_by_sys) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  int i = M.first[blockIdx.x] + threadIdx.x;
  if (i >= M.end[blockIdx.x]) return;
  double f = fac_by_sys[s];
  double4 v = A.vel[i];
  v.x *= f; v.y *= f; v.z *= f;
  A.vel[i] = v;
}

__global__ void k_zero_force(Arena A, BlockMap M) {
  int i = M.first[blockIdx.x] + threadIdx.x;
  if (i < M.end[blockIdx.x]) A.force[i] = make_double4(0, 0, 0, 0);
}

// ------------------------------------------------------------------ integrators
// ---- per-atom integrator updates, shared by the split and fused kernels
// velocity_verlet_b (src/Integration.F90:1171-1186)
__device__ __forceinline__ void vv_b_atom(double dt, double om, const double4& F, double4& v, double4& a) {
  const double adv = dt * 0.5;
  a.x = F.x * om; a.y = F.y * om; a.z = F.z * om;
  v.x = v.x + adv * a.x;
  v.y = v.y + adv * a.y;
  v.z = v.z + adv * a.z;
}

// ermak_b (src/Integration.F90:1013-1031)
__device__ __forceinline__ void ermak_b_atom(const SysDev& S, double om, const double4& F, const double4& vv,
                                             double4& v, double4& a) {
  const double c12 = S.cc1 - S.cc2;
  v.x = S.cc0 * v.x + c12 * a.x + S.cc2 * F.x * om + vv.x;
  v.y = S.cc0 * v.y + c12 * a.y + S.cc2 * F.y * om + vv.y;
  v.z = S.cc0 * v.z + c12 * a.z + S.cc2 * F.z * om + vv.z;
  a.x = F.x * om; a.y = F.y * om; a.z = F.z * om;
}

// velocity_verlet_a (src/Integration.F90:1150-1168)
__device__ __forceinline__ void vv_a_atom(double dt, double om, const double4& F, double4& x, double4& v,
                                          double4& a) {
  const double adv = dt * 0.5, adx = adv * dt;
  a.x = F.x * om; a.y = F.y * om; a.z = F.z * om;
  x.x = x.x + dt * v.x + adx * a.x;
  x.y = x.y + dt * v.y + adx * a.y;
  x.z = x.z + dt * v.z + adx * a.z;
  v.x = v.x + adv * a.x;
  v.y = v.y + adv * a.y;
  v.z = v.z + adv * a.z;
}

// nordsieck_predictor (src/Integration.F90:1192-1228): the fifth-order Gear
// predictor on the scaled derivatives (v dt, a = dt^2/2 F/m after a
// correction, a2..a4 the higher ones), summed left to right as written
__device__ __forceinline__ double nord_pred(double dt, double& x, double& v, double& a, double& a2, double& a3,
                                            double a4) {
  v = v * dt;
  const double p1 = a, p2 = a2, p4 = a3, p7 = a4;
  const double p3 = 3.0 * p2, p5 = 2.0 * p4, p6 = 2.0 * p5, p8 = 5.0 * p7, p9 = 2.0 * p8;
  x = p7 + p4 + p2 + p1 + v + x;
  v = p8 + p6 + p3 + p1 + p1 + v;
  a = p9 + p6 + p5 + p3 + p1;
  a2 = p9 + p6 + p2;
  a3 = p8 + p4;
  return x;
}

__device__ __forceinline__ void nord_a_atom(Arena& A, double dt, int i, double4& x, double4& v, double4& a) {
  double4 a2 = A.acel2[i], a3 = A.acel3[i];
  const double4 a4 = A.acel4[i];
  nord_pred(dt, x.x, v.x, a.x, a2.x, a3.x, a4.x);
  nord_pred(dt, x.y, v.y, a.y, a2.y, a3.y, a4.y);
  nord_pred(dt, x.z, v.z, a.z, a2.z, a3.z, a4.z);
  A.acel2[i] = a2;
  A.acel3[i] = a3;
}

// nordsieck_corrector (src/Integration.F90:1230-1268), Allen & Tildesley's
// coefficients for second-order equations: p = dt^2/2 F/m - a corrects
// every derivative, then v returns to normal units
__device__ __forceinline__ void nord_corr(double dt, double hm, double F, double& x, double& v, double& a,
                                          double& a2, double& a3, double& a4) {
  const double p = hm * F - a;
  x = x + p * (3.0 / 20.0);
  v = v + p * (251.0 / 360.0);
  a = a + p;
  a2 = a2 + p * (11.0 / 18.0);
  a3 = a3 + p * (1.0 / 6.0);
  a4 = a4 + p * (1.0 / 60.0);
  v = v / dt;
}

__device__ __forceinline__ void nord_b_atom(Arena& A, double dt, double om, int i, const double4& F, double4& x,
                                            double4& v, double4& a) {
  double4 a2 = A.acel2[i], a3 = A.acel3[i], a4 = A.acel4[i];
  const double hm = dt * dt / 2.0 * om;
  nord_corr(dt, hm, F.x, x.x, v.x, a.x, a2.x, a3.x, a4.x);
  nord_corr(dt, hm, F.y, x.y, v.y, a.y, a2.y, a3.y, a4.y);
  nord_corr(dt, hm, F.z, x.z, v.z, a.z, a2.z, a3.z, a4.z);
  A.acel2[i] = a2;
  A.acel3[i] = a3;
  A.acel4[i] = a4;
}

// ermak_a (src/Integration.F90:963-1011): position update and the velocity
// kick vel_v that ermak_b adds
__device__ __forceinline__ void ermak_a_atom(const Arena& A, const SysDev& S, const SysState& st, int i,
                                             double2 mi, const double4& v, const double4& a, double4& x,
                                             double4& vv) {
  double r[6];
  if (S.use_ext_normals) {
#pragma unroll
    for (int k = 0; k < 6; k++) r[k] = A.ext_normals[(size_t)6 * i + k];
  } else {
    normals6((uint32_t)(i - S.off), st.step, S.seed, r);
  }
  const double f_lan = S.skt * mi.y;
  const double pr = f_lan * S.sdr, pv = f_lan * S.sdv;
  vv.x = pv * (S.crv1 * r[0] + S.crv2 * r[1]);
  vv.y = pv * (S.crv1 * r[2] + S.crv2 * r[3]);
  vv.z = pv * (S.crv1 * r[4] + S.crv2 * r[5]);
  vv.w = 0.0;
  const double c2dt = S.cc2 * S.dt;
  x.x = x.x + S.cc1 * v.x + c2dt * a.x + pr * r[0];
  x.y = x.y + S.cc1 * v.y + c2dt * a.y + pr * r[2];
  x.z = x.z + S.cc1 * v.z + c2dt * a.z + pr * r[4];
}

// do_pbc_1 (src/Set_Properties.f90:444-470): a single wrap into [0, box)
__device__ __forceinline__ void wrap_atom(const SysDev& S, double4& x) {
  if (S.boxed) {
    if (S.pbc[0]) { if (x.x >= S.L[0]) x.x = x.x - S.L[0]; else if (x.x < 0.0) x.x = x.x + S.L[0]; }
    if (S.pbc[1]) { if (x.y >= S.L[1]) x.y = x.y - S.L[1]; else if (x.y < 0.0) x.y = x.y + S.L[1]; }
    if (S.pbc[2]) { if (x.z >= S.L[2]) x.z = x.z - S.L[2]; else if (x.z < 0.0) x.z = x.z + S.L[2]; }
  }
}

// lgf_stepa (src/Integration.F90:527-598) per atom, after k_lgf_sys moved
// the box: the noise displacement pos_v = fac0 / m r, acel = F / m, and
// x = (L / L_old) x + 2 L / (L_old + L) b dt (v + dt/2 acel + pos_v / 2)
// with b = 1 / (1 + dt/2 gamma / m)
__device__ __forceinline__ void lgf_a_atom(const Arena& A, const SysDev& S, const SysState& st, int i, double om,
                                           const double4& F, const double4& v, double4& a, double4& x,
                                           double4& pv) {
  double r0, r1, r2;
  if (S.use_ext_normals) {
    r0 = A.ext_normals[(size_t)6 * i];
    r1 = A.ext_normals[(size_t)6 * i + 2];
    r2 = A.ext_normals[(size_t)6 * i + 4];
  } else {
    double q[6];
    normals6((uint32_t)(i - S.off), st.step, S.seed, q);
    r0 = q[0], r1 = q[2], r2 = q[4];
  }
  const double b0 = 1.0 / (1.0 + S.lgf_facg0 * om);
  const double c = om * S.lgf_fac0;
  pv = make_double4(c * r0, c * r1, c * r2, 0.0);
  a.x = F.x * om; a.y = F.y * om; a.z = F.z * om;
  const double hdt = 0.5 * S.dt;
  x.x = st.lgf_sc[0] * x.x + st.lgf_f2[0] * b0 * S.dt * (v.x + hdt * a.x + 0.5 * pv.x);
  x.y = st.lgf_sc[1] * x.y + st.lgf_f2[1] * b0 * S.dt * (v.y + hdt * a.y + 0.5 * pv.y);
  x.z = st.lgf_sc[2] * x.z + st.lgf_f2[2] * b0 * S.dt * (v.z + hdt * a.z + 0.5 * pv.z);
}

// lgf_stepb (src/Integration.F90:600-650) per atom:
// v = a v + dt/2 (a acel + F / m) + b pos_v, a = (1 - dt/2 gamma / m) b
__device__ __forceinline__ void lgf_b_atom(const SysDev& S, double om, const double4& F, const double4& pv,
                                           double4& v, double4& a) {
  const double b0 = 1.0 / (1.0 + S.lgf_facg0 * om);
  const double a0 = (1.0 - S.lgf_facg0 * om) * b0;
  const double hdt = 0.5 * S.dt;
  v.x = a0 * v.x + hdt * (a0 * a.x + om * F.x) + b0 * pv.x;
  v.y = a0 * v.y + hdt * (a0 * a.y + om * F.y) + b0 * pv.y;
  v.z = a0 * v.z + hdt * (a0 * a.z + om * F.z) + b0 * pv.z;
  a.x = F.x * om; a.y = F.y * om; a.z = F.z * om;
}

// component D of a double4 (a compile-time index keeps it in registers)
template <int D>
__device__ __forceinline__ double& cmp(double4& v) {
  if constexpr (D == 0) return v.x;
  else if constexpr (D == 1) return v.y;
  else return v.z;
}
template <int D>
__device__ __forceinline__ double cmp(const double4& v) {
  if constexpr (D == 0) return v.x;
  else if constexpr (D == 1) return v.y;
  else return v.z;
}

// Half step a of coordinate D under its own integrator (IT_AXES):
// lgf_flex_stepa (src/Integration.F90:698-776) -- the same update as the
// isotropic piston on this coordinate alone -- or ermak_a_x (:1033-1082);
// r1, r2: this atom's normal pair for the coordinate.  pv receives the
// piston's noise displacement or Ermak's velocity kick.
template <int D>
__device__ __forceinline__ void axis_a(const SysDev& S, const SysState& st, double om, double osm, double r1,
                                       double r2, const double4& F, const double4& v, double4& a, double4& x,
                                       double4& pv) {
  const double* p = S.ax_p[D];
  if (S.ax_mode[D] == AX_FLEX) {
    const double b0 = 1.0 / (1.0 + p[1] * om);
    cmp<D>(pv) = om * p[0] * r1;
    cmp<D>(a) = cmp<D>(F) * om;
    cmp<D>(x) = st.lgf_sc[D] * cmp<D>(x) +
                st.lgf_f2[D] * b0 * S.dt * (cmp<D>(v) + 0.5 * S.dt * cmp<D>(a) + 0.5 * cmp<D>(pv));
  } else if (S.ax_mode[D] == AX_ERMAK) {
    const double f_lan = p[7] * osm;
    const double pr = f_lan * p[3] * r1;
    cmp<D>(pv) = f_lan * p[4] * (p[5] * r1 + p[6] * r2);
    cmp<D>(x) = cmp<D>(x) + p[1] * cmp<D>(v) + p[2] * S.dt * cmp<D>(a) + pr;
  }
}

// Half step b of coordinate D: lgf_flex_stepb (:778-830) or ermak_b_x
// (:1084-1105); a coordinate without an integrator keeps its velocity
template <int D>
__device__ __forceinline__ void axis_b(const SysDev& S, double om, const double4& F, const double4& pv, double4& v,
                                       double4& a) {
  const double* p = S.ax_p[D];
  if (S.ax_mode[D] == AX_FLEX) {
    const double b0 = 1.0 / (1.0 + p[1] * om);
    const double a0 = (1.0 - p[1] * om) * b0;
    cmp<D>(v) = a0 * cmp<D>(v) + 0.5 * S.dt * (a0 * cmp<D>(a) + om * cmp<D>(F)) + b0 * cmp<D>(pv);
    cmp<D>(a) = cmp<D>(F) * om;
  } else if (S.ax_mode[D] == AX_ERMAK) {
    cmp<D>(v) = p[0] * cmp<D>(v) + (p[1] - p[2]) * cmp<D>(a) + p[2] * cmp<D>(F) * om + cmp<D>(pv);
    cmp<D>(a) = cmp<D>(F) * om;
  }
}

__device__ __forceinline__ void axes_a_atom(const Arena& A, const SysDev& S, const SysState& st, int i,
                                            double2 mi, const double4& F, const double4& v, double4& a,
                                            double4& x, double4& pv) {
  double r[6];
  if (S.use_ext_normals) {
#pragma unroll
    for (int k = 0; k < 6; k++) r[k] = A.ext_normals[(size_t)6 * i + k];
  } else {
    normals6((uint32_t)(i - S.off), st.step, S.seed, r);
  }
  pv = make_double4(0, 0, 0, 0);
  axis_a<0>(S, st, mi.x, mi.y, r[0], r[1], F, v, a, x, pv);
  axis_a<1>(S, st, mi.x, mi.y, r[2], r[3], F, v, a, x, pv);
  axis_a<2>(S, st, mi.x, mi.y, r[4], r[5], F, v, a, x, pv);
}

// re-plan a moving box's cell grid for its new lengths (intergroup_setcells,
// cells no smaller than the list cut-off) within the cells allocated, with
// fewer, larger cells where the allocation is short; below three cells a
// dimension's stencil would visit a cell twice
// the fixed-point frame of the mixed kernels follows the box: periodic
// dimensions map [0, L) onto the 32-bit ring for the current L (the same
// arithmetic as the host's set-up), and the step kernel that moves every atom
// into the new box rewrites the fixed-point copies in it
__device__ __forceinline__ void fx_frame(SysDev& S) {
  for (int d = 0; d < 3; d++)
    if (S.fx_per[d]) {
      S.fx_scale[d] = 4294967296.0 / S.L[d];
      const double u = S.L[d] / 4294967296.0;
      S.fx_inv[d] = (float)u;
      S.fx_inv_lo[d] = (float)(u - (double)S.fx_inv[d]);
    }
}

__device__ __forceinline__ void regrid(SysDev& S, SysState& st) {
  fx_frame(S);
  if (!S.use_cells) return;
  int nc[3];
  for (int d = 0; d < 3; d++) nc[d] = (int)(S.L[d] / S.rlist);
  while ((int64_t)nc[0] * nc[1] * nc[2] > S.cell_cap) {
    int m = nc[1] > nc[0] ? 1 : 0;
    if (nc[2] > nc[m]) m = 2;
    nc[m]--;
  }
  if (nc[0] < 3 || nc[1] < 3 || nc[2] < 3) {
    atomicOr(&st.status, ST_BOX);
    return;
  }
  for (int d = 0; d < 3; d++) {
    S.nc[d] = nc[d];
    S.cell[d] = S.L[d] / nc[d];
    S.inv_cell[d] = 1.0 / S.cell[d];
  }
  S.ncell = nc[0] * nc[1] * nc[2];
}

// Per-coordinate pistons (IT_AXES), one thread per system: each closes its
// previous step (lgf_flex_stepb: pistonf from the virial's diagonal entry,
// pvel with the factor V / L) and moves its length (lgf_flex_stepa)
//   L' = L + b dt (pvel + (dt pistonf V / L + rangv) / (2 Q)),
// every piston with the volume of the step's start, as the reference
// updates the volume only once all of them have moved.
__device__ __forceinline__ void axes_sys(SysDev& S, SysState& st) {
  const double dt = S.dt;
  const double vol0 = S.L[0] * S.L[1] * S.L[2];
  double q[6];
  if (!S.use_ext_normals) normals6((uint32_t)S.n, st.step, S.seed, q);
  double Ln[3];
  for (int d = 0; d < 3; d++) {
    Ln[d] = S.L[d];
    if (S.ax_mode[d] != AX_FLEX) continue;
    const double* p = S.ax_p[d];
    const double pf = (st.vir[d] + p[2]) / vol0 - p[3];
    if (st.ax_phase[d] == 0) {
      st.ax_phase[d] = 1;
    } else {
      st.ax_pvel[d] = p[7] * st.ax_pvel[d] + 0.5 * p[4] * dt * (p[7] * st.ax_pf[d] + pf) * vol0 / S.L[d] +
                      p[5] * p[4] * st.ax_rangv[d];
    }
    st.ax_pf[d] = pf;
    const double rangv = (S.use_ext_normals ? st.ax_ext[d] : q[d]) * p[6];
    st.ax_rangv[d] = rangv;
    Ln[d] = S.L[d] + p[5] * dt * (st.ax_pvel[d] + 0.5 * p[4] * (dt * pf * vol0 / S.L[d] + rangv));
  }
  for (int d = 0; d < 3; d++) {
    if (!(Ln[d] > 0.0)) {
      atomicOr(&st.status, ST_BOX);
      Ln[d] = S.L[d];
    }
    const double Lo = S.L[d];
    st.lgf_sc[d] = Ln[d] / Lo;
    st.lgf_f2[d] = 2.0 * Ln[d] / (Lo + Ln[d]);
    S.L[d] = Ln[d];
    S.invL[d] = 1.0 / Ln[d];
  }
  regrid(S, st);
}

// ------------------------------------------------------------------ LKD
// Block sums of three per-atom values; true in thread 0 of the system's
// last block, which then holds the system's totals (added in block order).
__device__ __forceinline__ bool sys3_close(Arena& A, const BlockMap& M, int s, const double w[3], double t[3]) {
  double b[3];
#pragma unroll
  for (int k = 0; k < 3; k++) b[k] = block_sum(w[k]);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) A.blk_red[8 * (M.base + blockIdx.x) + k] = b[k];
  bool last = last_block(M, A.st, s, &A.st[s].ticket2);
  if (!last || threadIdx.x >= 32) return false;
  const int b0 = M.sys_blk0[s], nb = M.sys_nblk[s];
  for (int k = 0; k < 3; k++) t[k] = 0.0;
  for (int q = threadIdx.x; q < nb; q += 32)
#pragma unroll
    for (int k = 0; k < 3; k++) t[k] += __ldcg(&A.blk_red[8 * (b0 + q) + k]);
#pragma unroll
  for (int k = 0; k < 3; k++)
    for (int o = 16; o; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
  return threadIdx.x == 0;
}

// the LKD velocity half kick (lkd_stepa :385-398 / lkd_stepb :470-481):
// acel = F/m, v += dt/2 acel - dt/2 gamma0/m v + fac0/m r
__device__ __forceinline__ void lkd_kick(const SysDev& S, double om, const double4& F, const double r[3], double4& v,
                                         double4& a) {
  const double hdt = 0.5 * S.dt;
  const double c = om * S.lkd[0];
  a.x = F.x * om; a.y = F.y * om; a.z = F.z * om;
  v.x = v.x + hdt * a.x - hdt * S.lkd[3] * om * v.x + c * r[0];
  v.y = v.y + hdt * a.y - hdt * S.lkd[3] * om * v.y + c * r[1];
  v.z = v.z + hdt * a.z - hdt * S.lkd[3] * om * v.z + c * r[2];
}

// the LKD piston momentum step (lkd_stepa :400-411, lkd_stepb :458-468)
// from the diagonal kinetic sums K of the current velocities:
// P = mean_k (K_k + W_kk) / V, pvel += dt/2 (P - P0) - gammav dt/2 pvel/Q + facv r
__device__ __forceinline__ void lkd_piston(const SysDev& S, SysState& st, const double K[3], double r) {
  const double vol = S.L[0] * S.L[1] * S.L[2];
  const double press = ((K[0] + st.vir[0]) / vol + (K[1] + st.vir[1]) / vol + (K[2] + st.vir[2]) / vol) / 3;
  const double dt = S.dt;
  st.lgf_pvel = st.lgf_pvel + 0.5 * dt * (press - S.lkd[2]) - S.lkd[4] * 0.5 * dt * st.lgf_pvel / S.lkd[5] +
                S.lkd[1] * r;
}

// lkd_stepa, first part (Integration.F90:357-423): the velocity half kick
// of every atom, then, in the system's last block, the piston momentum from
// the pressure of the kicked velocities and the box's two half advances
//   L_h = L (1 + dt/2 pvel / (Q V))^(1/3),  L' = L_h (1 + dt/2 pvel / (Q V_h))^(1/3)
// (single-precision exponent 1./dd), which k_step_a applies to the atoms.
__global__ void __launch_bounds__(BLOCK) k_lkd_a(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  SysDev& S = A.sys[s];
  SysState& st = A.st[s];
  if (S.integ != IT_LKD) return;  // uniform per block
  const int i = M.first[blockIdx.x] + threadIdx.x;
  double w[3] = {0, 0, 0};
  if (i < M.end[blockIdx.x]) {
    double r[3];
    if (S.use_ext_normals) {
      for (int k = 0; k < 3; k++) r[k] = A.ext_normals[(size_t)6 * i + 2 * k];
    } else {
      double q[6];
      normals6((uint32_t)(i - S.off), st.step, S.seed, q);
      r[0] = q[0], r[1] = q[2], r[2] = q[4];
    }
    double4 v = A.vel[i], a;
    lkd_kick(S, A.minv[i].x, A.force[i], r, v, a);
    A.vel[i] = v;
    A.acel[i] = a;
    const double m = A.mass[i];
    w[0] = v.x * v.x * m;
    w[1] = v.y * v.y * m;
    w[2] = v.z * v.z * m;
  }
  double K[3];
  if (!sys3_close(A, M, s, w, K)) return;
  double rp;
  if (S.use_ext_normals) {
    rp = st.ax_ext[0];
  } else {
    double q[6];
    normals6((uint32_t)S.n, st.step, S.seed, q);
    rp = q[0];
  }
  lkd_piston(S, st, K, rp);
  const double expo = (double)(1.0f / 3.0f);
  const double dt = S.dt;
  double vol = S.L[0] * S.L[1] * S.L[2];
  for (int d = 0; d < 3; d++) {
    st.lkd_bo[d] = S.L[d];
    st.lkd_bh[d] = S.L[d] * pow(1.0 + 0.5 * dt * st.lgf_pvel / S.lkd[5] / vol, expo);
  }
  vol = st.lkd_bh[0] * st.lkd_bh[1] * st.lkd_bh[2];
  const double g = 1.0 + 0.5 * dt * st.lgf_pvel / S.lkd[5] / vol;
  if (!(vol > 0.0) || !(g > 0.0)) {
    atomicOr(&st.status, ST_BOX);
    for (int d = 0; d < 3; d++) st.lkd_bh[d] = st.lkd_bf[d] = st.lkd_bo[d];
    return;
  }
  for (int d = 0; d < 3; d++) {
    st.lkd_bf[d] = st.lkd_bh[d] * pow(g, expo);
    S.L[d] = st.lkd_bf[d];
    S.invL[d] = 1.0 / st.lkd_bf[d];
  }
  regrid(S, st);
}

// The G-JF piston of each constant-pressure system (one thread per system),
// ahead of the atoms' half step.  It first closes the previous step's
// piston (lgf_stepb: pistonf from the virial of the last force evaluation
// and pvel), which needs the whole system's virial and so waits for this
// launch, then moves the box (lgf_stepa): the volume
//   V = V0 + b dt (pvel + (dt pistonf + rangv) / (2 Q)),
// each length L (V / V0)^(1/3) with the single-precision exponent 1./dd of
// the reference, and the cell grid of the next rebuild re-planned for the
// new lengths within the cells allocated.  The first step takes pistonf
// from the virial of the initial interact and leaves pvel at 0.
__global__ void k_lgf_sys(Arena A, const int* sys, int nsys) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nsys) return;
  const int s = sys[k];
  if (s < 0) return;
  SysDev& S = A.sys[s];
  SysState& st = A.st[s];
  if (S.integ == IT_AXES) {
    axes_sys(S, st);
    return;
  }
  if (S.integ != IT_LGF) return;
  const double dt = S.dt;
  const double vol0 = S.L[0] * S.L[1] * S.L[2];
  const double sv = (st.vir[0] + st.vir[1] + st.vir[2]) / 3;
  const double pf = (sv + S.lgf_kin) / vol0 - S.lgf_press;
  if (st.lgf_phase == 0) {
    st.lgf_phase = 1;
  } else {
    st.lgf_pvel = S.lgf_av * st.lgf_pvel + 0.5 * S.lgf_ipm * dt * (S.lgf_av * st.lgf_pf + pf) +
                  S.lgf_bv * S.lgf_ipm * st.lgf_rangv;
  }
  st.lgf_pf = pf;
  double r;
  if (S.use_ext_normals) {
    r = st.ext_piston;
  } else {
    double q[6];
    normals6((uint32_t)S.n, st.step, S.seed, q);
    r = q[0];
  }
  const double rangv = r * S.lgf_facv;
  st.lgf_rangv = rangv;
  const double vol = vol0 + S.lgf_bv * dt * (st.lgf_pvel + 0.5 * S.lgf_ipm * (dt * pf + rangv));
  if (!(vol > 0.0)) {
    atomicOr(&st.status, ST_BOX);
    for (int d = 0; d < 3; d++) st.lgf_sc[d] = st.lgf_f2[d] = 1.0;
    return;
  }
  const double g = pow(vol / vol0, (double)(1.0f / 3.0f));
  for (int d = 0; d < 3; d++) {
    const double Lo = S.L[d], Ln = Lo * g;
    st.lgf_sc[d] = Ln / Lo;
    st.lgf_f2[d] = 2.0 * Ln / (Lo + Ln);
    S.L[d] = Ln;
    S.invL[d] = 1.0 / Ln;
  }
  regrid(S, st);
}

// the moved atom's outputs: position, fixed-point copy, skin displacement
// (xo = its position at the last rebuild, ty = its species)
__device__ __forceinline__ double moved_atom(Arena& A, const SysDev& S, SysState& st, int i, const double4& x,
                                             const double4& xo, int ty) {
  A.pos[i] = x;
  if (S.prec == PREC_MIXED || S.ff == FF_TERSOFF) {
    int bad = 0;
    write_fx(A, S, i, x, ty, bad);
    if (bad) atomicOr(&st.status, ST_LOST);
  }
  double d = disp2(S, x, xo);
  if (!(d == d)) atomicOr(&st.status, ST_NAN);
  return d;
}

// test_update (src/Neighbour.F90:1305-1346) over the system: block top-2 of
// the squared displacements, merged by the system's last block, which sets
// the rebuild flag (and raises the graph's rebuild condition) and closes
// the step's integrator bookkeeping.
// PISTON=false: a kernel that never sees a constant-pressure system
template <bool COND, bool PISTON = true>
__device__ __forceinline__ void skin_close(Arena& A, const BlockMap& M, int s, const SysDev& S, SysState& st,
                                           bool frozen, double2 t, cudaGraphConditionalHandle cond) {
  t = block_top2(t);
  if (threadIdx.x == 0) A.blk_top2[M.base + blockIdx.x] = t;
  if (last_block(M, A.st, s, &st.ticket)) {
    double2 w = sys_top2(A, M, s);
    if (threadIdx.x == 0) {
      // a moving box (constant pressure) shifts periodic images by up to
      // the change of its lengths since the build, on top of the atoms'
      // own displacements
      double box = 0.0;
      if (PISTON && (S.integ == IT_LGF || S.integ == IT_AXES || S.integ == IT_LKD))
        box = fabs(S.L[0] - st.box_b[0]) + fabs(S.L[1] - st.box_b[1]) + fabs(S.L[2] - st.box_b[2]);
      const double D = __dadd_rn(__dadd_rn(__dsqrt_rn(w.x), __dsqrt_rn(w.y)), box);
      int rb = D > S.skin;
      st.dmax = D;
      if (frozen) rb = 0;
      st.rebuild = rb;
      if (rb) {
        atomicOr(A.any_rebuild, 1);
        if constexpr (COND) cudaGraphSetConditional(cond, 1u);
      }
      if (((S.integ == IT_ERMAK || S.integ == IT_LGF || S.integ == IT_AXES || S.integ == IT_LKD ||
            S.integ == IT_BROWN) &&
           !S.use_ext_normals) ||
          S.thermo == TH_ANDERSEN)
        st.step++;
      if (S.integ == IT_FIRE) st.fire_zero = 0;
    }
  }
}

// integration_stepa (src/Integration.F90:243-262): the algorithm's half
// step, do_pbc (Set_Properties.f90:444-470), then the displacement test of
// test_update fused in (the list decision for this step's interact).
// When the step is replayed from a CUDA graph, `cond` is the handle of the
// conditional node that guards the rebuild kernels: any system that needs a
// rebuild raises it, so steps without a rebuild skip those launches.
// COND=false builds a copy without the device-side graph call, for plain
// launches (profilers do not replay kernels that contain it).
template <bool COND>
__global__ void __launch_bounds__(BLOCK) k_step_a(Arena A, BlockMap M, cudaGraphConditionalHandle cond) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  SysState& st = A.st[s];
  int i = M.first[blockIdx.x] + threadIdx.x;
  bool act = i < M.end[blockIdx.x];
  bool frozen = S.integ == IT_FIRE && st.fire_done;
  double2 t = make_double2(1.e-16, 1.e-16);
  if (act && S.integ != IT_NONE && !frozen) {
    double4 x = A.pos[i], v = A.vel[i], a = A.acel[i];
    const double2 mi = A.minv[i];
    if (S.integ == IT_VV || S.integ == IT_FIRE) {
      const double dt = S.integ == IT_FIRE ? st.fire_dt : S.dt;
      if (S.integ == IT_FIRE && st.fire_zero) v = make_double4(0, 0, 0, 0);
      vv_a_atom(dt, mi.x, A.force[i], x, v, a);
      A.acel[i] = a;
      A.vel[i] = v;
    } else if (S.integ == IT_ERMAK) {
      double4 vv;
      ermak_a_atom(A, S, st, i, mi, v, a, x, vv);
      A.vel_v[i] = vv;
    } else if (S.integ == IT_LGF) {
      double4 pv;
      lgf_a_atom(A, S, st, i, mi.x, A.force[i], v, a, x, pv);
      A.acel[i] = a;
      A.vel_v[i] = pv;
    } else if (S.integ == IT_AXES) {
      double4 pv;
      axes_a_atom(A, S, st, i, mi, A.force[i], v, a, x, pv);
      A.acel[i] = a;
      A.vel_v[i] = pv;
    } else if (S.integ == IT_LKD) {
      // lkd_stepa (:423-436): drift with the half-advanced box, then scale
      // positions and velocities to the final box (v was kicked by k_lkd_a)
      x.x = x.x + v.x * S.dt * st.lkd_bo[0] * st.lkd_bo[0] / (st.lkd_bh[0] * st.lkd_bh[0]);
      x.y = x.y + v.y * S.dt * st.lkd_bo[1] * st.lkd_bo[1] / (st.lkd_bh[1] * st.lkd_bh[1]);
      x.z = x.z + v.z * S.dt * st.lkd_bo[2] * st.lkd_bo[2] / (st.lkd_bh[2] * st.lkd_bh[2]);
      x.x = x.x * st.lkd_bf[0] / st.lkd_bo[0];
      x.y = x.y * st.lkd_bf[1] / st.lkd_bo[1];
      x.z = x.z * st.lkd_bf[2] / st.lkd_bo[2];
      v.x = v.x * st.lkd_bo[0] / st.lkd_bf[0];
      v.y = v.y * st.lkd_bo[1] / st.lkd_bf[1];
      v.z = v.z * st.lkd_bo[2] / st.lkd_bf[2];
      A.vel[i] = v;
    } else if (S.integ == IT_NORD) {
      // between the predictor and the corrector v holds v dt
      nord_a_atom(A, S.dt, i, x, v, a);
      A.acel[i] = a;
      A.vel[i] = v;
    }
    wrap_atom(S, x);
    t.x = moved_atom(A, S, st, i, x, A.pos_old[i], A.type[i]);
  }
  skin_close<COND>(A, M, s, S, st, frozen, t, cond);
}

// Atom i's step_b of one step and step_a of the next (velocity Verlet or
// Ermak; other integrators leave the atom alone) given its force F, in
// registers: the operations of k_step_b and k_step_a in their order.
// ba_store writes the result.
struct BaAtom {
  double4 x, v, a, vv;
  double d;  // squared displacement since the list build (1e-16: not moved)
  int ty;
  bool on;   // velocity Verlet or Ermak
};

__device__ __forceinline__ void ba_calc(const Arena& A, const SysDev& S, const SysState& st, int i, const double4& F,
                                        BaAtom& b) {
  const int integ = S.integ;
  b.on = integ == IT_VV || integ == IT_ERMAK;
  b.d = 1.e-16;
  if (!b.on) return;
  // every input is loaded before the first use, so all loads are in flight together
  b.x = A.pos[i];
  b.v = A.vel[i];
  b.a = A.acel[i];
  const double2 mi = A.minv[i];
  const double4 xo = A.pos_old[i];
  b.ty = A.type[i];
  const double4 vv0 = integ == IT_ERMAK ? A.vel_v[i] : make_double4(0, 0, 0, 0);
  if (integ == IT_VV) {
    vv_b_atom(S.dt, mi.x, F, b.v, b.a);
    vv_a_atom(S.dt, mi.x, F, b.x, b.v, b.a);
  } else {
    ermak_b_atom(S, mi.x, F, vv0, b.v, b.a);
    ermak_a_atom(A, S, st, i, mi, b.v, b.a, b.x, b.vv);
  }
  wrap_atom(S, b.x);
  b.d = disp2(S, b.x, xo);
}

__device__ __forceinline__ void ba_store(Arena& A, const SysDev& S, SysState& st, int i, const BaAtom& b) {
  if (!b.on) return;
  if (S.integ == IT_ERMAK) A.vel_v[i] = b.vv;
  A.acel[i] = b.a;
  A.vel[i] = b.v;
  A.pos[i] = b.x;
  if (S.prec == PREC_MIXED || S.ff == FF_TERSOFF) {
    int bad = 0;
    write_fx(A, S, i, b.x, b.ty, bad);
    if (bad) atomicOr(&st.status, ST_LOST);
  }
  if (!(b.d == b.d)) atomicOr(&st.status, ST_NAN);
}

// step_b of one step fused with step_a of the next, for velocity Verlet and
// Ermak systems (FIRE needs its system-wide P between the two and keeps the
// split kernels).  Per atom it is exactly k_step_b followed by k_step_a:
// the same operations in the same order, with each array read and written
// once instead of twice.
// APT atoms per thread (blocks of APT * BLOCK atoms, one after another):
// a large system's blocks then pay the skin test's block merge and ticket
// once per APT * BLOCK atoms.
template <bool COND, int APT>
__global__ void __launch_bounds__(BLOCK, 4) k_step_ba(Arena A, BlockMap M, cudaGraphConditionalHandle cond) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  SysState& st = A.st[s];
  double2 t = make_double2(1.e-16, 1.e-16);
#pragma unroll 1
  for (int k = 0; k < APT; k++) {
    const int i = M.first[blockIdx.x] + threadIdx.x + k * BLOCK;
    if (i < M.end[blockIdx.x]) {
      BaAtom b;
      b.on = false;
      ba_calc(A, S, st, i, A.force[i], b);
      t = top2_merge(t, make_double2(b.d, 1.e-16));
      ba_store(A, S, st, i, b);
    }
  }
  skin_close<COND, false>(A, M, s, S, st, false, t, cond);
}

// The force pass fused with the integrator: each atom's force, then its
// step_b and the next step's step_a (ba_calc), then the skin test of the
// system.  The force pass reads the neighbours' positions from the density
// pass's gather records (fxe, pose), never from pos / fxp, so moving an atom
// while others still gather is safe; the next density pass starts after
// this launch.  Velocity Verlet and Ermak systems; the sums and the step are
// those of the separate kernels, bit for bit.
template <int K, bool ONE, int MINB, bool COND>
__global__ void __launch_bounds__(BLOCK, MINB) k_smatb_force_mixed_ba(Arena A, BlockMap M,
                                                                       cudaGraphConditionalHandle cond) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  SysState& st = A.st[s];
  __shared__ SmF32 tab_sh[ONE ? 1 : MAXT * MAXT];
  const SmF32* tab = smf_table<ONE>(A, S, tab_sh);
  const int i = M.first[blockIdx.x] + threadIdx.x / K;
  const int lane = threadIdx.x % K;
  const bool act = i < M.end[blockIdx.x];
  double4 F;
  force_mixed_body<K, ONE, false, false>(A, M, s, S, tab, i, lane, act, F);
  double2 t = make_double2(1.e-16, 1.e-16);
  BaAtom b;
  b.on = false;
  if (act && lane == 0) {
    A.force[i] = make_double4(F.x, F.y, F.z, 0.0);
    A.epot[i] = F.w;
    ba_calc(A, S, st, i, make_double4(F.x, F.y, F.z, 0.0), b);
    t.x = b.d;
    ba_store(A, S, st, i, b);
  }
  skin_close<COND, false>(A, M, s, S, st, false, t, cond);
}

template <int K, bool COND>
__global__ void __launch_bounds__(BLOCK) k_smatb_force_fp64_ba(Arena A, BlockMap M, cudaGraphConditionalHandle cond) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  SysState& st = A.st[s];
  __shared__ SmFP64 tab_sh[MAXT * MAXT];
  const SmFP64* tab = sm_table(A, S, tab_sh);
  const int i = M.first[blockIdx.x] + threadIdx.x / K;
  const int lane = threadIdx.x % K;
  const bool act = i < M.end[blockIdx.x];
  double4 F;
  force_fp64_body<K, false, false>(A, M, s, S, tab, i, lane, act, F);
  double2 t = make_double2(1.e-16, 1.e-16);
  BaAtom b;
  b.on = false;
  if (act && lane == 0) {
    A.force[i] = make_double4(F.x, F.y, F.z, 0.0);
    A.epot[i] = F.w;
    ba_calc(A, S, st, i, make_double4(F.x, F.y, F.z, 0.0), b);
    t.x = b.d;
    ba_store(A, S, st, i, b);
  }
  skin_close<COND, false>(A, M, s, S, st, false, t, cond);
}

// integration_stepb (src/Integration.F90:264-301): velocity_verlet_b
// (:1171-1186), ermak_b (:1013-1031), the pistons' second halves or the
// Nordsieck corrector (:1230-1268) or cbrownian (:855-882); FIRE adds P = sum v.F, the per-atom
// mixing v = (1-a) v + a |v| F/|F| (FIRE.f90:99-114, with |v|) and the
// dt / alpha control (:116-131) in the system's last block.
// MOVES: the launch includes systems whose step b moves the atoms (the
// predictor-corrector, whose corrector also holds three more derivative
// vectors, and Brownian dynamics); the other integrators' copy stays leaner
template <bool MOVES>
__global__ void __launch_bounds__(BLOCK) k_step_b(Arena A, BlockMap M) {
  int s = blk_sys(M);
  if (s < 0) return;  // padding block of a fixed-capacity map
  const SysDev& S = A.sys[s];
  SysState& st = A.st[s];
  int i = M.first[blockIdx.x] + threadIdx.x;
  bool act = i < M.end[blockIdx.x];
  bool frozen = S.integ == IT_FIRE && st.fire_done;
  double P = 0.0, f2max = 0.0;
  double lkd_w[3] = {0, 0, 0};
  if (act && S.integ != IT_NONE && !frozen) {
    double4 v = A.vel[i], a = A.acel[i];
    const double4 F = A.force[i];
    const double om = A.minv[i].x;
    if (S.integ == IT_VV || S.integ == IT_FIRE) {
      vv_b_atom(S.integ == IT_FIRE ? st.fire_dt : S.dt, om, F, v, a);
      if (S.integ == IT_FIRE) {
        P = v.x * F.x + v.y * F.y + v.z * F.z;
        double fn2 = F.x * F.x + F.y * F.y + F.z * F.z;
        f2max = fn2;
        double vn = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
        double fn = sqrt(fn2);
        double al = st.fire_alpha;
        double mixf = fn > 0.0 ? al * vn / fn : 0.0;
        v.x = v.x * (1.0 - al) + mixf * F.x;
        v.y = v.y * (1.0 - al) + mixf * F.y;
        v.z = v.z * (1.0 - al) + mixf * F.z;
      }
    } else if (S.integ == IT_ERMAK) {
      ermak_b_atom(S, om, F, A.vel_v[i], v, a);
    } else if (S.integ == IT_LGF) {
      lgf_b_atom(S, om, F, A.vel_v[i], v, a);
    } else if (S.integ == IT_AXES) {
      const double4 pv = A.vel_v[i];
      axis_b<0>(S, om, F, pv, v, a);
      axis_b<1>(S, om, F, pv, v, a);
      axis_b<2>(S, om, F, pv, v, a);
    } else if (S.integ == IT_LKD) {
      // lkd_stepb (:438-484): the pressure of the velocities as they come
      // in (summed below), then the second half kick
      const double m = A.mass[i];
      lkd_w[0] = v.x * v.x * m;
      lkd_w[1] = v.y * v.y * m;
      lkd_w[2] = v.z * v.z * m;
      double r[3];
      if (S.use_ext_normals) {
        for (int k = 0; k < 3; k++) r[k] = A.ext_normals[(size_t)6 * i + 2 * k + 1];
      } else {
        double q[6];
        normals6((uint32_t)(i - S.off), st.step, S.seed, q);
        r[0] = q[1], r[1] = q[3], r[2] = q[5];
      }
      lkd_kick(S, om, F, r, v, a);
    } else if (MOVES && (S.integ == IT_NORD || S.integ == IT_BROWN)) {
      // the step moves the atom: do_pbc after integration_stepb
      // (src/Integration.F90:275-280); the next step's skin test sees it
      double4 x = A.pos[i];
      if (S.integ == IT_NORD) {
        nord_b_atom(A, S.dt, om, i, F, x, v, a);
      } else {
        // cbrownian (:855-882): one normal per coordinate, the first of a
        // rang pair (the parity stream's layout; Philox: the same slots)
        double r[3];
        if (S.use_ext_normals) {
          for (int k = 0; k < 3; k++) r[k] = A.ext_normals[(size_t)6 * i + 2 * k];
        } else {
          double q[6];
          normals6((uint32_t)(i - S.off), st.step, S.seed, q);
          r[0] = q[0], r[1] = q[2], r[2] = q[4];
        }
        const double osm = A.minv[i].y;
        const double4 xo = x;
        x.x = xo.x + om * S.bd_fac1 * F.x + osm * r[0] * S.bd_fac2;
        x.y = xo.y + om * S.bd_fac1 * F.y + osm * r[1] * S.bd_fac2;
        x.z = xo.z + om * S.bd_fac1 * F.z + osm * r[2] * S.bd_fac2;
        v.x = (x.x - xo.x) / S.dt;
        v.y = (x.y - xo.y) / S.dt;
        v.z = (x.z - xo.z) / S.dt;
      }
      wrap_atom(S, x);
      moved_atom(A, S, st, i, x, A.pos_old[i], A.type[i]);
    }
    A.vel[i] = v;
    A.acel[i] = a;
  }
  if (S.integ == IT_LKD) {  // uniform per block
    double K[3];
    if (sys3_close(A, M, s, lkd_w, K)) {
      double rp;
      if (S.use_ext_normals) {
        rp = st.ax_ext[1];
      } else {
        double q[6];
        normals6((uint32_t)S.n, st.step, S.seed, q);
        rp = q[1];
      }
      lkd_piston(S, st, K, rp);
    }
    return;
  }
  if (S.integ != IT_FIRE) return;  // uniform per block
  double Pb = block_sum(P);
  double Fb = block_max(f2max);
  if (threadIdx.x == 0) A.blk_red[2 * (M.base + blockIdx.x)] = Pb, A.blk_red[2 * (M.base + blockIdx.x) + 1] = Fb;
  if (last_block(M, A.st, s, &st.ticket2) && threadIdx.x < 32) {
    const int b0 = M.sys_blk0[s], nb = M.sys_nblk[s];
    double Pt = 0.0, Ft = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) {
      Pt += __ldcg(&A.blk_red[2 * (b0 + b)]);
      Ft = fmax(Ft, __ldcg(&A.blk_red[2 * (b0 + b) + 1]));
    }
    for (int o = 16; o; o >>= 1) {
      Pt += __shfl_xor_sync(0xffffffffu, Pt, o);
      Ft = fmax(Ft, __shfl_xor_sync(0xffffffffu, Ft, o));
    }
    if (threadIdx.x == 0 && !frozen) {
      st.fire_P = Pt;
      st.fmax2 = Ft;
      st.fire_iter++;
      const double alpha0 = 0.1, finc = 1.1, fdec = 0.5, falf = 0.99;
      if (Pt > 0.0) {
        st.fire_np++;
        if (st.fire_np > 5) {
          st.fire_dt = fmin(st.fire_dt * finc, S.fire_dtmax);
          st.fire_alpha = st.fire_alpha * falf;
        }
      } else {
        st.fire_np = 0;
        st.fire_dt = st.fire_dt * fdec;
        st.fire_alpha = alpha0;
        st.fire_zero = 1;  // velocities are zeroed by the next step_a
      }
      double fm = sqrt(Ft) * c_ui_ev();
      if (fm < S.fire_fmax || st.fire_iter >= S.fire_maxit) st.fire_done = 1;
    }
  }
}

// ------------------------------------------------------------------ reductions
// Per-system inquiry sums (inq_kin_energy / inq_temperature,
// src/Inq_Properties.F90:399-437) over the system's blocks of an atom map;
// each block's partials go to blk_red and the system's last block adds them
// in block order, so the sums are the same bits on every run.
//  PASS 0: Epot, the total mass and momentum (-> the centre-of-mass velocity),
//          max |F|^2 and the status: out[4s+0], out[4s+2], out[4s+3], and
//          v_cm in out[4 scap + 3s ..];
//  PASS 1: Ekin = 1/2 sum m |v - v_cm|^2 (the reference's sum, which keeps
//          its digits when the centre of mass drifts): out[4s+1].
template <int PASS>
__global__ void k_sys_reduce(Arena A, BlockMap M, int scap, double* out) {
  const int s = blk_sys(M);
  if (s < 0) return;
  const SysDev& S = A.sys[s];
  const int i = M.first[blockIdx.x] + threadIdx.x;
  const bool act = i < M.end[blockIdx.x];
  constexpr int NW = PASS == 0 ? 6 : 1;
  double w[NW];
#pragma unroll
  for (int k = 0; k < NW; k++) w[k] = 0.0;
  if (act) {
    const double4 v = A.vel[i];
    const double m = A.mass[i];
    if constexpr (PASS == 0) {
      const double4 F = A.force[i];
      w[0] = A.epot[i];
      w[1] = m;
      w[2] = m * v.x;
      w[3] = m * v.y;
      w[4] = m * v.z;
      w[5] = F.x * F.x + F.y * F.y + F.z * F.z;
    } else {
      const double* c = out + 4 * (size_t)scap + 3 * (size_t)s;
      const double a = v.x - c[0], b = v.y - c[1], d = v.z - c[2];
      w[0] = (a * a + b * b + d * d) * m;
    }
  }
  double bsum[NW];
#pragma unroll
  for (int k = 0; k < NW; k++) bsum[k] = (PASS == 0 && k == 5) ? block_max(w[k]) : block_sum(w[k]);
  if (threadIdx.x == 0)
    for (int k = 0; k < NW; k++) A.blk_red[8 * (M.base + blockIdx.x) + k] = bsum[k];
  if (last_block(M, A.st, s, &A.st[s].ticket2) && threadIdx.x < 32) {
    const int b0 = M.sys_blk0[s], nb = M.sys_nblk[s];
    double t[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) t[k] = 0.0;
    for (int q = threadIdx.x; q < nb; q += 32)
#pragma unroll
      for (int k = 0; k < NW; k++) {
        const double x = __ldcg(&A.blk_red[8 * (b0 + q) + k]);
        t[k] = (PASS == 0 && k == 5) ? fmax(t[k], x) : t[k] + x;
      }
#pragma unroll
    for (int k = 0; k < NW; k++)
      for (int o = 16; o; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, t[k], o);
        t[k] = (PASS == 0 && k == 5) ? fmax(t[k], x) : t[k] + x;
      }
    if (threadIdx.x == 0) {
      if constexpr (PASS == 0) {
        out[4 * (size_t)s + 0] = t[0];
        out[4 * (size_t)s + 2] = t[5];
        out[4 * (size_t)s + 3] = (double)A.st[s].status;
        double* c = out + 4 * (size_t)scap + 3 * (size_t)s;
        if (S.n == 1) {
          const double4 v = A.vel[S.off];
          c[0] = v.x; c[1] = v.y; c[2] = v.z;
        } else {
          c[0] = t[2] / t[1]; c[1] = t[3] / t[1]; c[2] = t[4] / t[1];
        }
      } else {
        out[4 * (size_t)s + 1] = 0.5 * t[0];
      }
    }
  }
}

}  // namespace gg
