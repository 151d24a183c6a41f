// gemsgpu.cu -- host runtime and C ABI of the B200 force/neighbour path.
//
// A context owns one CUDA stream and one HBM arena holding every system's
// atoms (structure of arrays).  Host records mirror the reference's
// intergroup / integrate objects; the device keeps all per-step state, so a
// molecular-dynamics step needs no host round trip (the rebuild decision of
// test_update is taken on the device).  gemsgpu_md_steps captures a chunk of
// steps in a CUDA graph and replays it.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gemsgpu.h"
#include "common.cuh"
#include "kernels.cuh"
#include "lbfgs.cuh"
#include "neb.cuh"

using namespace gg;

namespace {

constexpr double kB_ev = 8.617385e-05;  // src/Constants.F90:173
const double UI_EV = c_ui_ev();
const double EV_UI_H = 1.0 / c_ui_ev();
const double kB_ui = kB_ev * EV_UI_H;

struct DevMap {
  BlockMap m{};
  int* buf = nullptr;  // device storage of the map arrays
  int nblk = 0;
  std::vector<int> blk0, nblkv;  // host copies of sys_blk0 / sys_nblk
};

struct SysHost {
  bool alive = false;
  int off = 0, n = 0, ntypes = 1;
  int cell_off = 0, cell_cap = 0;
  int param_off = 0;
  bool first = true;        // next interact builds the list (update)
  bool pos_dirty = false;   // positions replaced from the host since the skin test
  bool has_forces = false;
  int lanes = 8;            // lanes per atom in the force kernels (autotuned)
  int variant = 1;          // 1: species table in shared memory, 0: constants in
                            //    registers (single-species mixed SMA-TB; autotuned)
  std::vector<PairP> prm;   // ntypes x ntypes
  std::vector<char> deaf;   // ntypes x ntypes: [a][b] = 1 once set_feels(b, a) left
                            //   type a deaf to type b (the pair acts on b only)
  SysDev d{};
  bool ff_set = false;
  double temp = 0.0;        // Ermak bath temperature (K)
  bool box_live = false;    // the device moved the box (constant pressure)
  std::vector<int> ax_order;  // IT_AXES: coordinates in the order their integrators were added
};

// a system whose box the device moves (a G-JF piston on the volume or on
// a length)
bool moving_box(const SysDev& d) {
  if (d.integ == IT_LGF || d.integ == IT_LKD) return true;
  if (d.integ != IT_AXES) return false;
  return d.ax_mode[0] == AX_FLEX || d.ax_mode[1] == AX_FLEX || d.ax_mode[2] == AX_FLEX;
}

// a pair of types that acts on one side only (`interact g1 feels g2`): its
// forces are not a pair virial
// write a pair's parameters both ways, except a direction set_feels
// turned off: that stays off whatever pair setter is called later
void put_pair(SysHost& h, int ti, int tj, const PairP& P) {
  if (h.deaf.size() != h.prm.size()) h.deaf.assign(h.prm.size(), 0);
  const int a = ti * h.ntypes + tj, b = tj * h.ntypes + ti;
  if (!h.deaf[a]) h.prm[a] = P;
  if (!h.deaf[b]) h.prm[b] = P;
}

bool one_sided(const SysHost& h) {
  auto on = [&](int a, int b) {
    const PairP& P = h.prm[a * h.ntypes + b];
    return P.v[0] != 0.0 || P.v[1] != 0.0;
  };
  if (h.d.ff != FF_LJ) return false;
  for (int a = 0; a < h.ntypes; a++)
    for (int b = 0; b < h.ntypes; b++)
      if (on(a, b) != on(b, a)) return true;
  return false;
}

struct Graph {
  cudaGraphExec_t exec = nullptr;
  uint64_t epoch = 0;
  int64_t nodes = 0;       // unconditional kernel nodes per replay
  int64_t body_nodes = 0;  // kernels of one conditional rebuild body
};

}  // namespace

struct gemsgpu_ctx {
  int device = 0;
  int nsm = 148;             // multiprocessors of the device
  cudaStream_t stream = nullptr;
  std::string err;
  // arena
  Arena A{};
  int64_t acap = 0;   // atoms
  int64_t ccap = 0;   // cells
  int scap = 0;       // systems
  int pcap = 0;       // pair-parameter slots
  int nblk_cap = 0;   // per-block scratch entries
  int64_t atoms_used = 0, cells_used = 0;
  int params_used = 0;
  std::vector<SysHost> sys;
  std::vector<std::pair<int64_t, int64_t>> free_atoms, free_cells;
  uint64_t epoch = 1;  // bumps when device pointers or maps change
  int64_t launches = 0;  // kernels issued (graph replays add their node count)
  bool use_cond = true;  // conditional graph nodes guard the rebuild chain
  bool fuse_forces = true;  // force pass + half steps in one kernel (GEMSGPU_NO_FUSED_FORCES=1: off)
  int64_t body_nodes = 0;  // kernels in one captured rebuild chain
  unsigned long long body_seen = 0;  // body_runs already accounted
  int64_t pending = 0;   // kernels recorded by the capture in progress
  // while a batched graph is captured as one branch per system: the batch;
  // a one-system map then is that system's blocks of the batch's map
  std::vector<int> view_set;
  int64_t bodies = 0;    // conditional rebuild bodies in the graph being built
  std::map<std::string, DevMap> maps;
  std::map<std::string, Graph> graphs;
  // pinned scratch for small readbacks
  double* h_red = nullptr;
  int h_red_cap = 0;
  double* d_red = nullptr;
  int* d_sys = nullptr;
  int d_sys_cap = 0;
  SysState* h_st = nullptr;
  double* stage = nullptr;      // 3 doubles per atom, host <-> device staging
  int64_t stage_cap = 0;
  int64_t snap_cap = 0;
  double4* snap = nullptr;      // pos, vel, acel, force [, acel2, acel3, acel4]
  int snap_arrays = 0;
  SysState* snap_st = nullptr;
  SysDev* snap_sys = nullptr;   // boxes moved by constant-pressure steps
  bool tersoff = false;         // a Tersoff system exists: rslot, tsmask, tsfb are kept
  // the L-BFGS workspace, kept between calls (freeing device memory can stall
  // for a long time, so a minimisation does not allocate and free its own)
  gg::LbWork lbw{};
  int lbw_m = 0, lbw_scap = 0;
  double* d_fac = nullptr;      // per-system velocity factors of gemsgpu_retemper
  int d_fac_cap = 0;
};

// A pool: a fixed-capacity batch of systems sharing one force-field kind and
// launch shape.  Its block maps live in device buffers sized for the
// capacity and padded with empty blocks, so one captured graph serves any
// active set -- changing the set rewrites the maps, not the graph.
struct gemsgpu_pool {
  gemsgpu_ctx* ctx = nullptr;
  int max_systems = 0;
  int64_t max_atoms = 0, max_cells = 0;
  int ff = 0, prec = 0, lanes = 8, variant = 1, chunk = 50;
  std::vector<int> active;  // system ids
  // map kinds: 0 atoms/256, 1 cells/256, 2 atoms/LIST_ATOMS, 3 cells/8, 4 atoms/(256/K)
  int cap[5] = {0, 0, 0, 0, 0};
  int* dmap[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int* dsys = nullptr;      // padded system array
  int scap = 0;             // system-id capacity of the per-system map arrays
  gg::BlockMap maps[5];
  bool maps_dirty = true;
  cudaGraphExec_t exec = nullptr;
  gg::Arena captured{};     // arena the graph was captured against
  int64_t nodes = 0, body_nodes = 0;
  std::vector<int> host_buf;
};

// Serving loop: jobs (FIRE relaxations, short Langevin runs) arrive at any
// time, wait in a queue, are admitted into the pool while memory and slots
// allow, advance together chunk by chunk, and leave when done.
struct ServerJob {
  int64_t id = 0;
  gemsgpu_job spec{};
  std::vector<double> pos;   // input copy, then the final positions
  int state = 0;             // GEMSGPU_JOB_*
  int sys = -1;
  int done_steps = 0;
  double epot_ev = 0.0, ekin_ev = 0.0, fmax_ev = 0.0;
  int iters = 0;
  int error = 0;
};

struct gemsgpu_server {
  gemsgpu_ctx* ctx = nullptr;
  gemsgpu_pool* pool = nullptr;
  int max_jobs = 0;
  int64_t max_atoms = 0;
  int chunk = 50;
  int64_t next_id = 1;
  int64_t atoms_in = 0;
  std::deque<int64_t> queue;
  std::vector<int64_t> running;
  std::map<int64_t, ServerJob> jobs;
};

namespace {

int fail(gemsgpu_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CU(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? GEMSGPU_ERR_OOM          \
                                                       : GEMSGPU_ERR_CUDA,        \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,      \
                  __LINE__);                                                      \
  } while (0)

#define CHK(expr)          \
  do {                     \
    int r_ = (expr);       \
    if (r_ != 0) return r_; \
  } while (0)

template <typename T>
int dalloc(gemsgpu_ctx* ctx, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  CU(cudaMalloc((void**)p, n * sizeof(T)));
  return 0;
}

// grow one device array keeping its first `keep` elements
template <typename T>
int dgrow(gemsgpu_ctx* ctx, T** p, size_t keep, size_t n) {
  T* q = nullptr;
  CHK(dalloc(ctx, &q, n));
  if (*p && keep) CU(cudaMemcpyAsync(q, *p, keep * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
  if (*p) {
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaFree(*p));
  }
  *p = q;
  return 0;
}

void drop_graphs(gemsgpu_ctx* c) {
  for (auto& kv : c->graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  c->graphs.clear();
}

void drop_maps(gemsgpu_ctx* c) {
  for (auto& kv : c->maps)
    if (kv.second.buf) cudaFree(kv.second.buf);
  c->maps.clear();
}

void invalidate(gemsgpu_ctx* c) {
  c->epoch++;
  drop_graphs(c);
}

// ------------------------------------------------------------- arena
int tersoff_records(gemsgpu_ctx* ctx);

int grow_atoms(gemsgpu_ctx* ctx, int64_t need) {
  if (need <= ctx->acap) return 0;
  int64_t nc = std::max<int64_t>(need, ctx->acap + ctx->acap / 2);
  nc = (nc + 255) / 256 * 256;
  int64_t keep = ctx->acap;
  Arena& A = ctx->A;
  CHK(dgrow(ctx, &A.pos, keep, nc));
  CHK(dgrow(ctx, &A.pos_old, keep, nc));
  CHK(dgrow(ctx, &A.vel, keep, nc));
  CHK(dgrow(ctx, &A.acel, keep, nc));
  CHK(dgrow(ctx, &A.force, keep, nc));
  CHK(dgrow(ctx, &A.vel_v, keep, nc));
  if (A.acel2) {
    CHK(dgrow(ctx, &A.acel2, keep, nc));
    CHK(dgrow(ctx, &A.acel3, keep, nc));
    CHK(dgrow(ctx, &A.acel4, keep, nc));
  }
  CHK(dgrow(ctx, &A.epot, keep, nc));
  CHK(dgrow(ctx, &A.band, keep, nc));
  CHK(dgrow(ctx, &A.eband, keep, nc));
  CHK(dgrow(ctx, &A.ebandf, keep, nc));
  CHK(dgrow(ctx, &A.fxp, keep, nc));
  CHK(dgrow(ctx, &A.pose, keep, nc));
  CHK(dgrow(ctx, &A.fxe, keep, nc));
  CHK(dgrow(ctx, &A.minv, keep, nc));
  CHK(dgrow(ctx, &A.mass, keep, nc));
  CHK(dgrow(ctx, &A.type, keep, nc));
  CHK(dgrow(ctx, &A.nn, keep, nc));
  CHK(dgrow(ctx, &A.hnn, keep, nc));
  CHK(dgrow(ctx, &A.ncut, keep, nc));
  CHK(dgrow(ctx, &A.cell_of, keep, nc));
  CHK(dgrow(ctx, &A.slot, keep, nc));
  CHK(dgrow(ctx, &A.cell_atoms, keep, nc));
  CHK(dgrow(ctx, &A.cell_pos, keep, nc));
  CHK(dgrow(ctx, &A.ext_normals, 6 * keep, 6 * nc));
  // the lists' leading dimension is the atom capacity: re-lay them out
  if (A.lcap > 0) {
    int** lists[2] = {&A.list, &A.flist};
    for (int q = 0; q < 2; q++) {
      int* nl = nullptr;
      CHK(dalloc(ctx, &nl, (size_t)A.lcap * nc));
      CU(cudaMemsetAsync(nl, 0, (size_t)A.lcap * nc * sizeof(int), ctx->stream));
      if (*lists[q] && keep)
        CU(cudaMemcpy2DAsync(nl, nc * sizeof(int), *lists[q], keep * sizeof(int), keep * sizeof(int), A.lcap,
                             cudaMemcpyDeviceToDevice, ctx->stream));
      CU(cudaStreamSynchronize(ctx->stream));
      if (*lists[q]) CU(cudaFree(*lists[q]));
      *lists[q] = nl;
    }
    unsigned char** bytes[2] = {&A.rslot, &A.tidx};
    for (auto pp : bytes) {
      if (!*pp) continue;
      unsigned char* nr = nullptr;
      CHK(dalloc(ctx, &nr, (size_t)A.lcap * nc));
      CU(cudaMemsetAsync(nr, 0xff, (size_t)A.lcap * nc, ctx->stream));
      if (keep) CU(cudaMemcpy2DAsync(nr, nc, *pp, keep, keep, A.lcap, cudaMemcpyDeviceToDevice, ctx->stream));
      CU(cudaStreamSynchronize(ctx->stream));
      CU(cudaFree(*pp));
      *pp = nr;
    }
  }
  ctx->acap = nc;
  A.cap = nc;
  // the Tersoff bond records are rewritten by every force evaluation
  if (ctx->tersoff) CHK(tersoff_records(ctx));
  invalidate(ctx);
  return 0;
}

// Tersoff scratch: per-step bond masks and records (TS_MAXB rows of the
// atom capacity), and the reverse list slots (one byte per list entry)
int tersoff_records(gemsgpu_ctx* ctx) {
  Arena& A = ctx->A;
  const size_t n = (size_t)std::max<int64_t>(ctx->acap, 1);
  CU(cudaStreamSynchronize(ctx->stream));
  if (A.tsmask) CU(cudaFree(A.tsmask));
  if (A.tsfb) CU(cudaFree(A.tsfb));
  if (A.tsfb32) CU(cudaFree(A.tsfb32));
  A.tsmask = nullptr;
  A.tsfb = nullptr;
  A.tsfb32 = nullptr;
  CHK(dalloc(ctx, &A.tsmask, n));
  CU(cudaMemsetAsync(A.tsmask, 0, n * sizeof(unsigned long long), ctx->stream));
  CHK(dalloc(ctx, &A.tsfb, (size_t)TS_MAXB * n));
  CHK(dalloc(ctx, &A.tsfb32, (size_t)TS_MAXB * n));
  if (!A.rslot && A.lcap > 0) {
    CHK(dalloc(ctx, &A.rslot, (size_t)A.lcap * n));
    CU(cudaMemsetAsync(A.rslot, 0xff, (size_t)A.lcap * n, ctx->stream));
    CHK(dalloc(ctx, &A.tidx, (size_t)A.lcap * n));
    CU(cudaMemsetAsync(A.tidx, 0xff, (size_t)A.lcap * n, ctx->stream));
  }
  return 0;
}

// dynamic shared memory of the two cell-list kernels for list capacity lcap
int list_smem_attr(gemsgpu_ctx* ctx, int lcap) {
  const size_t smem = list_smem(lcap), smemw = listw_smem<128>(lcap), smemw4 = listw_smem<512>(lcap);
  if (smem > 200 * 1024 || smemw > 200 * 1024 || smemw4 > 200 * 1024)
    return fail(ctx, GEMSGPU_ERR_ARG, "neighbour capacity %d too large", lcap);
  if (smem > 48 * 1024)
    CU(cudaFuncSetAttribute(k_list_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (smemw > 48 * 1024) {
    CU(cudaFuncSetAttribute(k_list_cells_w<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemw));
    CU(cudaFuncSetAttribute(k_list_cells_w<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemw));
  }
  if (smemw4 > 48 * 1024) {
    CU(cudaFuncSetAttribute(k_list_cells_w<512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemw4));
    CU(cudaFuncSetAttribute(k_list_cells_w<512, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemw4));
  }
  return 0;
}


int grow_list(gemsgpu_ctx* ctx, int lcap) {
  Arena& A = ctx->A;
  if (lcap <= A.lcap && A.list) return 0;
  lcap = (lcap + 7) / 8 * 8;
  const size_t ld = (size_t)std::max<int64_t>(ctx->acap, 1);
  int** lists[2] = {&A.list, &A.flist};
  for (int q = 0; q < 2; q++) {
    int* nl = nullptr;
    CHK(dalloc(ctx, &nl, (size_t)lcap * ld));
    CU(cudaMemsetAsync(nl, 0, (size_t)lcap * ld * sizeof(int), ctx->stream));
    // keep every system's current list: rows 0..lcap_old-1 are contiguous
    if (*lists[q] && A.lcap > 0)
      CU(cudaMemcpyAsync(nl, *lists[q], (size_t)A.lcap * ld * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (*lists[q]) CU(cudaFree(*lists[q]));
    *lists[q] = nl;
  }
  if (ctx->tersoff) {
    unsigned char** bytes[2] = {&A.rslot, &A.tidx};
    for (auto pp : bytes) {
      unsigned char* nr = nullptr;
      CHK(dalloc(ctx, &nr, (size_t)lcap * ld));
      CU(cudaMemsetAsync(nr, 0xff, (size_t)lcap * ld, ctx->stream));
      if (*pp && A.lcap > 0)
        CU(cudaMemcpyAsync(nr, *pp, (size_t)A.lcap * ld, cudaMemcpyDeviceToDevice, ctx->stream));
      CU(cudaStreamSynchronize(ctx->stream));
      if (*pp) CU(cudaFree(*pp));
      *pp = nr;
    }
  }
  A.lcap = lcap;
  CHK(list_smem_attr(ctx, lcap));
  invalidate(ctx);
  return 0;
}

int grow_cells(gemsgpu_ctx* ctx, int64_t need) {
  if (need <= ctx->ccap) return 0;
  int64_t nc = std::max<int64_t>(need, ctx->ccap + ctx->ccap / 2);
  nc = (nc + 255) / 256 * 256;
  Arena& A = ctx->A;
  int64_t keep = ctx->ccap;
  CHK(dgrow(ctx, &A.cell_count, keep, nc));
  if (keep < nc) CU(cudaMemsetAsync(A.cell_count + keep, 0, (nc - keep) * sizeof(int), ctx->stream));
  CHK(dgrow(ctx, &A.cell_n, keep, nc));
  CHK(dgrow(ctx, &A.cell_loc, keep, nc));
  CHK(dgrow(ctx, &A.cell_start, keep, nc));
  CHK(dgrow(ctx, &A.chunk_sum, keep / 256, nc / 256));
  ctx->ccap = nc;
  invalidate(ctx);
  return 0;
}

int grow_systems(gemsgpu_ctx* ctx, int need) {
  if (need <= ctx->scap) return 0;
  int nc = std::max(need, std::max(16, ctx->scap * 2));
  Arena& A = ctx->A;
  CHK(dgrow(ctx, &A.sys, ctx->scap, nc));
  CHK(dgrow(ctx, &A.st, ctx->scap, nc));
  CU(cudaMemsetAsync(A.st + ctx->scap, 0, (nc - ctx->scap) * sizeof(SysState), ctx->stream));
  if (ctx->h_st) cudaFreeHost(ctx->h_st);
  CU(cudaMallocHost((void**)&ctx->h_st, nc * sizeof(SysState)));
  if (ctx->snap_st) cudaFree(ctx->snap_st);
  CHK(dalloc(ctx, &ctx->snap_st, nc));
  if (ctx->snap_sys) cudaFree(ctx->snap_sys);
  CHK(dalloc(ctx, &ctx->snap_sys, nc));
  ctx->scap = nc;
  invalidate(ctx);
  return 0;
}

int grow_params(gemsgpu_ctx* ctx, int need) {
  if (need <= ctx->pcap) return 0;
  int nc = std::max(need, std::max(64, ctx->pcap * 2));
  CHK(dgrow(ctx, &ctx->A.prm, ctx->pcap, nc));
  ctx->pcap = nc;
  invalidate(ctx);
  return 0;
}

int grow_blocks(gemsgpu_ctx* ctx, int nblk) {
  if (nblk <= ctx->nblk_cap) return 0;
  int nc = std::max(nblk, ctx->nblk_cap * 2);
  CHK(dgrow(ctx, &ctx->A.blk_top2, 0, nc));
  CHK(dgrow(ctx, &ctx->A.blk_red, 0, 8 * (size_t)nc));
  ctx->nblk_cap = nc;
  invalidate(ctx);
  return 0;
}

// first-fit range allocation with a bump pointer
int64_t take_range(std::vector<std::pair<int64_t, int64_t>>& fr, int64_t& used, int64_t n,
                   int64_t align) {
  for (size_t k = 0; k < fr.size(); k++) {
    int64_t b = (fr[k].first + align - 1) / align * align;
    if (b + n <= fr[k].second) {
      int64_t e = fr[k].second;
      int64_t a0 = fr[k].first;
      fr.erase(fr.begin() + k);
      if (a0 < b) fr.push_back({a0, b});
      if (b + n < e) fr.push_back({b + n, e});
      return b;
    }
  }
  int64_t b = (used + align - 1) / align * align;
  used = b + n;
  return b;
}

// ------------------------------------------------------------- derived config
void derive(gemsgpu_ctx* ctx, SysHost& h) {
  SysDev& d = h.d;
  d.off = h.off;
  d.n = h.n;
  d.ntypes = h.ntypes;
  d.param_off = h.param_off;
  // rcut: max cut-off over the species pairs (intergroup rcut)
  double rc = 0.0;
  if (d.ff == FF_LJ)
    for (auto& p : h.prm) rc = std::max(rc, p.v[2]);
  if (d.ff == FF_SMATB)
    for (auto& p : h.prm)
      if (p.v[13] != 0.0) rc = std::max(rc, p.v[6]);
  if (d.ff == FF_TERSOFF) rc = d.ts.R + d.ts.D;
  d.rcut = rc;
  double rl = rc + d.skin;
  d.rlist = rl;
  d.rlist2 = rl * rl;
  for (int k = 0; k < 8; k++) {
    const double t = rc + 1e-4 + k * (d.skin / 7.0);
    d.ncut_r2[k] = (float)(t * t);
  }
  // the force order puts a pair potential's inner regime first (SMA-TB
  // r <= rci, Tersoff r <= R - D), so a warp's lanes meet the same branch
  // at the same slot; it only orders entries, so any value <= ncut_r2[0] is right
  double rin = 0.0;
  if (d.ff == FF_SMATB)
    for (auto& p : h.prm)
      if (p.v[13] != 0.0) rin = std::max(rin, p.v[5]);
  if (d.ff == FF_TERSOFF) rin = d.ts.R - d.ts.D;
  d.nsplit_r2 = std::min((float)(rin * rin), d.ncut_r2[0]);
  // intergroup_setcells (src/Neighbour.F90:587-664)
  d.use_cells = 0;
  for (int k = 0; k < 3; k++) {
    d.nc[k] = 1;
    d.invL[k] = d.boxed ? 1.0 / d.L[k] : 0.0;
  }
  if (d.boxed && rl > 0.0) {
    bool any4 = false;
    int nc[3];
    for (int k = 0; k < 3; k++) {
      nc[k] = (int)(d.L[k] / rl);
      if (nc[k] >= 4) any4 = true;
    }
    if (any4) {
      d.use_cells = 1;
      for (int k = 0; k < 3; k++) {
        d.nc[k] = nc[k];
        d.cell[k] = d.L[k] / nc[k];
        d.inv_cell[k] = 1.0 / d.cell[k];
      }
    }
  }
  d.ncell = d.use_cells ? d.nc[0] * d.nc[1] * d.nc[2] : 0;
  // list kernel: one warp per cell with a 128-candidate tile for cells of
  // about three atoms or fewer, a 512-candidate tile up to sixteen, else one
  // CTA per cell
  const double per_cell = d.use_cells ? (double)h.n / d.ncell : 0.0;
  d.list_warp = !d.use_cells ? 0 : per_cell < 3.5 ? 1 : per_cell <= 16.0 ? 2 : 0;
  // the list build's FP32 frame: stencil images when every periodic dim
  // has three cells or more (a constant-pressure box never shrinks below)
  d.list_img = 1;
  for (int k = 0; k < 3; k++)
    if (d.use_cells && d.pbc[k] && d.nc[k] < 3) d.list_img = 0;
  // fixed-point frame of the mixed kernels
  for (int k = 0; k < 3; k++) {
    bool per = d.boxed && d.pbc[k];
    d.fx_per[k] = per ? 1 : 0;
    if (per) {
      d.fx_scale[k] = 4294967296.0 / d.L[k];
      double u = d.L[k] / 4294967296.0;
      d.fx_inv[k] = (float)u;
      d.fx_inv_lo[k] = (float)(u - (double)d.fx_inv[k]);
      d.fx_origin[k] = 0.0;
    } else {
      d.fx_scale[k] = 4194304.0;  // 2^22 per Angstrom
      d.fx_inv[k] = (float)(1.0 / 4194304.0);
      d.fx_inv_lo[k] = 0.0f;
      d.fx_origin[k] = d.boxed ? 0.5 * d.L[k] : d.fx_origin[k];
    }
  }
}

// cells a system's grid may use: its grid, or for a constant-pressure box
// the grid of a box 15% longer in every dimension, which it may re-plan
// into as the box moves
int cells_needed(const SysHost& h) {
  if (!h.d.use_cells) return 0;
  if (!moving_box(h.d)) return h.d.ncell;
  int64_t m = 1;
  for (int k = 0; k < 3; k++) m *= std::max(h.d.nc[k], (int)(1.15 * h.d.L[k] / h.d.rlist));
  return (int)std::min<int64_t>(m, 1 << 26);
}

int alloc_cells(gemsgpu_ctx* ctx, SysHost& h) {
  int need = cells_needed(h);
  if (need <= h.cell_cap) {
    h.d.cell_off = h.cell_off;
    h.d.cell_cap = h.cell_cap;
    return 0;
  }
  if (h.cell_cap > 0) ctx->free_cells.push_back({h.cell_off, h.cell_off + h.cell_cap});
  int64_t cap = (need + 255) / 256 * 256;
  int64_t off = take_range(ctx->free_cells, ctx->cells_used, cap, 256);
  CHK(grow_cells(ctx, off + cap));
  h.cell_off = (int)off;
  h.cell_cap = (int)cap;
  h.d.cell_off = h.cell_off;
  h.d.cell_cap = h.cell_cap;
  invalidate(ctx);
  return 0;
}

// the box lengths a constant-pressure system has on the device
int live_box(gemsgpu_ctx* ctx, int s, double L[3]) {
  SysDev d;
  CU(cudaMemcpyAsync(&d, ctx->A.sys + s, sizeof(SysDev), cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < 3; k++) L[k] = d.L[k];
  return 0;
}

int push_sys(gemsgpu_ctx* ctx, int s) {
  SysHost& h = ctx->sys[s];
  if (h.box_live) CHK(live_box(ctx, s, h.d.L));  // keep the box the pistons moved
  derive(ctx, h);
  CHK(alloc_cells(ctx, h));
  CU(cudaMemcpyAsync(ctx->A.sys + s, &h.d, sizeof(SysDev), cudaMemcpyHostToDevice, ctx->stream));
  if (!h.prm.empty())
    CU(cudaMemcpyAsync(ctx->A.prm + h.param_off, h.prm.data(), h.prm.size() * sizeof(PairP),
                       cudaMemcpyHostToDevice, ctx->stream));
  return 0;
}

int check_sys(gemsgpu_ctx* ctx, int s) {
  if (!ctx) return GEMSGPU_ERR_ARG;
  if (s < 0 || s >= (int)ctx->sys.size() || !ctx->sys[s].alive)
    return fail(ctx, GEMSGPU_ERR_ARG, "unknown system %d", s);
  return 0;
}

// ------------------------------------------------------------- block maps
// kind 0: atoms, `apb` atoms per block; kind 1: cells, 256 cells per block.
std::string map_key(const std::vector<int>& ss, int apb, int kind) {
  std::string key = std::to_string(kind) + ":" + std::to_string(apb) + ":";
  for (int s : ss) key += std::to_string(s) + ",";
  return key;
}

// position of ss as a contiguous run inside the batch being captured, or -1
int view_run(const gemsgpu_ctx* ctx, const std::vector<int>& ss) {
  const std::vector<int>& vs = ctx->view_set;
  if (vs.size() <= ss.size() || ss.empty()) return -1;
  auto it = std::find(vs.begin(), vs.end(), ss[0]);
  if (it == vs.end() || (size_t)(vs.end() - it) < ss.size()) return -1;
  return std::equal(ss.begin(), ss.end(), it) ? (int)(it - vs.begin()) : -1;
}

int get_map(gemsgpu_ctx* ctx, const std::vector<int>& ss, int apb, int kind, BlockMap* out) {
  if (view_run(ctx, ss) >= 0) {
    // a branch of a batched graph: its systems' blocks of the batch's map
    std::vector<int> full;
    full.swap(ctx->view_set);
    BlockMap fm;
    int rc = get_map(ctx, full, apb, kind, &fm);
    full.swap(ctx->view_set);
    CHK(rc);
    const DevMap& dm = ctx->maps[map_key(ctx->view_set, apb, kind)];
    int b0 = -1, b1 = 0;
    for (int s : ss)
      if (dm.nblkv[s] > 0) {
        if (b0 < 0) b0 = dm.blk0[s];
        b1 = dm.blk0[s] + dm.nblkv[s];
      }
    if (b0 < 0) b0 = b1 = 0;
    const int nb = b1 - b0;
    BlockMap v = fm;
    v.nblk = nb;
    v.base = b0;
    v.sys = fm.sys + b0;
    v.first = fm.first + b0;
    v.end = fm.end + b0;
    *out = v;
    return 0;
  }
  std::string key = map_key(ss, apb, kind);
  auto it = ctx->maps.find(key);
  if (it != ctx->maps.end()) {
    *out = it->second.m;
    return 0;
  }
  std::vector<int> bs, bf, be;
  std::vector<int> blk0(ctx->scap, 0), nblk(ctx->scap, 0);
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    int lo, hi;
    if (kind == 0) {
      lo = h.off;
      hi = h.off + h.n;
    } else {
      if (!h.d.use_cells) continue;
      lo = h.cell_off;
      // a moving box re-plans its grid on the device within its allocation
      hi = h.cell_off + (moving_box(h.d) ? h.cell_cap : h.d.ncell);
    }
    blk0[s] = (int)bs.size();
    for (int a = lo; a < hi; a += apb) {
      bs.push_back(s);
      bf.push_back(a);
      be.push_back(std::min(hi, a + apb));
    }
    nblk[s] = (int)bs.size() - blk0[s];
  }
  int nb = (int)bs.size();
  CHK(grow_blocks(ctx, std::max(nb, 1)));
  std::vector<int> all;
  all.insert(all.end(), bs.begin(), bs.end());
  all.insert(all.end(), bf.begin(), bf.end());
  all.insert(all.end(), be.begin(), be.end());
  all.insert(all.end(), blk0.begin(), blk0.end());
  all.insert(all.end(), nblk.begin(), nblk.end());
  DevMap dm;
  CHK(dalloc(ctx, &dm.buf, all.size()));
  CU(cudaMemcpyAsync(dm.buf, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice,
                     ctx->stream));
  dm.m.nblk = nb;
  dm.m.apb = apb;
  dm.m.sys = dm.buf;
  dm.m.first = dm.buf + nb;
  dm.m.end = dm.buf + 2 * nb;
  dm.m.sys_blk0 = dm.buf + 3 * nb;
  dm.m.sys_nblk = dm.buf + 3 * nb + ctx->scap;
  dm.m.base = 0;
  dm.nblk = nb;
  dm.blk0 = blk0;
  dm.nblkv = nblk;
  ctx->maps[key] = dm;
  *out = dm.m;
  return 0;
}

int sys_array(gemsgpu_ctx* ctx, const std::vector<int>& ss, const int** out) {
  std::string key = "S:";
  for (int s : ss) key += std::to_string(s) + ",";
  auto it = ctx->maps.find(key);
  if (it == ctx->maps.end()) {
    DevMap dm;
    CHK(dalloc(ctx, &dm.buf, ss.size()));
    CU(cudaMemcpyAsync(dm.buf, ss.data(), ss.size() * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->stream));
    dm.nblk = (int)ss.size();
    it = ctx->maps.emplace(key, dm).first;
  }
  *out = it->second.buf;
  return 0;
}

// ------------------------------------------------------------- launches
// one SMA-TB pass (0: density, 1: force) for a block map of K lanes per atom.
// variant bit 0: species constants in shared memory (1) or registers (0,
// single species only); bit 1: register-capped build for more warps per SM
// (four 256-thread blocks); bit 2 with bit 1: the force pass capped at three
// blocks instead (no spills, fewer warps).
template <int K>
void smatb_pass_k(gemsgpu_ctx* ctx, int pass, int prec, bool regs, bool tight, bool tight3, bool vir,
                  const BlockMap& m) {
  cudaStream_t st = ctx->stream;
  const Arena& A = ctx->A;
  if (prec == PREC_MIXED) {
    if (pass == 0) {
      if (regs && tight) k_smatb_rho_mixed<K, true, 4><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else if (regs) k_smatb_rho_mixed<K, true, 1><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else if (tight) k_smatb_rho_mixed<K, false, 4><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else k_smatb_rho_mixed<K, false, 1><<<m.nblk, BLOCK, 0, st>>>(A, m);
    } else if (vir) {  // the virial build: uncapped
      if (regs) k_smatb_force_mixed<K, true, 1, true><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else k_smatb_force_mixed<K, false, 1, true><<<m.nblk, BLOCK, 0, st>>>(A, m);
    } else {
      if (regs && tight && tight3) k_smatb_force_mixed<K, true, 3><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else if (regs && tight) k_smatb_force_mixed<K, true, 4><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else if (regs) k_smatb_force_mixed<K, true, 1><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else if (tight && tight3) k_smatb_force_mixed<K, false, 3><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else if (tight) k_smatb_force_mixed<K, false, 4><<<m.nblk, BLOCK, 0, st>>>(A, m);
      else k_smatb_force_mixed<K, false, 1><<<m.nblk, BLOCK, 0, st>>>(A, m);
    }
  } else {
    if (pass == 0) k_smatb_rho_fp64<K><<<m.nblk, BLOCK, 0, st>>>(A, m);
    else if (vir) k_smatb_force_fp64<K, true><<<m.nblk, BLOCK, 0, st>>>(A, m);
    else k_smatb_force_fp64<K, false><<<m.nblk, BLOCK, 0, st>>>(A, m);
  }
  ++ctx->launches;
}

template <int K>
void lj_k(gemsgpu_ctx* ctx, int prec, bool vir, const BlockMap& m) {
  if (prec == PREC_MIXED && vir) k_lj_mixed<K, true><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m);
  else if (prec == PREC_MIXED) k_lj_mixed<K><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m);
  else if (vir) k_lj_fp64<K, true><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m);
  else k_lj_fp64<K, false><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m);
  ++ctx->launches;
}

void smatb_pass(gemsgpu_ctx* ctx, int pass, int prec, int variant, bool single, int K, const BlockMap& m,
                bool vir = false) {
  const bool regs = single && (variant & 1) == 0;
  const bool tight = (variant & 2) != 0;
  const bool tight3 = (variant & 4) != 0;
  switch (K) {
    case 1: smatb_pass_k<1>(ctx, pass, prec, regs, tight, tight3, vir, m); break;
    case 2: smatb_pass_k<2>(ctx, pass, prec, regs, tight, tight3, vir, m); break;
    case 4: smatb_pass_k<4>(ctx, pass, prec, regs, tight, tight3, vir, m); break;
    case 8: smatb_pass_k<8>(ctx, pass, prec, regs, tight, tight3, vir, m); break;
    case 16: smatb_pass_k<16>(ctx, pass, prec, regs, tight, tight3, vir, m); break;
    default: smatb_pass_k<32>(ctx, pass, prec, regs, tight, tight3, vir, m); break;
  }
}

// Tersoff forces: bond records per centre atom, then the per-atom gather,
// both on the system's map of BLOCK / lanes atoms per block (lanes = threads
// per atom of the bond kernel: 4, or 2 in mixed precision).  variant bit 1:
// the bond kernel built for four blocks per SM, with bit 2 for three
// (autotuned).
template <typename R, int TPA>
void tersoff_bonds_t(gemsgpu_ctx* ctx, int variant, const BlockMap& m) {
  const size_t sh = tsf_smem<R, TPA>();
  if ((variant & 6) == 6) k_tsf_bonds<R, 3, TPA><<<m.nblk, BLOCK, sh, ctx->stream>>>(ctx->A, m);
  else if (variant & 2) k_tsf_bonds<R, 4, TPA><<<m.nblk, BLOCK, sh, ctx->stream>>>(ctx->A, m);
  else k_tsf_bonds<R, 1, TPA><<<m.nblk, BLOCK, sh, ctx->stream>>>(ctx->A, m);
}

// the bond kernels' dynamic shared memory may exceed the default 48 KB
template <typename R, int TPA>
int tersoff_smem_attr_t() {
  const int sh = (int)tsf_smem<R, TPA>();
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tsf_bonds<R, 1, TPA>, cudaFuncAttributeMaxDynamicSharedMemorySize, sh);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tsf_bonds<R, 3, TPA>, cudaFuncAttributeMaxDynamicSharedMemorySize, sh);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tsf_bonds<R, 4, TPA>, cudaFuncAttributeMaxDynamicSharedMemorySize, sh);
  return e == cudaSuccess ? 0 : 1;
}

int tersoff_smem_attr(gemsgpu_ctx* ctx) {
  if (tersoff_smem_attr_t<float, 2>() || tersoff_smem_attr_t<float, 4>() || tersoff_smem_attr_t<double, 4>())
    return fail(ctx, GEMSGPU_ERR_CUDA, "Tersoff kernels: shared-memory size refused");
  return 0;
}

void tersoff_bonds(gemsgpu_ctx* ctx, int prec, int variant, const BlockMap& m) {
  // two threads per atom: float only (the FP64 bond arrays of 128 atoms
  // exceed the static shared memory)
  if (prec == PREC_MIXED && m.apb == BLOCK / 2) tersoff_bonds_t<float, 2>(ctx, variant, m);
  else if (prec == PREC_MIXED) tersoff_bonds_t<float, 4>(ctx, variant, m);
  else tersoff_bonds_t<double, 4>(ctx, variant, m);
  ++ctx->launches;
}

void tersoff_gather(gemsgpu_ctx* ctx, int prec, const BlockMap& m) {
  if (prec == PREC_MIXED) k_tsf_gather<float><<<m.nblk, m.apb, 0, ctx->stream>>>(ctx->A, m);
  else k_tsf_gather<double><<<m.nblk, m.apb, 0, ctx->stream>>>(ctx->A, m);
  ++ctx->launches;
}

void tersoff_pass(gemsgpu_ctx* ctx, int prec, int variant, const BlockMap& m) {
  tersoff_bonds(ctx, prec, variant, m);
  tersoff_gather(ctx, prec, m);
}

void lj_pass(gemsgpu_ctx* ctx, int prec, int K, bool vir, const BlockMap& m) {
  switch (K) {
    case 2: lj_k<2>(ctx, prec, vir, m); break;
    case 4: lj_k<4>(ctx, prec, vir, m); break;
    case 8: lj_k<8>(ctx, prec, vir, m); break;
    case 16: lj_k<16>(ctx, prec, vir, m); break;
    case 32: lj_k<32>(ctx, prec, vir, m); break;
    default: lj_k<1>(ctx, prec, vir, m); break;
  }
}

// threads per atom of a Tersoff system's bond kernel: its tuned lanes if
// valid for its precision, else TS_TPA
int tersoff_lanes(const SysHost& h) {
  return (h.lanes == 2 && h.d.prec == PREC_MIXED) ? 2 : TS_TPA;
}

// group systems by (ff, prec, lanes) and launch the force kernels
int launch_forces(gemsgpu_ctx* ctx, const std::vector<int>& ss) {
  std::map<std::tuple<int, int, int, int, int>, std::vector<int>> groups;
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    if (h.d.ff == FF_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "system %d has no force field", s);
    int K = h.d.ff == FF_TERSOFF ? tersoff_lanes(h) : h.lanes;
    int key = h.variant * 2 + (h.ntypes == 1 ? 1 : 0);
    groups[{h.d.ff, h.d.prec, K, key, h.d.virial}].push_back(s);
  }
  for (auto& kv : groups) {
    int ff = std::get<0>(kv.first), prec = std::get<1>(kv.first), K = std::get<2>(kv.first);
    const int variant = std::get<3>(kv.first) / 2;
    const bool single = (std::get<3>(kv.first) & 1) != 0;
    const bool vir = std::get<4>(kv.first) != 0;
    BlockMap m;
    CHK(get_map(ctx, kv.second, BLOCK / K, 0, &m));
    if (ff == FF_TERSOFF) {
      tersoff_pass(ctx, prec, variant, m);
      continue;
    }
    if (ff == FF_SMATB) {
      smatb_pass(ctx, 0, prec, variant, single, K, m);
      smatb_pass(ctx, 1, prec, variant, single, K, m, vir);
    } else if (ff == FF_LJ) {
      lj_pass(ctx, prec, K, vir, m);
    }
  }
  CU(cudaGetLastError());
  return 0;
}

// the rebuild chain; every kernel returns at once for systems whose
// rebuild flag is clear, so the chain can sit in a captured step.
// grid of the rebuild kernels that visit only flagged systems' blocks
int rebuild_grid(const gemsgpu_ctx* ctx, int nblk) { return std::max(1, std::min(nblk, 8 * ctx->nsm)); }

// the warp-per-cell list kernels for the systems of each tile size
// (t128 / t512) and frame ([0] integer, [1] image)
int launch_list_w(gemsgpu_ctx* ctx, const BlockMap& mc8, const bool* t128, const bool* t512) {
  cudaStream_t st = ctx->stream;
  const Arena& A = ctx->A;
  const int g = rebuild_grid(ctx, mc8.nblk);
  if (t128[1]) k_list_cells_w<128, true><<<g, BLOCK, listw_smem<128>(A.lcap), st>>>(A, mc8);
  if (t128[0]) k_list_cells_w<128, false><<<g, BLOCK, listw_smem<128>(A.lcap), st>>>(A, mc8);
  if (t512[1]) k_list_cells_w<512, true><<<g, BLOCK, listw_smem<512>(A.lcap), st>>>(A, mc8);
  if (t512[0]) k_list_cells_w<512, false><<<g, BLOCK, listw_smem<512>(A.lcap), st>>>(A, mc8);
  ctx->launches += t128[0] + t128[1] + t512[0] + t512[1];
  CU(cudaGetLastError());
  return 0;
}

int launch_rebuild(gemsgpu_ctx* ctx, const std::vector<int>& ss, int in_graph = 0) {
  BlockMap ma, mc, mc8, mc1;
  const int* sa;
  CHK(get_map(ctx, ss, BLOCK, 0, &ma));
  CHK(get_map(ctx, ss, 256, 1, &mc));
  CHK(get_map(ctx, ss, BLOCK / 32, 1, &mc8));
  CHK(get_map(ctx, ss, 1, 1, &mc1));
  CHK(sys_array(ctx, ss, &sa));
  cudaStream_t st = ctx->stream;
  const Arena& A = ctx->A;
  bool cells = mc.nblk > 0;
  bool n2 = false;
  for (int s : ss) n2 |= !ctx->sys[s].d.use_cells;
  if (cells) {
    k_bin<<<ma.nblk, BLOCK, 0, st>>>(A, ma); ++ctx->launches;
    k_scan1<<<mc.nblk, BLOCK, 0, st>>>(A, mc); ++ctx->launches;
    k_scan2<<<(int)ss.size(), BLOCK, 0, st>>>(A, sa, (int)ss.size()); ++ctx->launches;
    k_scatter<<<ma.nblk, BLOCK, 0, st>>>(A, ma); ++ctx->launches;
    k_sort_cells<<<rebuild_grid(ctx, mc8.nblk), BLOCK, 0, st>>>(A, mc8); ++ctx->launches;
    bool kind[3][2] = {};
    for (int s : ss)
      if (ctx->sys[s].d.use_cells) kind[ctx->sys[s].d.list_warp][ctx->sys[s].d.list_img] = true;
    if (kind[0][0] || kind[0][1]) {
      k_list_cells<<<rebuild_grid(ctx, mc1.nblk * LIST_SPLIT), BLOCK, list_smem(A.lcap), st>>>(A, mc1);
      ++ctx->launches;
    }
    CHK(launch_list_w(ctx, mc8, kind[1], kind[2]));
  }
  if (n2) {
    k_list_n2<<<rebuild_grid(ctx, ma.nblk), BLOCK, 0, st>>>(A, ma); ++ctx->launches;
  }
  bool ts = false;
  for (int s : ss) ts |= ctx->sys[s].d.ff == FF_TERSOFF;
  if (ts) {
    k_tsf_rslot<<<rebuild_grid(ctx, ma.nblk), BLOCK, 0, st>>>(A, ma); ++ctx->launches;
  }
  k_count_rebuild<<<((int)ss.size() + 255) / 256, 256, 0, st>>>(A, sa, (int)ss.size(), in_graph); ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

int launch_step_a(gemsgpu_ctx* ctx, const std::vector<int>& ss,
                  cudaGraphConditionalHandle cond = 0, int use_cond = 0) {
  BlockMap ma;
  CHK(get_map(ctx, ss, BLOCK, 0, &ma));
  bool piston = false, lkd = false;
  for (int s : ss) {
    piston |= ctx->sys[s].d.integ == IT_LGF || ctx->sys[s].d.integ == IT_AXES;
    lkd |= ctx->sys[s].d.integ == IT_LKD;
  }
  if (lkd) {
    k_lkd_a<<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma);
    ++ctx->launches;
    for (int s : ss)
      if (ctx->sys[s].d.integ == IT_LKD) ctx->sys[s].box_live = true;
  }
  if (piston) {
    const int* sa;
    CHK(sys_array(ctx, ss, &sa));
    k_lgf_sys<<<((int)ss.size() + 127) / 128, 128, 0, ctx->stream>>>(ctx->A, sa, (int)ss.size());
    ++ctx->launches;
    for (int s : ss)
      if (moving_box(ctx->sys[s].d)) ctx->sys[s].box_live = true;
  }
  if (use_cond) k_step_a<true><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
  else k_step_a<false><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
  ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

// atoms per thread of the fused integrator step: STEP_APT for launches of
// four or more full waves of one-atom blocks (four blocks per SM), else one
#ifndef STEP_APT
#define STEP_APT 2
#endif
int step_apt(const gemsgpu_ctx* ctx, const std::vector<int>& ss) {
  // a branch of a batched graph uses the batch's map: the batch decides
  const std::vector<int>& all = view_run(ctx, ss) >= 0 ? ctx->view_set : ss;
  int64_t n = 0;
  for (int s : all) n += ctx->sys[s].n;
  return n >= (int64_t)4 * 4 * BLOCK * ctx->nsm ? STEP_APT : 1;
}

int launch_step_ba(gemsgpu_ctx* ctx, const std::vector<int>& ss,
                   cudaGraphConditionalHandle cond = 0, int use_cond = 0) {
  BlockMap ma;
  const int apt = step_apt(ctx, ss);
  CHK(get_map(ctx, ss, apt * BLOCK, 0, &ma));
  if (apt == 4) {
    if (use_cond) k_step_ba<true, 4><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
    else k_step_ba<false, 4><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
  } else if (apt == 2) {
    if (use_cond) k_step_ba<true, 2><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
    else k_step_ba<false, 2><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
  } else {
    if (use_cond) k_step_ba<true, 1><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
    else k_step_ba<false, 1><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma, cond);
  }
  ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

// step_b of one step and step_a of the next fuse into one kernel when every
// system integrates with velocity Verlet or Ermak
bool can_fuse_steps(const gemsgpu_ctx* ctx, const std::vector<int>& ss) {
  for (int s : ss) {
    const int it = ctx->sys[s].d.integ;
    if (it != IT_VV && it != IT_ERMAK) return false;
    if (ctx->sys[s].d.thermo != TH_NONE) return false;  // it runs between the two
  }
  return true;
}

// the force pass and the next half steps run as one kernel
// (k_smatb_force_*_ba) when every system is a velocity-Verlet or Ermak SMA-TB
// system without the virial, in FP64 or in mixed precision with the species
// constants in registers
bool can_fuse_forces(const gemsgpu_ctx* ctx, const std::vector<int>& ss) {
  if (!ctx->fuse_forces || !can_fuse_steps(ctx, ss)) return false;
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    if (h.d.ff != FF_SMATB || h.d.virial) return false;
    if (h.d.prec == PREC_MIXED && (h.ntypes != 1 || (h.variant & 1))) return false;
  }
  return true;
}

template <int K, int MINB>
void force_mixed_ba(gemsgpu_ctx* ctx, const BlockMap& m, cudaGraphConditionalHandle cond, bool use_cond) {
  if (use_cond) k_smatb_force_mixed_ba<K, true, MINB, true><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, cond);
  else k_smatb_force_mixed_ba<K, true, MINB, false><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, cond);
}

template <int K>
void force_ba_k(gemsgpu_ctx* ctx, int prec, int variant, const BlockMap& m, cudaGraphConditionalHandle cond,
                bool use_cond) {
  if (prec == PREC_MIXED) {
    if ((variant & 2) && (variant & 4)) force_mixed_ba<K, 3>(ctx, m, cond, use_cond);
    else if (variant & 2) force_mixed_ba<K, 4>(ctx, m, cond, use_cond);
    else force_mixed_ba<K, 1>(ctx, m, cond, use_cond);
  } else if (use_cond) {
    k_smatb_force_fp64_ba<K, true><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, cond);
  } else {
    k_smatb_force_fp64_ba<K, false><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, cond);
  }
  ++ctx->launches;
}

// the density pass, then the force pass fused with step_b of this step and
// step_a of the next (which raises `cond` when a list must be rebuilt)
int launch_forces_ba(gemsgpu_ctx* ctx, const std::vector<int>& ss, cudaGraphConditionalHandle cond = 0,
                     int use_cond = 0) {
  std::map<std::tuple<int, int, int>, std::vector<int>> groups;
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    groups[{h.d.prec, h.lanes, h.variant}].push_back(s);
  }
  for (auto& kv : groups) {
    const int prec = std::get<0>(kv.first), K = std::get<1>(kv.first), variant = std::get<2>(kv.first);
    BlockMap m;
    CHK(get_map(ctx, kv.second, BLOCK / K, 0, &m));
    smatb_pass(ctx, 0, prec, variant, true, K, m);
    switch (K) {
      case 1: force_ba_k<1>(ctx, prec, variant, m, cond, use_cond != 0); break;
      case 2: force_ba_k<2>(ctx, prec, variant, m, cond, use_cond != 0); break;
      case 4: force_ba_k<4>(ctx, prec, variant, m, cond, use_cond != 0); break;
      case 8: force_ba_k<8>(ctx, prec, variant, m, cond, use_cond != 0); break;
      case 16: force_ba_k<16>(ctx, prec, variant, m, cond, use_cond != 0); break;
      default: force_ba_k<32>(ctx, prec, variant, m, cond, use_cond != 0); break;
    }
  }
  CU(cudaGetLastError());
  return 0;
}

int launch_step_b(gemsgpu_ctx* ctx, const std::vector<int>& ss) {
  BlockMap ma;
  CHK(get_map(ctx, ss, BLOCK, 0, &ma));
  bool moves = false, thermo = false, scal = false;
  for (int s : ss) {
    const SysDev& d = ctx->sys[s].d;
    moves |= d.integ == IT_NORD || d.integ == IT_BROWN;
    thermo |= d.thermo != TH_NONE;
    scal |= d.thermo == TH_SCALVEL || d.thermo == TH_SCALVEL_AFTER;
  }
  if (moves) k_step_b<true><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma);
  else k_step_b<false><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma);
  ++ctx->launches;
  // the thermostats after the integrator's stepb
  if (scal) {
    k_thermo_sum<0><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma);
    k_thermo_sum<1><<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma);
    ctx->launches += 2;
  }
  if (thermo) {
    k_thermo_apply<<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma);
    ++ctx->launches;
  }
  CU(cudaGetLastError());
  return 0;
}

int read_states(gemsgpu_ctx* ctx) {
  CU(cudaMemcpyAsync(ctx->h_st, ctx->A.st, ctx->scap * sizeof(SysState), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int clear_status(gemsgpu_ctx* ctx, const std::vector<int>& ss) {
  if (ss.empty()) return 0;
  const int* sa;
  CHK(sys_array(ctx, ss, &sa));
  k_clear_status<<<((int)ss.size() + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, sa, (int)ss.size());
  ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

int status_error(gemsgpu_ctx* ctx, int s, int st) {
  if (st & ST_NAN) return fail(ctx, GEMSGPU_ERR_NAN, "system %d: non-finite positions", s);
  if (st & ST_LOST)
    return fail(ctx, GEMSGPU_ERR_LOST, "system %d: atom outside the cell grid / fixed-point range", s);
  if (st & ST_BONDS)
    return fail(ctx, GEMSGPU_ERR_STATE,
                "system %d: a Tersoff atom has more than %d bonds (r <= R+D), or a bond beyond list slot 63",
                s, TS_MAXB);
  if (st & ST_OVERFLOW) return fail(ctx, GEMSGPU_ERR_OVERFLOW, "system %d: neighbour list overflow", s);
  if (st & ST_BOX)
    return fail(ctx, GEMSGPU_ERR_STATE,
                "system %d: the constant-pressure box left its cell grid (under three list cut-offs "
                "or a collapsed volume)", s);
  return 0;
}

// neighbour capacity estimate: 1.5x the ideal count at the system's density
int estimate_cap(const SysHost& h) {
  const SysDev& d = h.d;
  double rl = std::sqrt(d.rlist2);
  double vol;
  if (d.boxed)
    vol = d.L[0] * d.L[1] * d.L[2];
  else
    vol = h.n / 0.06;  // close-packed metals ~0.06 atoms / A^3
  double dens = h.n / std::max(vol, 1e-6);
  dens = std::max(dens, 0.06);
  double nb = 4.18879 * rl * rl * rl * dens;
  int cap = (int)(1.5 * nb) + 16;
  cap = std::min(cap, std::max(h.n, 16));
  return std::max(cap, 16);
}

// interact (src/Interaction.f90:135-241) for a set of systems, host-driven:
// rebuild if flagged (heal overflow by growing the list), then forces.
int interact_group(gemsgpu_ctx* ctx, const std::vector<int>& ss, bool sync_check) {
  std::vector<int> first, dirty;
  int need = 0;
  for (int s : ss) {
    SysHost& h = ctx->sys[s];
    if (h.first) first.push_back(s);
    else if (h.pos_dirty) dirty.push_back(s);
    need = std::max(need, estimate_cap(h));
  }
  if (ctx->A.lcap < need) CHK(grow_list(ctx, need));
  CHK(clear_status(ctx, ss));
  if (!first.empty()) {
    const int* sa;
    CHK(sys_array(ctx, first, &sa));
    k_force_rebuild<<<((int)first.size() + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, sa,
                                                                                 (int)first.size()); ++ctx->launches;
  }
  if (!dirty.empty()) {
    BlockMap m;
    CHK(get_map(ctx, dirty, BLOCK, 0, &m));
    k_skin<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  }
  CHK(launch_rebuild(ctx, ss));
  if (sync_check) {
    CHK(read_states(ctx));
    int grow = 0;
    for (int s : ss) {
      const SysState& st = ctx->h_st[s];
      if (st.status & ST_OVERFLOW) grow = std::max(grow, st.maxnn);
    }
    if (grow > 0) {
      CHK(grow_list(ctx, grow + grow / 4 + 8));
      CHK(clear_status(ctx, ss));
      const int* sa;
      CHK(sys_array(ctx, ss, &sa));
      k_force_rebuild<<<((int)ss.size() + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, sa,
                                                                              (int)ss.size()); ++ctx->launches;
      CHK(launch_rebuild(ctx, ss));
      CHK(read_states(ctx));
    }
    for (int s : ss) CHK(status_error(ctx, s, ctx->h_st[s].status & ~0));
  }
  CHK(launch_forces(ctx, ss));
  for (int s : ss) {
    SysHost& h = ctx->sys[s];
    h.first = false;
    h.pos_dirty = false;
    h.has_forces = true;
  }
  return 0;
}

// Epot, Ekin, max |F|^2 and the status of each system of ss (4 doubles per
// system, in the order of ss): two grid-wide passes over the atom map
int reduce_sys(gemsgpu_ctx* ctx, const std::vector<int>& ss, std::vector<double>& out) {
  const int n = (int)ss.size();
  const int sc = ctx->scap;
  if (sc > ctx->h_red_cap) {
    if (ctx->h_red) cudaFreeHost(ctx->h_red);
    if (ctx->d_red) cudaFree(ctx->d_red);
    ctx->h_red = nullptr;
    ctx->d_red = nullptr;
    CU(cudaMallocHost((void**)&ctx->h_red, 4 * sizeof(double) * sc));
    CHK(dalloc(ctx, &ctx->d_red, 7 * (size_t)sc));  // 4 results + the centre-of-mass velocity
    ctx->h_red_cap = sc;
  }
  BlockMap m;
  CHK(get_map(ctx, ss, BLOCK, 0, &m));
  if (m.nblk > 0) {
    k_sys_reduce<0><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, sc, ctx->d_red);
    k_sys_reduce<1><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, sc, ctx->d_red);
    ctx->launches += 2;
  }
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(ctx->h_red, ctx->d_red, 4 * sizeof(double) * sc, cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  out.assign(4 * (size_t)n, 0.0);
  for (int k = 0; k < n; k++)
    for (int q = 0; q < 4; q++) out[4 * (size_t)k + q] = ctx->h_red[4 * (size_t)ss[k] + q];
  return 0;
}

// one captured MD step for a set of systems
// n plain steps; with fusion, step k > 0 opens with step_b(k-1)+step_a(k)
// and only the last step closes with its own step_b
int record_steps(gemsgpu_ctx* ctx, const std::vector<int>& ss, int n) {
  if (ss.size() == 1 && can_fuse_forces(ctx, ss)) {
    // step_a, then per step: rebuild chain, density pass, force pass with
    // step_b + the next step_a; the last step closes with its own step_b
    CHK(launch_step_a(ctx, ss));
    for (int k = 0; k < n; k++) {
      CHK(launch_rebuild(ctx, ss));
      if (k < n - 1) {
        CHK(launch_forces_ba(ctx, ss));
      } else {
        CHK(launch_forces(ctx, ss));
        CHK(launch_step_b(ctx, ss));
      }
    }
    return 0;
  }
  const bool fuse = can_fuse_steps(ctx, ss);
  for (int k = 0; k < n; k++) {
    if (k == 0 || !fuse) CHK(launch_step_a(ctx, ss));
    else CHK(launch_step_ba(ctx, ss));
    CHK(launch_rebuild(ctx, ss));
    CHK(launch_forces(ctx, ss));
    if (!fuse || k == n - 1) CHK(launch_step_b(ctx, ss));
  }
  return 0;
}

// Capture `nsteps` MD steps into one graph.  Each step is
//   [step_a] -> IF(rebuild needed) { rebuild chain } -> [forces, step_b]
// where the IF node's handle is raised by k_step_a; the rebuild kernels
// therefore cost nothing on steps that keep their list.  For velocity
// Verlet and Ermak systems step_b and the next step_a are one kernel:
//   [step_a] IF [forces] ([step_ba] IF [forces])... [step_b]
int capture_into(gemsgpu_ctx* ctx, cudaGraph_t g, std::vector<cudaGraphNode_t>& deps,
                 int (*fn)(gemsgpu_ctx*, const std::vector<int>&, void*),
                 const std::vector<int>& ss, void* arg) {
  CU(cudaStreamBeginCaptureToGraph(ctx->stream, g, deps.empty() ? nullptr : deps.data(), nullptr,
                                   deps.size(), cudaStreamCaptureModeThreadLocal));
  int rc = fn(ctx, ss, arg);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* d = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(ctx->stream, &cs, nullptr, nullptr, &d, &nd);
  std::vector<cudaGraphNode_t> nd_copy;
  if (e == cudaSuccess) nd_copy.assign(d, d + nd);
  cudaGraph_t out = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &out);
  if (rc) return rc;
  if (e != cudaSuccess || e2 != cudaSuccess)
    return fail(ctx, GEMSGPU_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
  deps = nd_copy;
  return 0;
}

struct CondArg {
  cudaGraphConditionalHandle h;
};

int cap_step_a(gemsgpu_ctx* ctx, const std::vector<int>& ss, void* arg) {
  return launch_step_a(ctx, ss, ((CondArg*)arg)->h, 1);
}
int cap_step_ba(gemsgpu_ctx* ctx, const std::vector<int>& ss, void* arg) {
  return launch_step_ba(ctx, ss, ((CondArg*)arg)->h, 1);
}
int cap_rebuild(gemsgpu_ctx* ctx, const std::vector<int>& ss, void*) {
  const int64_t before = ctx->launches;
  int rc = launch_rebuild(ctx, ss, 1);
  ctx->body_nodes = ctx->launches - before;
  ctx->bodies++;
  return rc;
}
int cap_forces_b(gemsgpu_ctx* ctx, const std::vector<int>& ss, void*) {
  CHK(launch_forces(ctx, ss));
  return launch_step_b(ctx, ss);
}
int cap_forces(gemsgpu_ctx* ctx, const std::vector<int>& ss, void*) {
  return launch_forces(ctx, ss);
}
int cap_forces_ba(gemsgpu_ctx* ctx, const std::vector<int>& ss, void* arg) {
  return launch_forces_ba(ctx, ss, ((CondArg*)arg)->h, 1);
}
int cap_plain(gemsgpu_ctx* ctx, const std::vector<int>& ss, void* arg) {
  return record_steps(ctx, ss, *(int*)arg);
}

constexpr size_t MAX_BRANCHES = 16;  // branches of a batched MD graph

// A batch of several systems with one launch shape is captured as
// independent branches -- one per system, or up to 16 runs of consecutive
// systems for larger batches: each branch's steps, conditional rebuilds and
// force passes form their own chain, so the GPU overlaps one system's list
// build or kernel tail with the others' work.  A branch's launches use the
// batch's block maps (views of its systems' blocks), so each block keeps
// its own per-block scratch slot.
int build_chunk_graph(gemsgpu_ctx* ctx, const std::vector<int>& ss, int nsteps, cudaGraph_t* out) {
  cudaGraph_t g = nullptr;
  CU(cudaGraphCreate(&g, 0));
  int rc = 0;
  bool cond_ok = ctx->use_cond;
  // up to MAX_BRANCHES branches of consecutive systems
  std::vector<std::vector<int>> sets;
  bool uniform = true;
  for (int s : ss) {
    const SysHost& a = ctx->sys[s];
    const SysHost& b = ctx->sys[ss[0]];
    uniform &= a.d.ff == b.d.ff && a.d.prec == b.d.prec && a.lanes == b.lanes && a.variant == b.variant &&
               a.d.virial == b.d.virial && (a.ntypes == 1) == (b.ntypes == 1);
  }
  const size_t nb = uniform ? std::min(ss.size(), MAX_BRANCHES) : 1;
  for (size_t j = 0; j < nb; j++)
    sets.emplace_back(ss.begin() + j * ss.size() / nb, ss.begin() + (j + 1) * ss.size() / nb);
  std::vector<std::vector<cudaGraphNode_t>> deps(sets.size());
  if (sets.size() > 1) ctx->view_set = ss;
  ctx->bodies = 0;
  // the force pass fused with the half steps: [step_a] IF [rho, force+ba] IF ... [rho, force, step_b]
  std::vector<CondArg> next(sets.size());
  std::vector<char> fused(sets.size(), 0);
  // (fusion saves a launch and its tail per step: alone +7 % mixed, +4 %
  // FP64; a batch of eight 32k-atom SMA-TB replicas +3 %)
  for (size_t j = 0; j < sets.size(); j++) fused[j] = can_fuse_forces(ctx, sets[j]);
  auto add_if = [&](size_t j, const CondArg& ca) -> int {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = ca.h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cn;
    if (cudaGraphAddNode(&cn, g, deps[j].data(), deps[j].size(), &cp) != cudaSuccess) return -1;
    std::vector<cudaGraphNode_t> none;
    int r = capture_into(ctx, cp.conditional.phGraph_out[0], none, cap_rebuild, sets[j], nullptr);
    deps[j].assign(1, cn);
    return r;
  };
  for (int k = 0; k < nsteps && rc == 0 && cond_ok; k++) {
    for (size_t j = 0; j < sets.size() && rc == 0 && cond_ok; j++) {
      if (!fused[j]) continue;
      const std::vector<int>& sj = sets[j];
      if (k == 0) {
        CondArg ca{};
        if (cudaGraphConditionalHandleCreate(&ca.h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
          cond_ok = false;
          break;
        }
        if ((rc = capture_into(ctx, g, deps[j], cap_step_a, sj, &ca))) break;
        if ((rc = add_if(j, ca)) < 0) {
          cond_ok = false;
          rc = 0;
          break;
        }
        if (rc) break;
      }
      if (k < nsteps - 1) {
        CondArg ca{};
        if (cudaGraphConditionalHandleCreate(&ca.h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
          cond_ok = false;
          break;
        }
        if ((rc = capture_into(ctx, g, deps[j], cap_forces_ba, sj, &ca))) break;
        if ((rc = add_if(j, ca)) < 0) {
          cond_ok = false;
          rc = 0;
          break;
        }
      } else {
        rc = capture_into(ctx, g, deps[j], cap_forces_b, sj, nullptr);
      }
    }
    for (size_t j = 0; j < sets.size() && rc == 0 && cond_ok; j++) {
      if (fused[j]) continue;
      const std::vector<int>& sj = sets[j];
      const bool fuse = can_fuse_steps(ctx, sj);
      CondArg ca{};
      if (cudaGraphConditionalHandleCreate(&ca.h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
        cond_ok = false;
        break;
      }
      rc = capture_into(ctx, g, deps[j], (k == 0 || !fuse) ? cap_step_a : cap_step_ba, sj, &ca);
      if (rc) break;
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = ca.h;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t cn;
      if (cudaGraphAddNode(&cn, g, deps[j].data(), deps[j].size(), &cp) != cudaSuccess) {
        cond_ok = false;
        break;
      }
      std::vector<cudaGraphNode_t> none;
      rc = capture_into(ctx, cp.conditional.phGraph_out[0], none, cap_rebuild, sj, nullptr);
      if (rc) break;
      deps[j].assign(1, cn);
      rc = capture_into(ctx, g, deps[j], (fuse && k < nsteps - 1) ? cap_forces : cap_forces_b, sj, nullptr);
    }
  }
  ctx->view_set.clear();
  cudaGetLastError();
  if (rc == 0 && !cond_ok) {
    // conditional nodes unavailable: plain capture, rebuild kernels exit early
    cudaGraphDestroy(g);
    ctx->use_cond = false;
    CU(cudaGraphCreate(&g, 0));
    std::vector<cudaGraphNode_t> none;
    int n = nsteps;
    rc = capture_into(ctx, g, none, cap_plain, ss, &n);
  }
  if (rc) {
    cudaGraphDestroy(g);
    return rc;
  }
  *out = g;
  return 0;
}

int get_graph(gemsgpu_ctx* ctx, const std::vector<int>& ss, int nsteps, cudaGraphExec_t* out) {
  std::string key = "G" + std::to_string(nsteps) + ":";
  for (int s : ss) key += std::to_string(s) + ",";
  auto it = ctx->graphs.find(key);
  if (it != ctx->graphs.end() && it->second.epoch == ctx->epoch) {
    *out = it->second.exec;
    return 0;
  }
  // make sure every map exists before capture (map creation copies memory)
  {
    BlockMap m;
    const int* sa;
    CHK(get_map(ctx, ss, BLOCK, 0, &m));
    CHK(get_map(ctx, ss, step_apt(ctx, ss) * BLOCK, 0, &m));
    CHK(get_map(ctx, ss, 256, 1, &m));
    CHK(get_map(ctx, ss, BLOCK / 32, 1, &m));
    CHK(get_map(ctx, ss, 1, 1, &m));
    CHK(sys_array(ctx, ss, &sa));
    const size_t nbr = std::min(ss.size(), MAX_BRANCHES);
    for (size_t j = 0; j < nbr && ss.size() > 1; j++)
      CHK(sys_array(ctx, std::vector<int>(ss.begin() + j * ss.size() / nbr, ss.begin() + (j + 1) * ss.size() / nbr),
                    &sa));
    for (int s : ss) {
      const SysHost& h = ctx->sys[s];
      CHK(get_map(ctx, ss, BLOCK / h.lanes, 0, &m));
    }
    std::map<std::tuple<int, int, int>, std::vector<int>> groups;
    for (int s : ss) {
      const SysHost& h = ctx->sys[s];
      groups[{h.d.ff, h.d.prec, h.lanes}].push_back(s);
    }
    for (auto& kv : groups) {
      int K = std::get<2>(kv.first);
      CHK(get_map(ctx, kv.second, BLOCK / K, 0, &m));
    }
    CU(cudaStreamSynchronize(ctx->stream));
  }
  cudaGraph_t g = nullptr;
  const int64_t before = ctx->launches;
  ctx->body_nodes = 0;
  int rc = build_chunk_graph(ctx, ss, nsteps, &g);
  int64_t nodes = ctx->launches - before;
  const int64_t body = ctx->use_cond ? ctx->body_nodes : 0;
  if (ctx->use_cond) nodes -= body * ctx->bodies;  // the bodies run only on rebuild steps
  ctx->launches = before;  // captured, not executed
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  cudaError_t e;
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(ctx, GEMSGPU_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  if (it != ctx->graphs.end() && it->second.exec) cudaGraphExecDestroy(it->second.exec);
  ctx->graphs[key] = Graph{ex, ctx->epoch, nodes, body};
  *out = ex;
  return 0;
}

int launch_graph(gemsgpu_ctx* ctx, const std::vector<int>& ss, int nsteps) {
  cudaGraphExec_t ex;
  CHK(get_graph(ctx, ss, nsteps, &ex));
  CU(cudaGraphLaunch(ex, ctx->stream));
  std::string key = "G" + std::to_string(nsteps) + ":";
  for (int s : ss) key += std::to_string(s) + ",";
  ctx->launches += ctx->graphs[key].nodes;
  if (ctx->graphs[key].body_nodes) {
    unsigned long long runs = 0;
    CU(cudaMemcpyAsync(&runs, ctx->A.body_runs, sizeof(runs), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->launches += (int64_t)(runs - ctx->body_seen) * ctx->graphs[key].body_nodes;
    ctx->body_seen = runs;
  }
  return 0;
}

int snapshot(gemsgpu_ctx* ctx, bool restore) {
  int64_t n = ctx->acap;
  Arena& A = ctx->A;
  // the Nordsieck derivatives, once a system has them
  int na = A.acel2 ? 7 : 4;
  if (restore) na = std::min(na, ctx->snap_arrays);
  if (!restore && (ctx->snap_cap < n || ctx->snap_arrays < na)) {
    if (ctx->snap) cudaFree(ctx->snap);
    CHK(dalloc(ctx, &ctx->snap, na * (size_t)n));
    ctx->snap_cap = n;
    ctx->snap_arrays = na;
  }
  double4* arr[7] = {A.pos, A.vel, A.acel, A.force, A.acel2, A.acel3, A.acel4};
  for (int k = 0; k < na; k++) {
    if (restore)
      CU(cudaMemcpyAsync(arr[k], ctx->snap + k * n, n * sizeof(double4), cudaMemcpyDeviceToDevice,
                         ctx->stream));
    else
      CU(cudaMemcpyAsync(ctx->snap + k * n, arr[k], n * sizeof(double4), cudaMemcpyDeviceToDevice,
                         ctx->stream));
  }
  if (restore) {
    CU(cudaMemcpyAsync(A.st, ctx->snap_st, ctx->scap * sizeof(SysState), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    CU(cudaMemcpyAsync(A.sys, ctx->snap_sys, ctx->scap * sizeof(SysDev), cudaMemcpyDeviceToDevice,
                       ctx->stream));
  } else {
    CU(cudaMemcpyAsync(ctx->snap_st, A.st, ctx->scap * sizeof(SysState), cudaMemcpyDeviceToDevice,
                       ctx->stream));
    CU(cudaMemcpyAsync(ctx->snap_sys, A.sys, ctx->scap * sizeof(SysDev), cudaMemcpyDeviceToDevice,
                       ctx->stream));
  }
  return 0;
}

constexpr int CHUNK = 50;

// dinamic (src/Programs.f90:114-167) for a set of systems, device-resident:
// chunks of CHUNK captured steps; after each chunk the states are checked,
// and a chunk that overflowed a list is undone, the list grown and redone.
int md_group(gemsgpu_ctx* ctx, const std::vector<int>& ss, int nsteps) {
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    if (h.d.integ == IT_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "system %d has no integrator", s);
  }
  bool need_first = false;
  for (int s : ss) need_first |= ctx->sys[s].first || ctx->sys[s].pos_dirty || !ctx->sys[s].has_forces;
  if (need_first) CHK(interact_group(ctx, ss, true));
  int done = 0;
  int retries = 0;
  while (done < nsteps) {
    int k = std::min(CHUNK, nsteps - done);
    CHK(snapshot(ctx, false));
    CHK(clear_status(ctx, ss));
    CHK(launch_graph(ctx, ss, k));
    CHK(read_states(ctx));
    int grow = 0, bad = 0, bads = -1;
    for (int s : ss) {
      int st = ctx->h_st[s].status;
      if (st & ST_OVERFLOW) grow = std::max(grow, ctx->h_st[s].maxnn);
      if (st & ST_FATAL) { bad = st; bads = s; }
    }
    if (bad) return status_error(ctx, bads, bad);
    if (grow > 0) {
      if (++retries > 4) return fail(ctx, GEMSGPU_ERR_OVERFLOW, "neighbour list keeps overflowing");
      CHK(snapshot(ctx, true));
      {
        // the fixed-point copies were left at the undone chunk's positions
        BlockMap mr;
        CHK(get_map(ctx, ss, BLOCK, 0, &mr));
        k_refresh_fx<<<mr.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, mr); ++ctx->launches;
      }
      CHK(grow_list(ctx, grow + grow / 4 + 8));
      const int* sa;
      CHK(sys_array(ctx, ss, &sa));
      k_force_rebuild<<<((int)ss.size() + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, sa, (int)ss.size()); ++ctx->launches;
      CHK(clear_status(ctx, ss));
      CHK(launch_rebuild(ctx, ss));
      CHK(launch_forces(ctx, ss));
      continue;
    }
    done += k;
  }
  return 0;
}

int ensure_stage(gemsgpu_ctx* ctx, int64_t n) {
  if (ctx->stage_cap >= n) return 0;
  if (ctx->stage) CU(cudaFree(ctx->stage));
  ctx->stage = nullptr;
  CHK(dalloc(ctx, &ctx->stage, 3 * (size_t)n));
  ctx->stage_cap = n;
  return 0;
}

// host interleaved xyz -> arena double4 slots (one H2D copy + a repack kernel)
int h2d_xyz(gemsgpu_ctx* ctx, const double* src, double4* dst, int n) {
  CHK(ensure_stage(ctx, n));
  CU(cudaMemcpyAsync(ctx->stage, src, (size_t)3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  k_unpack3<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ctx->stage, dst, n); ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

// arena double4 slots -> host interleaved xyz (a pack kernel + one D2H copy)
int d2h_xyz(gemsgpu_ctx* ctx, const double4* src, double* dst, int n) {
  CHK(ensure_stage(ctx, n));
  k_pack3<<<(n + 255) / 256, 256, 0, ctx->stream>>>(src, ctx->stage, n); ++ctx->launches;
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(dst, ctx->stage, (size_t)3 * n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return 0;
}

void copy_interleaved_to_d4(const double* src, std::vector<double4>& dst, int n) {
  dst.resize(n);
  for (int i = 0; i < n; i++) dst[i] = make_double4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0);
}

// ------------------------------------------------------------- pools
int pool_kind_apb(const gemsgpu_pool* P, int kind) {
  switch (kind) {
    case 0: return BLOCK;
    case 1: return 256;
    case 2: return LIST_ATOMS;
    case 3: return BLOCK / 32;
    default: return BLOCK / P->lanes;
  }
}

int pool_alloc(gemsgpu_pool* P) {
  gemsgpu_ctx* ctx = P->ctx;
  for (int k = 0; k < 5; k++) {
    int64_t units = (k == 1 || k == 3) ? P->max_cells : P->max_atoms;
    int apb = pool_kind_apb(P, k);
    P->cap[k] = (int)((units + apb - 1) / apb + P->max_systems);
    if (P->cap[k] < 1) P->cap[k] = 1;
    // sys, first, end (cap each) + sys_blk0, sys_nblk (scap each)
    CHK(dalloc(ctx, &P->dmap[k], 3 * (size_t)P->cap[k] + 2 * (size_t)P->scap));
    BlockMap& m = P->maps[k];
    m.nblk = P->cap[k];
    m.apb = apb;
    m.sys = P->dmap[k];
    m.first = P->dmap[k] + P->cap[k];
    m.end = P->dmap[k] + 2 * P->cap[k];
    m.sys_blk0 = P->dmap[k] + 3 * P->cap[k];
    m.sys_nblk = P->dmap[k] + 3 * P->cap[k] + P->scap;
    m.base = 0;
  }
  CHK(dalloc(ctx, &P->dsys, P->max_systems));
  CHK(grow_blocks(ctx, *std::max_element(P->cap, P->cap + 5)));
  return 0;
}

// write the padded maps of the current active set
int pool_upload_maps(gemsgpu_pool* P) {
  gemsgpu_ctx* ctx = P->ctx;
  for (int k = 0; k < 5; k++) {
    const int cap = P->cap[k], apb = pool_kind_apb(P, k);
    std::vector<int>& b = P->host_buf;
    b.assign(3 * (size_t)cap + 2 * (size_t)P->scap, 0);
    int* bs = b.data();
    int* bf = bs + cap;
    int* be = bs + 2 * cap;
    int* b0 = bs + 3 * cap;
    int* nb = b0 + P->scap;
    int n = 0;
    for (int s : P->active) {
      const SysHost& h = ctx->sys[s];
      int lo, hi;
      if (k == 1 || k == 3) {
        if (!h.d.use_cells) continue;
        lo = h.cell_off;
        hi = h.cell_off + h.d.ncell;
      } else {
        lo = h.off;
        hi = h.off + h.n;
      }
      b0[s] = n;
      for (int a = lo; a < hi; a += apb) {
        if (n >= cap) return fail(ctx, GEMSGPU_ERR_FULL, "pool map capacity exceeded");
        bs[n] = s;
        bf[n] = a;
        be[n] = std::min(hi, a + apb);
        n++;
      }
      nb[s] = n - b0[s];
    }
    for (int q = n; q < cap; q++) bs[q] = -1;
    CU(cudaMemcpyAsync(P->dmap[k], b.data(), b.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  }
  std::vector<int> sa(P->max_systems, -1);
  for (size_t q = 0; q < P->active.size(); q++) sa[q] = P->active[q];
  CU(cudaMemcpyAsync(P->dsys, sa.data(), sa.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));  // host buffers are reused
  P->maps_dirty = false;
  return 0;
}

// kernels of one pooled step (capacity grids; padding blocks return at once)
int pool_step_a(gemsgpu_pool* P, cudaGraphConditionalHandle h, bool cond) {
  gemsgpu_ctx* ctx = P->ctx;
  const BlockMap& m = P->maps[0];
  if (cond) k_step_a<true><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, h);
  else k_step_a<false><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, h);
  ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

int pool_rebuild(gemsgpu_pool* P, int in_graph) {
  gemsgpu_ctx* ctx = P->ctx;
  cudaStream_t st = ctx->stream;
  const Arena& A = ctx->A;
  const BlockMap &ma = P->maps[0], &mc = P->maps[1], &mc8 = P->maps[3];
  const int ns = P->max_systems;
  k_bin<<<ma.nblk, BLOCK, 0, st>>>(A, ma); ++ctx->launches;
  k_scan1<<<mc.nblk, BLOCK, 0, st>>>(A, mc); ++ctx->launches;
  k_scan2<<<ns, BLOCK, 0, st>>>(A, P->dsys, ns); ++ctx->launches;
  k_scatter<<<ma.nblk, BLOCK, 0, st>>>(A, ma); ++ctx->launches;
  k_sort_cells<<<rebuild_grid(ctx, mc8.nblk), BLOCK, 0, st>>>(A, mc8); ++ctx->launches;
  k_list_cells<<<rebuild_grid(ctx, mc8.nblk * LIST_SPLIT), BLOCK, list_smem(A.lcap), st>>>(A, mc8);
  ++ctx->launches;
  const bool all[2] = {true, true};
  CHK(launch_list_w(ctx, mc8, all, all));
  k_list_n2<<<rebuild_grid(ctx, ma.nblk), BLOCK, 0, st>>>(A, ma); ++ctx->launches;
  if (P->ff == FF_TERSOFF) {
    k_tsf_rslot<<<rebuild_grid(ctx, ma.nblk), BLOCK, 0, st>>>(A, ma); ++ctx->launches;
  }
  k_count_rebuild<<<(ns + 255) / 256, 256, 0, st>>>(A, P->dsys, ns, in_graph); ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

int pool_forces(gemsgpu_pool* P) {
  gemsgpu_ctx* ctx = P->ctx;
  const BlockMap& mk = P->maps[4];
  if (P->ff == FF_SMATB) {
    // the graph is captured once: the register variant (bit 0 clear) is only
    // allowed for single-species members (checked in gemsgpu_pool_set)
    const bool single = (P->variant & 1) == 0;
    smatb_pass(ctx, 0, P->prec, P->variant, single, P->lanes, mk);
    smatb_pass(ctx, 1, P->prec, P->variant, single, P->lanes, mk);
  } else if (P->ff == FF_LJ) {
    lj_pass(ctx, P->prec, P->lanes, false, mk);
  } else if (P->ff == FF_TERSOFF) {
    tersoff_pass(ctx, P->prec, P->variant, mk);
  }
  CU(cudaGetLastError());
  return 0;
}

int pool_step_b(gemsgpu_pool* P) {
  gemsgpu_ctx* ctx = P->ctx;
  const BlockMap& m = P->maps[0];
  k_step_b<false><<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  CU(cudaGetLastError());
  return 0;
}

struct PoolArg {
  gemsgpu_pool* P;
  cudaGraphConditionalHandle h;
  int n;
};
int pcap_a(gemsgpu_ctx*, const std::vector<int>&, void* a) {
  PoolArg* q = (PoolArg*)a;
  return pool_step_a(q->P, q->h, true);
}
int pcap_rebuild(gemsgpu_ctx* ctx, const std::vector<int>&, void* a) {
  const int64_t before = ctx->launches;
  int rc = pool_rebuild(((PoolArg*)a)->P, 1);
  ((PoolArg*)a)->P->body_nodes = ctx->launches - before;
  return rc;
}
int pcap_fb(gemsgpu_ctx*, const std::vector<int>&, void* a) {
  CHK(pool_forces(((PoolArg*)a)->P));
  return pool_step_b(((PoolArg*)a)->P);
}
int pcap_plain(gemsgpu_ctx*, const std::vector<int>&, void* a) {
  PoolArg* q = (PoolArg*)a;
  for (int k = 0; k < q->n; k++) {
    CHK(pool_step_a(q->P, 0, false));
    CHK(pool_rebuild(q->P, 0));
    CHK(pool_forces(q->P));
    CHK(pool_step_b(q->P));
  }
  return 0;
}

int pool_capture(gemsgpu_pool* P) {
  gemsgpu_ctx* ctx = P->ctx;
  if (P->exec) {
    cudaGraphExecDestroy(P->exec);
    P->exec = nullptr;
  }
  cudaGraph_t g = nullptr;
  CU(cudaGraphCreate(&g, 0));
  const int64_t before = ctx->launches;
  std::vector<cudaGraphNode_t> deps;
  std::vector<int> none_ss;
  int rc = 0;
  bool cond = ctx->use_cond;
  P->body_nodes = 0;
  for (int k = 0; k < P->chunk && rc == 0 && cond; k++) {
    PoolArg pa{P, 0, 0};
    if (cudaGraphConditionalHandleCreate(&pa.h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
      cond = false;
      break;
    }
    rc = capture_into(ctx, g, deps, pcap_a, none_ss, &pa);
    if (rc) break;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = pa.h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cn;
    if (cudaGraphAddNode(&cn, g, deps.data(), deps.size(), &cp) != cudaSuccess) {
      cond = false;
      break;
    }
    std::vector<cudaGraphNode_t> none;
    rc = capture_into(ctx, cp.conditional.phGraph_out[0], none, pcap_rebuild, none_ss, &pa);
    if (rc) break;
    deps.assign(1, cn);
    rc = capture_into(ctx, g, deps, pcap_fb, none_ss, &pa);
  }
  cudaGetLastError();
  if (rc == 0 && !cond) {
    cudaGraphDestroy(g);
    CU(cudaGraphCreate(&g, 0));
    deps.clear();
    PoolArg pa{P, 0, P->chunk};
    P->body_nodes = 0;
    rc = capture_into(ctx, g, deps, pcap_plain, none_ss, &pa);
  }
  int64_t nodes = ctx->launches - before;
  ctx->launches = before;
  if (rc) {
    cudaGraphDestroy(g);
    return rc;
  }
  P->nodes = nodes - P->body_nodes * P->chunk;
  cudaError_t e = cudaGraphInstantiate(&P->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(ctx, GEMSGPU_ERR_CUDA, "pool graph instantiate: %s", cudaGetErrorString(e));
  P->captured = ctx->A;
  return 0;
}

bool same_arena(const Arena& a, const Arena& b) { return memcmp(&a, &b, sizeof(Arena)) == 0; }

// one pooled chunk: (re)capture if the arena moved, launch, check states;
// undo and redo a chunk whose lists overflowed.
int pool_chunk(gemsgpu_pool* P) {
  gemsgpu_ctx* ctx = P->ctx;
  if (P->active.empty()) return 0;
  if (P->maps_dirty) CHK(pool_upload_maps(P));
  for (int attempt = 0; attempt < 5; attempt++) {
    if (!P->exec || !same_arena(P->captured, ctx->A)) CHK(pool_capture(P));
    CHK(snapshot(ctx, false));
    k_clear_status<<<(P->max_systems + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, P->dsys, P->max_systems);
    ++ctx->launches;
    CU(cudaGraphLaunch(P->exec, ctx->stream));
    ctx->launches += P->nodes;
    if (P->body_nodes) {
      unsigned long long runs = 0;
      CU(cudaMemcpyAsync(&runs, ctx->A.body_runs, sizeof(runs), cudaMemcpyDeviceToHost, ctx->stream));
      CU(cudaStreamSynchronize(ctx->stream));
      ctx->launches += (int64_t)(runs - ctx->body_seen) * P->body_nodes;
      ctx->body_seen = runs;
    }
    CHK(read_states(ctx));
    int grow = 0;
    for (int s : P->active) {
      int st = ctx->h_st[s].status;
      if (st & ST_FATAL) return status_error(ctx, s, st);
      if (st & ST_OVERFLOW) grow = std::max(grow, ctx->h_st[s].maxnn);
    }
    if (!grow) return 0;
    CHK(snapshot(ctx, true));
    // the fixed-point copies were left at the undone chunk's positions
    k_refresh_fx<<<P->maps[0].nblk, BLOCK, 0, ctx->stream>>>(ctx->A, P->maps[0]); ++ctx->launches;
    CHK(grow_list(ctx, grow + grow / 4 + 8));
    CHK(list_smem_attr(ctx, ctx->A.lcap));
    k_force_rebuild<<<(P->max_systems + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, P->dsys, P->max_systems);
    ++ctx->launches;
    k_clear_status<<<(P->max_systems + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, P->dsys, P->max_systems);
    ++ctx->launches;
    CHK(pool_rebuild(P, 0));
    CHK(pool_forces(P));
  }
  return fail(ctx, GEMSGPU_ERR_OVERFLOW, "neighbour list keeps overflowing");
}

// systems entering a pool get their first list and forces (interact)
int pool_prepare(gemsgpu_pool* P, const std::vector<int>& fresh) {
  gemsgpu_ctx* ctx = P->ctx;
  if (fresh.empty()) return 0;
  for (int s : fresh) {
    SysHost& h = ctx->sys[s];
    if (h.d.ff != P->ff || h.d.prec != P->prec)
      return fail(ctx, GEMSGPU_ERR_STATE, "system %d does not match the pool's force field / precision", s);
    h.lanes = P->lanes;
    h.variant = P->variant;
  }
  return interact_group(ctx, fresh, true);
}

}  // namespace

// ============================================================== C ABI
extern "C" {

const char* gemsgpu_version(void) { return "gemsgpu 0.1 (sm_100a)"; }

int gemsgpu_create(int device, int64_t max_atoms, int max_systems, gemsgpu_ctx** out) {
  if (!out) return GEMSGPU_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GEMSGPU_ERR_NODEV;
  if (device < 0 || device >= ndev) return GEMSGPU_ERR_ARG;
  auto* ctx = new gemsgpu_ctx();
  ctx->device = device;
  // profilers cannot replay kernels of graphs with conditional nodes:
  // GEMSGPU_NO_COND=1 captures plain steps (rebuild kernels exit early)
  if (const char* e = getenv("GEMSGPU_NO_COND")) ctx->use_cond = !(e[0] == '1');
  if (const char* e = getenv("GEMSGPU_NO_FUSED_FORCES")) ctx->fuse_forces = !(e[0] == '1');
  int rc = 0;
  do {
    if (cudaSetDevice(device) != cudaSuccess) { rc = GEMSGPU_ERR_CUDA; break; }
    if (cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
      rc = GEMSGPU_ERR_CUDA;
      break;
    }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      rc = GEMSGPU_ERR_CUDA;
      break;
    }
    if ((rc = grow_systems(ctx, std::max(max_systems, 16)))) break;
    if ((rc = grow_atoms(ctx, std::max<int64_t>(max_atoms, 1024)))) break;
    if ((rc = grow_cells(ctx, 4096))) break;
    if ((rc = grow_params(ctx, 64))) break;
    if ((rc = grow_blocks(ctx, 1024))) break;
    if ((rc = dalloc(ctx, &ctx->A.any_rebuild, 1))) break;
    if ((rc = dalloc(ctx, &ctx->A.body_runs, 1))) break;
    cudaMemsetAsync(ctx->A.any_rebuild, 0, sizeof(int), ctx->stream);
    cudaMemsetAsync(ctx->A.body_runs, 0, sizeof(unsigned long long), ctx->stream);
  } while (0);
  if (rc) {
    gemsgpu_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return 0;
}

int gemsgpu_destroy(gemsgpu_ctx* ctx) {
  if (!ctx) return GEMSGPU_ERR_ARG;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  drop_maps(ctx);
  Arena& A = ctx->A;
  void* ptrs[] = {A.pos, A.pos_old, A.vel, A.acel, A.force, A.vel_v, A.acel2, A.acel3, A.acel4, A.epot, A.band, A.eband,
                  A.ebandf, A.fxp, A.pose, A.fxe, A.minv, A.mass, A.type, A.nn, A.hnn, A.ncut, A.list, A.flist, A.cell_of, A.slot,
                  A.cell_count, A.cell_n, A.cell_loc, A.cell_start, A.chunk_sum, A.cell_atoms,
                  A.cell_pos, A.rslot, A.tidx, A.tsmask, A.tsfb, A.tsfb32,
                  A.ext_normals, A.blk_top2, A.blk_red, A.sys, A.st, A.prm, A.any_rebuild, A.body_runs,
                  ctx->d_red, ctx->snap, ctx->snap_st, ctx->snap_sys, ctx->d_sys,
                  ctx->lbw.x0, ctx->lbw.g, ctx->lbw.gold, ctx->lbw.d, ctx->lbw.S, ctx->lbw.Y, ctx->lbw.st,
                  ctx->d_fac};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (ctx->h_red) cudaFreeHost(ctx->h_red);
  if (ctx->h_st) cudaFreeHost(ctx->h_st);
  if (ctx->stage) cudaFree(ctx->stage);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return 0;
}

int gemsgpu_last_error(gemsgpu_ctx* ctx, char* buf, int len) {
  if (!ctx || !buf || len <= 0) return GEMSGPU_ERR_ARG;
  snprintf(buf, len, "%s", ctx->err.c_str());
  return 0;
}

int gemsgpu_system_create(gemsgpu_ctx* ctx, int natoms, int ntypes, int* sys) {
  if (!ctx || !sys || natoms <= 0 || ntypes <= 0 || ntypes > MAXT)
    return fail(ctx, GEMSGPU_ERR_ARG, "system_create: natoms>0 and 1<=ntypes<=%d", MAXT);
  cudaSetDevice(ctx->device);
  int s = -1;
  for (size_t k = 0; k < ctx->sys.size(); k++)
    if (!ctx->sys[k].alive) { s = (int)k; break; }
  if (s < 0) {
    s = (int)ctx->sys.size();
    ctx->sys.emplace_back();
  }
  CHK(grow_systems(ctx, s + 1));
  SysHost& h = ctx->sys[s];
  h = SysHost();
  h.alive = true;
  h.n = natoms;
  h.ntypes = ntypes;
  int64_t off = take_range(ctx->free_atoms, ctx->atoms_used, natoms, 32);
  CHK(grow_atoms(ctx, off + natoms));
  h.off = (int)off;
  h.param_off = ctx->params_used;
  ctx->params_used += ntypes * ntypes;
  CHK(grow_params(ctx, ctx->params_used));
  h.prm.assign(ntypes * ntypes, PairP{});
  h.d = SysDev{};
  h.d.skin = 1.0;
  h.d.skin_mic = 1;
  h.d.dt = 0.002;
  h.d.fx_origin[0] = h.d.fx_origin[1] = h.d.fx_origin[2] = 0.0;
  SysState z{};
  CU(cudaMemcpyAsync(ctx->A.st + s, &z, sizeof(z), cudaMemcpyHostToDevice, ctx->stream));
  CHK(push_sys(ctx, s));
  invalidate(ctx);
  drop_maps(ctx);
  *sys = s;
  return 0;
}

int gemsgpu_system_destroy(gemsgpu_ctx* ctx, int sys) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  ctx->free_atoms.push_back({h.off, h.off + h.n});
  if (h.cell_cap) ctx->free_cells.push_back({h.cell_off, h.cell_off + h.cell_cap});
  h.alive = false;
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_upload(gemsgpu_ctx* ctx, int sys, const double* pos, const double* vel,
                   const double* mass, const int* type) {
  CHK(check_sys(ctx, sys));
  if (!pos || !mass) return fail(ctx, GEMSGPU_ERR_ARG, "upload: pos and mass are required");
  cudaSetDevice(ctx->device);
  SysHost& h = ctx->sys[sys];
  int n = h.n;
  std::vector<double4> b;
  copy_interleaved_to_d4(pos, b, n);
  // fixed-point origin of open dims: centroid of the first upload
  double cg[3] = {0, 0, 0};
  for (int i = 0; i < n; i++) {
    cg[0] += b[i].x; cg[1] += b[i].y; cg[2] += b[i].z;
  }
  for (int k = 0; k < 3; k++) {
    double c = cg[k] / n;
    if (!std::isfinite(c)) return fail(ctx, GEMSGPU_ERR_NAN, "upload: non-finite positions");
    if (!h.d.boxed) h.d.fx_origin[k] = c;
  }
  Arena& A = ctx->A;
  CU(cudaMemcpyAsync(A.pos + h.off, b.data(), n * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(A.pos_old + h.off, b.data(), n * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
  std::vector<double4> v(n, make_double4(0, 0, 0, 0));
  if (vel) copy_interleaved_to_d4(vel, v, n);
  CU(cudaMemcpyAsync(A.vel + h.off, v.data(), n * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
  std::vector<double4> z(n, make_double4(0, 0, 0, 0));
  CU(cudaMemcpyAsync(A.acel + h.off, z.data(), n * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(A.force + h.off, z.data(), n * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(A.vel_v + h.off, z.data(), n * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
  for (double4* d : {A.acel2, A.acel3, A.acel4})
    if (d) CU(cudaMemcpyAsync(d + h.off, z.data(), n * sizeof(double4), cudaMemcpyHostToDevice, ctx->stream));
  std::vector<double2> mi(n);
  std::vector<int> t(n, 0);
  for (int i = 0; i < n; i++) {
    // set_mass (src/Set_Properties.f90:168-191)
    double m = mass[i];
    if (m == 0.0) mi[i] = make_double2(0.0, 0.0);
    else {
      double om = 1.0 / m;
      mi[i] = make_double2(om, std::sqrt(om));
    }
    if (type) {
      if (type[i] < 0 || type[i] >= h.ntypes) return fail(ctx, GEMSGPU_ERR_ARG, "upload: type out of range");
      t[i] = type[i];
    }
  }
  CU(cudaMemcpyAsync(A.mass + h.off, mass, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(A.minv + h.off, mi.data(), n * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaMemcpyAsync(A.type + h.off, t.data(), n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  CHK(push_sys(ctx, sys));
  BlockMap m;
  CHK(get_map(ctx, {sys}, BLOCK, 0, &m));
  k_refresh_fx<<<m.nblk, BLOCK, 0, ctx->stream>>>(A, m); ++ctx->launches;
  h.first = true;
  h.has_forces = false;
  CU(cudaGetLastError());
  return 0;
}

int gemsgpu_set_positions(gemsgpu_ctx* ctx, int sys, const double* pos) {
  CHK(check_sys(ctx, sys));
  if (!pos) return fail(ctx, GEMSGPU_ERR_ARG, "set_positions: NULL");
  SysHost& h = ctx->sys[sys];
  CHK(h2d_xyz(ctx, pos, ctx->A.pos + h.off, h.n));
  BlockMap m;
  CHK(get_map(ctx, {sys}, BLOCK, 0, &m));
  k_refresh_fx<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  CU(cudaStreamSynchronize(ctx->stream));
  h.pos_dirty = true;
  h.has_forces = false;
  return 0;
}

static int set_d4(gemsgpu_ctx* ctx, int sys, const double* src, double4* dst) {
  CHK(check_sys(ctx, sys));
  if (!src) return fail(ctx, GEMSGPU_ERR_ARG, "NULL array");
  SysHost& h = ctx->sys[sys];
  CHK(h2d_xyz(ctx, src, dst + h.off, h.n));
  CU(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int gemsgpu_set_velocities(gemsgpu_ctx* ctx, int sys, const double* vel) {
  if (!ctx) return GEMSGPU_ERR_ARG;
  return set_d4(ctx, sys, vel, ctx->A.vel);
}
int gemsgpu_set_accelerations(gemsgpu_ctx* ctx, int sys, const double* acel) {
  if (!ctx) return GEMSGPU_ERR_ARG;
  return set_d4(ctx, sys, acel, ctx->A.acel);
}

static int get_d4(gemsgpu_ctx* ctx, const SysHost& h, const double4* src, double* dst) {
  CHK(d2h_xyz(ctx, src + h.off, dst, h.n));
  CU(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int gemsgpu_download(gemsgpu_ctx* ctx, int sys, double* pos, double* vel, double* force,
                     double* epot_atoms) {
  CHK(check_sys(ctx, sys));
  const SysHost& h = ctx->sys[sys];
  if (pos) CHK(get_d4(ctx, h, ctx->A.pos, pos));
  if (vel) CHK(get_d4(ctx, h, ctx->A.vel, vel));
  if (force) CHK(get_d4(ctx, h, ctx->A.force, force));
  if (epot_atoms) {
    CU(cudaMemcpyAsync(epot_atoms, ctx->A.epot + h.off, h.n * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

int gemsgpu_download_acel(gemsgpu_ctx* ctx, int sys, double* acel) {
  CHK(check_sys(ctx, sys));
  if (!acel) return fail(ctx, GEMSGPU_ERR_ARG, "NULL array");
  return get_d4(ctx, ctx->sys[sys], ctx->A.acel, acel);
}

int gemsgpu_set_box(gemsgpu_ctx* ctx, int sys, int boxed, const double L[3], const int pbc[3]) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (boxed) {
    if (!L) return fail(ctx, GEMSGPU_ERR_ARG, "set_box: L required");
    for (int k = 0; k < 3; k++)
      if (!(L[k] > 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "set_box: L must be positive");
  }
  if (moving_box(h.d) && !boxed) return fail(ctx, GEMSGPU_ERR_STATE, "set_box: a piston system keeps its box");
  h.box_live = false;  // the given box replaces the one the pistons moved
  h.d.boxed = boxed ? 1 : 0;
  for (int k = 0; k < 3; k++) {
    h.d.L[k] = boxed ? L[k] : 0.0;
    h.d.pbc[k] = (boxed && pbc) ? (pbc[k] ? 1 : 0) : 0;
  }
  CHK(push_sys(ctx, sys));
  h.first = true;
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_set_skin(gemsgpu_ctx* ctx, int sys, double skin) {
  CHK(check_sys(ctx, sys));
  if (!(skin >= 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "skin must be >= 0");
  ctx->sys[sys].d.skin = skin;
  CHK(push_sys(ctx, sys));
  ctx->sys[sys].first = true;
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_set_skin_mode(gemsgpu_ctx* ctx, int sys, int mic) {
  CHK(check_sys(ctx, sys));
  ctx->sys[sys].d.skin_mic = mic ? 1 : 0;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

int gemsgpu_set_list_mode(gemsgpu_ctx* ctx, int sys, int half) {
  CHK(check_sys(ctx, sys));
  ctx->sys[sys].d.half = half ? 1 : 0;
  ctx->sys[sys].first = true;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

int gemsgpu_set_precision(gemsgpu_ctx* ctx, int sys, int prec) {
  CHK(check_sys(ctx, sys));
  if (prec != GEMSGPU_PREC_FP64 && prec != GEMSGPU_PREC_MIXED)
    return fail(ctx, GEMSGPU_ERR_ARG, "unknown precision %d", prec);
  if (prec != GEMSGPU_PREC_FP64 && ctx->sys[sys].d.ff == FF_LJ)
    for (const PairP& P : ctx->sys[sys].prm)
      if (P.v[8] == 2.0) return fail(ctx, GEMSGPU_ERR_STATE, "set_precision: sm1 pairs are FP64 only");
  ctx->sys[sys].d.prec = prec;
  if (ctx->sys[sys].d.ff == FF_TERSOFF) ctx->sys[sys].lanes = TS_TPA;  // two lanes are mixed-only
  CHK(push_sys(ctx, sys));
  BlockMap m;
  CHK(get_map(ctx, {sys}, BLOCK, 0, &m));
  k_refresh_fx<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  ctx->sys[sys].has_forces = false;
  invalidate(ctx);
  return 0;
}

int gemsgpu_set_lj(gemsgpu_ctx* ctx, int sys, int ti, int tj, double eps, double sigma,
                   double rcut, int shifted_force, double eshift) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (ti < 0 || tj < 0 || ti >= h.ntypes || tj >= h.ntypes || !(rcut > 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_lj: bad type pair or cut-off");
  if (h.d.ff != FF_NONE && h.d.ff != FF_LJ)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lj: system already has another force field");
  h.d.ff = FF_LJ;
  PairP P{};
  P.v[0] = eps;
  P.v[1] = sigma;
  P.v[2] = rcut;
  P.v[3] = rcut * rcut;
  if (shifted_force) {
    // plj_set (src/Pairs.F90:282-291)
    double x = sigma / rcut, x3 = x * x * x, x6 = x3 * x3;
    P.v[4] = 4.0 * eps * (x6 * x6 - x6);
    double s3 = sigma * sigma * sigma, s6 = s3 * s3, s12 = s6 * s6;
    double r3 = rcut * rcut * rcut, r6 = r3 * r3, r7 = r6 * rcut, r13 = r6 * r6 * rcut;
    P.v[5] = 24.0 * eps * (2.0 * (s12 / r13) - (s6 / r7));
    P.v[7] = 1.0;
  }
  P.v[6] = eshift;
  put_pair(h, ti, tj, P);
  h.ff_set = true;
  h.first = true;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_set_smatb(gemsgpu_ctx* ctx, int sys, int ti, int tj, double A, double xi, double p,
                      double q, double r0, double rci, double rce) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (ti < 0 || tj < 0 || ti >= h.ntypes || tj >= h.ntypes || !(rce > rci) || !(r0 > 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_smatb: bad type pair or cut-offs");
  if (h.d.ff != FF_NONE && h.d.ff != FF_SMATB)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_smatb: system already has another force field");
  h.d.ff = FF_SMATB;
  // smatb_set (src/TB.F90:106-170): tail coefficients of Logsdail et al. 2012
  PairP P{};
  double dcut = rce - rci;
  double ab = -1.0 / (dcut * dcut * dcut);
  double bb = -(q / r0) / (dcut * dcut);
  double cb = -((q / r0) * (q / r0)) / dcut;
  double aux = xi * std::exp(-q * (rci / r0 - 1.0));
  P.v[7] = aux * (12.0 * ab - 6.0 * bb + cb) / (2.0 * (dcut * dcut));
  P.v[8] = aux * (15.0 * ab - 7.0 * bb + cb) / dcut;
  P.v[9] = aux * (20.0 * ab - 8.0 * bb + cb) / 2.0;
  aux = A * std::exp(-p * (rci / r0 - 1.0));
  bb = -(p / r0) / (dcut * dcut);
  cb = -((p / r0) * (p / r0)) / dcut;
  P.v[10] = aux * (12.0 * ab - 6.0 * bb + cb) / (2.0 * (dcut * dcut));
  P.v[11] = aux * (15.0 * ab - 7.0 * bb + cb) / dcut;
  P.v[12] = aux * (20.0 * ab - 8.0 * bb + cb) / 2.0;
  P.v[0] = A; P.v[1] = xi; P.v[2] = p; P.v[3] = q; P.v[4] = r0; P.v[5] = rci; P.v[6] = rce;
  P.v[13] = 1.0;
  h.prm[ti * h.ntypes + tj] = P;
  h.prm[tj * h.ntypes + ti] = P;
  h.ff_set = true;
  h.first = true;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_set_tersoff(gemsgpu_ctx* ctx, int sys, const double prm[12]) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (!prm) return fail(ctx, GEMSGPU_ERR_ARG, "set_tersoff: NULL");
  if (h.d.ff != FF_NONE && h.d.ff != FF_TERSOFF)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_tersoff: system already has another force field");
  h.d.ff = FF_TERSOFF;
  TersoffP& T = h.d.ts;
  T.A = prm[0]; T.B = prm[1]; T.l1 = prm[2]; T.l2 = prm[3]; T.beta = prm[4]; T.n = prm[5];
  T.c = prm[6]; T.d = prm[7]; T.h = prm[8]; T.R = prm[9]; T.D = prm[10]; T.chi = prm[11];
  h.lanes = TS_TPA;
  if (!ctx->tersoff) {
    ctx->tersoff = true;
    CHK(tersoff_smem_attr(ctx));
    CHK(tersoff_records(ctx));
  }
  h.ff_set = true;
  h.first = true;
  CHK(push_sys(ctx, sys));
  BlockMap m;
  CHK(get_map(ctx, {sys}, BLOCK, 0, &m));
  k_refresh_fx<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_forces(gemsgpu_ctx* ctx, int sys, double* epot, int* rebuilt) {
  CHK(check_sys(ctx, sys));
  cudaSetDevice(ctx->device);
  int64_t before = 0;
  if (rebuilt) {
    CHK(read_states(ctx));
    before = ctx->h_st[sys].nupd;
  }
  CHK(interact_group(ctx, {sys}, true));
  if (epot || rebuilt) {
    std::vector<double> r;
    CHK(reduce_sys(ctx, {sys}, r));
    if (epot) *epot = r[0];
    if (rebuilt) {
      CHK(read_states(ctx));
      *rebuilt = ctx->h_st[sys].nupd > before;
    }
  }
  return 0;
}

int gemsgpu_update(gemsgpu_ctx* ctx, int sys) {
  CHK(check_sys(ctx, sys));
  ctx->sys[sys].first = true;
  std::vector<int> ss{sys};
  int need = estimate_cap(ctx->sys[sys]);
  if (ctx->A.lcap < need) CHK(grow_list(ctx, need));
  CHK(clear_status(ctx, ss));
  const int* sa;
  CHK(sys_array(ctx, ss, &sa));
  k_force_rebuild<<<1, 256, 0, ctx->stream>>>(ctx->A, sa, 1); ++ctx->launches;
  CHK(launch_rebuild(ctx, ss));
  CHK(read_states(ctx));
  if (ctx->h_st[sys].status & ST_OVERFLOW) {
    CHK(grow_list(ctx, ctx->h_st[sys].maxnn + 8));
    CHK(clear_status(ctx, ss));
    k_force_rebuild<<<1, 256, 0, ctx->stream>>>(ctx->A, sa, 1); ++ctx->launches;
    CHK(launch_rebuild(ctx, ss));
    CHK(read_states(ctx));
  }
  CHK(status_error(ctx, sys, ctx->h_st[sys].status));
  ctx->sys[sys].first = false;
  ctx->sys[sys].pos_dirty = false;
  return 0;
}

int gemsgpu_get_list(gemsgpu_ctx* ctx, int sys, int* nn, int* list, int cap, int* cap_needed) {
  CHK(check_sys(ctx, sys));
  const SysHost& h = ctx->sys[sys];
  std::vector<int> hn(h.n);
  // a half-list system's `list` holds the half list (hnn entries); flist
  // holds the full list the force kernels use
  CU(cudaMemcpyAsync(hn.data(), (h.d.half ? ctx->A.hnn : ctx->A.nn) + h.off, h.n * sizeof(int),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  int mx = 0;
  for (int v : hn) mx = std::max(mx, v);
  if (cap_needed) *cap_needed = mx;
  if (nn) memcpy(nn, hn.data(), h.n * sizeof(int));
  if (list) {
    if (cap < mx) return fail(ctx, GEMSGPU_ERR_ARG, "get_list: cap %d < needed %d", cap, mx);
    int rows = std::min(mx, ctx->A.lcap);
    std::vector<int> tmp((size_t)rows * h.n);
    if (rows > 0)
      CU(cudaMemcpy2DAsync(tmp.data(), h.n * sizeof(int), ctx->A.list + h.off, ctx->acap * sizeof(int),
                           h.n * sizeof(int), rows, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (int m = 0; m < cap; m++)
      for (int i = 0; i < h.n; i++)
        list[(size_t)m * h.n + i] = (m < rows && m < hn[i]) ? tmp[(size_t)m * h.n + i] - h.off : 0;
  }
  return 0;
}

int gemsgpu_get_nupd(gemsgpu_ctx* ctx, int sys, int64_t* nupd) {
  CHK(check_sys(ctx, sys));
  CHK(read_states(ctx));
  if (nupd) *nupd = ctx->h_st[sys].nupd;
  return 0;
}

int gemsgpu_set_vv(gemsgpu_ctx* ctx, int sys, double dt) {
  CHK(check_sys(ctx, sys));
  if (!(dt > 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "dt must be > 0");
  SysHost& h = ctx->sys[sys];
  h.d.integ = IT_VV;
  h.d.dt = dt;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

// the Nordsieck derivative arrays, zero, on first use
static int ensure_nord(gemsgpu_ctx* ctx) {
  Arena& A = ctx->A;
  if (A.acel2) return 0;
  for (double4** d : {&A.acel2, &A.acel3, &A.acel4}) {
    CHK(dalloc(ctx, d, (size_t)ctx->acap));
    CU(cudaMemsetAsync(*d, 0, (size_t)ctx->acap * sizeof(double4), ctx->stream));
  }
  return 0;
}

// `evolve pred_corr_5` (src/Integration.F90:143-145): nordsieck_predictor
// as step a, nordsieck_corrector as step b.  The derivatives acel..acel4
// carry over as the reference's atoms keep them (zero for new atoms, or
// from a .chp file).
int gemsgpu_set_pred_corr(gemsgpu_ctx* ctx, int sys, double dt) {
  CHK(check_sys(ctx, sys));
  if (!(dt > 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "dt must be > 0");
  CHK(ensure_nord(ctx));
  SysHost& h = ctx->sys[sys];
  h.d.integ = IT_NORD;
  h.d.dt = dt;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

// `evolve scalvel temp steps` and `evolve scalvel_after temp steps upto`
// (src/Integration.F90:205-213, set_scalvel :1271-1298): after the system's
// integrator, v *= (T0/T)^(0.5/steps) every step (scalvel_after: only while
// |T - T0| > upto T0).  upto < 0 selects scalvel.
int gemsgpu_set_scalvel(gemsgpu_ctx* ctx, int sys, double temp, int steps, double upto) {
  CHK(check_sys(ctx, sys));
  if (!(temp >= 0.0) || steps < 1) return fail(ctx, GEMSGPU_ERR_ARG, "set_scalvel: T >= 0, steps >= 1");
  SysDev& d = ctx->sys[sys].d;
  d.thermo = upto < 0.0 ? TH_SCALVEL : TH_SCALVEL_AFTER;
  d.th[0] = temp;
  d.th[1] = 0.5 / steps;
  d.th[2] = upto;
  d.th[3] = kB_ui;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

// `evolve andersen temp [nu]` (src/Integration.F90:214-217, set_andersen
// :1343-1364): after the system's integrator, each atom collides with
// probability nu dt and takes new velocities of scale sqrt(kB T / (3N)^2)
// / sqrt(m) (the reference's factor), from a Philox stream keyed by seed.
int gemsgpu_set_andersen(gemsgpu_ctx* ctx, int sys, double temp, double nu, uint64_t seed) {
  CHK(check_sys(ctx, sys));
  if (!(temp >= 0.0) || !(nu >= 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "set_andersen: T >= 0, nu >= 0");
  SysHost& h = ctx->sys[sys];
  SysDev& d = h.d;
  d.thermo = TH_ANDERSEN;
  const double dof = 3.0 * h.n;
  d.th[0] = std::sqrt(kB_ui * temp / (dof * dof));
  d.th[1] = nu;
  d.th_seed = seed ^ 0x9E3779B97F4A7C15ull;  // apart from the integrator's stream
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

int gemsgpu_clear_thermostat(gemsgpu_ctx* ctx, int sys) {
  CHK(check_sys(ctx, sys));
  ctx->sys[sys].d.thermo = TH_NONE;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

// `evolve brownian temp gama` (src/Integration.F90:146-149): set_cbrownian
// (:834-853); step a does nothing, step b is cbrownian (:855-882)
int gemsgpu_set_brownian(gemsgpu_ctx* ctx, int sys, double dt, double temp, double gama, uint64_t seed) {
  CHK(check_sys(ctx, sys));
  if (!(dt > 0.0) || !(gama > 0.0) || !(temp >= 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_brownian: dt>0, gamma>0, T>=0");
  SysHost& h = ctx->sys[sys];
  SysDev& d = h.d;
  d.integ = IT_BROWN;
  d.dt = dt;
  d.bd_fac1 = dt / gama;
  d.bd_fac2 = std::sqrt(2.0 * kB_ui * temp * d.bd_fac1);
  h.temp = temp;
  d.seed = seed;
  d.use_ext_normals = 0;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

int gemsgpu_set_ermak(gemsgpu_ctx* ctx, int sys, double dt, double gama, double temp, uint64_t seed) {
  CHK(check_sys(ctx, sys));
  if (!(dt > 0.0) || !(gama > 0.0) || !(temp >= 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_ermak: dt>0, gamma>0, T>=0");
  SysHost& h = ctx->sys[sys];
  SysDev& d = h.d;
  // set_ermak (src/Integration.F90:909-961)
  d.integ = IT_ERMAK;
  d.dt = dt;
  d.cc0 = std::exp(-dt * gama);
  d.cc1 = (1.0 - d.cc0) / gama;
  d.cc2 = (1.0 - d.cc1 / dt) / gama;
  d.sdr = std::sqrt(dt / gama * (2.0 - (3.0 - 4.0 * d.cc0 + d.cc0 * d.cc0) / (dt * gama)));
  d.sdv = std::sqrt(1.0 - d.cc0 * d.cc0);
  d.crv1 = (1.0 - d.cc0) * (1.0 - d.cc0) / (gama * d.sdr * d.sdv);
  d.crv2 = std::sqrt(1.0 - (d.crv1 * d.crv1));
  d.skt = std::sqrt(kB_ui * temp);
  h.temp = temp;
  d.seed = seed;
  d.use_ext_normals = 0;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

int gemsgpu_set_ermak_normals(gemsgpu_ctx* ctx, int sys, const double* normals) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (!normals) {
    h.d.use_ext_normals = 0;
  } else {
    CU(cudaMemcpyAsync(ctx->A.ext_normals + (size_t)6 * h.off, normals, (size_t)6 * h.n * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
    h.d.use_ext_normals = 1;
  }
  CHK(push_sys(ctx, sys));
  CU(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int gemsgpu_set_fire(gemsgpu_ctx* ctx, int sys, double dt0, double dtmax) {
  CHK(check_sys(ctx, sys));
  if (!(dt0 > 0.0) || !(dtmax >= dt0)) return fail(ctx, GEMSGPU_ERR_ARG, "set_fire: 0 < dt0 <= dtmax");
  SysHost& h = ctx->sys[sys];
  h.d.integ = IT_FIRE;
  h.d.dt = dt0;
  h.d.fire_dtmax = dtmax;
  h.d.fire_fmax = 0.0;
  h.d.fire_maxit = 0x7fffffff;
  CHK(push_sys(ctx, sys));
  SysState z{};
  CHK(read_states(ctx));
  z.nupd = ctx->h_st[sys].nupd;
  z.fire_dt = dt0;
  z.fire_alpha = 0.1;
  CU(cudaMemcpyAsync(ctx->A.st + sys, &z, sizeof(z), cudaMemcpyHostToDevice, ctx->stream));
  std::vector<double4> zero(h.n, make_double4(0, 0, 0, 0));
  CU(cudaMemcpyAsync(ctx->A.vel + h.off, zero.data(), h.n * sizeof(double4), cudaMemcpyHostToDevice,
                     ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  invalidate(ctx);
  return 0;
}

// slj_set (src/Pairs.F90:374-401): LJ core to rs, then the tail
// sa4 (r - rc)^4 + sa8 (r - rc)^8 that reaches zero with zero slope at rc
int gemsgpu_set_slj(gemsgpu_ctx* ctx, int sys, int ti, int tj, double eps, double sigma, double rs) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (ti < 0 || tj < 0 || ti >= h.ntypes || tj >= h.ntypes || !(rs > 0.0) || !(sigma > 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_slj: bad type pair, sigma or rs");
  if (h.d.ff != FF_NONE && h.d.ff != FF_LJ)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_slj: system already has another force field");
  const double x = sigma / rs, x3 = x * x * x, s_dr = x3 * x3;
  const double urs = 4.0 * eps * (s_dr * s_dr - s_dr);
  const double dudrs = -eps * (48.0 * s_dr - 24.0) * s_dr / rs;
  const double rc = rs - 32.0 * urs / (11.0 * dudrs);
  if (!(rc > rs)) return fail(ctx, GEMSGPU_ERR_ARG, "set_slj: rs must lie in the attractive part of the core");
  const double d = rc - rs, d4 = d * d * d * d;
  h.d.ff = FF_LJ;
  PairP P{};
  P.v[0] = eps;
  P.v[1] = sigma;
  P.v[2] = rc;
  P.v[3] = rc * rc;
  P.v[8] = 1.0;
  P.v[9] = (8.0 * urs + d * dudrs) / (4 * d4);
  P.v[10] = -(4.0 * urs + d * dudrs) / (4 * (d4 * d4));
  P.v[11] = rs;
  put_pair(h, ti, tj, P);
  h.ff_set = true;
  h.first = true;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

// wca_set (src/Pairs.F90:495-506): LJ cut at 2**(1./6.) sigma, the
// exponent a single-precision literal, shifted up by eps (wca_interact,
// Pairs.F90:508-589)
int gemsgpu_set_wca(gemsgpu_ctx* ctx, int sys, int ti, int tj, double eps, double sigma) {
  if (!(sigma > 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "set_wca: sigma must be positive");
  return gemsgpu_set_lj(ctx, sys, ti, tj, eps, sigma, std::pow(2.0, (double)(1.0f / 6.0f)) * sigma, 0, -eps);
}

// sm1_set (src/Pairs.F90:916-923): a smooth step of depth eps (eV) from r1
// to r2 = the cut-off (sm1_interact, Pairs.F90:925-1011)
int gemsgpu_set_sm1(gemsgpu_ctx* ctx, int sys, int ti, int tj, double r1, double r2, double eps) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (ti < 0 || tj < 0 || ti >= h.ntypes || tj >= h.ntypes || !(r1 > 0.0) || !(r2 > r1))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_sm1: bad type pair or radii");
  if (h.d.ff != FF_NONE && h.d.ff != FF_LJ)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_sm1: system already has another force field");
  if (h.d.prec != PREC_FP64) return fail(ctx, GEMSGPU_ERR_STATE, "set_sm1: FP64 systems only");
  h.d.ff = FF_LJ;
  PairP P{};
  P.v[0] = eps;
  P.v[1] = r1;
  P.v[2] = r2;
  P.v[3] = r2 * r2;
  P.v[8] = 2.0;
  P.v[11] = r1;
  put_pair(h, ti, tj, P);
  h.ff_set = true;
  h.first = true;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

// `interact g1 feels g2` (src/Interaction.f90:69-76, 128-131): half and
// newton off, so only the atoms of g1 feel the pair; with one type per
// group, the pair (ti, tj) keeps acting on type ti and stops acting on tj
int gemsgpu_set_feels(gemsgpu_ctx* ctx, int sys, int ti, int tj) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (ti < 0 || tj < 0 || ti >= h.ntypes || tj >= h.ntypes)
    return fail(ctx, GEMSGPU_ERR_ARG, "set_feels: bad type pair");
  if (h.d.ff != FF_LJ) return fail(ctx, GEMSGPU_ERR_STATE, "set_feels: pair potentials only");
  if (h.d.virial) return fail(ctx, GEMSGPU_ERR_STATE, "set_feels: one-sided pairs have no pair virial");
  if (ti == tj) return 0;
  if (h.deaf.size() != h.prm.size()) h.deaf.assign(h.prm.size(), 0);
  h.deaf[tj * h.ntypes + ti] = 1;
  h.prm[tj * h.ntypes + ti] = PairP{};
  h.has_forces = false;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_set_virial(gemsgpu_ctx* ctx, int sys, int on) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (on && h.d.ff != FF_LJ && h.d.ff != FF_SMATB)
    return fail(ctx, GEMSGPU_ERR_STATE, "virial: lj, plj, slj and SMA-TB systems only");
  if (on && one_sided(h))
    return fail(ctx, GEMSGPU_ERR_STATE, "virial: one-sided (feels) pairs have no pair virial");
  if (!on && moving_box(h.d)) return fail(ctx, GEMSGPU_ERR_STATE, "virial: the piston needs it");
  h.d.virial = on ? 1 : 0;
  h.has_forces = false;
  CHK(push_sys(ctx, sys));
  invalidate(ctx);
  return 0;
}

namespace {
// pressure units (src/Constants.F90:186-193): atm -> internal on input,
// internal -> atm on output (write_pressure, src/Output.F90:767-770)
double atm_ui() { return 1.01325 * 1.e5 * ((1.0 / (UI_EV * 1.60219e-19)) * 1e-30); }
double ui_atm() { return 1.0 / ((1.0 / (UI_EV * 1.60219e-19)) * 1e-30) * 1e-5 * (1.0 / 1.01325); }
}  // namespace

// set_lgf (src/Integration.F90:486-525): the isotropic G-JF piston
int gemsgpu_set_lgf(gemsgpu_ctx* ctx, int sys, double dt, double temp, double press_atm, double pgama0,
                    double pgamav, double pmass, uint64_t seed) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (!(dt > 0.0) || !(temp >= 0.0) || !(pgama0 >= 0.0) || !(pgamav >= 0.0) || !(pmass > 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_lgf: dt>0, T>=0, gammas>=0, piston mass>0");
  if (!h.d.boxed || !h.d.pbc[0] || !h.d.pbc[1] || !h.d.pbc[2])
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lgf: the piston needs a box periodic in x, y and z");
  if (h.d.ff != FF_LJ && h.d.ff != FF_SMATB)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lgf: lj, plj, slj and SMA-TB systems only");
  if (one_sided(h))
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lgf: one-sided (feels) pairs have no pair virial");
  SysDev& d = h.d;
  d.integ = IT_LGF;
  d.dt = dt;
  d.lgf_fac0 = std::sqrt(2.0 * pgama0 * kB_ui * temp * dt);
  d.lgf_facg0 = 0.5 * dt * pgama0;
  d.lgf_kin = h.n * temp * kB_ui;
  d.lgf_press = press_atm * atm_ui();
  d.lgf_ipm = 1.0 / pmass;
  d.lgf_bv = 1.0 / (1.0 + 0.5 * dt * d.lgf_ipm * pgamav);
  d.lgf_facv = std::sqrt(2.0 * pgamav * kB_ui * temp * dt);
  d.lgf_av = (1.0 - 0.5 * dt * d.lgf_ipm * pgamav) * d.lgf_bv;
  d.virial = 1;
  d.seed = seed;
  d.use_ext_normals = 0;
  h.temp = temp;
  h.has_forces = false;  // the first piston step needs the virial
  CHK(push_sys(ctx, sys));
  CHK(read_states(ctx));
  SysState st = ctx->h_st[sys];
  st.lgf_phase = 0;
  st.lgf_pf = st.lgf_pvel = st.lgf_rangv = 0.0;
  for (int k = 0; k < 3; k++) st.box_b[k] = d.L[k];
  CU(cudaMemcpyAsync(ctx->A.st + sys, &st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

int gemsgpu_set_lgf_normals(gemsgpu_ctx* ctx, int sys, const double* normals) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (h.d.integ != IT_LGF && h.d.integ != IT_AXES && h.d.integ != IT_LKD)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lgf_normals: not a piston or per-coordinate system");
  if (!normals) {
    h.d.use_ext_normals = 0;
  } else if (h.d.integ == IT_LKD) {
    // stepa: a pair per atom coordinate, the piston's; stepb: the piston's,
    // a pair per atom coordinate (first values used)
    std::vector<double> nrm(6 * (size_t)h.n, 0.0);
    const double* q = normals;
    for (int i = 0; i < h.n; i++)
      for (int k = 0; k < 3; k++, q += 2) nrm[6 * (size_t)i + 2 * k] = q[0];
    double pist[3] = {q[0], q[2], 0.0};
    q += 4;
    for (int i = 0; i < h.n; i++)
      for (int k = 0; k < 3; k++, q += 2) nrm[6 * (size_t)i + 2 * k + 1] = q[0];
    CU(cudaMemcpyAsync(ctx->A.ext_normals + (size_t)6 * h.off, nrm.data(), nrm.size() * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->A.st[sys].ax_ext, pist, sizeof(pist), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    h.d.use_ext_normals = 1;
  } else if (h.d.integ == IT_AXES) {
    // the pairs in draw order, scattered to (atom, coordinate) slots
    std::vector<double> nrm(6 * (size_t)h.n, 0.0);
    double pist[3] = {0, 0, 0};
    const double* q = normals;
    for (int d : h.ax_order) {
      if (h.d.ax_mode[d] == AX_FLEX) {
        pist[d] = q[0];
        q += 2;
      }
      for (int i = 0; i < h.n; i++, q += 2) {
        nrm[6 * (size_t)i + 2 * d] = q[0];
        nrm[6 * (size_t)i + 2 * d + 1] = q[1];
      }
    }
    CU(cudaMemcpyAsync(ctx->A.ext_normals + (size_t)6 * h.off, nrm.data(), nrm.size() * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->A.st[sys].ax_ext, pist, sizeof(pist), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    h.d.use_ext_normals = 1;
  } else {
    CU(cudaMemcpyAsync(ctx->A.ext_normals + (size_t)6 * h.off, normals + 2, (size_t)6 * h.n * sizeof(double),
                       cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(&ctx->A.st[sys].ext_piston, normals, sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
    h.d.use_ext_normals = 1;
  }
  CHK(push_sys(ctx, sys));
  CU(cudaStreamSynchronize(ctx->stream));
  return 0;
}

// set_lkd (src/Integration.F90:329-355): the Langevin piston of Kolb &
// Dunweg
int gemsgpu_set_lkd(gemsgpu_ctx* ctx, int sys, double dt, double temp, double press_atm, double pgama0,
                    double pgamav, double pmass, uint64_t seed) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (!(dt > 0.0) || !(temp >= 0.0) || !(pgama0 >= 0.0) || !(pgamav >= 0.0) || !(pmass > 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "set_lkd: dt>0, T>=0, gammas>=0, piston mass>0");
  if (!h.d.boxed || !h.d.pbc[0] || !h.d.pbc[1] || !h.d.pbc[2])
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lkd: the piston needs a box periodic in x, y and z");
  if (h.d.ff != FF_LJ && h.d.ff != FF_SMATB)
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lkd: lj, plj, slj and SMA-TB systems only");
  if (one_sided(h))
    return fail(ctx, GEMSGPU_ERR_STATE, "set_lkd: one-sided (feels) pairs have no pair virial");
  SysDev& d = h.d;
  d.integ = IT_LKD;
  d.dt = dt;
  d.lkd[0] = std::sqrt(kB_ui * temp * dt * pgama0);
  d.lkd[1] = std::sqrt(kB_ui * temp * dt * pgamav);
  d.lkd[2] = press_atm * atm_ui();
  d.lkd[3] = pgama0;
  d.lkd[4] = pgamav;
  d.lkd[5] = pmass;
  d.virial = 1;
  d.seed = seed;
  d.use_ext_normals = 0;
  h.temp = temp;
  h.has_forces = false;  // the piston needs the virial
  CHK(push_sys(ctx, sys));
  CHK(read_states(ctx));
  SysState st = ctx->h_st[sys];
  st.lgf_pvel = 0.0;
  for (int k = 0; k < 3; k++) st.box_b[k] = d.L[k];
  CU(cudaMemcpyAsync(ctx->A.st + sys, &st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

// one per-coordinate integrator more (IT_AXES); a system that had another
// integrator starts an empty set
static int add_axis(gemsgpu_ctx* ctx, int sys, int axis, double dt, int mode, const double p[8], uint64_t seed) {
  SysHost& h = ctx->sys[sys];
  SysDev& d = h.d;
  if (d.integ != IT_AXES) {
    d.integ = IT_AXES;
    for (int k = 0; k < 3; k++) d.ax_mode[k] = AX_NONE;
    h.ax_order.clear();
    d.dt = dt;
  }
  if (d.ax_mode[axis] != AX_NONE)
    return fail(ctx, GEMSGPU_ERR_STATE, "coordinate %d already has an integrator", axis);
  if (dt != d.dt) return fail(ctx, GEMSGPU_ERR_ARG, "per-coordinate integrators share one dt");
  d.ax_mode[axis] = mode;
  for (int k = 0; k < 8; k++) d.ax_p[axis][k] = p[k];
  h.ax_order.push_back(axis);
  d.seed = seed;
  d.use_ext_normals = 0;
  if (mode == AX_FLEX) {
    d.virial = 1;
    h.has_forces = false;  // the first piston step needs the virial
  }
  CHK(push_sys(ctx, sys));
  CHK(read_states(ctx));
  SysState st = ctx->h_st[sys];
  st.ax_phase[axis] = 0;
  st.ax_pf[axis] = st.ax_pvel[axis] = st.ax_rangv[axis] = 0.0;
  for (int k = 0; k < 3; k++) st.box_b[k] = d.L[k];
  CU(cudaMemcpyAsync(ctx->A.st + sys, &st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
  CU(cudaStreamSynchronize(ctx->stream));
  invalidate(ctx);
  drop_maps(ctx);
  return 0;
}

// set_lgf_flex (src/Integration.F90:652-696): a G-JF piston on one length
int gemsgpu_add_lgf_axis(gemsgpu_ctx* ctx, int sys, int axis, double dt, double temp, double press_atm,
                         double pgama0, double pgamav, double pmass, uint64_t seed) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (axis < 0 || axis > 2) return fail(ctx, GEMSGPU_ERR_ARG, "add_lgf_axis: axis 0, 1 or 2");
  if (!(dt > 0.0) || !(temp >= 0.0) || !(pgama0 >= 0.0) || !(pgamav >= 0.0) || !(pmass > 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "add_lgf_axis: dt>0, T>=0, gammas>=0, piston mass>0");
  if (!h.d.boxed || !h.d.pbc[axis])
    return fail(ctx, GEMSGPU_ERR_STATE, "add_lgf_axis: the piston needs a box periodic along its axis");
  if (h.d.ff != FF_LJ && h.d.ff != FF_SMATB)
    return fail(ctx, GEMSGPU_ERR_STATE, "add_lgf_axis: lj, plj, slj and SMA-TB systems only");
  if (one_sided(h))
    return fail(ctx, GEMSGPU_ERR_STATE, "add_lgf_axis: one-sided (feels) pairs have no pair virial");
  double p[8];
  p[0] = std::sqrt(2.0 * pgama0 * kB_ui * temp * dt);
  p[1] = 0.5 * dt * pgama0;
  p[2] = h.n * temp * kB_ui;
  p[3] = press_atm * atm_ui();
  p[4] = 1.0 / pmass;
  p[5] = 1.0 / (1.0 + 0.5 * dt * p[4] * pgamav);
  p[6] = std::sqrt(2.0 * pgamav * kB_ui * temp * dt);
  p[7] = (1.0 - 0.5 * dt * p[4] * pgamav) * p[5];
  return add_axis(ctx, sys, axis, dt, AX_FLEX, p, seed);
}

// set_ermak with a coordinate (src/Integration.F90:909-961): Ermak
// dynamics of one coordinate
int gemsgpu_add_ermak_axis(gemsgpu_ctx* ctx, int sys, int axis, double dt, double gama, double temp,
                           uint64_t seed) {
  CHK(check_sys(ctx, sys));
  if (axis < 0 || axis > 2) return fail(ctx, GEMSGPU_ERR_ARG, "add_ermak_axis: axis 0, 1 or 2");
  if (!(dt > 0.0) || !(gama > 0.0) || !(temp >= 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "add_ermak_axis: dt>0, gamma>0, T>=0");
  double p[8];
  p[0] = std::exp(-dt * gama);
  p[1] = (1.0 - p[0]) / gama;
  p[2] = (1.0 - p[1] / dt) / gama;
  p[3] = std::sqrt(dt / gama * (2.0 - (3.0 - 4.0 * p[0] + p[0] * p[0]) / (dt * gama)));
  p[4] = std::sqrt(1.0 - p[0] * p[0]);
  p[5] = (1.0 - p[0]) * (1.0 - p[0]) / (gama * p[3] * p[4]);
  p[6] = std::sqrt(1.0 - (p[5] * p[5]));
  p[7] = std::sqrt(kB_ui * temp);
  return add_axis(ctx, sys, axis, dt, AX_ERMAK, p, seed);
}

int gemsgpu_get_box(gemsgpu_ctx* ctx, int sys, double L[3]) {
  CHK(check_sys(ctx, sys));
  if (!L) return fail(ctx, GEMSGPU_ERR_ARG, "get_box: NULL");
  SysHost& h = ctx->sys[sys];
  if (h.box_live) return live_box(ctx, sys, L);
  for (int k = 0; k < 3; k++) L[k] = h.d.L[k];
  return 0;
}

static void sym9(const double w[6], double f, double* out) {
  const int idx[9] = {0, 3, 4, 3, 1, 5, 4, 5, 2};
  for (int k = 0; k < 9; k++) out[k] = w[idx[k]] * f;
}

// inq_virial (src/Inq_Properties.F90:439-527) of the last force evaluation,
// eV, row-major 3x3
int gemsgpu_virial(gemsgpu_ctx* ctx, int sys, double* out9) {
  CHK(check_sys(ctx, sys));
  if (!out9) return fail(ctx, GEMSGPU_ERR_ARG, "virial: NULL");
  const SysHost& h = ctx->sys[sys];
  if (!h.d.virial || (h.d.ff != FF_LJ && h.d.ff != FF_SMATB) || !h.has_forces)
    return fail(ctx, GEMSGPU_ERR_STATE, "virial: not computed (set_virial, forces)");
  CHK(read_states(ctx));
  sym9(ctx->h_st[sys].vir, UI_EV, out9);
  return 0;
}

// inq_pressure (src/Inq_Properties.F90:529-573): (sum m v v + W) / V, atm
int gemsgpu_pressure(gemsgpu_ctx* ctx, int sys, double* out9) {
  CHK(check_sys(ctx, sys));
  if (!out9) return fail(ctx, GEMSGPU_ERR_ARG, "pressure: NULL");
  const SysHost& h = ctx->sys[sys];
  if (!h.d.virial || (h.d.ff != FF_LJ && h.d.ff != FF_SMATB) || !h.has_forces)
    return fail(ctx, GEMSGPU_ERR_STATE, "pressure: virial not computed");
  if (!h.d.boxed) return fail(ctx, GEMSGPU_ERR_STATE, "pressure: no box");
  BlockMap m;
  CHK(get_map(ctx, {sys}, BLOCK, 0, &m));
  k_kin_tensor<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  CU(cudaGetLastError());
  CHK(read_states(ctx));
  double L[3];
  CHK(gemsgpu_get_box(ctx, sys, L));
  const SysState& st = ctx->h_st[sys];
  double w[6];
  for (int k = 0; k < 6; k++) w[k] = st.ktens[k] + st.vir[k];
  sym9(w, ui_atm() / (L[0] * L[1] * L[2]), out9);
  return 0;
}

int gemsgpu_step_a(gemsgpu_ctx* ctx, int sys) {
  CHK(check_sys(ctx, sys));
  SysHost& h = ctx->sys[sys];
  if (h.d.integ == IT_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "no integrator");
  CHK(launch_step_a(ctx, {sys}));
  h.pos_dirty = false;
  return 0;
}

int gemsgpu_step_b(gemsgpu_ctx* ctx, int sys) {
  CHK(check_sys(ctx, sys));
  if (ctx->sys[sys].d.integ == IT_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "no integrator");
  CHK(launch_step_b(ctx, {sys}));
  CU(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int gemsgpu_md_steps(gemsgpu_ctx* ctx, int sys, int nsteps) {
  CHK(check_sys(ctx, sys));
  if (nsteps < 0) return fail(ctx, GEMSGPU_ERR_ARG, "nsteps < 0");
  cudaSetDevice(ctx->device);
  return md_group(ctx, {sys}, nsteps);
}

int gemsgpu_energy(gemsgpu_ctx* ctx, int sys, double* epot_ev, double* ekin_ev, double* temp) {
  CHK(check_sys(ctx, sys));
  std::vector<double> r;
  CHK(reduce_sys(ctx, {sys}, r));
  const SysHost& h = ctx->sys[sys];
  if (epot_ev) *epot_ev = r[0] * UI_EV;
  if (ekin_ev) *ekin_ev = r[1] * UI_EV;
  if (temp) *temp = 2.0 * r[1] / (kB_ui * (3.0 * h.n));
  return 0;
}

int gemsgpu_fmax(gemsgpu_ctx* ctx, int sys, double* fmax_ev) {
  CHK(check_sys(ctx, sys));
  std::vector<double> r;
  CHK(reduce_sys(ctx, {sys}, r));
  if (fmax_ev) *fmax_ev = std::sqrt(r[2]) * UI_EV;
  return 0;
}

static int sys_list(gemsgpu_ctx* ctx, const int* sys, int nsys, std::vector<int>& ss) {
  if (!ctx || !sys || nsys <= 0) return fail(ctx, GEMSGPU_ERR_ARG, "empty system list");
  ss.assign(sys, sys + nsys);
  for (int s : ss) CHK(check_sys(ctx, s));
  std::vector<int> t = ss;
  std::sort(t.begin(), t.end());
  if (std::unique(t.begin(), t.end()) != t.end())
    return fail(ctx, GEMSGPU_ERR_ARG, "duplicate system in batch");
  return 0;
}

int gemsgpu_batch_md_steps(gemsgpu_ctx* ctx, const int* sys, int nsys, int nsteps) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  cudaSetDevice(ctx->device);
  return md_group(ctx, ss, nsteps);
}

int gemsgpu_batch_fire(gemsgpu_ctx* ctx, const int* sys, int nsys, double fmax, int maxit, int* iters) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  if (!(fmax > 0.0) || maxit <= 0) return fail(ctx, GEMSGPU_ERR_ARG, "batch_fire: fmax>0, maxit>0");
  cudaSetDevice(ctx->device);
  for (int s : ss) {
    SysHost& h = ctx->sys[s];
    if (h.d.integ != IT_FIRE) return fail(ctx, GEMSGPU_ERR_STATE, "system %d is not set up for FIRE", s);
    h.d.fire_fmax = fmax;
    h.d.fire_maxit = maxit;
    CHK(push_sys(ctx, s));
  }
  invalidate(ctx);
  // converged systems freeze on the device; poll between chunks
  CHK(interact_group(ctx, ss, true));
  {
    std::vector<double> r;
    CHK(reduce_sys(ctx, ss, r));
    CHK(read_states(ctx));
    for (size_t k = 0; k < ss.size(); k++) {
      SysState st = ctx->h_st[ss[k]];
      st.fire_done = std::sqrt(r[4 * k + 2]) * UI_EV < fmax ? 1 : 0;
      CU(cudaMemcpyAsync(ctx->A.st + ss[k], &st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
    }
  }
  int total = 0;
  bool uniform = true;
  int64_t atoms = 0, cells = 0;
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    uniform &= h.d.ff == ctx->sys[ss[0]].d.ff && h.d.prec == ctx->sys[ss[0]].d.prec &&
               h.lanes == ctx->sys[ss[0]].lanes && h.variant == ctx->sys[ss[0]].variant;
    atoms += h.n;
    cells += h.d.use_cells ? h.d.ncell : 0;
  }
  if (uniform) {
    // converged systems leave the pool's active set between chunks
    const SysHost& h0 = ctx->sys[ss[0]];
    gemsgpu_pool* P = nullptr;
    CHK(gemsgpu_pool_create(ctx, (int)ss.size(), atoms, cells, h0.d.ff, h0.d.prec, h0.lanes, h0.variant,
                            CHUNK, &P));
    int rc = 0;
    for (;;) {
      if ((rc = read_states(ctx))) break;
      std::vector<int> act;
      for (int s : ss)
        if (!ctx->h_st[s].fire_done) act.push_back(s);
      if (act.empty() || total >= maxit) break;
      if ((rc = gemsgpu_pool_set(P, act.data(), (int)act.size()))) break;
      if ((rc = gemsgpu_pool_run(P, 1))) break;
      total += CHUNK;
    }
    gemsgpu_pool_destroy(P);
    CHK(rc);
  } else {
    for (;;) {
      CHK(read_states(ctx));
      bool all = true;
      for (int s : ss) all &= ctx->h_st[s].fire_done != 0;
      if (all || total >= maxit) break;
      int k = std::min(CHUNK, maxit - total);
      CHK(clear_status(ctx, ss));
      CHK(launch_graph(ctx, ss, k));
      total += k;
      CHK(read_states(ctx));
      for (int s : ss) {
        int st = ctx->h_st[s].status;
        if (st & ST_FATAL) return status_error(ctx, s, st);
        if (st & ST_OVERFLOW) {
          CHK(grow_list(ctx, ctx->h_st[s].maxnn + 16));
          const int* sa;
          CHK(sys_array(ctx, ss, &sa));
          k_force_rebuild<<<((int)ss.size() + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, sa, (int)ss.size());
          ++ctx->launches;
          CHK(clear_status(ctx, ss));
          CHK(launch_rebuild(ctx, ss));
          CHK(launch_forces(ctx, ss));
          break;
        }
      }
    }
  }
  CHK(read_states(ctx));
  if (iters)
    for (size_t k = 0; k < ss.size(); k++) iters[k] = ctx->h_st[ss[k]].fire_iter;
  return 0;
}

int gemsgpu_batch_energy(gemsgpu_ctx* ctx, const int* sys, int nsys, double* epot_ev, double* ekin_ev,
                         double* temp) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  std::vector<double> r;
  CHK(reduce_sys(ctx, ss, r));
  for (int k = 0; k < nsys; k++) {
    if (epot_ev) epot_ev[k] = r[4 * k] * UI_EV;
    if (ekin_ev) ekin_ev[k] = r[4 * k + 1] * UI_EV;
    if (temp) temp[k] = 2.0 * r[4 * k + 1] / (kB_ui * (3.0 * ctx->sys[ss[k]].n));
  }
  return 0;
}

// Host <-> device state of many systems in one call: every copy and repack
// is queued on the context's stream and the call synchronises once (the
// per-system calls synchronise each time).  The staging buffer holds two
// regions of 3 doubles per atom of the whole set, so no copy waits for
// another's repack.
int gemsgpu_batch_set_state(gemsgpu_ctx* ctx, const int* sys, int nsys, const double* const* pos,
                            const double* const* vel) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  if (!pos && !vel) return fail(ctx, GEMSGPU_ERR_ARG, "batch_set_state: nothing to set");
  cudaSetDevice(ctx->device);
  int64_t total = 0;
  for (int s : ss) total += ctx->sys[s].n;
  CHK(ensure_stage(ctx, 2 * total));
  int64_t o = 0;
  std::vector<int> moved;
  for (int k = 0; k < nsys; k++) {
    SysHost& h = ctx->sys[ss[k]];
    double* sp = ctx->stage + 3 * o;
    double* sv = ctx->stage + 3 * (total + o);
    if (pos && pos[k]) {
      CU(cudaMemcpyAsync(sp, pos[k], (size_t)3 * h.n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      k_unpack3<<<(h.n + 255) / 256, 256, 0, ctx->stream>>>(sp, ctx->A.pos + h.off, h.n); ++ctx->launches;
      moved.push_back(ss[k]);
    }
    if (vel && vel[k]) {
      CU(cudaMemcpyAsync(sv, vel[k], (size_t)3 * h.n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      k_unpack3<<<(h.n + 255) / 256, 256, 0, ctx->stream>>>(sv, ctx->A.vel + h.off, h.n); ++ctx->launches;
    }
    o += h.n;
  }
  if (!moved.empty()) {
    BlockMap m;
    CHK(get_map(ctx, moved, BLOCK, 0, &m));
    k_refresh_fx<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  }
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(ctx->stream));
  for (int s : moved) {
    ctx->sys[s].pos_dirty = true;
    ctx->sys[s].has_forces = false;
  }
  return 0;
}

int gemsgpu_batch_get_state(gemsgpu_ctx* ctx, const int* sys, int nsys, double* const* pos, double* const* vel,
                            double* epot_ev, double* ekin_ev, double* temp) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  cudaSetDevice(ctx->device);
  int64_t total = 0;
  for (int s : ss) total += ctx->sys[s].n;
  CHK(ensure_stage(ctx, 2 * total));
  int64_t o = 0;
  for (int k = 0; k < nsys; k++) {
    const SysHost& h = ctx->sys[ss[k]];
    double* sp = ctx->stage + 3 * o;
    double* sv = ctx->stage + 3 * (total + o);
    if (pos && pos[k]) {
      k_pack3<<<(h.n + 255) / 256, 256, 0, ctx->stream>>>(ctx->A.pos + h.off, sp, h.n); ++ctx->launches;
      CU(cudaMemcpyAsync(pos[k], sp, (size_t)3 * h.n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (vel && vel[k]) {
      k_pack3<<<(h.n + 255) / 256, 256, 0, ctx->stream>>>(ctx->A.vel + h.off, sv, h.n); ++ctx->launches;
      CU(cudaMemcpyAsync(vel[k], sv, (size_t)3 * h.n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    o += h.n;
  }
  CU(cudaGetLastError());
  if (epot_ev || ekin_ev || temp) {
    std::vector<double> r;
    CHK(reduce_sys(ctx, ss, r));  // synchronises the stream
    for (int k = 0; k < nsys; k++) {
      if (epot_ev) epot_ev[k] = r[4 * k] * UI_EV;
      if (ekin_ev) ekin_ev[k] = r[4 * k + 1] * UI_EV;
      if (temp) temp[k] = 2.0 * r[4 * k + 1] / (kB_ui * (3.0 * ctx->sys[ss[k]].n));
    }
  } else {
    CU(cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

static int sys_list(gemsgpu_ctx* ctx, const int* sys, int nsys, std::vector<int>& ss);

// time launch_forces over the candidate shapes for a set of systems that
// share one force field / precision, keep the fastest for all of them
static int autotune_set(gemsgpu_ctx* ctx, const std::vector<int>& ss, int reps, int* lanes_out, int* variant_out,
                        double* best_ms) {
  if (reps <= 0) reps = 10;
  cudaSetDevice(ctx->device);
  const SysHost& h0 = ctx->sys[ss[0]];
  bool single = true;
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    if (h.d.ff == FF_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "autotune: no force field");
    if (h.d.ff != h0.d.ff || h.d.prec != h0.d.prec)
      return fail(ctx, GEMSGPU_ERR_ARG, "autotune: systems differ in force field or precision");
    single &= h.ntypes == 1;
  }
  std::vector<int> need;
  for (int s : ss)
    if (ctx->sys[s].first || ctx->sys[s].pos_dirty || !ctx->sys[s].has_forces) need.push_back(s);
  if (!need.empty()) CHK(interact_group(ctx, need, true));
  std::vector<std::pair<int, int>> cand;
  if (h0.d.ff == FF_TERSOFF) {
    for (int K : {TS_TPA, 2}) {
      if (K == 2 && h0.d.prec != PREC_MIXED) continue;
      cand.push_back({K, 1});
      cand.push_back({K, 3});
      cand.push_back({K, 7});
    }
  } else {
    for (int K : {1, 2, 4, 8, 16, 32}) {
      cand.push_back({K, 1});
      if (h0.d.ff == FF_SMATB && h0.d.prec == PREC_MIXED) {
        cand.push_back({K, 3});
        cand.push_back({K, 7});
        if (single) {
          cand.push_back({K, 0});
          cand.push_back({K, 2});
          cand.push_back({K, 6});
        }
      }
    }
  }
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  double best = 1e30;
  std::pair<int, int> pick = {h0.lanes, h0.variant};
  for (auto c : cand) {
    for (int s : ss) {
      ctx->sys[s].lanes = c.first;
      ctx->sys[s].variant = c.second;
    }
    CHK(launch_forces(ctx, ss));  // warm-up (and map creation)
    CU(cudaEventRecord(e0, ctx->stream));
    for (int r = 0; r < reps; r++) CHK(launch_forces(ctx, ss));
    CU(cudaEventRecord(e1, ctx->stream));
    CU(cudaEventSynchronize(e1));
    float ms;
    CU(cudaEventElapsedTime(&ms, e0, e1));
    if (ms / reps < best) {
      best = ms / reps;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int s : ss) {
    ctx->sys[s].lanes = pick.first;
    ctx->sys[s].variant = pick.second;
  }
  invalidate(ctx);
  if (lanes_out) *lanes_out = pick.first;
  if (variant_out) *variant_out = pick.second;
  if (best_ms) *best_ms = best;
  return 0;
}

int gemsgpu_autotune(gemsgpu_ctx* ctx, int sys, int reps, int* lanes_out, int* variant_out,
                     double* best_ms) {
  CHK(check_sys(ctx, sys));
  return autotune_set(ctx, {sys}, reps, lanes_out, variant_out, best_ms);
}

int gemsgpu_batch_autotune(gemsgpu_ctx* ctx, const int* sys, int nsys, int reps, int* lanes_out,
                           int* variant_out, double* best_ms) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  return autotune_set(ctx, ss, reps, lanes_out, variant_out, best_ms);
}

int gemsgpu_set_lanes(gemsgpu_ctx* ctx, int sys, int lanes, int variant) {
  CHK(check_sys(ctx, sys));
  if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    return fail(ctx, GEMSGPU_ERR_ARG, "lanes must be a power of two <= 32");
  if (variant < 0 || variant > 7 || variant == 4 || variant == 5)
    return fail(ctx, GEMSGPU_ERR_ARG, "variant must be 0..3, 6 or 7");
  SysHost& h = ctx->sys[sys];
  if (h.d.ff == FF_TERSOFF && lanes != TS_TPA && !(lanes == 2 && h.d.prec == PREC_MIXED))
    return fail(ctx, GEMSGPU_ERR_ARG, "Tersoff: lanes 4, or 2 in mixed precision");
  h.lanes = lanes;
  h.variant = variant;
  invalidate(ctx);
  return 0;
}

// parallel_tempering2 (src/ReplicaExchange.f90:55-138): in round ns the
// temperature index k pairs with k+par (even k) or k-par (odd k), par = +1
// for even ns and -1 for odd ns; the lower index accepts with
// min(1, exp(-(beta_k - beta_k')(U_k' - U_k))).  Host arithmetic only, so
// every rank of a multi-GPU run reaches the same decisions from the same
// energies.
int gemsgpu_remd_decide(int nrep, const double* epot_ev, const double* temps, int round, uint64_t seed,
                        const double* uniforms, int* partner, int* accepted) {
  if (nrep <= 0 || !epot_ev || !temps || !partner) return GEMSGPU_ERR_ARG;
  for (int k = 0; k < nrep; k++) {
    if (!(temps[k] > 0.0)) return GEMSGPU_ERR_ARG;
    partner[k] = k;
  }
  const double kB_ev = 8.617385e-5;
  const int par = (round % 2 == 0) ? 1 : -1;
  int nacc = 0;
  for (int k = 0; k < nrep; k++) {
    int p = (k % 2 == 0) ? k + par : k - par;
    if (p < 0 || p >= nrep || p < k) continue;  // k is the lower index of the pair
    double bk = 1.0 / (kB_ev * temps[k]), bp = 1.0 / (kB_ev * temps[p]);
    double du = (epot_ev[p] - epot_ev[k]) * (bk - bp);
    bool swap = true;
    if (du > 0.0) {
      double u;
      if (uniforms) {
        u = uniforms[k];
      } else {
        uint4 q = philox10(make_uint4((uint32_t)k, (uint32_t)round, (uint32_t)((uint64_t)round >> 32), 7u),
                           make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
        u = ((double)(q.x >> 5) * 67108864.0 + (double)(q.y >> 6)) / 9007199254740992.0;
      }
      swap = u < std::exp(-du);
    }
    if (!swap) continue;
    nacc++;
    partner[k] = p;
    partner[p] = k;
  }
  if (accepted) *accepted = nacc;
  return 0;
}

// each system takes its new Ermak temperature; velocities scale by
// sqrt(T_new / T_old) (the reference rescales after exchanging configurations)
int gemsgpu_retemper(gemsgpu_ctx* ctx, int nsys, const int* sys, const double* temps) {
  if (!ctx || nsys <= 0 || !sys || !temps) return fail(ctx, GEMSGPU_ERR_ARG, "retemper: arguments");
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  for (int k = 0; k < nsys; k++) {
    if (ctx->sys[ss[k]].d.integ != IT_ERMAK)
      return fail(ctx, GEMSGPU_ERR_STATE, "retemper: system %d is not an Ermak system", ss[k]);
    if (!(temps[k] > 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "retemper: temperatures > 0");
  }
  cudaSetDevice(ctx->device);
  std::vector<double> fac(ctx->scap, 1.0);
  bool any = false;
  for (int k = 0; k < nsys; k++) {
    SysHost& h = ctx->sys[ss[k]];
    if (h.temp != temps[k]) {
      fac[ss[k]] = std::sqrt(temps[k] / h.temp);
      h.d.skt = std::sqrt(kB_ui * temps[k]);
      h.temp = temps[k];
      CHK(push_sys(ctx, ss[k]));
      any = true;
    }
  }
  if (any) {
    if (ctx->d_fac_cap < ctx->scap) {
      CU(cudaStreamSynchronize(ctx->stream));
      if (ctx->d_fac) cudaFree(ctx->d_fac);
      ctx->d_fac = nullptr;
      CHK(dalloc(ctx, &ctx->d_fac, ctx->scap));
      ctx->d_fac_cap = ctx->scap;
    }
    CU(cudaMemcpyAsync(ctx->d_fac, fac.data(), ctx->scap * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    BlockMap m;
    CHK(get_map(ctx, ss, BLOCK, 0, &m));
    k_scale_vel<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m, ctx->d_fac); ++ctx->launches;
    CU(cudaStreamSynchronize(ctx->stream));  // the host vector `fac` is released on return
  }
  return 0;
}

int gemsgpu_replica_exchange(gemsgpu_ctx* ctx, int nrep, int* sys_of_temp, const double* temps,
                             int round, uint64_t seed, const double* uniforms, int* accepted) {
  if (!ctx || nrep <= 0 || !sys_of_temp || !temps) return fail(ctx, GEMSGPU_ERR_ARG, "replica_exchange: arguments");
  std::vector<int> ss(sys_of_temp, sys_of_temp + nrep);
  for (int k = 0; k < nrep; k++) {
    CHK(check_sys(ctx, ss[k]));
    if (ctx->sys[ss[k]].d.integ != IT_ERMAK)
      return fail(ctx, GEMSGPU_ERR_STATE, "replica_exchange: system %d is not an Ermak system", ss[k]);
    if (!(temps[k] > 0.0)) return fail(ctx, GEMSGPU_ERR_ARG, "replica_exchange: temperatures > 0");
  }
  {
    std::vector<int> t = ss;
    std::sort(t.begin(), t.end());
    if (std::unique(t.begin(), t.end()) != t.end()) return fail(ctx, GEMSGPU_ERR_ARG, "duplicate replica");
  }
  // inq_pot_energy of every replica at its current configuration (eV, as
  // gemsgpu_batch_energy reports it)
  std::vector<double> ep(nrep);
  CHK(gemsgpu_batch_energy(ctx, ss.data(), nrep, ep.data(), nullptr, nullptr));
  std::vector<int> partner(nrep);
  int nacc = 0;
  if (gemsgpu_remd_decide(nrep, ep.data(), temps, round, seed, uniforms, partner.data(), &nacc))
    return fail(ctx, GEMSGPU_ERR_ARG, "replica_exchange: decision arguments");
  // the replica at temperature partner[k] moves to temperature k
  for (int k = 0; k < nrep; k++) sys_of_temp[k] = ss[partner[k]];
  CHK(gemsgpu_retemper(ctx, nrep, sys_of_temp, temps));
  if (accepted) *accepted = nacc;
  return 0;
}

int gemsgpu_pool_create(gemsgpu_ctx* ctx, int max_systems, int64_t max_atoms, int64_t max_cells, int ff,
                        int prec, int lanes, int variant, int chunk_steps, gemsgpu_pool** out) {
  if (!ctx || !out || max_systems <= 0 || max_atoms <= 0 || max_cells < 0 || chunk_steps <= 0)
    return fail(ctx, GEMSGPU_ERR_ARG, "pool_create: arguments");
  if (ff < FF_LJ || ff > FF_TERSOFF || (prec != PREC_FP64 && prec != PREC_MIXED))
    return fail(ctx, GEMSGPU_ERR_ARG, "pool_create: force field / precision");
  if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    return fail(ctx, GEMSGPU_ERR_ARG, "pool_create: lanes");
  cudaSetDevice(ctx->device);
  auto* P = new gemsgpu_pool();
  P->ctx = ctx;
  P->max_systems = max_systems;
  P->max_atoms = max_atoms;
  P->max_cells = max_cells;
  P->ff = ff;
  P->prec = prec;
  P->lanes = ff == FF_TERSOFF ? TS_TPA : lanes;
  P->variant = (variant >= 0 && variant <= 7 && variant != 4 && variant != 5) ? variant : 1;
  P->chunk = chunk_steps;
  int rc = grow_systems(ctx, std::max((int)ctx->sys.size(), 0) + max_systems + 1);
  P->scap = ctx->scap;
  if (!rc) rc = pool_alloc(P);
  if (rc) {
    gemsgpu_pool_destroy(P);
    return rc;
  }
  *out = P;
  return 0;
}

int gemsgpu_pool_destroy(gemsgpu_pool* P) {
  if (!P) return GEMSGPU_ERR_ARG;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  for (int k = 0; k < 5; k++)
    if (P->dmap[k]) cudaFree(P->dmap[k]);
  if (P->dsys) cudaFree(P->dsys);
  delete P;
  return 0;
}

int gemsgpu_pool_set(gemsgpu_pool* P, const int* sys, int nsys) {
  if (!P) return GEMSGPU_ERR_ARG;
  gemsgpu_ctx* ctx = P->ctx;
  if (nsys < 0 || nsys > P->max_systems || (nsys > 0 && !sys))
    return fail(ctx, GEMSGPU_ERR_ARG, "pool_set: 0 <= nsys <= %d", P->max_systems);
  std::vector<int> ss(sys, sys + nsys);
  int64_t atoms = 0;
  for (int s : ss) {
    CHK(check_sys(ctx, s));
    if (s >= P->scap) return fail(ctx, GEMSGPU_ERR_FULL, "system id beyond the pool's capacity");
    if ((P->variant & 1) == 0 && ctx->sys[s].ntypes != 1)
      return fail(ctx, GEMSGPU_ERR_STATE, "pool variant %d needs single-species systems", P->variant);
    const SysDev& d = ctx->sys[s].d;
    if (moving_box(d) || d.virial)
      return fail(ctx, GEMSGPU_ERR_STATE, "pool_set: pools run fixed boxes without the virial");
    if (d.ff != P->ff || d.prec != P->prec)
      return fail(ctx, GEMSGPU_ERR_STATE, "pool_set: system %d has another force field or precision", s);
    // the pool's captured step runs k_step_a / k_step_b<false> and no
    // thermostat kernels: velocity Verlet, Ermak and FIRE only
    if (d.integ != IT_VV && d.integ != IT_ERMAK && d.integ != IT_FIRE)
      return fail(ctx, GEMSGPU_ERR_STATE,
                  "pool_set: system %d: pools run velocity Verlet, Ermak or FIRE systems only", s);
    if (d.thermo != TH_NONE)
      return fail(ctx, GEMSGPU_ERR_STATE, "pool_set: system %d has a thermostat; pools run none", s);
    atoms += ctx->sys[s].n;
  }
  if (atoms > P->max_atoms) return fail(ctx, GEMSGPU_ERR_FULL, "pool_set: %lld atoms > capacity", (long long)atoms);
  std::vector<int> fresh;
  for (int s : ss)
    if (std::find(P->active.begin(), P->active.end(), s) == P->active.end() &&
        (ctx->sys[s].first || ctx->sys[s].pos_dirty || !ctx->sys[s].has_forces))
      fresh.push_back(s);
  CHK(pool_prepare(P, fresh));
  P->active = ss;
  P->maps_dirty = true;
  return 0;
}

int gemsgpu_pool_run(gemsgpu_pool* P, int nchunks) {
  if (!P || nchunks < 0) return GEMSGPU_ERR_ARG;
  cudaSetDevice(P->ctx->device);
  for (int c = 0; c < nchunks; c++) CHK(pool_chunk(P));
  return 0;
}

int gemsgpu_server_create(gemsgpu_ctx* ctx, int max_jobs, int64_t max_atoms, int prec, int lanes,
                          int variant, int chunk_steps, gemsgpu_server** out) {
  if (!ctx || !out || max_jobs <= 0 || max_atoms <= 0 || chunk_steps <= 0)
    return fail(ctx, GEMSGPU_ERR_ARG, "server_create: arguments");
  cudaSetDevice(ctx->device);
  auto* S = new gemsgpu_server();
  S->ctx = ctx;
  S->max_jobs = max_jobs;
  S->max_atoms = max_atoms;
  S->chunk = chunk_steps;
  // room for every admitted job without moving the arena (no re-capture)
  int rc = grow_atoms(ctx, ctx->atoms_used + max_atoms + 32 * (int64_t)max_jobs);
  if (!rc) rc = gemsgpu_pool_create(ctx, max_jobs, max_atoms, 1, FF_SMATB, prec, lanes, variant, chunk_steps,
                                    &S->pool);
  if (rc) {
    delete S;
    return rc;
  }
  *out = S;
  return 0;
}

int gemsgpu_server_destroy(gemsgpu_server* S) {
  if (!S) return GEMSGPU_ERR_ARG;
  for (int64_t id : S->running) {
    ServerJob& j = S->jobs[id];
    if (j.sys >= 0) gemsgpu_system_destroy(S->ctx, j.sys);
  }
  if (S->pool) gemsgpu_pool_destroy(S->pool);
  delete S;
  return 0;
}

int gemsgpu_server_submit(gemsgpu_server* S, const gemsgpu_job* job, int64_t* id) {
  if (!S || !job || !job->pos || job->natoms <= 0) return GEMSGPU_ERR_ARG;
  gemsgpu_ctx* ctx = S->ctx;
  if (job->natoms > S->max_atoms) return fail(ctx, GEMSGPU_ERR_FULL, "job larger than the server's atom budget");
  if ((job->kind != GEMSGPU_JOB_FIRE && job->kind != GEMSGPU_JOB_MD) || job->steps <= 0 || !(job->dt > 0.0))
    return fail(ctx, GEMSGPU_ERR_ARG, "submit: kind, steps > 0, dt > 0");
  ServerJob j;
  j.id = S->next_id++;
  j.spec = *job;
  j.pos.assign(job->pos, job->pos + 3 * (size_t)job->natoms);
  j.spec.pos = nullptr;
  j.state = GEMSGPU_JOB_QUEUED;
  S->jobs[j.id] = std::move(j);
  S->queue.push_back(S->jobs.rbegin()->first);
  if (id) *id = S->queue.back();
  return 0;
}

static int server_admit(gemsgpu_server* S, int64_t id) {
  gemsgpu_ctx* ctx = S->ctx;
  ServerJob& j = S->jobs[id];
  const gemsgpu_job& q = j.spec;
  int sys = -1;
  CHK(gemsgpu_system_create(ctx, q.natoms, 1, &sys));
  j.sys = sys;
  std::vector<double> m(q.natoms, q.mass);
  CHK(gemsgpu_upload(ctx, sys, j.pos.data(), nullptr, m.data(), nullptr));
  CHK(gemsgpu_set_smatb(ctx, sys, 0, 0, q.smatb[0], q.smatb[1], q.smatb[2], q.smatb[3], q.smatb[4], q.smatb[5],
                        q.smatb[6]));
  CHK(gemsgpu_set_precision(ctx, sys, S->pool->prec));
  if (q.kind == GEMSGPU_JOB_FIRE) {
    CHK(gemsgpu_set_fire(ctx, sys, q.dt, 10.0 * q.dt));
    SysHost& h = ctx->sys[sys];
    h.d.fire_fmax = q.fmax;
    h.d.fire_maxit = q.steps;
    CHK(push_sys(ctx, sys));
  } else {
    CHK(gemsgpu_set_ermak(ctx, sys, q.dt, q.gamma, q.temp, q.seed));
  }
  j.state = GEMSGPU_JOB_RUNNING;
  S->atoms_in += q.natoms;
  S->running.push_back(id);
  return 0;
}

static int server_retire(gemsgpu_server* S, int64_t id, const SysState& st) {
  gemsgpu_ctx* ctx = S->ctx;
  ServerJob& j = S->jobs[id];
  double ep = 0, ek = 0, t = 0, fm = 0;
  CHK(gemsgpu_energy(ctx, j.sys, &ep, &ek, &t));
  CHK(gemsgpu_fmax(ctx, j.sys, &fm));
  j.epot_ev = ep;
  j.ekin_ev = ek;
  j.fmax_ev = fm;
  j.iters = j.spec.kind == GEMSGPU_JOB_FIRE ? st.fire_iter : j.done_steps;
  CHK(gemsgpu_download(ctx, j.sys, j.pos.data(), nullptr, nullptr, nullptr));
  CHK(gemsgpu_system_destroy(ctx, j.sys));
  S->atoms_in -= j.spec.natoms;
  j.sys = -1;
  j.state = GEMSGPU_JOB_DONE;
  return 0;
}

int gemsgpu_server_step(gemsgpu_server* S, int* n_running, int* n_queued, int* n_finished) {
  if (!S) return GEMSGPU_ERR_ARG;
  gemsgpu_ctx* ctx = S->ctx;
  cudaSetDevice(ctx->device);
  // admission by memory footprint: first fit over the queue (FIFO order)
  bool changed = false;
  for (auto it = S->queue.begin(); it != S->queue.end();) {
    if ((int)S->running.size() >= S->max_jobs) break;
    ServerJob& j = S->jobs[*it];
    if (S->atoms_in + j.spec.natoms > S->max_atoms) {
      ++it;
      continue;
    }
    int rc = server_admit(S, *it);
    if (rc) {
      j.state = GEMSGPU_JOB_FAILED;
      j.error = rc;
      if (j.sys >= 0) {
        gemsgpu_system_destroy(ctx, j.sys);
        j.sys = -1;
      }
    }
    changed = true;
    it = S->queue.erase(it);
  }
  int finished = 0;
  if (!S->running.empty()) {
    std::vector<int> act;
    for (int64_t id : S->running) act.push_back(S->jobs[id].sys);
    if (changed || act.size() != S->pool->active.size() || !std::equal(act.begin(), act.end(),
                                                                        S->pool->active.begin()))
      CHK(gemsgpu_pool_set(S->pool, act.data(), (int)act.size()));
    CHK(gemsgpu_pool_run(S->pool, 1));
    CHK(read_states(ctx));
    std::vector<int64_t> keep;
    for (int64_t id : S->running) {
      ServerJob& j = S->jobs[id];
      j.done_steps += S->chunk;
      const SysState st = ctx->h_st[j.sys];
      bool done = j.spec.kind == GEMSGPU_JOB_FIRE ? st.fire_done != 0 : j.done_steps >= j.spec.steps;
      if (done) {
        CHK(server_retire(S, id, st));
        finished++;
      } else {
        keep.push_back(id);
      }
    }
    if (keep.size() != S->running.size()) {
      S->running = keep;
      std::vector<int> act2;
      for (int64_t id : S->running) act2.push_back(S->jobs[id].sys);
      CHK(gemsgpu_pool_set(S->pool, act2.data(), (int)act2.size()));
    }
  }
  if (n_running) *n_running = (int)S->running.size();
  if (n_queued) *n_queued = (int)S->queue.size();
  if (n_finished) *n_finished = finished;
  return 0;
}

int gemsgpu_server_poll(gemsgpu_server* S, int64_t id, int* state, double* epot_ev, double* fmax_ev,
                        int* iters, double* pos_out) {
  if (!S) return GEMSGPU_ERR_ARG;
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return fail(S->ctx, GEMSGPU_ERR_ARG, "unknown job %lld", (long long)id);
  ServerJob& j = it->second;
  if (state) *state = j.state;
  if (j.state == GEMSGPU_JOB_DONE) {
    if (epot_ev) *epot_ev = j.epot_ev;
    if (fmax_ev) *fmax_ev = j.fmax_ev;
    if (iters) *iters = j.iters;
    if (pos_out) memcpy(pos_out, j.pos.data(), j.pos.size() * sizeof(double));
  }
  if (j.state == GEMSGPU_JOB_FAILED) return j.error;
  return 0;
}

int gemsgpu_server_forget(gemsgpu_server* S, int64_t id) {
  if (!S) return GEMSGPU_ERR_ARG;
  auto it = S->jobs.find(id);
  if (it == S->jobs.end() || (it->second.state != GEMSGPU_JOB_DONE && it->second.state != GEMSGPU_JOB_FAILED))
    return GEMSGPU_ERR_ARG;
  S->jobs.erase(it);
  return 0;
}

// ------------------------------------------------------------ checkpoints
// write_chp / read_chp (src/Checkpoint.F90:154-244): the per-system state a
// run resumes from -- positions, velocities, accelerations and the Nordsieck
// derivatives acel2..acel4 (GEMS layout; version 3 files, without the
// derivatives, still load), the Ermak/Philox step counter, the FIRE state and
// the rebuild count.  Resuming
// forces a neighbour rebuild, as the reference's interact does after
// read_chp (src/Checkpoint.F90:232-241).
namespace {
struct ChpHeader {
  char magic[8];
  int32_t version, n, ff, integ;
  uint64_t step;
  int64_t nupd;
  double fire_dt, fire_alpha;
  int32_t fire_np, fire_done, fire_iter, fire_zero;
  // the box and the G-JF piston (force, velocity, last noise, phase)
  double box[3];
  double lgf_pf, lgf_pvel, lgf_rangv;
  int32_t lgf_phase, pad;
  double ax_pf[3], ax_pvel[3], ax_rangv[3];
  int32_t ax_phase[3], pad2;
};
}  // namespace

int gemsgpu_checkpoint_size(gemsgpu_ctx* ctx, int sys, size_t* bytes) {
  CHK(check_sys(ctx, sys));
  if (!bytes) return fail(ctx, GEMSGPU_ERR_ARG, "checkpoint_size: NULL");
  *bytes = sizeof(ChpHeader) + 18 * sizeof(double) * (size_t)ctx->sys[sys].n;
  return 0;
}

int gemsgpu_checkpoint_save(gemsgpu_ctx* ctx, int sys, void* buf, size_t bytes) {
  size_t need = 0;
  CHK(gemsgpu_checkpoint_size(ctx, sys, &need));
  if (!buf || bytes < need) return fail(ctx, GEMSGPU_ERR_ARG, "checkpoint_save: buffer of %zu bytes needed", need);
  const SysHost& h = ctx->sys[sys];
  CHK(read_states(ctx));
  const SysState& st = ctx->h_st[sys];
  ChpHeader hd{};
  memcpy(hd.magic, "GEMSGPU", 8);
  hd.version = 4;
  hd.n = h.n;
  hd.ff = h.d.ff;
  hd.integ = h.d.integ;
  hd.step = st.step;
  hd.nupd = st.nupd;
  hd.fire_dt = st.fire_dt;
  hd.fire_alpha = st.fire_alpha;
  hd.fire_np = st.fire_np;
  hd.fire_done = st.fire_done;
  hd.fire_iter = st.fire_iter;
  hd.fire_zero = st.fire_zero;
  CHK(gemsgpu_get_box(ctx, sys, hd.box));
  hd.lgf_pf = st.lgf_pf;
  hd.lgf_pvel = st.lgf_pvel;
  hd.lgf_rangv = st.lgf_rangv;
  hd.lgf_phase = st.lgf_phase;
  for (int k = 0; k < 3; k++) {
    hd.ax_pf[k] = st.ax_pf[k];
    hd.ax_pvel[k] = st.ax_pvel[k];
    hd.ax_rangv[k] = st.ax_rangv[k];
    hd.ax_phase[k] = st.ax_phase[k];
  }
  char* p = static_cast<char*>(buf);
  memcpy(p, &hd, sizeof(hd));
  double* x = reinterpret_cast<double*>(p + sizeof(hd));
  CHK(get_d4(ctx, h, ctx->A.pos, x));
  CHK(get_d4(ctx, h, ctx->A.vel, x + 3 * (size_t)h.n));
  CHK(get_d4(ctx, h, ctx->A.acel, x + 6 * (size_t)h.n));
  if (ctx->A.acel2) {
    CHK(get_d4(ctx, h, ctx->A.acel2, x + 9 * (size_t)h.n));
    CHK(get_d4(ctx, h, ctx->A.acel3, x + 12 * (size_t)h.n));
    CHK(get_d4(ctx, h, ctx->A.acel4, x + 15 * (size_t)h.n));
  } else {
    std::fill(x + 9 * (size_t)h.n, x + 18 * (size_t)h.n, 0.0);
  }
  return 0;
}

int gemsgpu_checkpoint_load(gemsgpu_ctx* ctx, int sys, const void* buf, size_t bytes) {
  CHK(check_sys(ctx, sys));
  if (!buf || bytes < sizeof(ChpHeader)) return fail(ctx, GEMSGPU_ERR_ARG, "checkpoint_load: no header");
  SysHost& h = ctx->sys[sys];
  ChpHeader hd;
  memcpy(&hd, buf, sizeof(hd));
  if (memcmp(hd.magic, "GEMSGPU", 8) != 0 || (hd.version != 3 && hd.version != 4))
    return fail(ctx, GEMSGPU_ERR_ARG, "checkpoint_load: not a checkpoint of this library");
  if (hd.n != h.n) return fail(ctx, GEMSGPU_ERR_ARG, "checkpoint_load: %d atoms, system has %d", hd.n, h.n);
  const size_t per_atom = hd.version == 4 ? 18 : 9;
  const size_t need = sizeof(ChpHeader) + per_atom * sizeof(double) * (size_t)h.n;
  if (bytes < need) return fail(ctx, GEMSGPU_ERR_ARG, "checkpoint_load: %zu bytes expected", need);
  if (h.d.boxed && (moving_box(h.d) || hd.integ == IT_LGF || hd.integ == IT_AXES || hd.integ == IT_LKD)) {
    // the box the piston had reached
    h.box_live = false;
    for (int k = 0; k < 3; k++) h.d.L[k] = hd.box[k];
    CHK(push_sys(ctx, sys));
    drop_maps(ctx);
    invalidate(ctx);
  }
  const double* x = reinterpret_cast<const double*>(static_cast<const char*>(buf) + sizeof(hd));
  CHK(h2d_xyz(ctx, x, ctx->A.pos + h.off, h.n));
  CHK(h2d_xyz(ctx, x + 3 * (size_t)h.n, ctx->A.vel + h.off, h.n));
  CHK(h2d_xyz(ctx, x + 6 * (size_t)h.n, ctx->A.acel + h.off, h.n));
  std::vector<double> hi(9 * (size_t)h.n, 0.0);
  if (hd.version == 4) std::copy(x + 9 * (size_t)h.n, x + 18 * (size_t)h.n, hi.begin());
  bool any_hi = false;
  for (double q : hi) any_hi |= q != 0.0;
  if (any_hi) CHK(ensure_nord(ctx));
  if (ctx->A.acel2) {
    CHK(h2d_xyz(ctx, hi.data(), ctx->A.acel2 + h.off, h.n));
    CHK(h2d_xyz(ctx, hi.data() + 3 * (size_t)h.n, ctx->A.acel3 + h.off, h.n));
    CHK(h2d_xyz(ctx, hi.data() + 6 * (size_t)h.n, ctx->A.acel4 + h.off, h.n));
  }
  CHK(read_states(ctx));
  SysState st = ctx->h_st[sys];
  st.step = hd.step;
  st.nupd = hd.nupd;
  st.fire_dt = hd.fire_dt;
  st.fire_alpha = hd.fire_alpha;
  st.fire_np = hd.fire_np;
  st.fire_done = hd.fire_done;
  st.fire_iter = hd.fire_iter;
  st.fire_zero = hd.fire_zero;
  st.lgf_pf = hd.lgf_pf;
  st.lgf_pvel = hd.lgf_pvel;
  st.lgf_rangv = hd.lgf_rangv;
  st.lgf_phase = hd.lgf_phase;
  for (int k = 0; k < 3; k++) {
    st.box_b[k] = h.d.L[k];
    st.ax_pf[k] = hd.ax_pf[k];
    st.ax_pvel[k] = hd.ax_pvel[k];
    st.ax_rangv[k] = hd.ax_rangv[k];
    st.ax_phase[k] = hd.ax_phase[k];
  }
  st.status = 0;
  CU(cudaMemcpyAsync(ctx->A.st + sys, &st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
  BlockMap m;
  CHK(get_map(ctx, {sys}, BLOCK, 0, &m));
  k_refresh_fx<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  CU(cudaStreamSynchronize(ctx->stream));
  h.first = true;        // the resumed interact rebuilds the list
  h.has_forces = false;
  return 0;
}

// ------------------------------------------------------------------ GEMS .chp
// write_chp / read_chp (src/Checkpoint.F90:154-244) lay a checkpoint out as
// Fortran unformatted sequential records, each framed by its byte length as
// a 4-byte integer before and after (the gfortran layout):
//   current, step, nsteps, nlocal            4 x int32
//   tbox(3,3)                                9 x float64, column-major
//   'lcg' | 'std', then the generator state  (write_chpseed, Random.F90:178-184)
//   piston(3)                                3 x logical(4)
//   ppos(i), pvel(i), pistonf(i)             one float64 record each, per piston i
//   nframe, time, dm_steps, pnframe, ptime, frame   5 x float64 + int32
//   per atom: pos, vel, acel, acel2, acel3, acel4    3 x float64 each
// (write_chppiston / read_chppiston, Integration.F90:1488-1520).  The
// library writes the 'lcg' form with the caller's generator state; the
// higher derivatives acel2..4 are the Nordsieck predictor-corrector's (zero
// until a system of the context has used it).
namespace {
struct ChpOut {
  std::vector<unsigned char> b;
  void raw(const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    b.insert(b.end(), c, c + n);
  }
  void rec(const void* p, size_t n) {
    const int32_t m = (int32_t)n;
    raw(&m, 4);
    raw(p, n);
    raw(&m, 4);
  }
};

struct ChpIn {
  const unsigned char* p;
  size_t n, at = 0;
  bool ok = true;
  // the next record's payload (nullptr if the framing is broken)
  const unsigned char* rec(size_t* len) {
    int32_t m0, m1;
    if (at + 4 > n) return ok = false, nullptr;
    memcpy(&m0, p + at, 4);
    if (m0 < 0 || at + 8 + (size_t)m0 > n) return ok = false, nullptr;
    memcpy(&m1, p + at + 4 + m0, 4);
    if (m1 != m0) return ok = false, nullptr;
    const unsigned char* q = p + at + 4;
    at += 8 + (size_t)m0;
    *len = (size_t)m0;
    return q;
  }
  bool getb(void* out, size_t size) {
    size_t len = 0;
    const unsigned char* q = rec(&len);
    if (!q || len != size) return ok = false;
    memcpy(out, q, len);
    return true;
  }
  bool get(int32_t* out, size_t count) { return getb(out, 4 * count); }
  bool get(double* out, size_t count) { return getb(out, 8 * count); }
};

// The piston values the reference holds after a step: the library closes a
// G-JF piston step at the start of the next one (it needs the whole
// system's virial), so the step just taken is closed here, as lgf_stepb /
// lgf_flex_stepb (Integration.F90:600-650, 778-830) would have.
void chp_pistons(const SysDev& d, const SysState& st, const double L[3], int flag[3], double pvel[3], double pf[3]) {
  for (int k = 0; k < 3; k++) flag[k] = 0, pvel[k] = 0.0, pf[k] = 0.0;
  const double vol = L[0] * L[1] * L[2];
  if (d.integ == IT_LGF) {
    for (int k = 0; k < 3; k++) flag[k] = 1;
    if (st.lgf_phase) {
      const double pfn = ((st.vir[0] + st.vir[1] + st.vir[2]) / 3 + d.lgf_kin) / vol - d.lgf_press;
      pvel[0] = d.lgf_av * st.lgf_pvel + 0.5 * d.lgf_ipm * d.dt * (d.lgf_av * st.lgf_pf + pfn) +
                d.lgf_bv * d.lgf_ipm * st.lgf_rangv;
      pf[0] = pfn;
    } else {
      pvel[0] = st.lgf_pvel;
    }
  } else if (d.integ == IT_AXES) {
    for (int k = 0; k < 3; k++) {
      if (d.ax_mode[k] != AX_FLEX) continue;
      const double* q = d.ax_p[k];
      flag[k] = 1;
      if (st.ax_phase[k]) {
        const double pfn = (st.vir[k] + q[2]) / vol - q[3];
        pvel[k] = q[7] * st.ax_pvel[k] + 0.5 * q[4] * d.dt * (q[7] * st.ax_pf[k] + pfn) * vol / L[k] +
                  q[5] * q[4] * st.ax_rangv[k];
        pf[k] = pfn;
      } else {
        pvel[k] = st.ax_pvel[k];
      }
    }
  } else if (d.integ == IT_LKD) {
    for (int k = 0; k < 3; k++) flag[k] = 1;
    pvel[0] = st.lgf_pvel;
  }
}
}  // namespace

int gemsgpu_chp_write(gemsgpu_ctx* ctx, int sys, const gemsgpu_chp_info* info, void* buf, size_t bytes,
                      size_t* written) {
  CHK(check_sys(ctx, sys));
  if (!info) return fail(ctx, GEMSGPU_ERR_ARG, "chp_write: info required");
  const SysHost& h = ctx->sys[sys];
  if (h.pos_dirty || !h.has_forces)
    return fail(ctx, GEMSGPU_ERR_STATE, "chp_write: evaluate the forces at these positions first");
  double L[3];
  CHK(gemsgpu_get_box(ctx, sys, L));
  CHK(read_states(ctx));
  const SysState& st = ctx->h_st[sys];
  std::vector<double> x(3 * (size_t)h.n), v(3 * (size_t)h.n), a(3 * (size_t)h.n);
  CHK(get_d4(ctx, h, ctx->A.pos, x.data()));
  CHK(get_d4(ctx, h, ctx->A.vel, v.data()));
  CHK(get_d4(ctx, h, ctx->A.acel, a.data()));
  std::vector<double> hi(ctx->A.acel2 ? 9 * (size_t)h.n : 0);
  if (ctx->A.acel2) {
    CHK(get_d4(ctx, h, ctx->A.acel2, hi.data()));
    CHK(get_d4(ctx, h, ctx->A.acel3, hi.data() + 3 * (size_t)h.n));
    CHK(get_d4(ctx, h, ctx->A.acel4, hi.data() + 6 * (size_t)h.n));
  }
  ChpOut o;
  const int32_t head[4] = {info->current, info->step, info->nsteps, h.n};
  o.rec(head, sizeof(head));
  double tbox[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < 3; k++) tbox[4 * k] = h.d.boxed ? L[k] : 0.0;
  o.rec(tbox, sizeof(tbox));
  o.rec("lcg", 3);
  o.rec(info->rng, 3 * sizeof(int32_t));
  int flag[3];
  double pvel[3], pf[3];
  chp_pistons(h.d, st, L, flag, pvel, pf);
  const int32_t fl[3] = {flag[0], flag[1], flag[2]};
  o.rec(fl, sizeof(fl));
  for (int k = 0; k < 3; k++)
    if (flag[k]) {
      const double zero = 0.0;
      o.rec(&zero, 8);
      o.rec(&pvel[k], 8);
      o.rec(&pf[k], 8);
    }
  const double fr[5] = {info->nframe, info->time, info->dm_steps, info->pnframe, info->ptime};
  unsigned char frec[5 * 8 + 4];
  memcpy(frec, fr, sizeof(fr));
  memcpy(frec + sizeof(fr), &info->frame, 4);
  o.rec(frec, sizeof(frec));
  const double z3[3] = {0, 0, 0};
  for (int i = 0; i < h.n; i++) {
    o.rec(&x[3 * (size_t)i], 24);
    o.rec(&v[3 * (size_t)i], 24);
    o.rec(&a[3 * (size_t)i], 24);
    for (int k = 0; k < 3; k++) o.rec(hi.empty() ? z3 : &hi[3 * ((size_t)k * h.n + i)], 24);
  }
  if (written) *written = o.b.size();
  if (!buf) return 0;  // size query
  if (bytes < o.b.size()) return fail(ctx, GEMSGPU_ERR_ARG, "chp_write: buffer of %zu bytes needed", o.b.size());
  memcpy(buf, o.b.data(), o.b.size());
  return 0;
}

int gemsgpu_chp_read(gemsgpu_ctx* ctx, int sys, const void* buf, size_t bytes, gemsgpu_chp_info* info) {
  CHK(check_sys(ctx, sys));
  if (!buf) return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: NULL buffer");
  SysHost& h = ctx->sys[sys];
  ChpIn in{static_cast<const unsigned char*>(buf), bytes};
  int32_t head[4];
  double tbox[9];
  if (!in.get(head, 4) || !in.get(tbox, 9)) return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: not a GEMS checkpoint");
  if (head[3] != h.n)
    return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: %d atoms in the checkpoint, %d in the system", head[3], h.n);
  gemsgpu_chp_info got{};
  got.current = head[0];
  got.step = head[1];
  got.nsteps = head[2];
  size_t len = 0;
  const unsigned char* tag = in.rec(&len);
  if (!tag || len != 3) return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: generator record missing");
  if (memcmp(tag, "lcg", 3) == 0) {
    if (!in.get(got.rng, 3)) return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: lcg state");
  } else if (memcmp(tag, "std", 3) == 0) {
    int32_t sz = 0;
    if (!in.get(&sz, 1) || sz < 0 || !in.rec(&len) || len != 4 * (size_t)sz)
      return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: std seed");
  } else {
    return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: checkpoint file corrupted");
  }
  int32_t fl[3];
  if (!in.get(fl, 3)) return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: piston flags");
  double pvel[3] = {0, 0, 0};
  for (int k = 0; k < 3; k++)
    if (fl[k]) {
      double ppos, pf;
      if (!in.get(&ppos, 1) || !in.get(&pvel[k], 1) || !in.get(&pf, 1))
        return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: piston %d", k);
    }
  size_t flen = 0;
  const unsigned char* fr = in.rec(&flen);
  if (!fr || flen != 44) return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: frame record");
  double f5[5];
  memcpy(f5, fr, 40);
  memcpy(&got.frame, fr + 40, 4);
  got.nframe = f5[0], got.time = f5[1], got.dm_steps = f5[2], got.pnframe = f5[3], got.ptime = f5[4];
  std::vector<double> x(3 * (size_t)h.n), v(3 * (size_t)h.n), a(3 * (size_t)h.n), hi(9 * (size_t)h.n);
  for (int i = 0; i < h.n; i++) {
    if (!in.get(&x[3 * (size_t)i], 3) || !in.get(&v[3 * (size_t)i], 3) || !in.get(&a[3 * (size_t)i], 3) ||
        !in.get(&hi[3 * (size_t)i], 3) || !in.get(&hi[3 * ((size_t)h.n + i)], 3) ||
        !in.get(&hi[3 * (2 * (size_t)h.n + i)], 3))
      return fail(ctx, GEMSGPU_ERR_ARG, "chp_read: atom %d", i);
  }
  bool any_hi = false;
  for (double q : hi) any_hi |= q != 0.0;
  // the box the checkpoint had reached (box_setvars after read(chpunit) tbox)
  if (h.d.boxed) {
    h.box_live = false;
    for (int k = 0; k < 3; k++) h.d.L[k] = tbox[4 * k];
    CHK(push_sys(ctx, sys));
    drop_maps(ctx);
    invalidate(ctx);
  }
  CHK(h2d_xyz(ctx, x.data(), ctx->A.pos + h.off, h.n));
  CHK(h2d_xyz(ctx, v.data(), ctx->A.vel + h.off, h.n));
  CHK(h2d_xyz(ctx, a.data(), ctx->A.acel + h.off, h.n));
  if (any_hi) CHK(ensure_nord(ctx));
  if (ctx->A.acel2) {
    CHK(h2d_xyz(ctx, hi.data(), ctx->A.acel2 + h.off, h.n));
    CHK(h2d_xyz(ctx, hi.data() + 3 * (size_t)h.n, ctx->A.acel3 + h.off, h.n));
    CHK(h2d_xyz(ctx, hi.data() + 6 * (size_t)h.n, ctx->A.acel4 + h.off, h.n));
  }
  CHK(read_states(ctx));
  SysState st = ctx->h_st[sys];
  // a piston resumes as the reference's does after read_chp: pvel from the
  // file, pistonf from the virial of the first force evaluation
  if (h.d.integ == IT_LGF || h.d.integ == IT_LKD) {
    st.lgf_pvel = pvel[0];
    st.lgf_phase = 0;
  } else if (h.d.integ == IT_AXES) {
    for (int k = 0; k < 3; k++)
      if (h.d.ax_mode[k] == AX_FLEX) {
        st.ax_pvel[k] = pvel[k];
        st.ax_phase[k] = 0;
      }
  }
  for (int k = 0; k < 3; k++) st.box_b[k] = h.d.L[k];
  st.status = 0;
  CU(cudaMemcpyAsync(ctx->A.st + sys, &st, sizeof(st), cudaMemcpyHostToDevice, ctx->stream));
  BlockMap m;
  CHK(get_map(ctx, {sys}, BLOCK, 0, &m));
  k_refresh_fx<<<m.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, m); ++ctx->launches;
  CU(cudaStreamSynchronize(ctx->stream));
  h.first = true;  // the resumed interact rebuilds the list, as read_chp's interact does
  h.has_forces = false;
  h.pos_dirty = false;
  if (info) *info = got;
  return 0;
}

// ------------------------------------------------------------------ L-BFGS
// lbfgs_minimizator (src/Quasi_Newton.f90:77-160) for nsys systems at once;
// the kernels and the method are in lbfgs.cuh.  Rounds of function
// evaluations run in chunks; after each chunk the host reads the systems'
// phases, drops finished systems from the launches, and heals a list
// overflow by growing the list and restarting the affected searches from
// their current points (the L-BFGS history is then discarded).
// (re)allocate the context's L-BFGS workspace for the current arena and
// system capacity and at least m history pairs
int lbfgs_workspace(gemsgpu_ctx* ctx, int m) {
  LbWork& W = ctx->lbw;
  CU(cudaStreamSynchronize(ctx->stream));
  void* old[7] = {W.x0, W.g, W.gold, W.d, W.S, W.Y, W.st};
  for (void* p : old)
    if (p) cudaFree(p);
  W = LbWork{};
  ctx->lbw_m = 0;
  ctx->lbw_scap = 0;
  const int64_t cap = ctx->acap;
  const int mm = std::max(m, 5);  // at least GEMS's default history, so a later m = 5 call reuses it
  CHK(dalloc(ctx, &W.x0, cap));
  CHK(dalloc(ctx, &W.g, cap));
  CHK(dalloc(ctx, &W.gold, cap));
  CHK(dalloc(ctx, &W.d, cap));
  CHK(dalloc(ctx, &W.S, (size_t)mm * cap));
  CHK(dalloc(ctx, &W.Y, (size_t)mm * cap));
  CHK(dalloc(ctx, &W.st, ctx->scap));
  W.cap = cap;
  ctx->lbw_m = mm;
  ctx->lbw_scap = ctx->scap;
  return 0;
}

int gemsgpu_batch_lbfgs(gemsgpu_ctx* ctx, const int* sys, int nsys, int m, double eps, double xtol, int itermax,
                        int* iters, int* nfun, int* status, double* emin_ev) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  if (m < 1 || m > LB_MAXM) return fail(ctx, GEMSGPU_ERR_ARG, "lbfgs: m must be 1..%d", LB_MAXM);
  if (!(eps > 0.0) || !(xtol >= 0.0) || itermax < 1) return fail(ctx, GEMSGPU_ERR_ARG, "lbfgs: eps, xtol, itermax");
  for (int s : ss)
    if (ctx->sys[s].d.ff == FF_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "lbfgs: system %d has no force field", s);
  cudaSetDevice(ctx->device);
  // workspace, indexed like the arena: the context's, grown when the arena,
  // the history length or the system capacity outgrew it
  const int64_t cap = ctx->acap;
  int rc = 0;
  if (cap > ctx->lbw.cap || m > ctx->lbw_m || ctx->scap > ctx->lbw_scap) CHK(lbfgs_workspace(ctx, m));
  const LbWork W = ctx->lbw;
  std::vector<LbState> hs(ctx->scap);
  for (auto& L : hs) {
    L = LbState{};
    L.phase = LB_IDLE;
    L.m = m;
    L.eps = eps;
    L.xtol = xtol;
    L.itermax = itermax;
  }
  auto fail_clean = [&](int code) { return code; };
  if (cudaMemcpyAsync(W.st, hs.data(), hs.size() * sizeof(LbState), cudaMemcpyHostToDevice, ctx->stream) !=
      cudaSuccess)
    return fail_clean(fail(ctx, GEMSGPU_ERR_CUDA, "lbfgs: state upload"));
  if ((rc = interact_group(ctx, ss, true))) return fail_clean(rc);
  const int* sa;
  if ((rc = sys_array(ctx, ss, &sa))) return fail_clean(rc);
  k_lb_init<<<(int)ss.size(), LB_THREADS, 0, ctx->stream>>>(ctx->A, W, sa, 0); ++ctx->launches;
  const int ROUND = 16;
  const int64_t budget = (int64_t)itermax * (LB_MAXFEV + 1) + ROUND;
  std::vector<int> active = ss;
  int heals = 0;
  for (int64_t rounds = 0; rounds < budget && !active.empty(); rounds += ROUND) {
    BlockMap ma;
    if ((rc = get_map(ctx, active, BLOCK, 0, &ma)) || (rc = sys_array(ctx, active, &sa)) ||
        (rc = clear_status(ctx, active)))
      return fail_clean(rc);
    const int na = (int)active.size();
    for (int r = 0; r < ROUND; r++) {
      k_lb_dir<<<na, LB_THREADS, 0, ctx->stream>>>(ctx->A, W, sa); ++ctx->launches;
      k_lb_move<<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, W, ma); ++ctx->launches;
      k_skin<<<ma.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, ma); ++ctx->launches;
      if ((rc = launch_rebuild(ctx, active)) || (rc = launch_forces(ctx, active))) return fail_clean(rc);
      k_lb_eval<<<na, LB_THREADS, 0, ctx->stream>>>(ctx->A, W, sa); ++ctx->launches;
    }
    if (cudaMemcpyAsync(hs.data(), W.st, hs.size() * sizeof(LbState), cudaMemcpyDeviceToHost, ctx->stream) !=
        cudaSuccess)
      return fail_clean(fail(ctx, GEMSGPU_ERR_CUDA, "lbfgs: state readback"));
    if ((rc = read_states(ctx))) return fail_clean(rc);
    int grow = 0;
    for (int s : active) {
      const int st = ctx->h_st[s].status;
      if (st & ST_FATAL) return fail_clean(status_error(ctx, s, st));
      if (st & ST_OVERFLOW) grow = std::max(grow, ctx->h_st[s].maxnn);
    }
    if (grow > 0) {
      // forces of this chunk may come from truncated lists: grow, rebuild,
      // and restart the unfinished searches from where they stand
      if (++heals > 4) return fail_clean(fail(ctx, GEMSGPU_ERR_OVERFLOW, "lbfgs: neighbour list keeps overflowing"));
      if ((rc = grow_list(ctx, grow + grow / 4 + 8))) return fail_clean(rc);
      for (int s : active) ctx->sys[s].first = true;
      if ((rc = interact_group(ctx, active, true)) || (rc = sys_array(ctx, active, &sa))) return fail_clean(rc);
      k_lb_init<<<(int)active.size(), LB_THREADS, 0, ctx->stream>>>(ctx->A, W, sa, 1); ++ctx->launches;
      continue;
    }
    std::vector<int> next;
    for (int s : active) {
      const int ph = hs[s].phase;
      if (ph == LB_EVAL || ph == LB_ACCEPT) next.push_back(s);
    }
    active.swap(next);
  }
  CU(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < nsys; k++) {
    const LbState& L = hs[ss[k]];
    SysHost& h = ctx->sys[ss[k]];
    h.has_forces = true;  // the last evaluation was at the final positions
    h.pos_dirty = false;
    if (iters) iters[k] = L.iter;
    if (nfun) nfun[k] = L.nfun;
    if (status) status[k] = L.phase == LB_DONE ? 0 : (L.phase == LB_FAIL ? -1 : 1);
    if (emin_ev) emin_ev[k] = L.f;
  }
  return 0;
}

int gemsgpu_lbfgs(gemsgpu_ctx* ctx, int sys, int m, double eps, double xtol, int itermax, int* iters, int* nfun,
                  int* status, double* emin_ev) {
  CHK(check_sys(ctx, sys));
  return gemsgpu_batch_lbfgs(ctx, &sys, 1, m, eps, xtol, itermax, iters, nfun, status, emin_ev);
}

// ------------------------------------------------------------------ NEB
// neb (src/NEB.f90:58-220) over nimg image systems; kernels in neb.cuh.
// Reproduced as the reference runs it: the last image's energy is not
// evaluated before the final report (its loop ends at nimg-1, :110), so it
// enters the tangent choice as 0; the time step is set once from the RMS
// NEB force of the interpolated band, dt = sqrt(2 m 5e-5 / F_rms) (:133).
int gemsgpu_neb(gemsgpu_ctx* ctx, const int* sys, int nimg, const int* fixed, int nfixed, double k_ev, int iters,
                double* dt_out, double* eimg_ev) {
  if (!ctx || nimg < 3 || !fixed || nfixed < 2 || iters < 0)
    return fail(ctx, GEMSGPU_ERR_ARG, "neb: nimg >= 3, two or more fixed images, iters >= 0");
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nimg, ss));
  const SysHost& h0 = ctx->sys[ss[0]];
  for (int s : ss) {
    const SysHost& h = ctx->sys[s];
    if (h.d.ff == FF_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "neb: system %d has no force field", s);
    if (h.n != h0.n || h.ntypes != h0.ntypes || h.d.ff != h0.d.ff)
      return fail(ctx, GEMSGPU_ERR_ARG, "neb: the images must be systems of the same atoms and force field");
  }
  for (int j = 0; j < nfixed; j++) {
    if (fixed[j] < 0 || fixed[j] >= nimg || (j > 0 && fixed[j] <= fixed[j - 1]))
      return fail(ctx, GEMSGPU_ERR_ARG, "neb: fixed images must be increasing indices in [0, nimg)");
  }
  cudaSetDevice(ctx->device);
  const int n = h0.n;
  std::vector<int> off(nimg);
  for (int k = 0; k < nimg; k++) off[k] = ctx->sys[ss[k]].off;
  int *d_sys = nullptr, *d_off = nullptr;
  double *d_e = nullptr, *d_f = nullptr;
  auto release = [&]() {
    cudaFree(d_sys);
    cudaFree(d_off);
    cudaFree(d_e);
    cudaFree(d_f);
  };
  int rc = 0;
  if ((rc = dalloc(ctx, &d_sys, nimg)) || (rc = dalloc(ctx, &d_off, nimg)) || (rc = dalloc(ctx, &d_e, nimg)) ||
      (rc = dalloc(ctx, &d_f, nimg))) {
    release();
    return rc;
  }
  auto bail = [&](int code) {
    release();
    return code;
  };
  if (cudaMemcpyAsync(d_sys, ss.data(), nimg * sizeof(int), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
      cudaMemcpyAsync(d_off, off.data(), nimg * sizeof(int), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
      cudaMemsetAsync(d_e, 0, nimg * sizeof(double), ctx->stream) != cudaSuccess ||
      cudaMemsetAsync(d_f, 0, nimg * sizeof(double), ctx->stream) != cudaSuccess)
    return bail(fail(ctx, GEMSGPU_ERR_CUDA, "neb: set-up copies"));
  NebDev N{d_sys, d_off, d_e, d_f, nimg, n, k_ev / c_ui_ev()};
  // neb_linin, then unit masses at rest
  for (int j = 0; j + 1 < nfixed; j++) {
    if (fixed[j + 1] - fixed[j] < 2) continue;
    k_neb_interp<<<(3 * n + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, N, fixed[j], fixed[j + 1]);
    ++ctx->launches;
  }
  for (int k = 1; k < nimg - 1; k++) {
    if (cudaMemsetAsync(ctx->A.vel + off[k], 0, (size_t)n * sizeof(double4), ctx->stream) != cudaSuccess)
      return bail(fail(ctx, GEMSGPU_ERR_CUDA, "neb: velocity reset"));
    ctx->sys[ss[k]].pos_dirty = true;
  }
  {
    BlockMap mr;
    std::vector<int> inner(ss.begin() + 1, ss.end() - 1);
    if ((rc = get_map(ctx, inner, BLOCK, 0, &mr))) return bail(rc);
    k_refresh_fx<<<mr.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, mr); ++ctx->launches;
  }
  // forces and energies of images 0 .. nimg-2 (:110-118), the NEB force, dt
  std::vector<int> first(ss.begin(), ss.end() - 1);
  if ((rc = interact_group(ctx, first, true))) return bail(rc);
  k_neb_energy<<<nimg - 1, LB_THREADS, 0, ctx->stream>>>(ctx->A, N, 0); ++ctx->launches;
  k_neb_force<<<nimg - 2, LB_THREADS, 0, ctx->stream>>>(ctx->A, N); ++ctx->launches;
  std::vector<double> fsum(nimg);
  if (cudaMemcpyAsync(fsum.data(), d_f, nimg * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return bail(fail(ctx, GEMSGPU_ERR_CUDA, "neb: force readback"));
  double fprom = 0.0;
  for (int k = 1; k < nimg - 1; k++) fprom += fsum[k];
  fprom = std::sqrt(fprom / ((double)(nimg - 2) * (double)(3 * n)));
  if (!(fprom > 0.0)) return bail(fail(ctx, GEMSGPU_ERR_STATE, "neb: the band has no force"));
  const double mass = 1.0;
  const double dt = std::sqrt(2.0 * mass * 5e-5 / fprom);
  std::vector<int> inner(ss.begin() + 1, ss.end() - 1);
  const int ni = nimg - 2;
  const int vv_grid = (int)(((int64_t)ni * n + 255) / 256);
  for (int it = 0; it < iters; it++) {
    BlockMap mi;
    if ((rc = get_map(ctx, inner, BLOCK, 0, &mi)) || (rc = clear_status(ctx, inner))) return bail(rc);
    k_neb_vel<<<ni, LB_THREADS, 0, ctx->stream>>>(ctx->A, N); ++ctx->launches;
    k_neb_vv<true><<<vv_grid, 256, 0, ctx->stream>>>(ctx->A, N, dt); ++ctx->launches;
    k_skin<<<mi.nblk, BLOCK, 0, ctx->stream>>>(ctx->A, mi); ++ctx->launches;
    if ((rc = launch_rebuild(ctx, inner))) return bail(rc);
    if ((rc = read_states(ctx))) return bail(rc);
    int grow = 0;
    for (int s : inner) {
      const int st = ctx->h_st[s].status;
      if (st & ST_FATAL) return bail(status_error(ctx, s, st));
      if (st & ST_OVERFLOW) grow = std::max(grow, ctx->h_st[s].maxnn);
    }
    if (grow > 0) {  // the lists of this step would be truncated: grow and rebuild them
      if ((rc = grow_list(ctx, grow + grow / 4 + 8))) return bail(rc);
      for (int s : inner) ctx->sys[s].first = true;
      if ((rc = interact_group(ctx, inner, true))) return bail(rc);
    } else if ((rc = launch_forces(ctx, inner))) {
      return bail(rc);
    }
    k_neb_energy<<<ni, LB_THREADS, 0, ctx->stream>>>(ctx->A, N, 1); ++ctx->launches;
    k_neb_force<<<ni, LB_THREADS, 0, ctx->stream>>>(ctx->A, N); ++ctx->launches;
    k_neb_vel<<<ni, LB_THREADS, 0, ctx->stream>>>(ctx->A, N); ++ctx->launches;
    k_neb_vv<false><<<vv_grid, 256, 0, ctx->stream>>>(ctx->A, N, dt); ++ctx->launches;
  }
  // write_neb (:376-414): every image's forces and energy at the final band
  for (int s : ss) ctx->sys[s].pos_dirty = true;
  if ((rc = interact_group(ctx, ss, true))) return bail(rc);
  k_neb_energy<<<nimg, LB_THREADS, 0, ctx->stream>>>(ctx->A, N, 0); ++ctx->launches;
  std::vector<double> e(nimg);
  if (cudaMemcpyAsync(e.data(), d_e, nimg * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return bail(fail(ctx, GEMSGPU_ERR_CUDA, "neb: energy readback"));
  if (eimg_ev)
    for (int k = 0; k < nimg; k++) eimg_ev[k] = e[k] * c_ui_ev();
  if (dt_out) *dt_out = dt;
  release();
  return 0;
}

int gemsgpu_get_stream(gemsgpu_ctx* ctx, void** stream) {
  if (!ctx || !stream) return GEMSGPU_ERR_ARG;
  *stream = (void*)ctx->stream;
  return 0;
}

int gemsgpu_get_launch_count(gemsgpu_ctx* ctx, int64_t* launches) {
  if (!ctx || !launches) return GEMSGPU_ERR_ARG;
  *launches = ctx->launches;
  return 0;
}

static int time_kernels_set(gemsgpu_ctx* ctx, const std::vector<int>& ss, int reps, double* out_ms) {
  if (reps <= 0 || !out_ms) return fail(ctx, GEMSGPU_ERR_ARG, "time_kernels: reps > 0, out_ms");
  cudaSetDevice(ctx->device);
  const SysHost& h = ctx->sys[ss[0]];
  for (int s : ss) {
    const SysHost& q = ctx->sys[s];
    if (q.d.ff == FF_NONE) return fail(ctx, GEMSGPU_ERR_STATE, "no force field");
    if (q.d.ff != h.d.ff || q.d.prec != h.d.prec || q.lanes != h.lanes || q.variant != h.variant)
      return fail(ctx, GEMSGPU_ERR_ARG, "time_kernels: systems differ in force field or launch shape");
  }
  std::vector<int> need;
  for (int s : ss)
    if (ctx->sys[s].first || ctx->sys[s].pos_dirty || !ctx->sys[s].has_forces) need.push_back(s);
  if (!need.empty()) CHK(interact_group(ctx, need, true));
  const int K = h.lanes;
  bool single = true;
  for (int s : ss) single &= ctx->sys[s].ntypes == 1;
  BlockMap m;
  CHK(get_map(ctx, ss, BLOCK / K, 0, &m));
  const int* sa;
  CHK(sys_array(ctx, ss, &sa));
  cudaEvent_t ev[4];
  for (auto& e : ev) CU(cudaEventCreate(&e));
  const bool ts = h.d.ff == FF_TERSOFF;
  auto first_kernel = [&]() {
    if (h.d.ff == FF_SMATB) smatb_pass(ctx, 0, h.d.prec, h.variant, single, K, m);
    else if (ts) tersoff_bonds(ctx, h.d.prec, h.variant, m);
    else launch_forces(ctx, ss);
  };
  auto second_kernel = [&]() {
    if (h.d.ff == FF_SMATB) smatb_pass(ctx, 1, h.d.prec, h.variant, single, K, m);
    else if (ts) tersoff_gather(ctx, h.d.prec, m);
  };
  first_kernel();
  second_kernel();
  CU(cudaEventRecord(ev[0], ctx->stream));
  for (int r = 0; r < reps; r++) first_kernel();
  CU(cudaEventRecord(ev[1], ctx->stream));
  for (int r = 0; r < reps; r++) second_kernel();
  CU(cudaEventRecord(ev[2], ctx->stream));
  for (int r = 0; r < reps; r++) {
    k_force_rebuild<<<((int)ss.size() + 255) / 256, 256, 0, ctx->stream>>>(ctx->A, sa, (int)ss.size());
    ++ctx->launches;
    CHK(launch_rebuild(ctx, ss));
  }
  CU(cudaEventRecord(ev[3], ctx->stream));
  // the Tersoff gather adds to the forces: one untimed evaluation leaves them right
  if (ts) tersoff_pass(ctx, h.d.prec, h.variant, m);
  CU(cudaEventSynchronize(ev[3]));
  float t[3];
  CU(cudaEventElapsedTime(&t[0], ev[0], ev[1]));
  CU(cudaEventElapsedTime(&t[1], ev[1], ev[2]));
  CU(cudaEventElapsedTime(&t[2], ev[2], ev[3]));
  for (int k = 0; k < 3; k++) out_ms[k] = t[k] / reps;
  for (auto& e : ev) cudaEventDestroy(e);
  CU(cudaGetLastError());
  return 0;
}

int gemsgpu_time_kernels(gemsgpu_ctx* ctx, int sys, int reps, double* out_ms) {
  CHK(check_sys(ctx, sys));
  return time_kernels_set(ctx, {sys}, reps, out_ms);
}

int gemsgpu_batch_time_kernels(gemsgpu_ctx* ctx, const int* sys, int nsys, int reps, double* out_ms) {
  std::vector<int> ss;
  CHK(sys_list(ctx, sys, nsys, ss));
  return time_kernels_set(ctx, ss, reps, out_ms);
}

}  // extern "C"
