// noalloc.cu -- SMA-TB forces for callers that cannot allocate device memory.
//
// Some callers of this library may not allocate: a host program that owns a
// fixed device-memory budget and hands the library only its own buffers, or
// one that evaluates forces inside a region where cudaMalloc / cudaFree are
// not allowed (they synchronise the whole device, and are refused while a
// stream is being captured into a CUDA graph).  For them this file provides
// gemsgpu_smatb_forces_noalloc: the SMA-TB density and force passes over
// caller-owned device buffers, with the only scratch (the per-atom density
// rho_i and 1/sqrt(rho_i) carried from the first pass to the second) in a
// fixed file-scope device array.  Nothing here allocates.
//
// The neighbourhood is all pairs within rce (minimum image on periodic
// dimensions), so no neighbour list -- and no list memory -- is needed; the
// result equals the list-based SMA-TB kernels' up to summation order.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/gemsgpu.h"
#include "common.cuh"

namespace {

constexpr int NA_MAX = GEMSGPU_NOALLOC_MAX_ATOMS;
constexpr int NA_BLOCK = 128;
constexpr int NA_MAXDEV = 64;

// rho_i in [0, NA_MAX), 1/sqrt(rho_i) in [NA_MAX, 2 NA_MAX): 256 KiB that
// every GPU which loads the library holds until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[2 * NA_MAX];

// Device address of g_noalloc_scratch per device.  In host code the symbol
// is only a host-side stand-in, so its device address is looked up once per
// device (with that device current) and passed to the kernels.  The cached
// address belongs to the device's current context: after cudaDeviceReset
// (or anything else that destroys and re-creates the primary context) the
// module may load elsewhere, so a process that resets a device must not
// call gemsgpu_smatb_forces_noalloc on it again.
std::mutex g_na_mutex;
double* g_na_addr[NA_MAXDEV] = {nullptr};

cudaError_t scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= NA_MAXDEV) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_na_mutex);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_na_addr[dev] = static_cast<double*>(p);
  }
  *out = g_na_addr[dev];
  return cudaSuccess;
}

struct NaBox {
  double L[3], invL[3];
  int pbc[3];
};

// smatb_set (src/TB.F90:106-170) constants for one species pair
struct NaSm {
  double A, eps2, p, q, r0, rci, rce, b1, b2, b3, r1, r2, r3;
};

__device__ __forceinline__ void na_vd(const NaBox& B, const double* x, int i, int j, double& v0,
                                      double& v1, double& v2) {
  v0 = x[3 * j] - x[3 * i];
  v1 = x[3 * j + 1] - x[3 * i + 1];
  v2 = x[3 * j + 2] - x[3 * i + 2];
  if (B.pbc[0]) v0 = v0 - B.L[0] * round(v0 * B.invL[0]);
  if (B.pbc[1]) v1 = v1 - B.L[1] * round(v1 * B.invL[1]);
  if (B.pbc[2]) v2 = v2 - B.L[2] * round(v2 * B.invL[2]);
}

// density pass (smatb_preinteraction, src/TB.F90:367-455) into the scratch
__global__ void __launch_bounds__(NA_BLOCK) k_na_rho(const double* __restrict__ x, int n, NaBox B,
                                                     NaSm c, double* __restrict__ scratch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double band = 0.0;
  for (int j = 0; j < n; j++) {
    if (j == i) continue;
    double v0, v1, v2;
    na_vd(B, x, i, j, v0, v1, v2);
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
  }
  scratch[i] = band;                 // every entry < n is written: no clearing
  scratch[NA_MAX + i] = 1.0 / sqrt(band);
}

// force pass (smatb_interact, src/TB.F90:457-586) from the scratch
__global__ void __launch_bounds__(NA_BLOCK) k_na_force(const double* __restrict__ x, int n, NaBox B,
                                                       NaSm c, const double* __restrict__ scratch,
                                                       double ev_ui, double* __restrict__ force,
                                                       double* __restrict__ epot) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double ebi = scratch[NA_MAX + i];
  double f0 = 0.0, f1 = 0.0, f2 = 0.0, ep = 0.0;
  for (int j = 0; j < n; j++) {
    if (j == i) continue;
    double v0, v1, v2;
    na_vd(B, x, i, j, v0, v1, v2);
    double dr = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    if (dr > c.rce) continue;
    double ebs = ebi + scratch[NA_MAX + j];
    double factor, repul;
    if (dr <= c.rci) {
      double t = dr / c.r0 - 1.0;
      repul = c.A * exp(-c.p * t);
      factor = 2.0 * repul * (c.p / c.r0) - c.eps2 * 0.5 * exp(-2.0 * c.q * t) * (2.0 * c.q / c.r0) * ebs;
    } else {
      double d = dr - c.rce, d2 = d * d, d3 = d2 * d, d4 = d3 * d;
      double P = (c.b1 * d2 + c.b2 * d + c.b3) * d3;
      double dP = 5.0 * c.b1 * d4 + 4.0 * c.b2 * d3 + 3.0 * c.b3 * d2;
      double dR = 5.0 * c.r1 * d4 + 4.0 * c.r2 * d3 + 3.0 * c.r3 * d2;
      factor = P * dP * ebs - 2.0 * dR;
      repul = (c.r1 * d2 + c.r2 * d + c.r3) * d3;
    }
    double fr = factor * ev_ui / dr;
    f0 -= fr * v0;
    f1 -= fr * v1;
    f2 -= fr * v2;
    ep += repul;
  }
  force[3 * i] = f0;
  force[3 * i + 1] = f1;
  force[3 * i + 2] = f2;
  epot[i] = (ep - sqrt(scratch[i])) * ev_ui;
}

}  // namespace

extern "C" int gemsgpu_smatb_forces_noalloc(const double* d_pos, int n, int boxed, const double L[3],
                                            const int pbc[3], double A, double xi, double p, double q,
                                            double r0, double rci, double rce, double* d_force,
                                            double* d_epot, void* stream) {
  if (!d_pos || !d_force || !d_epot || n <= 0) return GEMSGPU_ERR_ARG;
  if (n > NA_MAX) return GEMSGPU_ERR_FULL;
  if (!(rce > rci) || !(r0 > 0.0)) return GEMSGPU_ERR_ARG;
  NaBox B{};
  for (int k = 0; k < 3; k++) {
    bool per = boxed && L && pbc && pbc[k];
    if (per && !(L[k] > 0.0)) return GEMSGPU_ERR_ARG;
    B.pbc[k] = per ? 1 : 0;
    B.L[k] = per ? L[k] : 0.0;
    B.invL[k] = per ? 1.0 / L[k] : 0.0;
  }
  // smatb_set tail coefficients (Logsdail et al. 2012)
  NaSm c{};
  const double dcut = rce - rci;
  const double ab = -1.0 / (dcut * dcut * dcut);
  double bb = -(q / r0) / (dcut * dcut);
  double cb = -((q / r0) * (q / r0)) / dcut;
  double aux = xi * std::exp(-q * (rci / r0 - 1.0));
  c.b1 = aux * (12.0 * ab - 6.0 * bb + cb) / (2.0 * (dcut * dcut));
  c.b2 = aux * (15.0 * ab - 7.0 * bb + cb) / dcut;
  c.b3 = aux * (20.0 * ab - 8.0 * bb + cb) / 2.0;
  aux = A * std::exp(-p * (rci / r0 - 1.0));
  bb = -(p / r0) / (dcut * dcut);
  cb = -((p / r0) * (p / r0)) / dcut;
  c.r1 = aux * (12.0 * ab - 6.0 * bb + cb) / (2.0 * (dcut * dcut));
  c.r2 = aux * (15.0 * ab - 7.0 * bb + cb) / dcut;
  c.r3 = aux * (20.0 * ab - 8.0 * bb + cb) / 2.0;
  c.A = A;
  c.eps2 = xi * xi;
  c.p = p;
  c.q = q;
  c.r0 = r0;
  c.rci = rci;
  c.rce = rce;
  double* scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) return GEMSGPU_ERR_CUDA;
  double ev_ui = EV_UI;  // GEMS internal energy unit
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid((n + NA_BLOCK - 1) / NA_BLOCK), block(NA_BLOCK);
  // cudaLaunchKernel returns this launch's own status, so an error left
  // behind by the caller's earlier work is not reported as this call's
  void* rho_args[] = {(void*)&d_pos, (void*)&n, (void*)&B, (void*)&c, (void*)&scratch};
  if (cudaLaunchKernel((const void*)k_na_rho, grid, block, rho_args, 0, st) != cudaSuccess)
    return GEMSGPU_ERR_CUDA;
  const double* scr = scratch;
  void* force_args[] = {(void*)&d_pos, (void*)&n, (void*)&B, (void*)&c, (void*)&scr, (void*)&ev_ui,
                        (void*)&d_force, (void*)&d_epot};
  if (cudaLaunchKernel((const void*)k_na_force, grid, block, force_args, 0, st) != cudaSuccess)
    return GEMSGPU_ERR_CUDA;
  return GEMSGPU_OK;
}
