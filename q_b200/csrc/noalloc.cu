// noalloc.cu -- water-water energy and gradient of one water sphere on
// caller-owned device buffers, without any device allocation.
//
// Some callers cannot allocate device memory: a host that hands the library
// only buffers from its own pool (a framework caching allocator, a
// pre-sized arena in a long-running service) or that forbids cudaMalloc on
// its thread.  This entry point serves them.  Its one piece of scratch memory,
// the water neighbour list, is a fixed file-scope __device__ array, so every
// GPU that loads this library holds QB_STATIC_WW_SCRATCH_BYTES of device
// memory until the process exits.  The computation is the library's SPC
// water-water pair kernel (the same math as the batch engine's), for systems
// of up to QB_STATIC_WW_MAX_WATERS waters with up to
// QB_STATIC_WW_MAX_NEIGHBOURS neighbours each.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "qb.h"

namespace qb {
void set_error(const std::string &m);
}

namespace {

constexpr int kMaxW = QB_STATIC_WW_MAX_WATERS;
constexpr int kMaxNb = QB_STATIC_WW_MAX_NEIGHBOURS;
constexpr unsigned kFull = 0xffffffffu;

// neighbour lists: kMaxW rows of kMaxNb water indices, then kMaxW counts
static __device__ __align__(256) int g_ww_scratch[kMaxW * kMaxNb + kMaxW];

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// One warp per water: every other water whose O lies within the cut-off.
__global__ void k_static_ww_list(const double *__restrict__ x, int nwat, double rc2,
                                 const unsigned char *__restrict__ excl, int *scratch, int *status) {
  int iw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (iw >= nwat) return;
  int *row = scratch + (size_t)iw * kMaxNb;
  int *count = scratch + (size_t)kMaxW * kMaxNb;
  int cnt = 0;
  if (!(excl && excl[iw])) {
    double xi = x[9 * iw], yi = x[9 * iw + 1], zi = x[9 * iw + 2];
    for (int base = 0; base < nwat; base += 32) {
      int jw = base + lane;
      bool ok = false;
      if (jw < nwat && jw != iw && !(excl && excl[jw])) {
        double dx = xi - x[9 * jw], dy = yi - x[9 * jw + 1], dz = zi - x[9 * jw + 2];
        ok = dx * dx + dy * dy + dz * dz <= rc2;
      }
      unsigned bal = __ballot_sync(kFull, ok);
      if (ok) {
        int pos = cnt + __popc(bal & ((1u << lane) - 1u));
        if (pos < kMaxNb) row[pos] = jw;
      }
      cnt += __popc(bal);
    }
  }
  if (lane == 0) {
    if (cnt > kMaxNb) { atomicExch(status, (int)QB_ERR_LIST_OVERFLOW); cnt = kMaxNb; }
    count[iw] = cnt;
  }
}

// SPC/TIP3P water-water terms (reference routine nonbond_ww_spc,
// src/q6/md.f90:11823): one warp per water, lanes over its neighbours, the
// water's 9 gradient components reduced with warp shuffles; every pair is seen
// from both waters, so each side adds half of the pair energy.
__global__ void k_static_ww_force(const double *__restrict__ x, int nwat, float qo, float qh, double A_OO,
                                  double B_OO, const int *__restrict__ scratch, double *grad, double *energy) {
  int iw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  bool active = iw < nwat;
  double f[9];
#pragma unroll
  for (int k = 0; k < 9; k++) f[k] = 0.0;
  double el = 0.0, vdw = 0.0;
  if (active) {
    const int *row = scratch + (size_t)iw * kMaxNb;
    int n = scratch[(size_t)kMaxW * kMaxNb + iw];
    double xi[9];
#pragma unroll
    for (int k = 0; k < 9; k++) xi[k] = x[9 * iw + k];
    const float qoo = qo * qo, qoh = qo * qh, qhh = qh * qh;
    for (int k = lane; k < n; k += 32) {
      int jw = row[k];
      double xj[9];
#pragma unroll
      for (int c = 0; c < 9; c++) xj[c] = x[9 * jw + c];
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
          double dx = xj[3 * b] - xi[3 * a], dy = xj[3 * b + 1] - xi[3 * a + 1], dz = xj[3 * b + 2] - xi[3 * a + 2];
          double rinv = sqrt(1.0 / (dx * dx + dy * dy + dz * dz));
          double r2 = rinv * rinv;
          float qq = (a == 0 && b == 0) ? qoo : ((a == 0 || b == 0) ? qoh : qhh);
          double Vel = (double)qq * rinv, dv;
          if (a == 0 && b == 0) {
            double r6 = r2 * r2 * r2;
            double Va = A_OO * r6 * r6, Vb = B_OO * r6;
            vdw += Va - Vb;
            dv = r2 * (-Vel - 12. * Va + 6. * Vb);
          } else {
            dv = r2 * (-Vel);
          }
          el += Vel;
          f[3 * a] -= dv * dx;
          f[3 * a + 1] -= dv * dy;
          f[3 * a + 2] -= dv * dz;
        }
    }
  }
#pragma unroll
  for (int k = 0; k < 9; k++) f[k] = wsum(f[k]);
  el = wsum(el);
  vdw = wsum(vdw);
  if (active && lane == 0) {
#pragma unroll
    for (int k = 0; k < 9; k++) grad[9 * iw + k] = f[k];
    atomicAdd(&energy[0], 0.5 * el);
    atomicAdd(&energy[1], 0.5 * vdw);
  }
}

// Device address of the scratch array, looked up once per device and CUDA
// context.  The context is part of the key: after a cudaDeviceReset the
// device's new primary context holds a new copy of the array, and the address
// cached for the old context would no longer be valid.
constexpr int kMaxDevices = 64;
std::mutex g_mutex;
int *g_scratch_ptr[kMaxDevices] = {nullptr};
void *g_scratch_ctx[kMaxDevices] = {nullptr};

// The current context (driver call cuCtxGetCurrent, reached through the
// runtime's entry-point table so the library needs no link to libcuda).
void *current_context() {
  using Fn = int (*)(void **);
  static Fn fn = nullptr;
  static bool looked = false;
  if (!looked) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<Fn>(p);
    looked = true;
  }
  void *ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

}  // namespace

extern "C" int qb_ww_energy_static(const double *x, int nwat, float crg_ow, float crg_hw, double A_OO,
                                   double B_OO, double cutoff, const unsigned char *excl, double *grad,
                                   double *energy, int *status, void *stream) {
  if (nwat < 0 || nwat > kMaxW) {
    qb::set_error("qb_ww_energy_static: " + std::to_string(nwat) + " waters exceeds the static limit of " +
                  std::to_string(kMaxW));
    return QB_ERR_ARG;
  }
  if (!x || !grad || !energy || !status || !(cutoff > 0)) {
    qb::set_error("qb_ww_energy_static: null buffer or non-positive cut-off");
    return QB_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    qb::set_error("qb_ww_energy_static: no current CUDA device");
    return QB_ERR_CUDA;
  }
  int *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    void *ctx = current_context();
    if (!g_scratch_ptr[dev] || !ctx || g_scratch_ctx[dev] != ctx) {
      // first call on this device: the symbol's device address, with the
      // device current (the host-side name is not a device address)
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_ww_scratch);
      if (e != cudaSuccess) {
        qb::set_error(std::string("qb_ww_energy_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return QB_ERR_CUDA;
      }
      g_scratch_ptr[dev] = static_cast<int *>(p);
      // the lookup made the device's primary context current if none was
      g_scratch_ctx[dev] = current_context();
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(energy, 0, 2 * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) {
    qb::set_error(std::string("qb_ww_energy_static: ") + cudaGetErrorString(e));
    return QB_ERR_CUDA;
  }
  if (nwat == 0) return QB_OK;
  int blocks = (nwat * 32 + 255) / 256;
  k_static_ww_list<<<blocks, 256, 0, s>>>(x, nwat, cutoff * cutoff, excl, scratch, status);
  k_static_ww_force<<<blocks, 256, 0, s>>>(x, nwat, crg_ow, crg_hw, A_OO, B_OO, scratch, grad, energy);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    qb::set_error(std::string("qb_ww_energy_static: launch: ") + cudaGetErrorString(e));
    return QB_ERR_CUDA;
  }
  return QB_OK;
}
