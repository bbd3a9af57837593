// mlp.cu -- the lambda-placement network: a 12 -> 64 -> 64 -> 11 perceptron
// with SiLU, run and trained on the 5th-generation tensor cores (tcgen05).
//
// One CTA of 128 threads works on tiles of 128 samples; thread t owns sample
// row t, which is TMEM lane t of every accumulator.  Each GEMM is one M = 128
// tcgen05.mma.kind::f16 chain (BF16 operands in shared memory, FP32
// accumulators in TMEM), issued by thread 0 and completed through an
// mbarrier.  Operands are K-major in the canonical no-swizzle layout: 8-row x
// 16-byte core matrices, the two 8-element halves of a 16-wide K slice 128
// bytes apart (leading byte offset), 8-row groups K*2*8 bytes apart (stride
// byte offset).  The backward GEMMs that contract over the batch take
// transposed copies written by the threads, so every operand has that one
// layout.  Training (Adam) runs all its iterations inside one launch; the
// FP32 master weights and moments live in global memory, their BF16 copies
// (and the transposes the backward pass needs) in shared memory.
//
// Every wait on the tensor cores is bounded: on time-out the kernel records
// QB_ERR_TIMEOUT, stops issuing work, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "qb_mlp.h"
#include "qsystem.hpp"

namespace qb {
void set_error(const std::string &m);

namespace mlp {

constexpr int IN = QB_MLP_IN, HID = QB_MLP_HIDDEN, OUT = QB_MLP_OUT;
constexpr int KIN = 16, NOUT = 16;   // padded input features / outputs
constexpr int ROWS = 128;            // samples per tile = TMEM lanes
constexpr int THREADS = 128;

// parameter vector offsets (floats)
constexpr int OW1 = 0, OB1 = OW1 + HID * IN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID, OW3 = OB2 + HID,
              OB3 = OW3 + OUT * HID, NPARAM = OB3 + OUT;
static_assert(NPARAM == QB_MLP_NPARAM, "parameter layout");

// shared-memory tiles (bytes): K-major canonical layout of R rows x K columns
constexpr int tile_bytes(int R, int K) { return R * K * 2; }
constexpr int S_X = 0;                                   // A  128 x 16  (x)
constexpr int S_W1 = S_X + tile_bytes(ROWS, KIN);        // B   64 x 16  (W1)
constexpr int S_H1 = S_W1 + tile_bytes(HID, KIN);        // A  128 x 64  (h1)
constexpr int S_W2 = S_H1 + tile_bytes(ROWS, HID);       // B   64 x 64  (W2)
constexpr int S_H2 = S_W2 + tile_bytes(HID, HID);        // A  128 x 64  (h2)
constexpr int S_W3 = S_H2 + tile_bytes(ROWS, HID);       // B   16 x 64  (W3, rows 11..15 zero)
constexpr int S_D3 = S_W3 + tile_bytes(NOUT, HID);       // A  128 x 16  (dz3, cols 11..15 zero)
constexpr int S_W3T = S_D3 + tile_bytes(ROWS, NOUT);     // B   64 x 16  (W3^T, cols 11..15 zero)
constexpr int S_D2 = S_W3T + tile_bytes(HID, NOUT);      // A  128 x 64  (dz2)
constexpr int S_W2T = S_D2 + tile_bytes(ROWS, HID);      // B   64 x 64  (W2^T)
constexpr int S_AT = S_W2T + tile_bytes(HID, HID);       // A  128 x 128 (dz^T: features x samples)
constexpr int S_BT = S_AT + tile_bytes(ROWS, ROWS);      // B   64 x 128 (activations^T)
constexpr int S_END = S_BT + tile_bytes(HID, ROWS);
constexpr int S_MISC = S_END;                            // mbarrier, TMEM address, bias gradients, loss
constexpr int SMEM_BYTES = S_MISC + 1024;

// TMEM columns of the accumulators (128 lanes x 512 columns allocated)
constexpr int T_Z1 = 0, T_Z2 = 64, T_Z3 = 128, T_DH2 = 144, T_DW3 = 208, T_DH1 = 272, T_DW2 = 336, T_DW1 = 400;
constexpr int TMEM_COLS = 512;
constexpr long long WAIT_LIMIT = 1LL << 26;   // try_wait polls before giving up (seconds)

// byte offset of element (r, k) in a K-major tile with K columns
__device__ __forceinline__ int kmaj(int r, int k, int K) {
  return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor of the 16-wide K slice s of a tile
__device__ __forceinline__ uint64_t sdesc(uint32_t tile_addr, int K, int s) {
  const uint32_t a = tile_addr + (uint32_t)s * 256u;
  uint64_t d = 0;
  d |= (uint64_t)((a >> 4) & 0x3FFFu);
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;                  // leading byte offset: K halves
  d |= (uint64_t)(((uint32_t)K * 16u >> 4) & 0x3FFFu) << 32;     // stride byte offset: 8-row groups
  d |= (uint64_t)1 << 46;                                         // descriptor version (sm_100)
  return d;                                                       // base offset 0, no swizzle
}

// instruction descriptor: D F32, A and B BF16, both K-major, M = 128, N
__host__ __device__ constexpr uint32_t idesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(ROWS >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// D[128 x N] (+)= A[128 x K] * B[N x K]^T over K/16 MMAs
__device__ __forceinline__ void gemm(uint32_t tmem_d, uint32_t a_tile, int Ka, uint32_t b_tile, int N, bool accumulate) {
  const uint32_t id = idesc(N);
  for (int s = 0; s < Ka / 16; s++)
    mma(tmem_d, sdesc(a_tile, Ka, s), sdesc(b_tile, Ka, s), id, (accumulate || s > 0) ? 1u : 0u);
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void st_bf16(uint8_t *sm, int tile, int r, int k, int K, float v) {
  *reinterpret_cast<__nv_bfloat16 *>(sm + tile + kmaj(r, k, K)) = __float2bfloat16_rn(v);
}
__device__ __forceinline__ float ld_bf16(const uint8_t *sm, int tile, int r, int k, int K) {
  return __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(sm + tile + kmaj(r, k, K)));
}

// add v, summed over the warp's 32 rows, to *acc (one shared atomic per warp)
__device__ __forceinline__ void warp_col_add(float *acc, float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(acc, v);
}

__device__ __forceinline__ float sigmoidf_(float z) { return 1.0f / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigmoidf_(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigmoidf_(z);
  return s * (1.0f + z * (1.0f - s));
}

struct Args {
  float *params;       // [NPARAM] FP32 master weights (updated in place when training)
  const float *x;      // [n x IN]
  const float *t;      // [n x OUT] targets (loss / training)
  int n;
  int mode;            // 0 forward, 1 loss + gradient, 2 train
  int iters;
  float lr, beta1, beta2, eps, wd;
  float *y;            // [n x OUT] outputs (forward)
  float *grad;         // [NPARAM] (mode 1)
  float *loss;         // [1] (mode 1) or [iters] (mode 2)
  float *adam_m, *adam_v;   // [NPARAM] (mode 2)
  int *status;
  long long wait_limit;     // try_wait polls of each tensor-core wait before it gives up
};

// BF16 copies of the weights: W1, W2, W3 as B operands, W2^T and W3^T for
// the backward data GEMMs.  Thread j < 64 writes row j of W1 and W2 (and
// column j of their transposes); thread j < 11 writes row j of W3.
__device__ void stage_weights(uint8_t *sm, const float *P, int j) {
  if (j < HID) {
    for (int i = 0; i < KIN; i++) st_bf16(sm, S_W1, j, i, KIN, i < IN ? P[OW1 + j * IN + i] : 0.0f);
    for (int i = 0; i < HID; i++) {
      const float w = P[OW2 + j * HID + i];     // W2[out j][in i]
      st_bf16(sm, S_W2, j, i, HID, w);
      st_bf16(sm, S_W2T, i, j, HID, w);         // W2^T: row = in i, K = out j
    }
  }
  if (j < NOUT)
    for (int i = 0; i < HID; i++) {
      const float w = j < OUT ? P[OW3 + j * HID + i] : 0.0f;
      st_bf16(sm, S_W3, j, i, HID, w);
      st_bf16(sm, S_W3T, i, j, NOUT, w);        // W3^T: row = hidden i, K = out j
    }
}

__global__ void __launch_bounds__(THREADS, 1) k_mlp(Args A) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int tid = threadIdx.x, warp = tid >> 5;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + S_MISC);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + S_MISC + 8);
  int *fail = reinterpret_cast<int *>(sm + S_MISC + 12);
  float *gb1 = reinterpret_cast<float *>(sm + S_MISC + 16);   // bias gradients
  float *gb2 = gb1 + HID;
  float *gb3 = gb2 + HID;
  float *red = gb3 + NOUT;                                     // [4] per-warp loss
  const uint32_t smb = smem_u32(sm);
  const uint32_t barp = smem_u32(bar);

  for (int k = tid * 16; k < S_END; k += THREADS * 16) *reinterpret_cast<uint4 *>(sm + k) = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    *fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barp) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);   // this warp's TMEM lanes
  uint32_t phase = 0;
  uint32_t late_phase = 2;   // the phase a wait gave up on (2: none)

  // issue on thread 0 after every thread's shared-memory writes, wait for completion
  auto run = [&](auto issue) -> bool {
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    if (tid == 0) {
      issue();
      commit(barp);
    }
    bool ok = wait_bar(barp, phase, A.wait_limit);
    if (!ok) late_phase = phase;
    phase ^= 1u;
    ok = __syncthreads_and(ok);
    tc_after();
    if (!ok && tid == 0) *fail = 1;
    return ok;
  };

  float *P = A.params;
  stage_weights(sm, P, tid);
  const int ntile = (A.n + ROWS - 1) / ROWS;
  const int iters = A.mode == 2 ? A.iters : 1;
  const float gscale = 2.0f / ((float)A.n * (float)OUT);   // d(mean squared error)/dy
  bool ok = true;

  for (int it = 0; it < iters && ok; it++) {
    if (tid < HID) { gb1[tid] = 0.f; gb2[tid] = 0.f; }
    if (tid < NOUT) gb3[tid] = 0.f;
    float lsum = 0.f;
    for (int tile = 0; tile < ntile && ok; tile++) {
      const int row = tile * ROWS + tid;
      const bool valid = row < A.n;
      // ---- forward
      for (int i = 0; i < KIN; i++) st_bf16(sm, S_X, tid, i, KIN, (valid && i < IN) ? A.x[(size_t)row * IN + i] : 0.f);
      ok = run([&] { gemm(tmem + T_Z1, smb + S_X, KIN, smb + S_W1, HID, false); });
      if (!ok) break;
      for (int c = 0; c < HID; c += 16) {
        float z[16];
        tld16(lane_base + T_Z1 + c, z);
        for (int k = 0; k < 16; k++) st_bf16(sm, S_H1, tid, c + k, HID, silu(z[k] + P[OB1 + c + k]));
      }
      ok = run([&] { gemm(tmem + T_Z2, smb + S_H1, HID, smb + S_W2, HID, false); });
      if (!ok) break;
      for (int c = 0; c < HID; c += 16) {
        float z[16];
        tld16(lane_base + T_Z2 + c, z);
        for (int k = 0; k < 16; k++) st_bf16(sm, S_H2, tid, c + k, HID, silu(z[k] + P[OB2 + c + k]));
      }
      ok = run([&] { gemm(tmem + T_Z3, smb + S_H2, HID, smb + S_W3, NOUT, false); });
      if (!ok) break;
      float y[16];
      tld16(lane_base + T_Z3, y);
      for (int k = 0; k < OUT; k++) y[k] += P[OB3 + k];
      if (A.mode == 0) {
        if (valid)
          for (int k = 0; k < OUT; k++) A.y[(size_t)row * OUT + k] = y[k];
        continue;
      }
      // ---- output gradient (mean squared error)
      for (int k = 0; k < NOUT; k++) {
        float d = 0.f;
        if (valid && k < OUT) {
          const float e = y[k] - A.t[(size_t)row * OUT + k];
          lsum += e * e;
          d = gscale * e;
        }
        st_bf16(sm, S_D3, tid, k, NOUT, d);
        st_bf16(sm, S_AT, k, tid, ROWS, d);             // dz3^T: row = output k, K = sample
        warp_col_add(&gb3[k], d);
      }
      for (int h = 0; h < HID; h++) st_bf16(sm, S_BT, h, tid, ROWS, ld_bf16(sm, S_H2, tid, h, HID));
      // dh2 = dz3 W3 ; dW3 += dz3^T h2
      ok = run([&] {
        gemm(tmem + T_DH2, smb + S_D3, NOUT, smb + S_W3T, HID, false);
        gemm(tmem + T_DW3, smb + S_AT, ROWS, smb + S_BT, HID, tile > 0);
      });
      if (!ok) break;
      for (int c = 0; c < HID; c += 16) {
        float g[16], z[16];
        tld16(lane_base + T_DH2 + c, g);
        tld16(lane_base + T_Z2 + c, z);
        for (int k = 0; k < 16; k++) {
          const float d = valid ? g[k] * dsilu(z[k] + P[OB2 + c + k]) : 0.f;
          st_bf16(sm, S_D2, tid, c + k, HID, d);
          st_bf16(sm, S_AT, c + k, tid, ROWS, d);       // dz2^T
          warp_col_add(&gb2[c + k], d);
        }
      }
      for (int h = 0; h < HID; h++) st_bf16(sm, S_BT, h, tid, ROWS, ld_bf16(sm, S_H1, tid, h, HID));
      // dh1 = dz2 W2 ; dW2 += dz2^T h1
      ok = run([&] {
        gemm(tmem + T_DH1, smb + S_D2, HID, smb + S_W2T, HID, false);
        gemm(tmem + T_DW2, smb + S_AT, ROWS, smb + S_BT, HID, tile > 0);
      });
      if (!ok) break;
      for (int c = 0; c < HID; c += 16) {
        float g[16], z[16];
        tld16(lane_base + T_DH1 + c, g);
        tld16(lane_base + T_Z1 + c, z);
        for (int k = 0; k < 16; k++) {
          const float d = valid ? g[k] * dsilu(z[k] + P[OB1 + c + k]) : 0.f;
          st_bf16(sm, S_AT, c + k, tid, ROWS, d);       // dz1^T
          warp_col_add(&gb1[c + k], d);
        }
      }
      for (int i = 0; i < KIN; i++) st_bf16(sm, S_BT, i, tid, ROWS, ld_bf16(sm, S_X, tid, i, KIN));
      // dW1 += dz1^T x
      ok = run([&] { gemm(tmem + T_DW1, smb + S_AT, ROWS, smb + S_BT, KIN, tile > 0); });
      if (!ok) break;
    }
    if (!ok || A.mode == 0) break;
    // ---- loss of this pass
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((tid & 31) == 0) red[warp] = lsum;
    __syncthreads();
    if (tid == 0) {
      const float L = (red[0] + red[1] + red[2] + red[3]) / ((float)A.n * (float)OUT);
      A.loss[A.mode == 2 ? it : 0] = L;
    }
    // ---- weight gradients from TMEM: thread j holds row j of dW1, dW2 (j < 64), dW3 (j < 11)
    float g1[16], g2[HID], g3[HID];
    tld16(lane_base + T_DW1, g1);
    for (int c = 0; c < HID; c += 16) tld16(lane_base + T_DW2 + c, g2 + c);
    for (int c = 0; c < HID; c += 16) tld16(lane_base + T_DW3 + c, g3 + c);
    const int j = tid;
    if (A.mode == 1) {
      if (j < HID) {
        for (int i = 0; i < IN; i++) A.grad[OW1 + j * IN + i] = g1[i];
        for (int i = 0; i < HID; i++) A.grad[OW2 + j * HID + i] = g2[i];
        A.grad[OB1 + j] = gb1[j];
        A.grad[OB2 + j] = gb2[j];
      }
      if (j < OUT) {
        for (int i = 0; i < HID; i++) A.grad[OW3 + j * HID + i] = g3[i];
        A.grad[OB3 + j] = gb3[j];
      }
      break;
    }
    // ---- Adam step on the FP32 master weights, then fresh BF16 copies
    const float t1 = (float)(it + 1);
    const float c1 = 1.0f / (1.0f - powf(A.beta1, t1)), c2 = 1.0f / (1.0f - powf(A.beta2, t1));
    // decoupled weight decay on the weight matrices, not on the biases
    auto adam = [&](int p, float g, float wd) {
      const float m = A.beta1 * A.adam_m[p] + (1.0f - A.beta1) * g;
      const float v = A.beta2 * A.adam_v[p] + (1.0f - A.beta2) * g * g;
      A.adam_m[p] = m;
      A.adam_v[p] = v;
      P[p] -= A.lr * ((m * c1) / (sqrtf(v * c2) + A.eps) + wd * P[p]);
    };
    if (j < HID) {
      for (int i = 0; i < IN; i++) adam(OW1 + j * IN + i, g1[i], A.wd);
      for (int i = 0; i < HID; i++) adam(OW2 + j * HID + i, g2[i], A.wd);
      adam(OB1 + j, gb1[j], 0.f);
      adam(OB2 + j, gb2[j], 0.f);
    }
    if (j < OUT) {
      for (int i = 0; i < HID; i++) adam(OW3 + j * HID + i, g3[i], A.wd);
      adam(OB3 + j, gb3[j], 0.f);
    }
    __threadfence_block();
    tc_before();
    __syncthreads();
    tc_after();
    stage_weights(sm, P, tid);
  }

  // ---- after a wait that gave up, the MMAs it waited for may still run:
  // wait for their commit once more (with the full limit) before the TMEM
  // they write is released
  if (late_phase != 2) wait_bar(barp, late_phase, WAIT_LIMIT);
  // ---- release TMEM (all tensor-core work has completed or timed out)
  tc_before();
  __syncthreads();
  if (*fail && tid == 0) atomicExch(A.status, (int)QB_ERR_TIMEOUT);
  if (warp == 0) {
    tc_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// ------------------------------------------------------------------ host

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

// polls of every tensor-core wait (qb_mlp_set_wait_limit); the default gives
// up after seconds
long long g_wait_limit = WAIT_LIMIT;

int call(int mode, float *params, const float *x, const float *t, int n, int iters, const qb_mlp_adam *adam,
         float *y, float *grad, float *loss, int device) {
  if (!params || !x || n <= 0 || n > QB_MLP_MAX_SAMPLES || (mode > 0 && !t) || (mode == 0 && !y) ||
      (mode == 1 && (!grad || !loss)) || (mode == 2 && (iters <= 0 || !adam || !loss))) {
    set_error("invalid argument");
    return QB_ERR_ARG;
  }
  auto cuda = [](cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw Error(QB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  try {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
      throw Error(QB_ERR_CUDA, "no such CUDA device");
    cuda(cudaSetDevice(device), "cudaSetDevice");
    const size_t np = NPARAM * sizeof(float), nx = (size_t)n * IN * sizeof(float), ny = (size_t)n * OUT * sizeof(float);
    const int nloss = mode == 2 ? iters : 1;
    DevBuf dP, dX, dT, dY, dG, dL, dM, dV, dS;
    cuda(cudaMalloc(&dP.p, np), "cudaMalloc");
    cuda(cudaMalloc(&dX.p, nx), "cudaMalloc");
    cuda(cudaMalloc(&dT.p, ny), "cudaMalloc");
    cuda(cudaMalloc(&dY.p, ny), "cudaMalloc");
    cuda(cudaMalloc(&dG.p, np), "cudaMalloc");
    cuda(cudaMalloc(&dL.p, nloss * sizeof(float)), "cudaMalloc");
    cuda(cudaMalloc(&dM.p, np), "cudaMalloc");
    cuda(cudaMalloc(&dV.p, np), "cudaMalloc");
    cuda(cudaMalloc(&dS.p, sizeof(int)), "cudaMalloc");
    cuda(cudaMemcpy(dP.p, params, np, cudaMemcpyHostToDevice), "upload");
    cuda(cudaMemcpy(dX.p, x, nx, cudaMemcpyHostToDevice), "upload");
    if (t) cuda(cudaMemcpy(dT.p, t, ny, cudaMemcpyHostToDevice), "upload");
    cuda(cudaMemset(dM.p, 0, np), "memset");
    cuda(cudaMemset(dV.p, 0, np), "memset");
    cuda(cudaMemset(dS.p, 0, sizeof(int)), "memset");
    Args a{};
    a.params = (float *)dP.p; a.x = (const float *)dX.p; a.t = (const float *)dT.p; a.n = n; a.mode = mode;
    a.iters = iters; a.y = (float *)dY.p; a.grad = (float *)dG.p; a.loss = (float *)dL.p;
    a.adam_m = (float *)dM.p; a.adam_v = (float *)dV.p; a.status = (int *)dS.p;
    a.wait_limit = g_wait_limit;
    if (adam) { a.lr = adam->lr; a.beta1 = adam->beta1; a.beta2 = adam->beta2; a.eps = adam->eps; a.wd = adam->weight_decay; }
    cuda(cudaFuncSetAttribute(k_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES), "smem attribute");
    k_mlp<<<1, THREADS, SMEM_BYTES>>>(a);
    cuda(cudaGetLastError(), "launch of mlp kernel");
    cuda(cudaDeviceSynchronize(), "mlp kernel");
    int st = 0;
    cuda(cudaMemcpy(&st, dS.p, sizeof(int), cudaMemcpyDeviceToHost), "status");
    if (st) throw Error(st, "tensor-core wait timed out in the mlp kernel");
    if (mode == 0) cuda(cudaMemcpy(y, dY.p, ny, cudaMemcpyDeviceToHost), "download");
    if (mode == 1) cuda(cudaMemcpy(grad, dG.p, np, cudaMemcpyDeviceToHost), "download");
    if (mode == 2) cuda(cudaMemcpy(params, dP.p, np, cudaMemcpyDeviceToHost), "download");
    if (mode > 0) cuda(cudaMemcpy(loss, dL.p, nloss * sizeof(float), cudaMemcpyDeviceToHost), "download");
    return QB_OK;
  } catch (const Error &e) {
    set_error(e.what());
    return e.code;
  }
}

}  // namespace mlp
}  // namespace qb

extern "C" {

int qb_mlp_forward(const float *params, const float *x, int n, float *y, int device) {
  return qb::mlp::call(0, const_cast<float *>(params), x, nullptr, n, 0, nullptr, y, nullptr, nullptr, device);
}

int qb_mlp_loss_grad(const float *params, const float *x, const float *t, int n, float *loss, float *grad,
                     int device) {
  return qb::mlp::call(1, const_cast<float *>(params), x, t, n, 0, nullptr, nullptr, grad, loss, device);
}

int qb_mlp_train(float *params, const float *x, const float *t, int n, int iters, const qb_mlp_adam *adam,
                 float *loss_history, int device) {
  return qb::mlp::call(2, params, x, t, n, iters, adam, nullptr, nullptr, loss_history, device);
}

int qb_mlp_set_wait_limit(long long polls) {
  if (polls < 0) { qb::set_error("negative wait limit"); return QB_ERR_ARG; }
  qb::mlp::g_wait_limit = polls > 0 ? polls : 0;
  return QB_OK;
}

}  // extern "C"
