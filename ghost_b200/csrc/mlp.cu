// mlp.cu -- the learned subgrid-stress closure: a 10 -> 64 -> 64 -> 6 MLP
// (GELU, tanh form) evaluated and trained with 5th-generation tensor cores.
//
// Per CTA tile of 128 grid points (rows):
//   forward   Z1 = X W1^T + b1, H1 = gelu(Z1); Z2 = H1 W2^T + b2, H2 = gelu(Z2);
//             Y = H2 W3^T + b3
//   backward  dY = 2 (Y - T) / (B * 6); dH2 = dY W3; dZ2 = dH2 gelu'(Z2);
//             dH1 = dZ2 W2; dZ1 = dH1 gelu'(Z1)
// Every product above is one or more tcgen05.mma (kind::f16, BF16 operands
// in shared memory, FP32 accumulators in tensor memory, M = 128 rows,
// K = 16 per instruction) issued by one thread and completed through an
// mbarrier; rows come back with tcgen05.ld (thread = row).  The weight
// gradients (a reduction over the batch) are accumulated in FP32 on the CUDA
// cores from the same BF16 activations, per CTA, and summed over CTAs in a
// fixed order by the Adam kernel.
#include <cuda_bf16.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <vector>

#include "../../include/ghost_b200.h"
#include "pipeline.cuh"

namespace gb {
int fail(int code, const char *fmt, ...);
}
using gb::fail;

namespace mlp {

constexpr int NIN = GHOST_MLP_NIN, NH = GHOST_MLP_NHID, NOUT = GHOST_MLP_NOUT;
constexpr int KIN = 16, KOUT = 16;  // padded widths of the input and output layers
constexpr int ROWS = 128;           // M of every MMA: one tile of grid points
constexpr int THREADS = 128;        // thread = row
// parameter vector offsets (FP32 master weights)
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH,
              OB3 = OW3 + NOUT * NH, NPARAM = OB3 + NOUT;
static_assert(NPARAM == GHOST_MLP_NPARAM, "parameter count");

#define MLP_CUDA(call)                                                                            \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return fail(GHOST_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------------
// K-major operand tile (rows x K bf16) in the canonical no-swizzle layout:
// 8x8 core matrices (8 rows of 16 bytes), core matrices adjacent along K
// 128 bytes apart (LBO), 8-row groups (K/8)*128 bytes apart (SBO).
__host__ __device__ constexpr int core_off(int r, int k, int K) {
  return (r >> 3) * (K >> 3) * 64 + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);  // in elements
}

__device__ __forceinline__ uint64_t smem_desc(const void *base, int K) {
  const uint64_t addr = (uint64_t)gb::smem_u32(base);
  uint64_t d = 0;
  d |= (addr & 0x3FFFFull) >> 4;                    // start address
  d |= (uint64_t)(128 >> 4) << 16;                   // LBO: next core matrix along K
  d |= (uint64_t)(((K >> 3) * 128) >> 4) << 32;     // SBO: next 8-row group
  d |= 1ull << 46;                                   // descriptor version (sm_100)
  return d;                                          // base offset 0, no swizzle
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, K-major A and B
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4)                  // D format F32
         | (1u << 7) | (1u << 10)   // A, B format BF16
         | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int accum) {
  uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   gb::smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// 16 FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// GELU in its tanh form (Hendrycks and Gimpel, 2016):
//   gelu(z) = z/2 (1 + tanh(c (z + a z^3))), c = sqrt(2/pi), a = 0.044715,
// with the hardware tanh (relative error about 2^-11, below the BF16
// resolution of the activations it feeds).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluC = 0.7978845608028654f, kGeluA = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_hw(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * z * (1.f + t);
}
__device__ __forceinline__ float gelu_d(float z) {
  const float t = tanh_hw(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * kGeluC * (1.f + 3.f * kGeluA * z * z);
}

// Eight consecutive K entries of one row are 16 contiguous bytes of a core
// matrix: round them to BF16 and store them with one 16-byte write.
__device__ __forceinline__ void store8_bf16(__nv_bfloat16 *dst, const float *v) {
  uint4 u;
  __nv_bfloat162 p;
  p = __floats2bfloat162_rn(v[0], v[1]);
  u.x = *reinterpret_cast<uint32_t *>(&p);
  p = __floats2bfloat162_rn(v[2], v[3]);
  u.y = *reinterpret_cast<uint32_t *>(&p);
  p = __floats2bfloat162_rn(v[4], v[5]);
  u.z = *reinterpret_cast<uint32_t *>(&p);
  p = __floats2bfloat162_rn(v[6], v[7]);
  u.w = *reinterpret_cast<uint32_t *>(&p);
  *reinterpret_cast<uint4 *>(dst) = u;
}

struct Smem {
  __nv_bfloat16 w1[NH * KIN];   // B operands (N x K)
  __nv_bfloat16 w2[NH * NH];
  __nv_bfloat16 w3[KOUT * NH];
  __nv_bfloat16 w3t[NH * KOUT];  // W3^T: N = 64 hidden, K = 16 outputs
  __nv_bfloat16 w2t[NH * NH];    // W2^T
  __nv_bfloat16 x[ROWS * KIN];   // A operands (M x K)
  __nv_bfloat16 h1[ROWS * NH];
  __nv_bfloat16 h2[ROWS * NH];
  __nv_bfloat16 dy[ROWS * KOUT];
  __nv_bfloat16 dz2[ROWS * NH];
  __nv_bfloat16 dz1[ROWS * NH];  // row-major: only the CUDA-core reductions read it
  float g1[ROWS * NH];           // gelu'(Z1), gelu'(Z2), row-major
  float g2[ROWS * NH];
  float b1[NH], b2[NH], b3[KOUT];
  uint64_t bar;
  uint32_t tmem;
  double loss;
};

constexpr int TMEM_COLS = 256;  // D1/D5 at 0, D2/D4 at 64, D3 at 128

// Loads the FP32 master weights as BF16 operands (with the transposed
// copies of the backward products when BWD).
template <class S, bool BWD> __device__ void load_weights(S &s, const float *__restrict__ P) {
  for (int q = threadIdx.x; q < NH * KIN; q += blockDim.x) {
    const int n = q / KIN, k = q % KIN;
    s.w1[core_off(n, k, KIN)] = __float2bfloat16_rn(k < NIN ? P[OW1 + n * NIN + k] : 0.f);
  }
  for (int q = threadIdx.x; q < NH * NH; q += blockDim.x) {
    const int n = q / NH, k = q % NH;
    s.w2[core_off(n, k, NH)] = __float2bfloat16_rn(P[OW2 + n * NH + k]);
    if constexpr (BWD) s.w2t[core_off(n, k, NH)] = __float2bfloat16_rn(P[OW2 + k * NH + n]);
  }
  for (int q = threadIdx.x; q < KOUT * NH; q += blockDim.x) {
    const int n = q / NH, k = q % NH;  // w3: N = outputs (padded), K = hidden
    s.w3[core_off(n, k, NH)] = __float2bfloat16_rn(n < NOUT ? P[OW3 + n * NH + k] : 0.f);
  }
  if constexpr (BWD) {
    for (int q = threadIdx.x; q < NH * KOUT; q += blockDim.x) {
      const int n = q / KOUT, k = q % KOUT;  // w3t: N = hidden, K = outputs
      s.w3t[core_off(n, k, KOUT)] = __float2bfloat16_rn(k < NOUT ? P[OW3 + k * NH + n] : 0.f);
    }
  }
  for (int q = threadIdx.x; q < NH; q += blockDim.x) {
    s.b1[q] = P[OB1 + q];
    s.b2[q] = P[OB2 + q];
  }
  for (int q = threadIdx.x; q < KOUT; q += blockDim.x) s.b3[q] = q < NOUT ? P[OB3 + q] : 0.f;
}

// One MMA chain D (tmem col `dcol`) = A (rows x K) * B^T (N x K), waited for
// by the whole CTA.  A K step of 16 is two core matrices, 256 bytes further
// along both operands.  On a timeout every thread agrees to give up, the
// status word is set, and the CTA waits (bounded) for the MMAs in flight so
// that the tensor memory can be released.
template <class S>
__device__ bool run_mma(S &s, uint32_t dcol, const __nv_bfloat16 *A, const __nv_bfloat16 *B, int K, int N,
                        uint32_t &phase, uint32_t cap, int *status) {
  // operands written by all threads (generic proxy) -> visible to the tensor cores
  gb::fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    const uint32_t idesc = instr_desc(ROWS, N);
    for (int ks = 0; ks < K / 16; ++ks)
      mma_bf16(s.tmem + dcol, smem_desc(A + ks * 128, K), smem_desc(B + ks * 128, K), idesc, ks > 0);
    mma_commit(&s.bar);
  }
  bool ok = gb::mbar_wait(&s.bar, phase, cap);
  ok = __syncthreads_and(ok);
  if (!ok) {
    if (threadIdx.x == 0) gb::record_timeout(status);
    gb::mbar_wait(&s.bar, phase, gb::kDrainPolls);
    __syncthreads();
  }
  phase ^= 1u;
  tc_fence_after();
  return ok;
}

// Reads this row's N accumulators of D at column dcol into v (N multiple of 16).
template <int N, class S> __device__ void read_row(const S &s, uint32_t dcol, float (&v)[N]) {
  const uint32_t lane_base = (uint32_t)(threadIdx.x & ~31) << 16;
#pragma unroll
  for (int c = 0; c < N; c += 16) {
    float t[16];
    tmem_ld16(s.tmem + lane_base + dcol + c, t);
#pragma unroll
    for (int q = 0; q < 16; ++q) v[c + q] = t[q];
  }
}

struct Gmlp {
  const float *P;  // parameters
  const float *x;  // B x NIN
  const float *t;  // B x NOUT (training)
  float *y;        // B x NOUT (inference), may be null
  float *grad;     // per-CTA gradient partials [gridDim.x][NPARAM + 1] (training), or null
  int B;
  float inv_count;  // 2 / (B * NOUT)
  int *status;
  uint32_t cap;
};

// Loss and gradients of one batch: forward, backward-data and weight-gradient
// sums per CTA (one CTA per SM).
__global__ void __launch_bounds__(THREADS, 1) mlp_train_kernel(Gmlp g) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  Smem &s = *reinterpret_cast<Smem *>(smem_raw);
  constexpr uint32_t COLS = TMEM_COLS;
  constexpr uint32_t D3 = 128;  // column of the layer-3 accumulator
  const int r = threadIdx.x;
  if (threadIdx.x < 32) {  // warp 0 owns the tensor memory
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(gb::smem_u32(&s.tmem)),
                 "r"(COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    gb::mbar_init(&s.bar, 1);
    gb::fence_barrier_init();
    s.loss = 0.0;
  }
  load_weights<Smem, true>(s, g.P);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  uint32_t phase = 0;
  // FP32 gradient accumulators: thread r owns entries q = r + THREADS*m of
  // the parameter vector (all rows of the tile summed per entry)
  constexpr int NOWN = (NPARAM + THREADS - 1) / THREADS;
  float acc[NOWN];
  {
#pragma unroll
    for (int m = 0; m < NOWN; ++m) acc[m] = 0.f;
  }
  double lacc = 0.0;
  const int ntiles = (g.B + ROWS - 1) / ROWS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row = tile * ROWS + r;
    const bool live = row < g.B;
    // ---- X
    {
      float xv[KIN];
#pragma unroll
      for (int k = 0; k < KIN; ++k) xv[k] = live && k < NIN ? g.x[(size_t)row * NIN + k] : 0.f;
#pragma unroll
      for (int k = 0; k < KIN; k += 8) store8_bf16(&s.x[core_off(r, k, KIN)], xv + k);
    }
    // ---- layer 1
    if (!run_mma(s, 0, s.x, s.w1, KIN, NH, phase, g.cap, g.status)) break;
    {
      float z[NH];
      read_row<NH>(s, 0, z);
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const float zz = z[h] + s.b1[h];
        z[h] = gelu(zz);
        s.g1[r * NH + h] = gelu_d(zz);
      }
#pragma unroll
      for (int h = 0; h < NH; h += 8) store8_bf16(&s.h1[core_off(r, h, NH)], z + h);
    }
    // ---- layer 2
    if (!run_mma(s, 64, s.h1, s.w2, NH, NH, phase, g.cap, g.status)) break;
    {
      float z[NH];
      read_row<NH>(s, 64, z);
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const float zz = z[h] + s.b2[h];
        z[h] = gelu(zz);
        s.g2[r * NH + h] = gelu_d(zz);
      }
#pragma unroll
      for (int h = 0; h < NH; h += 8) store8_bf16(&s.h2[core_off(r, h, NH)], z + h);
    }
    // ---- layer 3
    if (!run_mma(s, D3, s.h2, s.w3, NH, KOUT, phase, g.cap, g.status)) break;
    float yv[KOUT];
    read_row<KOUT>(s, D3, yv);
#pragma unroll
    for (int o = 0; o < KOUT; ++o) yv[o] += s.b3[o];
    {
      // ---- loss and dY
      float dyv[KOUT];
#pragma unroll
      for (int o = 0; o < KOUT; ++o) {
        float d = 0.f;
        if (live && o < NOUT) {
          const float e = yv[o] - g.t[(size_t)row * NOUT + o];
          lacc += (double)e * (double)e;
          d = e * g.inv_count;
        }
        dyv[o] = d;
      }
#pragma unroll
      for (int o = 0; o < KOUT; o += 8) store8_bf16(&s.dy[core_off(r, o, KOUT)], dyv + o);
      // ---- dH2 = dY W3  (A = dY: 128 x 16, B = W3^T: 64 x 16)
      if (!run_mma(s, 64, s.dy, s.w3t, KOUT, NH, phase, g.cap, g.status)) break;
      {
        float dh[NH];
        read_row<NH>(s, 64, dh);
#pragma unroll
        for (int h = 0; h < NH; ++h) dh[h] *= s.g2[r * NH + h];
#pragma unroll
        for (int h = 0; h < NH; h += 8) store8_bf16(&s.dz2[core_off(r, h, NH)], dh + h);
      }
      // ---- dH1 = dZ2 W2  (B = W2^T)
      if (!run_mma(s, 0, s.dz2, s.w2t, NH, NH, phase, g.cap, g.status)) break;
      {
        float dh[NH];
        read_row<NH>(s, 0, dh);
#pragma unroll
        for (int h = 0; h < NH; ++h) s.dz1[r * NH + h] = __float2bfloat16_rn(dh[h] * s.g1[r * NH + h]);
      }
      tc_fence_before();
      __syncthreads();
      // ---- weight gradients: sums over the tile's rows (FP32)
#pragma unroll 1
      for (int m = 0; m < NOWN; ++m) {
        const int q = r + THREADS * m;
        if (q >= NPARAM) break;
        float a = 0.f;
        if (q < OB1) {  // dW1[h][i] = sum dZ1[h] X[i]
          const int h = q / NIN, i = q % NIN;
          for (int rr = 0; rr < ROWS; ++rr)
            a += __bfloat162float(s.dz1[rr * NH + h]) * __bfloat162float(s.x[core_off(rr, i, KIN)]);
        } else if (q < OW2) {
          const int h = q - OB1;
          for (int rr = 0; rr < ROWS; ++rr) a += __bfloat162float(s.dz1[rr * NH + h]);
        } else if (q < OB2) {  // dW2[h2][h1] = sum dZ2[h2] H1[h1]
          const int h2 = (q - OW2) / NH, h1 = (q - OW2) % NH;
          for (int rr = 0; rr < ROWS; ++rr)
            a += __bfloat162float(s.dz2[core_off(rr, h2, NH)]) * __bfloat162float(s.h1[core_off(rr, h1, NH)]);
        } else if (q < OW3) {
          const int h = q - OB2;
          for (int rr = 0; rr < ROWS; ++rr) a += __bfloat162float(s.dz2[core_off(rr, h, NH)]);
        } else if (q < OB3) {  // dW3[o][h] = sum dY[o] H2[h]
          const int o = (q - OW3) / NH, h = (q - OW3) % NH;
          for (int rr = 0; rr < ROWS; ++rr)
            a += __bfloat162float(s.dy[core_off(rr, o, KOUT)]) * __bfloat162float(s.h2[core_off(rr, h, NH)]);
        } else {
          const int o = q - OB3;
          for (int rr = 0; rr < ROWS; ++rr) a += __bfloat162float(s.dy[core_off(rr, o, KOUT)]);
        }
        acc[m] += a;
      }
      __syncthreads();
    }
  }
  if (g.grad) {
    float *dst = g.grad + (size_t)blockIdx.x * (NPARAM + 1);
#pragma unroll
    for (int m = 0; m < NOWN; ++m) {
      const int q = r + THREADS * m;
      if (q < NPARAM) dst[q] = acc[m];
    }
    // loss: fixed-order sum over the CTA's rows
    __syncthreads();
    for (int w = 0; w < THREADS; ++w) {
      if (r == w) s.loss += lacc;
      __syncthreads();
    }
    if (r == 0) dst[NPARAM] = (float)s.loss;
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(s.tmem), "r"(COLS) : "memory");
}

// Inference on two tiles per CTA (256 threads; warps 0-3 take tile slot 0,
// warps 4-7 slot 1): one barrier and one MMA completion per layer serve both
// tiles.  Slot u accumulates in tensor-memory columns u*128 + (0: D1 and D3,
// 64: D2); the lanes are the rows, so both slots use lanes 0-127.
struct SmemF2 {
  __nv_bfloat16 w1[NH * KIN];
  __nv_bfloat16 w2[NH * NH];
  __nv_bfloat16 w3[KOUT * NH];
  __nv_bfloat16 x[2][ROWS * KIN];
  __nv_bfloat16 h1[2][ROWS * NH];
  __nv_bfloat16 h2[2][ROWS * NH];
  float b1[NH], b2[NH], b3[KOUT];
  uint64_t bar;
  uint32_t tmem;
};

__device__ bool run_mma2(SmemF2 &s, uint32_t dcol, const __nv_bfloat16 *A0, const __nv_bfloat16 *A1,
                         const __nv_bfloat16 *B, int K, int N, uint32_t &phase, uint32_t cap, int *status) {
  gb::fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x == 0) {
    const uint32_t idesc = instr_desc(ROWS, N);
    for (int u = 0; u < 2; ++u) {
      const __nv_bfloat16 *A = u ? A1 : A0;
      for (int ks = 0; ks < K / 16; ++ks)
        mma_bf16(s.tmem + u * 128 + dcol, smem_desc(A + ks * 128, K), smem_desc(B + ks * 128, K), idesc, ks > 0);
    }
    mma_commit(&s.bar);
  }
  bool ok = gb::mbar_wait(&s.bar, phase, cap);
  ok = __syncthreads_and(ok);
  if (!ok) {
    if (threadIdx.x == 0) gb::record_timeout(status);
    gb::mbar_wait(&s.bar, phase, gb::kDrainPolls);
    __syncthreads();
  }
  phase ^= 1u;
  tc_fence_after();
  return ok;
}

template <int N> __device__ void read_row2(const SmemF2 &s, uint32_t dcol, float (&v)[N]) {
  const uint32_t u = threadIdx.x >> 7;
  const uint32_t lane_base = (uint32_t)((threadIdx.x & 127) & ~31) << 16;
#pragma unroll
  for (int c = 0; c < N; c += 16) {
    float t[16];
    tmem_ld16(s.tmem + lane_base + u * 128 + dcol + c, t);
#pragma unroll
    for (int q = 0; q < 16; ++q) v[c + q] = t[q];
  }
}

__global__ void __launch_bounds__(2 * THREADS, 2) mlp_infer2_kernel(Gmlp g) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  SmemF2 &s = *reinterpret_cast<SmemF2 *>(smem_raw);
  constexpr uint32_t COLS = 256;
  const int r = threadIdx.x & 127, u = threadIdx.x >> 7;
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(gb::smem_u32(&s.tmem)),
                 "r"(COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    gb::mbar_init(&s.bar, 1);
    gb::fence_barrier_init();
  }
  load_weights<SmemF2, false>(s, g.P);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  uint32_t phase = 0;
  const int ntiles = (g.B + ROWS - 1) / ROWS;
  const int npairs = (ntiles + 1) / 2;
  for (int pair = blockIdx.x; pair < npairs; pair += gridDim.x) {
    const int row = (2 * pair + u) * ROWS + r;
    const bool live = row < g.B;
    {
      float xv[KIN];
#pragma unroll
      for (int k = 0; k < KIN; ++k) xv[k] = live && k < NIN ? g.x[(size_t)row * NIN + k] : 0.f;
#pragma unroll
      for (int k = 0; k < KIN; k += 8) store8_bf16(&s.x[u][core_off(r, k, KIN)], xv + k);
    }
    if (!run_mma2(s, 0, s.x[0], s.x[1], s.w1, KIN, NH, phase, g.cap, g.status)) break;
    {
      float z[NH];
      read_row2<NH>(s, 0, z);
#pragma unroll
      for (int h = 0; h < NH; ++h) z[h] = gelu(z[h] + s.b1[h]);
#pragma unroll
      for (int h = 0; h < NH; h += 8) store8_bf16(&s.h1[u][core_off(r, h, NH)], z + h);
    }
    if (!run_mma2(s, 64, s.h1[0], s.h1[1], s.w2, NH, NH, phase, g.cap, g.status)) break;
    {
      float z[NH];
      read_row2<NH>(s, 64, z);
#pragma unroll
      for (int h = 0; h < NH; ++h) z[h] = gelu(z[h] + s.b2[h]);
#pragma unroll
      for (int h = 0; h < NH; h += 8) store8_bf16(&s.h2[u][core_off(r, h, NH)], z + h);
    }
    if (!run_mma2(s, 0, s.h2[0], s.h2[1], s.w3, NH, KOUT, phase, g.cap, g.status)) break;
    float yv[KOUT];
    read_row2<KOUT>(s, 0, yv);
    if (live && g.y)
#pragma unroll
      for (int o = 0; o < NOUT; ++o) g.y[(size_t)row * NOUT + o] = yv[o] + s.b3[o];
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(s.tmem), "r"(COLS) : "memory");
}

// Sums the per-CTA partials in block order and applies Adam to the FP32
// master weights (grad = sum of the partials).
__global__ void adam_kernel(float *P, float *M, float *V, const float *partials, int nparts, int step, float lr,
                            float b1, float b2, float eps, float *grad_out, double *loss_out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < NPARAM) {
    float gq = 0.f;
    for (int c = 0; c < nparts; ++c) gq += partials[(size_t)c * (NPARAM + 1) + q];
    if (grad_out) grad_out[q] = gq;
    if (step > 0) {
      const float m = b1 * M[q] + (1.f - b1) * gq;
      const float v = b2 * V[q] + (1.f - b2) * gq * gq;
      M[q] = m;
      V[q] = v;
      const float mh = m / (1.f - powf(b1, (float)step));
      const float vh = v / (1.f - powf(b2, (float)step));
      P[q] -= lr * mh / (sqrtf(vh) + eps);
    }
  }
  if (q == 0 && loss_out) {
    double l = 0.0;
    for (int c = 0; c < nparts; ++c) l += (double)partials[(size_t)c * (NPARAM + 1) + NPARAM];
    *loss_out = l;
  }
}

}  // namespace mlp

using namespace mlp;

struct ghost_mlp {
  float *P = nullptr, *M = nullptr, *V = nullptr, *partials = nullptr, *grad = nullptr;
  double *loss = nullptr;
  int nparts = 0;
  int step = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  int *status = nullptr;
  uint32_t cap = 1u << 22;
};

static int mlp_launch(ghost_mlp *m, const float *x, const float *t, float *y, int B, bool train) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  const int ntiles = (B + ROWS - 1) / ROWS;
  Gmlp g{m->P, x, t, y, train ? m->partials : nullptr, B, 2.f / ((float)B * (float)NOUT), m->status, m->cap};
  if (train) {
    // one CTA per SM; the per-CTA gradient partials are summed by the Adam kernel
    const int grid = std::max(1, std::min(ntiles, nsm));
    const size_t smem = sizeof(Smem) + 1024;
    MLP_CUDA(cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mlp_train_kernel<<<grid, THREADS, smem, m->stream>>>(g);
    m->nparts = grid;
  } else {
    // two tiles per CTA, two CTAs per SM
    const int npairs = (ntiles + 1) / 2;
    const int grid = std::max(1, std::min(npairs, 2 * nsm));
    const size_t smem = sizeof(SmemF2) + 1024;
    MLP_CUDA(cudaFuncSetAttribute(mlp_infer2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mlp_infer2_kernel<<<grid, 2 * THREADS, smem, m->stream>>>(g);
  }
  MLP_CUDA(cudaGetLastError());
  return GHOST_OK;
}

static bool dev_ptr(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static int mlp_check_status(ghost_mlp *m) {
  int st = 0;
  MLP_CUDA(cudaMemcpy(&st, m->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemset(m->status, 0, sizeof(int));
    return fail(GHOST_ERR_TIMEOUT, "an MMA completion wait gave up");
  }
  return GHOST_OK;
}

extern "C" {

int ghost_mlp_create(int seed, ghost_mlp **out) {
  if (!out) return fail(GHOST_ERR_ARG, "null output");
  *out = nullptr;
  ghost_mlp *m = new ghost_mlp();
  cudaGetDevice(&m->device);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  const size_t pb = sizeof(float) * NPARAM;
  if (cudaMalloc(&m->P, pb) != cudaSuccess || cudaMalloc(&m->M, pb) != cudaSuccess ||
      cudaMalloc(&m->V, pb) != cudaSuccess || cudaMalloc(&m->grad, pb) != cudaSuccess ||
      cudaMalloc(&m->partials, sizeof(float) * (size_t)nsm * (NPARAM + 1)) != cudaSuccess ||
      cudaMalloc(&m->loss, sizeof(double)) != cudaSuccess || cudaMalloc(&m->status, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    ghost_mlp_destroy(m);
    return fail(GHOST_ERR_ALLOC, "MLP buffers");
  }
  // Glorot-uniform weights, zero biases (host RNG, seeded)
  std::vector<float> h(NPARAM, 0.f);
  std::mt19937 rng((uint32_t)seed);
  auto fill = [&](int off, int fan_out, int fan_in) {
    const float a = sqrtf(6.f / (float)(fan_in + fan_out));
    std::uniform_real_distribution<float> u(-a, a);
    for (int q = 0; q < fan_out * fan_in; ++q) h[off + q] = u(rng);
  };
  fill(OW1, NH, NIN);
  fill(OW2, NH, NH);
  fill(OW3, NOUT, NH);
  cudaMemcpy(m->P, h.data(), pb, cudaMemcpyHostToDevice);
  cudaMemset(m->M, 0, pb);
  cudaMemset(m->V, 0, pb);
  cudaMemset(m->status, 0, sizeof(int));
  *out = m;
  return GHOST_OK;
}

int ghost_mlp_destroy(ghost_mlp *m) {
  if (!m) return GHOST_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->P);
  cudaFree(m->M);
  cudaFree(m->V);
  cudaFree(m->grad);
  cudaFree(m->partials);
  cudaFree(m->loss);
  cudaFree(m->status);
  delete m;
  return GHOST_OK;
}

int ghost_mlp_set_stream(ghost_mlp *m, void *stream) {
  if (!m) return fail(GHOST_ERR_ARG, "null mlp");
  m->stream = (cudaStream_t)stream;
  return GHOST_OK;
}

int ghost_mlp_get_params(ghost_mlp *m, float *host) {
  if (!m || !host) return fail(GHOST_ERR_ARG, "null argument");
  MLP_CUDA(cudaStreamSynchronize(m->stream));
  MLP_CUDA(cudaMemcpy(host, m->P, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  return GHOST_OK;
}

int ghost_mlp_set_params(ghost_mlp *m, const float *host) {
  if (!m || !host) return fail(GHOST_ERR_ARG, "null argument");
  MLP_CUDA(cudaStreamSynchronize(m->stream));
  MLP_CUDA(cudaMemcpy(m->P, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
  MLP_CUDA(cudaMemset(m->M, 0, sizeof(float) * NPARAM));
  MLP_CUDA(cudaMemset(m->V, 0, sizeof(float) * NPARAM));
  m->step = 0;
  return GHOST_OK;
}

int ghost_mlp_forward(ghost_mlp *m, const float *x, float *y, int B) {
  if (!m || !x || !y || B < 1) return fail(GHOST_ERR_ARG, "bad argument");
  if (!dev_ptr(x) || !dev_ptr(y)) return fail(GHOST_ERR_ARG, "ghost_mlp_forward needs device arrays");
  return mlp_launch(m, x, nullptr, y, B, false);
}

int ghost_mlp_gradients(ghost_mlp *m, const float *x, const float *t, int B, float *grad_host, double *loss) {
  if (!m || !x || !t || B < 1) return fail(GHOST_ERR_ARG, "bad argument");
  if (!dev_ptr(x) || !dev_ptr(t)) return fail(GHOST_ERR_ARG, "ghost_mlp_gradients needs device arrays");
  int st = mlp_launch(m, x, t, nullptr, B, true);
  if (st) return st;
  adam_kernel<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->P, m->M, m->V, m->partials, m->nparts, 0, 0.f, 0.9f,
                                                            0.999f, 1e-8f, m->grad, m->loss);
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaStreamSynchronize(m->stream));
  if (grad_host) MLP_CUDA(cudaMemcpy(grad_host, m->grad, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  if (loss) {
    MLP_CUDA(cudaMemcpy(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost));
    *loss /= (double)B * NOUT;
  }
  return mlp_check_status(m);
}

int ghost_mlp_train_step(ghost_mlp *m, const float *x, const float *t, int B, float lr, double *loss) {
  if (!m || !x || !t || B < 1) return fail(GHOST_ERR_ARG, "bad argument");
  if (!dev_ptr(x) || !dev_ptr(t)) return fail(GHOST_ERR_ARG, "ghost_mlp_train_step needs device arrays");
  int st = mlp_launch(m, x, t, nullptr, B, true);
  if (st) return st;
  m->step += 1;
  adam_kernel<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->P, m->M, m->V, m->partials, m->nparts, m->step, lr,
                                                            0.9f, 0.999f, 1e-8f, nullptr, m->loss);
  MLP_CUDA(cudaGetLastError());
  if (loss) {
    MLP_CUDA(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MLP_CUDA(cudaStreamSynchronize(m->stream));
    *loss /= (double)B * NOUT;
    return mlp_check_status(m);
  }
  return GHOST_OK;
}

}  // extern "C"
