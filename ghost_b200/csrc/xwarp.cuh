// xwarp.cuh -- plain x transforms with one warp per x line.
//
// GHOST's fftp3d_real_to_complex / fftp3d_complex_to_real x stage (the
// real-to-complex and complex-to-real FFTW plans of fftp-3/fftp3D.fpp) for
// FP32 data and x lines of NX = 512 points: each line is a 256-point
// complex transform held by the 32 lanes of one warp, 8 values per lane, so
// the transform's shared-memory exchanges go through a buffer private to
// the warp and need __syncwarp only.
//
// Shared-memory layouts (8-byte complex elements):
//   tiles  element (k, l) of a kx-row tile (row k = 8 z-values, 64 bytes)
//          at byte 64k + 8l with the 16-byte chunk index XORed by
//          (k >> 1) & 3: the TMA SWIZZLE_64B pattern (every tile base is
//          1024-byte aligned and every box starts on 16 rows);
//   lines  element i of a warp's exchange buffer at
//          i ^ ((i >> 4) & 7) ^ ((i >> 3) & 8): the transform's exchange
//          patterns (t + 32e reads, radix-8 stage writes 8t + r and
//          64(t/8) + (t%8) + 8r) then touch 16 distinct 8-byte slots per
//          half-warp, the minimum for 8-byte accesses.
// The mirror element X_{M-k} (pack) and Z_{M-k} (unpack) of k = t + 32e is
// register 7-e of lane 32-t (lane 0: its own register 8-e), fetched by
// shuffles.
#pragma once
#include "fft_core.cuh"
#include "passes.cuh"
#include "pipeline.cuh"

namespace gb {

__device__ __forceinline__ int xw_line_swz(int i) { return i ^ ((i >> 4) & 7) ^ ((i >> 3) & 8); }
// byte offset of element (k, l) of a 64-byte-row tile under SWIZZLE_64B
__device__ __forceinline__ uint32_t xw_tile_off(int k, int l) {
  return ((uint32_t)k << 6) + (((uint32_t)(l >> 1) ^ ((uint32_t)(k >> 1) & 3u)) << 4) + ((uint32_t)(l & 1) << 3);
}

// pack for the inverse: Z_k = (X_k + conj X_{M-k}) + i e^{+2 pi i k/NX} (X_k - conj X_{M-k})
__device__ __forceinline__ float2 xw_pack(float2 xk, float2 xm, float2 w) {
  const float2 a = mk(xk.x + xm.x, xk.y - xm.y);
  const float2 b = mk(xk.x - xm.x, xk.y + xm.y);
  const float2 wb = cmulc(b, w);
  return mk(a.x - wb.y, a.y + wb.x);
}

__device__ __forceinline__ float2 shfl2(float2 v, int src) {
  return mk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// ====================================================================
// Plain x transforms (fftp3d_real_to_complex / fftp3d_complex_to_real,
// fftp-3/fftp3D.fpp), FP32, NX = 512, one warp per x line, persistent CTAs
// over tiles of 8 z-values at one y.  Both stream their input through a
// STAGES-deep TMA ring refilled by the last warp to read a slot.
//   r2c  real rows (x fastest, 2 KB each) arrive line-major, so a warp reads
//        its line without bank conflicts; the half spectrum is unpacked
//        into a swizzled kx-row tile and copied out after a CTA barrier.
//   c2r  the half spectrum arrives as SWIZZLE_64B kx-row tiles; each lane
//        stores its real pairs straight from registers (a warp writes 256
//        contiguous bytes per store).
// A timed-out wait records GHOST_ERR_TIMEOUT; the CTA then finishes its
// schedule with bounded waits (no early exit is needed: no CTA barrier
// waits on a warp that gave up).
// ====================================================================
template <int NX, int STAGES> struct XWPlainGeom {
  static constexpr int M = NX / 2, BZ = 8;
  static constexpr int SROWS = M + 32;
  static constexpr int OROWS = M + 32;  // two 144-row store boxes
  static constexpr size_t r2c_in = (size_t)BZ * M * 8;  // line-major real rows
  static constexpr size_t c2r_in = (size_t)SROWS * 64;  // kx-row tile
  static constexpr size_t out_bytes = (size_t)OROWS * 64;
  static constexpr size_t tail(size_t off_xw) { return off_xw + (size_t)BZ * M * 8 + NX * 8 + (STAGES + 1) * 8 + STAGES * 8 + 1024; }
  static constexpr size_t r2c_bytes = tail(STAGES * r2c_in + 2 * out_bytes);
  static constexpr size_t c2r_bytes = tail(STAGES * c2r_in);
};

// Shared tail of both kernels' shared memory: exchange buffers, twiddles,
// barriers, arrival counters, last issued loads.
struct XWRing {
  float2 *xw, *tw;
  uint64_t *full, *never;
  unsigned *cnt;
  int *last;
  __device__ __forceinline__ XWRing(unsigned char *base, int M, int NX, int STAGES, int l) {
    xw = reinterpret_cast<float2 *>(base) + (size_t)l * M;
    tw = reinterpret_cast<float2 *>(base) + (size_t)8 * M;
    full = reinterpret_cast<uint64_t *>(tw + NX);
    never = full + STAGES;
    cnt = reinterpret_cast<unsigned *>(never + 1);
    last = reinterpret_cast<int *>(cnt + STAGES);
  }
};

// bounded wait for load k of slot k % STAGES; a timed-out wait records the
// status, then waits (bounded) once more so that the slot stays in step
template <int STAGES>
__device__ __forceinline__ void xw_wait(const XWRing &rg, int k, const PipeCtl &ctl) {
  const int s = k % STAGES;
  const uint32_t par = (uint32_t)(k / STAGES) & 1u;
  const bool got = (!ctl.stall || k > 0 || injected_stall_wait(rg.never, ctl.cap)) && mbar_wait(&rg.full[s], par, ctl.cap);
  if (!got) {
    if ((threadIdx.x & 31) == 0) record_timeout(ctl.status);
    mbar_wait(&rg.full[s], par, kDrainPolls);
  }
}

// The half spectrum of a tile leaves by TMA tensor stores (two boxes of
// 144 kx rows, SWIZZLE_64B) issued by thread 0 from two alternating
// output tiles; before a tile is written again thread 0 has waited for the
// store that read it, so the other warps never wait on the stores.
template <int NX, int STAGES>
__global__ void __launch_bounds__(256, 2) xwarp_r2c_kernel(const __grid_constant__ CUtensorMap rmap,
                                                           const __grid_constant__ CUtensorMap cmap,
                                                           const float2 *__restrict__ twg, int ny, int nz, int rb,
                                                           PipeCtl ctl) {
  using C = float2;
  using G = XWPlainGeom<NX, STAGES>;
  constexpr int M = NX / 2, E = 8, T = 32, BZ = G::BZ;
  static_assert(M == E * T, "one warp per line: NX = 512");
  extern __shared__ unsigned char smem_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char *obuf = sm + STAGES * G::r2c_in;
  const int tid = threadIdx.x, lane = tid & 31, l = tid >> 5;
  XWRing rg(obuf + 2 * G::out_bytes, M, NX, STAGES, l);
  const int nzb = nz / BZ, ntiles = nzb * ny;
  if (tid == 0) {
    mbar_init(rg.never, 1);
    for (int q = 0; q < STAGES; ++q) {
      mbar_init(&rg.full[q], 1);
      rg.cnt[q] = 0;
    }
    fence_barrier_init();
  }
  for (int e = tid; e < NX; e += 256) rg.tw[e] = twg[e];
  __syncthreads();
  auto issue = [&](int k) {
    const int tile = blockIdx.x + k * gridDim.x;
    if (tile >= ntiles) return;
    const int s = k % STAGES;
    fence_proxy_async();
    mbar_arrive_expect_tx(&rg.full[s], (uint32_t)G::r2c_in);
    tma_load_3d(sm + (size_t)s * G::r2c_in, &rmap, 0, tile / nzb, (tile % nzb) * BZ, &rg.full[s]);
  };
  if (tid == 0)
    for (int k = 0; k < STAGES; ++k) issue(k);
  float2 *xw = rg.xw;
  const float2 *tw = rg.tw;
  auto buf = [xw](int idx) -> C & { return xw[xw_line_swz(idx)]; };
  auto wsync = [] { __syncwarp(); };
  const int src = (32 - lane) & 31;
  for (int k = 0;; ++k) {
    const int tile = blockIdx.x + k * gridDim.x;
    if (tile >= ntiles) break;
    const int s = k % STAGES;
    xw_wait<STAGES>(rg, k, ctl);
    const C *line = reinterpret_cast<const C *>(sm + (size_t)s * G::r2c_in) + (size_t)l * M + lane;
    C x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = line[T * e];
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&rg.cnt[s], 1u) % BZ == BZ - 1) {
        __threadfence_block();
        issue(k + STAGES);
      }
    }
    line_fft<C, M, E, -1, 2>(x, lane, tw, buf, wsync);
    unsigned char *ob = obuf + (size_t)(k & 1) * G::out_bytes;
    unsigned char *ob0 = ob + xw_tile_off(lane, l);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const C zm = shfl2(lane == 0 ? x[(8 - e) & 7] : x[7 - e], src);  // Z_{(M-k) mod M}
      *reinterpret_cast<C *>(ob0 + 2048 * e) = r2c_unpack(x[e], zm, tw[lane + T * e]);
      if (e == 0 && lane == 0)
        *reinterpret_cast<C *>(ob0 - xw_tile_off(0, l) + xw_tile_off(M, l)) = r2c_unpack(x[0], zm, mk(-1.f, 0.f));
    }
    fence_proxy_async();  // the tile's generic writes, before the async-proxy store reads them
    if (tid == 0) bulk_wait_read_all();  // the store of tile k-1 has read its buffer
    __syncthreads();
    if (tid == 0) {
      for (int q = 0; q < 2; ++q) tma_store_3d(&cmap, ob + (size_t)q * rb * 64, (tile % nzb) * BZ, tile / nzb, q * rb);
      bulk_commit();
    }
  }
  if (tid == 0) bulk_wait_all();
}

template <int NX, int STAGES>
__global__ void __launch_bounds__(256, 2) xwarp_c2r_kernel(const __grid_constant__ CUtensorMap cmap, float *__restrict__ out,
                                                           const float2 *__restrict__ twg, int ny, int nz, int nbox,
                                                           int rb, PipeCtl ctl) {
  using C = float2;
  using G = XWPlainGeom<NX, STAGES>;
  constexpr int M = NX / 2, E = 8, T = 32, BZ = G::BZ;
  static_assert(M == E * T, "one warp per line: NX = 512");
  extern __shared__ unsigned char smem_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, lane = tid & 31, l = tid >> 5;
  XWRing rg(sm + STAGES * G::c2r_in, M, NX, STAGES, l);
  const int nzb = nz / BZ, ntiles = nzb * ny;
  if (tid == 0) {
    mbar_init(rg.never, 1);
    for (int q = 0; q < STAGES; ++q) {
      mbar_init(&rg.full[q], 1);
      rg.cnt[q] = 0;
    }
    fence_barrier_init();
  }
  for (int e = tid; e < NX; e += 256) rg.tw[e] = twg[e];
  __syncthreads();
  auto issue = [&](int k) {
    const int tile = blockIdx.x + k * gridDim.x;
    if (tile >= ntiles) return;
    const int s = k % STAGES;
    fence_proxy_async();
    mbar_arrive_expect_tx(&rg.full[s], (uint32_t)(nbox * rb) * 64u);
    unsigned char *dst = sm + (size_t)s * G::c2r_in;
    for (int q = 0; q < nbox; ++q)
      tma_load_3d(dst + (size_t)q * rb * 64, &cmap, (tile % nzb) * BZ, tile / nzb, q * rb, &rg.full[s]);
  };
  if (tid == 0)
    for (int k = 0; k < STAGES; ++k) issue(k);
  float2 *xw = rg.xw;
  const float2 *tw = rg.tw;
  auto buf = [xw](int idx) -> C & { return xw[xw_line_swz(idx)]; };
  auto wsync = [] { __syncwarp(); };
  const int src = (32 - lane) & 31;
  const bool l0 = lane == 0;
  for (int k = 0;; ++k) {
    const int tile = blockIdx.x + k * gridDim.x;
    if (tile >= ntiles) break;
    const int s = k % STAGES;
    xw_wait<STAGES>(rg, k, ctl);
    const unsigned char *tb = sm + (size_t)s * G::c2r_in + xw_tile_off(lane, l);
    C x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = *reinterpret_cast<const C *>(tb + 2048 * e);
    const C xM = l0 ? *reinterpret_cast<const C *>(tb - xw_tile_off(0, l) + xw_tile_off(M, l)) : mk(0.f, 0.f);
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&rg.cnt[s], 1u) % BZ == BZ - 1) {
        __threadfence_block();
        issue(k + STAGES);
      }
    }
    // pack in pairs (e, 7-e), X_{M-k} as in the fused pass
    C carry = xM;
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      const C a = x[e], b = x[E - 1 - e];
      const C pa = shfl2(b, src), pb = shfl2(a, src);
      C xa = a, ma = l0 ? carry : pa;
      const C mb = l0 ? (e == E / 2 - 1 ? b : x[e + 1]) : pb;
      carry = b;
      if (e == 0 && l0) {
        xa.y = 0.f;
        ma.y = 0.f;
      }
      x[e] = xw_pack(xa, ma, tw[lane + T * e]);
      x[E - 1 - e] = xw_pack(b, mb, tw[lane + T * (E - 1 - e)]);
    }
    line_fft<C, M, E, +1, 2>(x, lane, tw, buf, wsync);
    C *row = reinterpret_cast<C *>(out + (size_t)NX * ((size_t)(tile / nzb) + (size_t)ny * ((tile % nzb) * BZ + l))) + lane;
#pragma unroll
    for (int e = 0; e < E; ++e) row[T * e] = x[e];
  }
}

}  // namespace gb
