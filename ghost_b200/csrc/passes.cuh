// passes.cuh -- the three 1D FFT passes of a 3D transform, with GHOST's
// spectral operators fused into their prologues and epilogues.
//
// Spectral fields live in GHOST's transposed layout a(k,j,i) (z fastest).
//   Z pass: lines along z are contiguous.  Thread t of a line owns
//           z = t + T*e; lines of one CTA are consecutive (j,i) lines.
//   Y pass: lines along y have stride nz.  A CTA takes BZ consecutive z
//           lines at one kx; thread (l,t) (l fastest) owns y = t + T*e of
//           line z0+l, so a warp touches BZ consecutive z per y row.
//   X pass: lines along kx have stride nz*ny.  A CTA takes BZ consecutive
//           z lines at one y; the nx/2+1 rows of BZ values are staged in
//           shared memory by cp.async, then each line runs the half-length
//           complex transform of a real-to-complex / complex-to-real pair.
// Real-space data never touch HBM on the HD path: the X pass goes
// spectral -> real (6 fields) -> omega x v -> spectral (3 fields).
#pragma once
#include "common.cuh"
#include "pipeline.cuh"

namespace gb {

template <typename R> struct Fields {
  cx<R> *p[12];
};
template <typename R> struct CFields {
  const cx<R> *p[12];
};

// --------------------------------------------------------------------
// cp.async helpers (16-byte global -> shared copies)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ====================================================================
// Z pass: persistent CTAs stream tiles of LPB z-lines (each line one bulk
// copy of N values per loaded field) through STAGES shared-memory buffers.
// ====================================================================
template <typename R, int N, int E, int LPB, int NL> struct ZGeom {
  static constexpr int T = N / E;
  static constexpr int NT = LPB * T;
  static constexpr int NP = N + N / 8;  // padded exchange line: idx + idx/8 spreads strided writes
  static constexpr size_t stage_elems = (size_t)NL * LPB * N;
  static constexpr size_t smem_bytes(int stages) {
    return (stages * stage_elems + N + 2 * (size_t)LPB * NP) * sizeof(cx<R>) + 8 * (stages + 1);
  }
};

// One 3D tensor map per field: (z in 8-byte units, y, kx).
struct FieldMaps {
  CUtensorMap m[9];
};

struct PipeCtl {
  int *status;    // device status word (GHOST_ERR_TIMEOUT on a timed-out wait)
  uint32_t cap;   // polls before a wait gives up
  int stall;      // fault injection: wait on a barrier nothing completes
};

// lines != nullptr: the pass covers the listed (j,i) lines only (entries
// < 0 pad the list); otherwise lines 0..nlines-1.  The body takes the CTA's
// index vb among the nvb CTAs working on this pass (blockIdx.x / gridDim.x
// for a launch of its own; a share of a launch shared by several grids).
template <typename R, int N, int E, int LPB, int STAGES, class Op>
__device__ __forceinline__ void zpipe_body(int vb, int nvb, const Op &op, const cx<R> *__restrict__ twg,
                                           const int *__restrict__ lines, int nlines, PipeCtl ctl) {
  using C = cx<R>;
  using G = ZGeom<R, N, E, LPB, Op::NLOAD>;
  constexpr int T = G::T, NT = G::NT, NP = G::NP, NL = Op::NLOAD;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C *stage = reinterpret_cast<C *>(smem_raw);
  C *tw = stage + STAGES * G::stage_elems;
  C *xb = tw + N;
  uint64_t *bars = reinterpret_cast<uint64_t *>(xb + 2 * LPB * NP);
  const int tid = threadIdx.x, lq = tid / T, t = tid - lq * T;
  const int ntiles = (nlines + LPB - 1) / LPB;
  if (tid == 0) {
    for (int q = 0; q <= STAGES; ++q) mbar_init(&bars[q], 1);  // bars[STAGES]: never completed
    fence_barrier_init();
  }
  for (int e = tid; e < N; e += NT) tw[e] = twg[e];
  __syncthreads();
  auto line_of = [&](int tile, int l) -> long {
    const long idx = (long)tile * LPB + l;
    if (idx >= nlines) return -1;
    return lines ? (long)lines[idx] : idx;
  };
  auto issue = [&](int k) {
    const int tile = vb + k * nvb;
    if (tile >= ntiles) return;
    const int s = k % STAGES;
    if (tid == 0) {
      uint32_t bytes = 0;
      for (int l = 0; l < LPB; ++l)
        if (line_of(tile, l) >= 0) bytes += NL * N * (uint32_t)sizeof(C);
      mbar_arrive_expect_tx(&bars[s], bytes);
    }
    for (int q = tid; q < NL * LPB; q += NT) {
      const int f = q / LPB, l = q - f * LPB;
      const long line = line_of(tile, l);
      if (line >= 0)
        bulk_g2s(stage + ((size_t)(s * NL + f) * LPB + l) * N, op.load_src(f) + (size_t)line * N,
                 N * (uint32_t)sizeof(C), &bars[s]);
    }
  };
  for (int k = 0; k < STAGES - 1; ++k) issue(k);
  C *mine = xb + lq * NP;
  int ph = 0;
  auto buf = dual_buf<C>([mine](int idx, int h) -> C & { return mine[h * (LPB * NP) + idx + (idx >> 3)]; }, &ph);
  auto sync = [] { __syncthreads(); };
  for (int k = 0;; ++k) {
    const int tile = vb + k * nvb;
    if (tile >= ntiles) break;
    fence_proxy_async();
    issue(k + STAGES - 1);
    const int s = k % STAGES;
    const bool ok = (!ctl.stall || injected_stall_wait(&bars[STAGES], ctl.cap)) &&
                    mbar_wait(&bars[s], (uint32_t)(k / STAGES) & 1u, ctl.cap);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) record_timeout(ctl.status);
      for (int kk = k; kk < k + STAGES; ++kk)
        if (vb + kk * nvb < ntiles) mbar_wait(&bars[kk % STAGES], (uint32_t)(kk / STAGES) & 1u, kDrainPolls);
      return;
    }
    const long line = line_of(tile, lq);
    const bool act = line >= 0;
    const C *in0 = stage + ((size_t)(s * NL) * LPB + lq) * N;
    auto in = [in0](int f) -> const C * { return in0 + (size_t)f * LPB * N; };
    op.template body<N, E>(act ? line : 0, act, t, tw, buf, sync, in);
    // the stage is refilled at the top of the next tile: the transforms'
    // exchange barriers follow every read of it, except without exchanges
    if constexpr (fft_exchanges<N, E>() == 0) __syncthreads();
  }
}

template <typename R, int N, int E, int LPB, int STAGES, int MINB, class Op>
__global__ void __launch_bounds__(LPB *(N / E), MINB) zpipe_kernel(Op op, const cx<R> *__restrict__ twg,
                                                              const int *__restrict__ lines, int nlines,
                                                              PipeCtl ctl) {
  zpipe_body<R, N, E, LPB, STAGES>(blockIdx.x, gridDim.x, op, twg, lines, nlines, ctl);
}

// Plain c2c along z of NF fields (in -> out, may alias).
template <typename R, int S, int NF> struct ZC2C {
  using C = cx<R>;
  static constexpr int NLOAD = NF;
  CFields<R> in;
  Fields<R> out;
  __device__ __forceinline__ const C *load_src(int f) const { return in.p[f]; }
  template <int N, int E, class Buf, class Sync, class In>
  __device__ __forceinline__ void body(long line, bool act, int t, const C *tw, Buf buf, Sync sync, In src) const {
    constexpr int T = N / E;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = src(f)[t + T * e];
      line_fft<C, N, E, S>(x, t, tw, buf, sync);
      if (act) {
        C *dst = out.p[f] + (size_t)line * N;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[t + T * e] = x[e];
      }
    }
  }
};

// Inverse prologue of the fused substep: from v (and theta for the
// Boussinesq solver) it forms per mode the fields the real-space products
// need and runs the inverse z transform of each:
//   PHYS 0 (HD):    v, curl v                       (prodre3 inputs)
//   PHYS 1 (BOUSS): v, curl v, i k theta            (prodre3 + advect3 inputs)
// curl as rotor3 (pseudospec3D_hd.f90:124-200), i k theta as derivk3.
// With copy != 0 it also stores the RK1 copies C = v (theta).
template <typename R, int PHYS> struct ZInv {
  using C = cx<R>;
  static constexpr int NIN = PHYS == 0 ? 3 : 4;
  static constexpr int NOUT = PHYS == 0 ? 6 : 9;
  static constexpr int NLOAD = NIN;
  CFields<R> v;   // NIN
  Fields<R> w;    // NOUT outputs
  Fields<R> cpy;  // NIN (when copy)
  KParams<R> kp;
  int copy;
  __device__ __forceinline__ const C *load_src(int f) const { return v.p[f]; }
  template <int N, int E, class Buf, class Sync, class In>
  __device__ __forceinline__ void body(long line, bool act, int t, const C *tw, Buf buf, Sync sync, In src) const {
    constexpr int T = N / E;
    const int j = (int)(line % kp.ny), ir = (int)(line / kp.ny), i = ir % kp.nxh + kp.i0;
    const R kx = kx_of(kp, i), ky = ky_of(kp, j);
    if (copy && act) {
#pragma unroll
      for (int c = 0; c < NIN; ++c)
#pragma unroll
        for (int e = 0; e < E; ++e) cpy.p[c][(size_t)line * N + t + T * e] = src(c)[t + T * e];
    }
#pragma unroll
    for (int f = 0; f < NOUT; ++f) {
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = t + T * e;
        const R kz = kz_of(kp, k);
        if (f < 3) {
          x[e] = src(f)[k];
        } else if (f < 6) {
          // i k a = (-k a.y, k a.x)
          if (f == 3) {
            const C vy = src(1)[k], vz = src(2)[k];
            x[e] = mk((-ky * vz.y) - (-kz * vy.y), (ky * vz.x) - (kz * vy.x));
          } else if (f == 4) {
            const C vx = src(0)[k], vz = src(2)[k];
            x[e] = mk((-kz * vx.y) - (-kx * vz.y), (kz * vx.x) - (kx * vz.x));
          } else {
            const C vx = src(0)[k], vy = src(1)[k];
            x[e] = mk((-kx * vy.y) - (-ky * vx.y), (kx * vy.x) - (ky * vx.x));
          }
        } else {
          const C th = src(NIN - 1)[k];
          const R kd = f == 6 ? kx : (f == 7 ? ky : kz);
          x[e] = mk(-(kd * th.y), kd * th.x);
        }
      }
      line_fft<C, N, E, +1>(x, t, tw, buf, sync);
      if (act) {
        C *dst = w.p[f] + (size_t)line * N;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[t + T * e] = x[e];
      }
    }
  }
};

// The nine velocity gradients (derivk3 of each component along each axis,
// pseudospec3D_hd.f90:22-88) with their inverse z transforms:
// w[3a+b] = i k_b v_a, for the inputs of the LES closure.
template <typename R> struct ZGrad {
  using C = cx<R>;
  static constexpr int NLOAD = 3;
  CFields<R> v;  // 3
  Fields<R> w;   // 9 outputs
  KParams<R> kp;
  __device__ __forceinline__ const C *load_src(int f) const { return v.p[f]; }
  template <int N, int E, class Buf, class Sync, class In>
  __device__ __forceinline__ void body(long line, bool act, int t, const C *tw, Buf buf, Sync sync, In src) const {
    constexpr int T = N / E;
    const int j = (int)(line % kp.ny), i = (int)(line / kp.ny) % kp.nxh + kp.i0;
    const R kx = kx_of(kp, i), ky = ky_of(kp, j);
#pragma unroll
    for (int f = 0; f < 9; ++f) {
      const int a = f / 3, b = f % 3;
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int k = t + T * e;
        const R kd = b == 0 ? kx : (b == 1 ? ky : kz_of(kp, k));
        const C u = src(a)[k];
        x[e] = mk(-(kd * u.y), kd * u.x);
      }
      line_fft<C, N, E, +1>(x, t, tw, buf, sync);
      if (act) {
        C *dst = w.p[f] + (size_t)line * N;
#pragma unroll
        for (int e = 0; e < E; ++e) dst[t + T * e] = x[e];
      }
    }
  }
};

// HD forward epilogue: forward z transform of the three components of
// omega x v, then nonlhd3 x3 (pseudospec3D_hd.f90:399-509), laplak3 and
// the truncated RK update of include/hd_rkstep2.f90:18-38, written to v.
template <typename R> struct ZFwdHD {
  using C = cx<R>;
  static constexpr int NLOAD = 3;
  CFields<R> nl;  // 3 (x and y transformed)
  Fields<R> v;    // 3 in/out
  CFields<R> c0;  // C1..C3
  CFields<R> f;   // forcing or null
  KParams<R> kp;
  R dt, nu, rmp;
  __device__ __forceinline__ const C *load_src(int q) const { return nl.p[q]; }
  template <int N, int E, class Buf, class Sync, class In>
  __device__ __forceinline__ void body(long line, bool act, int t, const C *tw, Buf buf, Sync sync, In src) const {
    constexpr int T = N / E;
    const int j = (int)(line % kp.ny), ir = (int)(line / kp.ny), i = ir % kp.nxh + kp.i0;
    const R kx = kx_of(kp, i), ky = ky_of(kp, j);
    const R nuv = kp.nu_run ? kp.nu_run[ir / kp.nxh] : nu;
    const bool forced = f.p[0] != nullptr;
    // The kept modes are known before the transforms: their v, C and f
    // values are prefetched into L2 while the three lines are transformed.
    bool keep[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const R kn2 = kn2_of(kp, i, j, t + T * e);
      keep[e] = act && kn2 <= kp.kmax && kn2 >= kp.tiny;
    }
    {
      const size_t base = (size_t)line * N + t;
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (keep[e]) {
          const size_t p = base + (size_t)T * e;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            prefetch_l2(v.p[c] + p);
            prefetch_l2(c0.p[c] + p);
            if (forced) prefetch_l2(f.p[c] + p);
          }
        }
    }
    C g[3][E];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int e = 0; e < E; ++e) g[c][e] = src(c)[t + T * e];
      line_fft<C, N, E, -1>(g[c], t, tw, buf, sync);
    }
    if (!act) return;
    // The projected nonlinear term replaces g in place; then, component by
    // component, all of the line's operands (v, C, f at the kept modes) are
    // loaded before any result is stored, so a thread waits for one round
    // of loads per component rather than one per element.
    R kk2e[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = t + T * e;
      kk2e[e] = (R)0;
      if (keep[e]) {
        const R kz = kz_of(kp, k);
        const R kk2 = kk2_of(kp, i, j, k);
        kk2e[e] = kk2;
        const C a = g[0][e], b = g[1][e], cc = g[2][e];
        const C s = mk(kx * a.x + ky * b.x + kz * cc.x, kx * a.y + ky * b.y + kz * cc.y);
        g[0][e] = (i == 0) ? mk(-a.x, -a.y) : mk(-a.x + (kx * s.x) / kk2, -a.y + (kx * s.y) / kk2);
        g[1][e] = (j == 0) ? mk(-b.x, -b.y) : mk(-b.x + (ky * s.x) / kk2, -b.y + (ky * s.y) / kk2);
        g[2][e] = (k == 0) ? mk(-cc.x, -cc.y) : mk(-cc.x + (kz * s.x) / kk2, -cc.y + (kz * s.y) / kk2);
      }
    }
    const size_t base = (size_t)line * N + t;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      C vv[E], ff[E], cc0[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        vv[e] = mk((R)0, (R)0);
        ff[e] = mk((R)0, (R)0);
        cc0[e] = mk((R)0, (R)0);
        if (keep[e]) {
          const size_t p = base + (size_t)T * e;
          vv[e] = v.p[c][p];
          cc0[e] = c0.p[c][p];
          if (forced) ff[e] = f.p[c][p];
        }
      }
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const size_t p = base + (size_t)T * e;
        if (keep[e]) {
          const R kk2 = kk2e[e];
          const C lap = mk(-kk2 * vv[e].x, -kk2 * vv[e].y);
          C sum = mk(nuv * lap.x + g[c][e].x, nuv * lap.y + g[c][e].y);
          if (forced) sum = mk(sum.x + ff[e].x, sum.y + ff[e].y);
          v.p[c][p] = mk(cc0[e].x + (dt * sum.x) * rmp, cc0[e].y + (dt * sum.y) * rmp);
        } else {
          v.p[c][p] = mk((R)0, (R)0);
        }
      }
    }
  }
};

// Boussinesq forward epilogue (include/rotbouss_rkstep2.f90:12-83):
// forward z transform of omega x v and of -v.grad(theta), Coriolis and
// buoyancy added before the projection, the heat current xtemp*vz, the
// Laplacians and the three-way truncated update (theta keeps its mean).
template <typename R> struct ZFwdBouss {
  using C = cx<R>;
  static constexpr int NLOAD = 4;
  CFields<R> nl;  // 4: (w x v)_xyz, -v.grad(theta)
  Fields<R> v;    // 4 in/out: vx, vy, vz, theta
  CFields<R> c0;  // C1..C3, C20
  CFields<R> f;   // fx, fy, fz, fs (any null: zero)
  KParams<R> kp;
  R dt, nu, kappa, omegaz, xmom, xtemp, rmp;
  __device__ __forceinline__ const C *load_src(int q) const { return nl.p[q]; }
  template <int N, int E, class Buf, class Sync, class In>
  __device__ __forceinline__ void body(long line, bool act, int t, const C *tw, Buf buf, Sync sync, In src) const {
    constexpr int T = N / E;
    const int j = (int)(line % kp.ny), i = (int)(line / kp.ny) % kp.nxh + kp.i0;
    const R kx = kx_of(kp, i), ky = ky_of(kp, j);
    const bool forced = f.p[0] != nullptr, sforced = f.p[3] != nullptr;
    const size_t base = (size_t)line * N + t;
    // mode 0: kept mode; 1: truncated (all zero); 2: kn2 < tiny (theta
    // keeps its mean).  Known before the transforms: the kept modes' v, C
    // and f values are prefetched into L2 while the lines are transformed.
    int mode[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const R kn2 = kn2_of(kp, i, j, t + T * e);
      mode[e] = (kn2 <= kp.kmax && kn2 >= kp.tiny) ? 0 : (kn2 > kp.kmax ? 1 : 2);
      if (act && mode[e] == 0) {
        const size_t p = base + (size_t)T * e;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          prefetch_l2(v.p[c] + p);
          prefetch_l2(c0.p[c] + p);
          if (c < 3 ? forced : sforced) prefetch_l2(f.p[c] + p);
        }
      }
    }
    C g[4][E];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
#pragma unroll
      for (int e = 0; e < E; ++e) g[c][e] = src(c)[t + T * e];
      line_fft<C, N, E, -1>(g[c], t, tw, buf, sync);
    }
    if (!act) return;
    const R two_om = (R)2 * omegaz;
    // As in ZFwdHD: all loads of a round before any store.  The velocity
    // and theta values enter the projection and the Laplacians, which are
    // folded into g there, so they are dead before the update loads C and f.
    C vv[4][E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
#pragma unroll
      for (int c = 0; c < 4; ++c) vv[c][e] = mk((R)0, (R)0);
      if (mode[e] == 0) {
        const size_t p = base + (size_t)T * e;
#pragma unroll
        for (int c = 0; c < 4; ++c) vv[c][e] = v.p[c][p];
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if (mode[e] != 0) continue;
      const int k = t + T * e;
      const R kz = kz_of(kp, k);
      const R kk2 = kk2_of(kp, i, j, k);
      const C a = mk(g[0][e].x - two_om * vv[1][e].x, g[0][e].y - two_om * vv[1][e].y);
      const C b = mk(g[1][e].x + two_om * vv[0][e].x, g[1][e].y + two_om * vv[0][e].y);
      const C cc = mk(g[2][e].x + xmom * vv[3][e].x, g[2][e].y + xmom * vv[3][e].y);
      const C s = mk(kx * a.x + ky * b.x + kz * cc.x, kx * a.y + ky * b.y + kz * cc.y);
      g[0][e] = (i == 0) ? mk(-a.x, -a.y) : mk(-a.x + (kx * s.x) / kk2, -a.y + (kx * s.y) / kk2);
      g[1][e] = (j == 0) ? mk(-b.x, -b.y) : mk(-b.x + (ky * s.x) / kk2, -b.y + (ky * s.y) / kk2);
      g[2][e] = (k == 0) ? mk(-cc.x, -cc.y) : mk(-cc.x + (kz * s.x) / kk2, -cc.y + (kz * s.y) / kk2);
      g[3][e] = mk(g[3][e].x + xtemp * vv[2][e].x, g[3][e].y + xtemp * vv[2][e].y);
#pragma unroll
      for (int c = 0; c < 4; ++c) {  // + dif * Laplacian
        const R dif = c < 3 ? nu : kappa;
        const C lap = mk(-kk2 * vv[c][e].x, -kk2 * vv[c][e].y);
        g[c][e] = mk(dif * lap.x + g[c][e].x, dif * lap.y + g[c][e].y);
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const bool fc = c < 3 ? forced : sforced;
      C ff[E], cc0[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        ff[e] = mk((R)0, (R)0);
        cc0[e] = mk((R)0, (R)0);
        const size_t p = base + (size_t)T * e;
        if (mode[e] == 0) {
          cc0[e] = c0.p[c][p];
          if (fc) ff[e] = f.p[c][p];
        } else if (mode[e] == 2 && c == 3) {
          cc0[e] = c0.p[3][p];
        }
      }
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const size_t p = base + (size_t)T * e;
        if (mode[e] == 0) {
          C sum = g[c][e];
          if (fc) sum = mk(sum.x + ff[e].x, sum.y + ff[e].y);
          v.p[c][p] = mk(cc0[e].x + (dt * sum.x) * rmp, cc0[e].y + (dt * sum.y) * rmp);
        } else {
          v.p[c][p] = (mode[e] == 2 && c == 3) ? cc0[e] : mk((R)0, (R)0);
        }
      }
    }
  }
};

// ====================================================================
// Y pass: persistent CTAs stream tiles of BZ z-lines x N y-rows of one
// field at one kx index (row j: BZ contiguous values, one bulk copy).  The
// tile's stage buffer then serves as the line-interleaved FFT exchange
// buffer, so a tile costs one trip through shared memory.
// With jpos/jneg (pruned passes) only rows j < jpos[i] or j >= N - jneg[i]
// can be non-zero: the inverse pass loads only those, the forward pass
// writes only those (the rest are never read).
// ====================================================================
// DUAL: the exchanges alternate between a second buffer of the same size
// and the tile's own stage buffer, one barrier per exchange and none other
// than the tile's first (the stage refill is issued after it).  The tile's
// result then leaves by TMA tensor stores (omaps, boxes of rbo rows) from
// whichever of the two buffers the last exchange did not use; one thread
// issues them and, before the next tile's first barrier, waits until they
// have read shared memory.
// KB > 1 (short lines, and only without DUAL): a tile holds BZ z-lines of
// KB consecutive kx indices, one block of BZ x N per kx, so that a CTA of
// KB BZ N/E threads has enough threads; thread (l, t, kb) with l fastest.
template <typename R, int N, int E, int BZ, bool DUAL = false, int KB = 1> struct YGeom {
  static constexpr int T = N / E;
  static constexpr int NT = KB * BZ * T;
  static constexpr size_t stage_elems = (size_t)KB * BZ * N;
  static constexpr size_t smem_bytes(int stages) {
    return ((stages + (DUAL ? 1 : 0)) * stage_elems + N) * sizeof(cx<R>) + 8 * (stages + 1);
  }
};

template <typename R, int N, int E, int BZ, int STAGES, int S, bool DUAL = false, int KB = 1>
__device__ __forceinline__ void ypipe_body(int vb, int nvb, const FieldMaps &maps, const FieldMaps &omaps,
                                           const Fields<R> &fld, const cx<R> *__restrict__ twg, int nz, int ni,
                                           int nf, int nruns, int nxh, const int *__restrict__ jpos,
                                           const int *__restrict__ jneg, int rb, int rbo, PipeCtl ctl) {
  static_assert(KB == 1 || !DUAL, "several kx per tile only without the second buffer");
  using C = cx<R>;
  using G = YGeom<R, N, E, BZ, DUAL, KB>;
  constexpr int T = G::T, NT = G::NT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C *stage = reinterpret_cast<C *>(smem_raw);
  C *xb = stage + STAGES * G::stage_elems;  // second exchange buffer (DUAL)
  C *tw = xb + (DUAL ? G::stage_elems : 0);
  uint64_t *bars = reinterpret_cast<uint64_t *>(tw + N);
  // with one kx per tile the kx offset is the constant 0 and every line is live
  const int tid = threadIdx.x, l = tid % BZ, t = KB == 1 ? tid / BZ : (tid / BZ) % T;
  const int kb = KB == 1 ? 0 : tid / (BZ * T);
  const int nzb = nz / BZ;
  const int nig = (ni + KB - 1) / KB;  // groups of KB kx indices
  const int ntiles = nzb * nig * nruns * nf;
  if (tid == 0) {
    for (int q = 0; q <= STAGES; ++q) mbar_init(&bars[q], 1);  // bars[STAGES]: never completed
    fence_barrier_init();
  }
  for (int e = tid; e < N; e += NT) tw[e] = twg[e];
  __syncthreads();
  struct Tile {
    int zb, ii, i, f;  // ii: first kx index of the tile within the run, i: its plane of the batched field
  };
  auto tile_of = [&](int tile) {
    Tile r;
    r.zb = tile % nzb;
    int q = tile / nzb;
    r.ii = (q % nig) * KB;
    q /= nig;
    r.i = (q % nruns) * nxh + r.ii;
    r.f = q / nruns;
    return r;
  };
  auto rows_of = [&](int i, int &jp, int &jn) {
    if (jpos && S > 0) {
      jp = jpos[i];
      jn = jneg[i];
    } else {
      jp = N;
      jn = 0;
    }
  };
  // one thread issues TMA tensor loads of rb-row boxes covering the live
  // rows of each of the tile's kx: [0, jp) from the top and [N - jn, N) from
  // the bottom (boxes may overlap or overrun into rows that are masked out below)
  constexpr int U = (int)sizeof(C) / 8;
  auto issue = [&](int k) {
    const int tile = vb + k * nvb;
    if (tile >= ntiles || tid != 0) return;
    const Tile tl = tile_of(tile);
    const int s = k % STAGES;
    // live rows of each kx of the tile, read once (none past the last kx)
    int jp[KB], jn[KB];
    uint32_t nbox = 0;
#pragma unroll
    for (int b = 0; b < KB; ++b) {
      jp[b] = jn[b] = 0;
      if (KB == 1 || tl.ii + b < ni) rows_of(tl.ii + b, jp[b], jn[b]);
      nbox += (jp[b] + rb - 1) / rb + (jn[b] + rb - 1) / rb;
    }
    fence_proxy_async();
    mbar_arrive_expect_tx(&bars[s], nbox * (uint32_t)rb * BZ * (uint32_t)sizeof(C));
#pragma unroll
    for (int b = 0; b < KB; ++b) {
      C *dst = stage + (size_t)s * G::stage_elems + (size_t)b * BZ * N;
      const int nb_top = (jp[b] + rb - 1) / rb, nb_bot = (jn[b] + rb - 1) / rb;
      for (int q = 0; q < nb_top; ++q)
        tma_load_3d(dst + (size_t)q * rb * BZ, &maps.m[tl.f], tl.zb * BZ * U, q * rb, tl.i + b, &bars[s]);
      for (int q = 0; q < nb_bot; ++q) {
        const int r0 = N - (q + 1) * rb;
        tma_load_3d(dst + (size_t)r0 * BZ, &maps.m[tl.f], tl.zb * BZ * U, r0, tl.i + b, &bars[s]);
      }
    }
  };
  for (int k = 0; k < STAGES - 1; ++k) issue(k);
  auto sync = [] { __syncthreads(); };
  for (int k = 0;; ++k) {
    const int tile = vb + k * nvb;
    if (tile >= ntiles) break;
    // DUAL: the refill of the previous tile's slot waits for this tile's
    // first barrier, which follows every read of that slot (so no barrier
    // closes a tile)
    if constexpr (!DUAL) issue(k + STAGES - 1);
    const int s = k % STAGES;
    const bool ok = (!ctl.stall || injected_stall_wait(&bars[STAGES], ctl.cap)) &&
                    mbar_wait(&bars[s], (uint32_t)(k / STAGES) & 1u, ctl.cap);
    // DUAL: the previous tile's stores have read their buffer before anyone
    // writes it again (this barrier orders every later write)
    if (DUAL && tid == 0) bulk_wait_read_all();
    if (__syncthreads_or(!ok)) {
      if (tid == 0) record_timeout(ctl.status);
      for (int kk = k; kk < k + STAGES - (DUAL ? 1 : 0); ++kk)
        if (vb + kk * nvb < ntiles) mbar_wait(&bars[kk % STAGES], (uint32_t)(kk / STAGES) & 1u, kDrainPolls);
      if (DUAL && tid == 0) bulk_wait_all();
      return;
    }
    if constexpr (DUAL) issue(k + STAGES - 1);
    const Tile tl = tile_of(tile);
    // this thread's kx: beyond the last one (a short last group) its line is
    // transformed from zeros and not stored
    const bool act = KB == 1 || tl.ii + kb < ni;
    int jp = N, jn = 0;
    if (jpos && act) {
      jp = jpos[tl.ii + kb];
      jn = jneg[tl.ii + kb];
    }
    C *sb = stage + (size_t)s * G::stage_elems + (size_t)kb * BZ * N;
    C x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int jj = t + T * e;
      const bool live = act && ((S < 0) || jj < jp || jj >= N - jn);
      x[e] = live ? sb[jj * BZ + l] : mk((R)0, (R)0);
    }
    if constexpr (DUAL) {
      // The exchanges alternate between the second buffer (half 1, first) and
      // this tile's stage buffer (half 0): the first exchange barrier follows
      // every thread's reads of the stage, so the second exchange may write
      // it, and the second buffer's last reads come before the next tile's
      // first barrier.
      int ph = 1;
      auto buf = dual_buf<C>([sb, xb, l](int idx, int h) -> C & { return (h ? xb : sb)[idx * BZ + l]; }, &ph);
      line_fft<C, N, E, S>(x, t, tw, buf, sync);
      // the exchanges used xb, sb, xb, ...: the result goes to the buffer the
      // last one did not use (its last reads came before that exchange's barrier)
      C *ob = (fft_exchanges<N, E>() % 2 == 1) ? sb : xb;
#pragma unroll
      for (int e = 0; e < E; ++e) ob[(t + T * e) * BZ + l] = x[e];
      fence_proxy_async();
      __syncthreads();
      if (tid == 0) {
        // rows written: all of them, or (pruned forward pass) boxes covering
        // the live rows; the extra rows of a box hold the transform's own
        // values, in rows nothing reads
        if (S > 0 || (jp == N && jn == 0)) {
          for (int r0 = 0; r0 < N; r0 += rbo) tma_store_3d(&omaps.m[tl.f], ob + (size_t)r0 * BZ, tl.zb * BZ * U, r0, tl.i);
        } else {
          for (int r0 = 0; r0 < jp; r0 += rbo) tma_store_3d(&omaps.m[tl.f], ob + (size_t)r0 * BZ, tl.zb * BZ * U, r0, tl.i);
          for (int q = 0; q * rbo < jn; ++q) {
            const int r0 = N - (q + 1) * rbo;
            tma_store_3d(&omaps.m[tl.f], ob + (size_t)r0 * BZ, tl.zb * BZ * U, r0, tl.i);
          }
        }
        bulk_commit();
      }
    } else {
      __syncthreads();  // every read of the stage before the exchanges overwrite it
      auto buf = [sb, l](int idx) -> C & { return sb[idx * BZ + l]; };
      line_fft<C, N, E, S>(x, t, tw, buf, sync);
      C *base = fld.p[tl.f] + (size_t)tl.zb * BZ + l + (size_t)nz * N * (tl.i + kb);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int jj = t + T * e;
        if (act && (S > 0 || jj < jp || jj >= N - jn)) base[(size_t)nz * jj] = x[e];
      }
      __syncthreads();  // the stage is read before the next refill
    }
  }
  if (DUAL && tid == 0) bulk_wait_all();
}

template <typename R, int N, int E, int BZ, int STAGES, int S, bool DUAL = false, int KB = 1>
__global__ void __launch_bounds__(KB *BZ *(N / E), 2) ypipe_kernel(const __grid_constant__ FieldMaps maps,
                                                                 const __grid_constant__ FieldMaps omaps,
                                                                 const __grid_constant__ Fields<R> fld,
                                                                 const cx<R> *__restrict__ twg, int nz, int ni,
                                                                 int nf, int nruns, int nxh,
                                                                 const int *__restrict__ jpos,
                                                                 const int *__restrict__ jneg, int rb, int rbo,
                                                                 PipeCtl ctl) {
  ypipe_body<R, N, E, BZ, STAGES, S, DUAL, KB>(blockIdx.x, gridDim.x, maps, omaps, fld, twg, nz, ni, nf, nruns, nxh,
                                                jpos, jneg, rb, rbo, ctl);
}

// ====================================================================
// X pass helpers
// ====================================================================
// Stage the (M+1) x BZ tile of kx rows at (z0.., j) of one field.
template <typename C, int BZ>
__device__ __forceinline__ void x_tile_load(C *tile, const C *src, int rows, size_t rowstride, int tid, int nthr) {
  constexpr int CH = BZ * (int)sizeof(C) / 16;  // 16-byte chunks per row
  const int nch = rows * CH;
  for (int q = tid; q < nch; q += nthr) {
    const int row = q / CH, c = q - row * CH;
    cp_async16(reinterpret_cast<unsigned char *>(tile + row * BZ) + 16 * c,
               reinterpret_cast<const unsigned char *>(src + rowstride * row) + 16 * c);
  }
}

// complex-to-real packing of the half spectrum for the M = nx/2 point
// inverse transform:  Z_k = (X_k + conj X_{M-k}) + i e^{+2 pi i k/nx} (X_k - conj X_{M-k}),
// with only the real parts of X_0 and X_M taken.
// rows: kx rows present in the tile (the rest are zero)
template <typename C>
__device__ __forceinline__ C c2r_pack(const C *tile, int bz, int l, int k, int M, int rows, const C *tw) {
  typedef decltype(C{}.x) R;
  C xk = k < rows ? tile[k * bz + l] : mk((R)0, (R)0);
  C xm = (M - k) < rows ? tile[(M - k) * bz + l] : mk((R)0, (R)0);
  if (k == 0) {
    xk.y = 0;
    xm.y = 0;
  }
  const C a = mk(xk.x + xm.x, xk.y - xm.y);  // xk + conj(xm)
  const C b = mk(xk.x - xm.x, xk.y + xm.y);  // xk - conj(xm)
  const C w = tw[k];                          // e^{-2 pi i k/nx}
  const C wb = cmulc(b, w);                   // b * e^{+2 pi i k/nx}
  return mk(a.x - wb.y, a.y + wb.x);          // a + i*wb
}

// real-to-complex unpacking: X_k = (Z_k + conj Z_{M-k})/2 + e^{-2 pi i k/nx} (Z_k - conj Z_{M-k})/(2i)
template <typename C> __device__ __forceinline__ C r2c_unpack(C zk, C zm, C w) {
  typedef decltype(zk.x) R;
  const R h = (R)0.5;
  const C F = mk(h * (zk.x + zm.x), h * (zk.y - zm.y));
  const C d = mk(zk.x - zm.x, zk.y + zm.y);
  const C G = mk(h * d.y, -h * d.x);
  const C wg = cmul(w, G);
  return mk(F.x + wg.x, F.y + wg.y);
}

// ====================================================================
// X pass of the fused substep: complex-to-real lines of every input
// field, the real-space products in registers, real-to-complex lines of
// the products.
//   PHYS 0 (HD):    in v, curl v (6)        -> out omega x v (3)
//                   (prodre3, pseudospec3D_hd.f90:316-396)
//   PHYS 1 (BOUSS): in v, curl v, grad theta (9)
//                   -> out omega x v (3), -v.grad(theta) (1)
//                   (prodre3 + advect3, pseudospec3D_phd.f90:23-114)
// A persistent CTA walks (z-block, y) tiles.  Every input field of a tile
// is one TMA tensor load (nbox boxes of rb kx-rows x BZ z-values) into a
// STAGES-deep ring, so the next fields (and the next tile) stream in while
// the current field is transformed.  scale is 1/(nx ny nz)^2; outputs may
// alias the inputs; only kx rows < rows are read (the rest are zero) and
// written (the rest are never read).
// ====================================================================
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}

// YB > 1 (short lines): a tile holds the BZ z-values of YB consecutive y
// rows, so that a CTA of YB BZ (NX/2)/E threads has enough threads; the
// stage holds rows [kx][y][z] (one TMA box of BZ x YB x rb per field) and
// the lines (y, z) interleave in the exchange buffer.
template <typename R, int NX, int BZ, int YB = 1> struct XGeom {
  static constexpr int M = NX / 2;
  // TMA boxes may overrun the M+1 rows by a few (zero-filled) rows
  static constexpr size_t stage_elems = (size_t)(M + 8) * BZ * YB;
  static constexpr size_t smem_bytes(int stages) {
    return (stages * stage_elems + NX + 2 * (size_t)M * BZ * YB) * sizeof(cx<R>) + 8 * (stages + 1);
  }
};



template <typename R, int NX, int E, int BZ, int PHYS, int STAGES, int YB = 1>
__device__ __forceinline__ void xpipe_nl_body(int vb, int nvb, const FieldMaps &maps, const Fields<R> &out,
                                              const cx<R> *__restrict__ twg, int ny, int nz, R scale, int rows,
                                              int nbox, int rb, int nruns, int nxh, PipeCtl ctl) {
  using C = cx<R>;
  using G = XGeom<R, NX, BZ, YB>;
  constexpr int M = NX / 2, T = M / E, NT = YB * BZ * T;
  constexpr int LW = YB * BZ;  // lines of a tile: (y, z) with z fastest
  constexpr int NIN = PHYS == 0 ? 6 : 9, NOUT = PHYS == 0 ? 3 : 4;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C *stage = reinterpret_cast<C *>(smem_raw);
  C *tw = stage + STAGES * G::stage_elems;
  C *xb = tw + NX;
  uint64_t *bars = reinterpret_cast<uint64_t *>(xb + 2 * (size_t)M * LW);
  const int tid = threadIdx.x, l = tid % BZ, t = YB == 1 ? tid / BZ : (tid / BZ) % T;
  const int yb = YB == 1 ? 0 : tid / (BZ * T);
  const int lw = yb * BZ + l;  // this thread's line within the tile
  const int nzb = nz / BZ, nyg = ny / YB;
  const int ntiles = nzb * nyg * nruns;
  const size_t rowstride = (size_t)nz * ny;
  if (tid == 0) {
    for (int q = 0; q <= STAGES; ++q) mbar_init(&bars[q], 1);  // bars[STAGES]: never completed
    fence_barrier_init();
  }
  for (int e = tid; e < NX; e += NT) tw[e] = twg[e];
  __syncthreads();
  // one thread issues nbox tensor loads of rb kx-rows x BZ z-values
  constexpr int U = (int)sizeof(C) / 8;
  auto issue = [&](int L) {
    const int k = L / NIN, f = L - k * NIN;
    const int tile = vb + k * nvb;
    if (tile >= ntiles || tid != 0) return;
    const int s = L % STAGES;
    fence_proxy_async();
    mbar_arrive_expect_tx(&bars[s], (uint32_t)(nbox * rb) * LW * (uint32_t)sizeof(C));
    C *dst = stage + (size_t)s * G::stage_elems;
    for (int q = 0; q < nbox; ++q)
      tma_load_3d(dst + (size_t)q * rb * LW, &maps.m[f], (tile % nzb) * BZ * U, ((tile / nzb) % nyg) * YB,
                  (tile / nzb / nyg) * nxh + q * rb, &bars[s]);
  };
  for (int L = 0; L < STAGES - 1; ++L) issue(L);
  int ph = 0;
  auto buf = dual_buf<C>([xb, lw](int idx, int h) -> C & { return xb[(size_t)h * (M * LW) + idx * LW + lw]; }, &ph);
  auto sync = [] { __syncthreads(); };
  for (int k = 0;; ++k) {
    const int tile = vb + k * nvb;
    if (tile >= ntiles) break;
    C V[3][E], P[NOUT][E];
    bool failed = false;
#pragma unroll
    for (int f = 0; f < NIN; ++f) {
      const int L = k * NIN + f;
      issue(L + STAGES - 1);
      const bool ok = (!ctl.stall || L > 0 || injected_stall_wait(&bars[STAGES], ctl.cap)) &&
                      mbar_wait(&bars[L % STAGES], (uint32_t)(L / STAGES) & 1u, ctl.cap);
      const C *sb = stage + (size_t)(L % STAGES) * G::stage_elems;
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = c2r_pack(sb, LW, lw, t + T * e, M, rows, tw);
      // The CTA agrees on the wait at the transform's first exchange barrier,
      // which also orders every read of the stage before its next refill (the
      // exchange halves alternate, so that barrier needs nothing before it).
      // A stage that timed out is read in bounds and its transform discarded.
      bool bad;
      if constexpr (fft_exchanges<M, E>() == 0) {
        bad = __syncthreads_or(!ok);
        line_fft<C, M, E, +1, 2>(x, t, tw, buf, sync);
      } else {
        line_fft_first<C, M, E, +1, 2>(x, t, tw, buf, [&] { bad = __syncthreads_or(!ok); }, sync);
      }
      if (bad) {
        if (tid == 0) record_timeout(ctl.status);
        for (int LL = L; LL < L + STAGES; ++LL)
          if (vb + (LL / NIN) * nvb < ntiles)
            mbar_wait(&bars[LL % STAGES], (uint32_t)(LL / STAGES) & 1u, kDrainPolls);
        failed = true;
        break;
      }
      // x[e] = (r_{2m}, r_{2m+1}) at m = t + T*e
      if (f < 3) {
#pragma unroll
        for (int e = 0; e < E; ++e) V[f][e] = x[e];
      } else if (f == 3) {  // wx: (w x v)_y = wz vx - vz wx ; (w x v)_z = wx vy - vx wy
#pragma unroll
        for (int e = 0; e < E; ++e) {
          P[1][e] = mk(-(V[2][e].x * x[e].x), -(V[2][e].y * x[e].y));
          P[2][e] = mk(x[e].x * V[1][e].x, x[e].y * V[1][e].y);
        }
      } else if (f == 4) {  // wy: (w x v)_x = wy vz - vy wz
#pragma unroll
        for (int e = 0; e < E; ++e) {
          P[0][e] = mk(x[e].x * V[2][e].x, x[e].y * V[2][e].y);
          P[2][e] = mk(P[2][e].x - V[0][e].x * x[e].x, P[2][e].y - V[0][e].y * x[e].y);
        }
      } else if (f == 5) {  // wz
#pragma unroll
        for (int e = 0; e < E; ++e) {
          P[0][e] = mk((P[0][e].x - V[1][e].x * x[e].x) * scale, (P[0][e].y - V[1][e].y * x[e].y) * scale);
          P[1][e] = mk((x[e].x * V[0][e].x + P[1][e].x) * scale, (x[e].y * V[0][e].y + P[1][e].y) * scale);
          P[2][e] = mk(P[2][e].x * scale, P[2][e].y * scale);
        }
      } else if constexpr (NOUT > 3) {
        // advect3 accumulates vx th_x + vy th_y + vz th_z, then times -1/(nx ny nz)^2
        if (f == 6) {
#pragma unroll
          for (int e = 0; e < E; ++e) P[NOUT - 1][e] = mk(V[0][e].x * x[e].x, V[0][e].y * x[e].y);
        } else if (f == 7) {
#pragma unroll
          for (int e = 0; e < E; ++e)
            P[NOUT - 1][e] = mk(P[NOUT - 1][e].x + V[1][e].x * x[e].x, P[NOUT - 1][e].y + V[1][e].y * x[e].y);
        } else {
#pragma unroll
          for (int e = 0; e < E; ++e)
            P[NOUT - 1][e] = mk((P[NOUT - 1][e].x + V[2][e].x * x[e].x) * -scale,
                                (P[NOUT - 1][e].y + V[2][e].y * x[e].y) * -scale);
        }
      }
    }
    if (failed) return;
    // forward: real-to-complex lines of the products
    C *obase = nullptr;
#pragma unroll
    for (int c = 0; c < NOUT; ++c) {
      line_fft<C, M, E, -1, 2>(P[c], t, tw, buf, sync);
#pragma unroll
      for (int e = 0; e < E; ++e) buf(t + T * e) = P[c][e];
      __syncthreads();
      obase = out.p[c] + (size_t)(tile % nzb) * BZ + (size_t)nz * (((tile / nzb) % nyg) * YB + yb) +
              rowstride * (size_t)((tile / nzb / nyg) * nxh) + l;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int kk = t + T * e;
        const C zk = buf(kk), zm = buf((M - kk) & (M - 1));
        if (kk < rows) obase[rowstride * kk] = r2c_unpack(zk, zm, tw[kk]);
        if (kk == 0 && M < rows) obase[rowstride * M] = r2c_unpack(zk, zm, mk((R)-1, (R)0));
      }
      buf.flip();  // the next write goes to the other half
    }
  }
}

template <typename R, int NX, int E, int BZ, int PHYS, int STAGES, int MINB = 2, int YB = 1>
__global__ void __launch_bounds__(YB *BZ *(NX / 2) / E, MINB) xpipe_nl_kernel(const __grid_constant__ FieldMaps maps,
                                                                         Fields<R> out, const cx<R> *__restrict__ twg,
                                                                         int ny, int nz, R scale, int rows, int nbox,
                                                                         int rb, int nruns, int nxh, PipeCtl ctl) {
  xpipe_nl_body<R, NX, E, BZ, PHYS, STAGES, YB>(blockIdx.x, gridDim.x, maps, out, twg, ny, nz, scale, rows, nbox, rb,
                                                nruns, nxh, ctl);
}

// ====================================================================
// X pass for the plain transforms (fftp3d_*), real data in GHOST's
// x-fastest layout.  The real lines go through shared memory so that
// global accesses stay coalesced in both layouts.
// ====================================================================
template <typename R, int NX, int E, int BZ>
__global__ void __launch_bounds__(BZ *(NX / 2) / E) xpass_c2r_kernel(const cx<R> *__restrict__ in,
                                                                     R *__restrict__ out,
                                                                     const cx<R> *__restrict__ twg, int ny,
                                                                     int nz) {
  using C = cx<R>;
  constexpr int M = NX / 2, T = M / E, NT = BZ * T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *tile = tw + NX;
  C *xb = tile + (M + 1) * BZ;
  const int tid = threadIdx.x, l = tid % BZ, t = tid / BZ;
  const int z0 = blockIdx.x * BZ, j = blockIdx.y;
  const size_t rowstride = (size_t)nz * ny;
  for (int e = tid; e < NX; e += NT) tw[e] = twg[e];
  x_tile_load<C, BZ>(tile, in + (size_t)z0 + (size_t)nz * j, M + 1, rowstride, tid, NT);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  auto buf = [xb, l](int idx) -> C & { return xb[idx * BZ + l]; };
  auto sync = [] { __syncthreads(); };
  C x[E];
#pragma unroll
  for (int e = 0; e < E; ++e) x[e] = c2r_pack(tile, BZ, l, t + T * e, M, M + 1, tw);
  line_fft<C, M, E, +1, 2>(x, t, tw, buf, sync);
  // line-major staging: line l, pair m at xb[l*M + m]
#pragma unroll
  for (int e = 0; e < E; ++e) xb[l * M + t + T * e] = x[e];
  __syncthreads();
  for (int q = tid; q < BZ * M; q += NT) {
    const int ll = q / M, m = q - ll * M;
    const C v = xb[q];
    R *row = out + (size_t)NX * ((size_t)j + (size_t)ny * (z0 + ll));
    row[2 * m] = v.x;
    row[2 * m + 1] = v.y;
  }
}

// Complex-to-real x lines of nine fields written straight into the LES
// closure's input rows: x[q][f] = (real value / (nx ny nz)) * gs for grid
// point q (real layout, x fastest), f = 0..8, and x[q][9] = delta.
template <typename R, int NX, int E, int BZ>
__global__ void __launch_bounds__(BZ *(NX / 2) / E) xpass_c2r_features_kernel(const __grid_constant__ Fields<R> in,
                                                                              float *__restrict__ xrows,
                                                                              const cx<R> *__restrict__ twg, int ny,
                                                                              int nz, R inv_n, float gs, float delta) {
  using C = cx<R>;
  constexpr int M = NX / 2, T = M / E, NT = BZ * T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *tile = tw + NX;
  C *xb = tile + (M + 1) * BZ;
  const int tid = threadIdx.x, l = tid % BZ, t = tid / BZ;
  const int z0 = blockIdx.x * BZ, j = blockIdx.y;
  const size_t rowstride = (size_t)nz * ny;
  for (int e = tid; e < NX; e += NT) tw[e] = twg[e];
  auto buf = [xb, l](int idx) -> C & { return xb[idx * BZ + l]; };
  auto sync = [] { __syncthreads(); };
  for (int f = 0; f < 9; ++f) {
    x_tile_load<C, BZ>(tile, in.p[f] + (size_t)z0 + (size_t)nz * j, M + 1, rowstride, tid, NT);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    C x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = c2r_pack(tile, BZ, l, t + T * e, M, M + 1, tw);
    line_fft<C, M, E, +1, 2>(x, t, tw, buf, sync);
#pragma unroll
    for (int e = 0; e < E; ++e) xb[l * M + t + T * e] = x[e];
    __syncthreads();
    for (int q = tid; q < BZ * M; q += NT) {
      const int ll = q / M, m = q - ll * M;
      const C v = xb[q];
      float *row = xrows + (size_t)10 * ((size_t)NX * ((size_t)j + (size_t)ny * (z0 + ll)) + 2 * m);
      row[f] = (float)(v.x * inv_n) * gs;
      row[10 + f] = (float)(v.y * inv_n) * gs;
      if (f == 8) {
        row[9] = delta;
        row[19] = delta;
      }
    }
    __syncthreads();  // the tile and the staging buffer are reused by the next field
  }
}

template <typename R, int NX, int E, int BZ>
__global__ void __launch_bounds__(BZ *(NX / 2) / E) xpass_r2c_kernel(const R *__restrict__ in,
                                                                     cx<R> *__restrict__ out,
                                                                     const cx<R> *__restrict__ twg, int ny,
                                                                     int nz) {
  using C = cx<R>;
  constexpr int M = NX / 2, T = M / E, NT = BZ * T;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *xb = tw + NX;  // BZ*M
  const int tid = threadIdx.x, l = tid % BZ, t = tid / BZ;
  const int z0 = blockIdx.x * BZ, j = blockIdx.y;
  const size_t rowstride = (size_t)nz * ny;
  for (int e = tid; e < NX; e += NT) tw[e] = twg[e];
  for (int q = tid; q < BZ * M; q += NT) {
    const int ll = q / M, m = q - ll * M;
    const R *row = in + (size_t)NX * ((size_t)j + (size_t)ny * (z0 + ll));
    xb[q] = mk(row[2 * m], row[2 * m + 1]);
  }
  __syncthreads();
  C x[E];
#pragma unroll
  for (int e = 0; e < E; ++e) x[e] = xb[l * M + t + T * e];
  __syncthreads();
  auto buf = [xb, l](int idx) -> C & { return xb[idx * BZ + l]; };
  auto sync = [] { __syncthreads(); };
  line_fft<C, M, E, -1, 2>(x, t, tw, buf, sync);
#pragma unroll
  for (int e = 0; e < E; ++e) buf(t + T * e) = x[e];
  __syncthreads();
  C *dst = out + (size_t)z0 + (size_t)nz * j;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int k = t + T * e;
    const C zk = buf(k), zm = buf((M - k) & (M - 1));
    dst[rowstride * k + l] = r2c_unpack(zk, zm, tw[k]);
    if (k == 0) dst[rowstride * M + l] = r2c_unpack(zk, zm, mk((R)-1, (R)0));
  }
}

}  // namespace gb
