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
// Z pass
// ====================================================================
template <int N, int E> struct ZShape {
  static constexpr int T = N / E;
  static constexpr int NP = N + N / 8;  // padded line: idx + idx/8 spreads strided writes over banks
};

// Generic shell: twiddles to shared memory, per-line buffer accessor, then
// the operation's body.  nlines must be a multiple of LPB (host checks).
template <typename R, int N, int E, class Op>
__global__ void __launch_bounds__(256) zpass_kernel(Op op, const cx<R> *__restrict__ twg, int lpb) {
  using C = cx<R>;
  constexpr int T = ZShape<N, E>::T, NP = ZShape<N, E>::NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *xb = tw + N;
  const int tid = threadIdx.x, lq = tid / T, t = tid - lq * T;
  for (int e = tid; e < N; e += blockDim.x) tw[e] = twg[e];
  __syncthreads();
  const long line = (long)blockIdx.x * lpb + lq;
  C *mine = xb + lq * NP;
  auto buf = [mine](int idx) -> C & { return mine[idx + (idx >> 3)]; };
  auto sync = [] { __syncthreads(); };
  op.template body<N, E>(line, t, tw, buf, sync);
}

// In-place (or out-of-place) c2c along z of nf fields.
template <typename R, int S> struct ZC2C {
  using C = cx<R>;
  CFields<R> in;
  Fields<R> out;
  int nf, nz;
  template <int N, int E, class Buf, class Sync>
  __device__ __forceinline__ void body(long line, int t, const C *tw, Buf buf, Sync sync) const {
    constexpr int T = N / E;
    for (int f = 0; f < nf; ++f) {
      const C *src = in.p[f] + (size_t)line * N;
      C *dst = out.p[f] + (size_t)line * N;
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = src[t + T * e];
      line_fft<C, N, E, S>(x, t, tw, buf, sync);
#pragma unroll
      for (int e = 0; e < E; ++e) dst[t + T * e] = x[e];
    }
  }
};

// Inverse prologue of the fused substep: reads v (and theta for the
// Boussinesq solver), forms per mode the fields the real-space products
// need and runs the inverse z transform of each:
//   PHYS 0 (HD):    v, curl v                       (prodre3 inputs)
//   PHYS 1 (BOUSS): v, curl v, i k theta            (prodre3 + advect3 inputs)
// curl as rotor3 (pseudospec3D_hd.f90:124-200), i k theta as derivk3.
// With copy != 0 it also stores the RK1 copies C = v (theta).
template <typename R, int PHYS> struct ZInv {
  using C = cx<R>;
  static constexpr int NIN = PHYS == 0 ? 3 : 4;
  static constexpr int NOUT = PHYS == 0 ? 6 : 9;
  CFields<R> v;   // NIN
  Fields<R> w;    // NOUT outputs
  Fields<R> cpy;  // NIN (when copy)
  KParams<R> kp;
  int copy;
  template <int N, int E, class Buf, class Sync>
  __device__ __forceinline__ void body(long line, int t, const C *tw, Buf buf, Sync sync) const {
    constexpr int T = N / E;
    const int j = (int)(line % kp.ny), i = (int)(line / kp.ny);
    const R kx = kx_of(kp, i), ky = ky_of(kp, j);
    C a[NIN][E];
#pragma unroll
    for (int c = 0; c < NIN; ++c)
#pragma unroll
      for (int e = 0; e < E; ++e) a[c][e] = v.p[c][(size_t)line * N + t + T * e];
    if (copy) {
#pragma unroll
      for (int c = 0; c < NIN; ++c)
#pragma unroll
        for (int e = 0; e < E; ++e) cpy.p[c][(size_t)line * N + t + T * e] = a[c][e];
    }
#pragma unroll 1
    for (int f = 0; f < NOUT; ++f) {
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const R kz = kz_of(kp, t + T * e);
        if (f < 3) {
          x[e] = a[f][e];
        } else if (f < 6) {
          // i k a = (-k a.y, k a.x)
          const C vx = a[0][e], vy = a[1][e], vz = a[2][e];
          if (f == 3) x[e] = mk((-ky * vz.y) - (-kz * vy.y), (ky * vz.x) - (kz * vy.x));
          else if (f == 4) x[e] = mk((-kz * vx.y) - (-kx * vz.y), (kz * vx.x) - (kx * vz.x));
          else x[e] = mk((-kx * vy.y) - (-ky * vx.y), (kx * vy.x) - (ky * vx.x));
        } else {
          const C th = a[NIN - 1][e];
          const R kd = f == 6 ? kx : (f == 7 ? ky : kz);
          x[e] = mk(-(kd * th.y), kd * th.x);
        }
      }
      line_fft<C, N, E, +1>(x, t, tw, buf, sync);
      C *dst = w.p[f] + (size_t)line * N;
#pragma unroll
      for (int e = 0; e < E; ++e) dst[t + T * e] = x[e];
    }
  }
};

// HD forward epilogue: forward z transform of the three components of
// omega x v, then nonlhd3 x3 (pseudospec3D_hd.f90:399-509), laplak3 and
// the truncated RK update of include/hd_rkstep2.f90:18-38, written to v.
template <typename R> struct ZFwdHD {
  using C = cx<R>;
  CFields<R> nl;  // 3 (x and y transformed)
  Fields<R> v;    // 3 in/out
  CFields<R> c0;  // C1..C3
  CFields<R> f;   // forcing or null
  KParams<R> kp;
  R dt, nu, rmp;
  template <int N, int E, class Buf, class Sync>
  __device__ __forceinline__ void body(long line, int t, const C *tw, Buf buf, Sync sync) const {
    constexpr int T = N / E;
    const int j = (int)(line % kp.ny), i = (int)(line / kp.ny);
    const R kx = kx_of(kp, i), ky = ky_of(kp, j);
    C g[3][E];
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = nl.p[c][(size_t)line * N + t + T * e];
      line_fft<C, N, E, -1>(x, t, tw, buf, sync);
#pragma unroll
      for (int e = 0; e < E; ++e) g[c][e] = x[e];
    }
    const bool forced = f.p[0] != nullptr;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = t + T * e;
      const size_t p = (size_t)line * N + k;
      const R kz = kz_of(kp, k);
      const R kn2 = kn2_of(kp, i, j, k);
      if (kn2 <= kp.kmax && kn2 >= kp.tiny) {
        const R kk2 = kk2_of(kp, i, j, k);
        const C a = g[0][e], b = g[1][e], cc = g[2][e];
        const C s = mk(kx * a.x + ky * b.x + kz * cc.x, kx * a.y + ky * b.y + kz * cc.y);
        C nl3[3];
        nl3[0] = (i == 0) ? mk(-a.x, -a.y) : mk(-a.x + (kx * s.x) / kk2, -a.y + (kx * s.y) / kk2);
        nl3[1] = (j == 0) ? mk(-b.x, -b.y) : mk(-b.x + (ky * s.x) / kk2, -b.y + (ky * s.y) / kk2);
        nl3[2] = (k == 0) ? mk(-cc.x, -cc.y) : mk(-cc.x + (kz * s.x) / kk2, -cc.y + (kz * s.y) / kk2);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const C vv = v.p[c][p];
          const C lap = mk(-kk2 * vv.x, -kk2 * vv.y);
          C sum = mk(nu * lap.x + nl3[c].x, nu * lap.y + nl3[c].y);
          if (forced) {
            const C ff = f.p[c][p];
            sum = mk(sum.x + ff.x, sum.y + ff.y);
          }
          const C cc0 = c0.p[c][p];
          v.p[c][p] = mk(cc0.x + (dt * sum.x) * rmp, cc0.y + (dt * sum.y) * rmp);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) v.p[c][p] = mk((R)0, (R)0);
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
  CFields<R> nl;  // 4: (w x v)_xyz, -v.grad(theta)
  Fields<R> v;    // 4 in/out: vx, vy, vz, theta
  CFields<R> c0;  // C1..C3, C20
  CFields<R> f;   // fx, fy, fz, fs (any null: zero)
  KParams<R> kp;
  R dt, nu, kappa, omegaz, xmom, xtemp, rmp;
  template <int N, int E, class Buf, class Sync>
  __device__ __forceinline__ void body(long line, int t, const C *tw, Buf buf, Sync sync) const {
    constexpr int T = N / E;
    const int j = (int)(line % kp.ny), i = (int)(line / kp.ny);
    const R kx = kx_of(kp, i), ky = ky_of(kp, j);
    C g[4][E];
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      C x[E];
#pragma unroll
      for (int e = 0; e < E; ++e) x[e] = nl.p[c][(size_t)line * N + t + T * e];
      line_fft<C, N, E, -1>(x, t, tw, buf, sync);
#pragma unroll
      for (int e = 0; e < E; ++e) g[c][e] = x[e];
    }
    const bool forced = f.p[0] != nullptr, sforced = f.p[3] != nullptr;
    const R two_om = (R)2 * omegaz;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = t + T * e;
      const size_t p = (size_t)line * N + k;
      const R kn2 = kn2_of(kp, i, j, k);
      if (kn2 <= kp.kmax && kn2 >= kp.tiny) {
        const R kz = kz_of(kp, k);
        const R kk2 = kk2_of(kp, i, j, k);
        C vv[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) vv[c] = v.p[c][p];
        const C a = mk(g[0][e].x - two_om * vv[1].x, g[0][e].y - two_om * vv[1].y);
        const C b = mk(g[1][e].x + two_om * vv[0].x, g[1][e].y + two_om * vv[0].y);
        const C cc = mk(g[2][e].x + xmom * vv[3].x, g[2][e].y + xmom * vv[3].y);
        const C s = mk(kx * a.x + ky * b.x + kz * cc.x, kx * a.y + ky * b.y + kz * cc.y);
        C rhs[4];
        rhs[0] = (i == 0) ? mk(-a.x, -a.y) : mk(-a.x + (kx * s.x) / kk2, -a.y + (kx * s.y) / kk2);
        rhs[1] = (j == 0) ? mk(-b.x, -b.y) : mk(-b.x + (ky * s.x) / kk2, -b.y + (ky * s.y) / kk2);
        rhs[2] = (k == 0) ? mk(-cc.x, -cc.y) : mk(-cc.x + (kz * s.x) / kk2, -cc.y + (kz * s.y) / kk2);
        rhs[3] = mk(g[3][e].x + xtemp * vv[2].x, g[3][e].y + xtemp * vv[2].y);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const R dif = c < 3 ? nu : kappa;
          const C lap = mk(-kk2 * vv[c].x, -kk2 * vv[c].y);
          C sum = mk(dif * lap.x + rhs[c].x, dif * lap.y + rhs[c].y);
          if (c < 3 ? forced : sforced) {
            const C ff = f.p[c][p];
            sum = mk(sum.x + ff.x, sum.y + ff.y);
          }
          const C cc0 = c0.p[c][p];
          v.p[c][p] = mk(cc0.x + (dt * sum.x) * rmp, cc0.y + (dt * sum.y) * rmp);
        }
      } else if (kn2 > kp.kmax) {
#pragma unroll
        for (int c = 0; c < 4; ++c) v.p[c][p] = mk((R)0, (R)0);
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) v.p[c][p] = mk((R)0, (R)0);
        v.p[3][p] = c0.p[3][p];
      }
    }
  }
};

// ====================================================================
// Y pass: in place c2c along y of nf fields
// ====================================================================
template <typename R, int N, int E, int S>
__global__ void __launch_bounds__(1024) ypass_kernel(Fields<R> fld, const cx<R> *__restrict__ twg, int nz,
                                                     int bz) {
  using C = cx<R>;
  constexpr int T = N / E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *xb = tw + N;
  const int tid = threadIdx.x, l = tid % bz, t = tid / bz;
  for (int e = tid; e < N; e += blockDim.x) tw[e] = twg[e];
  __syncthreads();
  const int z = blockIdx.x * bz + l, i = blockIdx.y;
  C *base = fld.p[blockIdx.z] + (size_t)z + (size_t)nz * N * i;
  C x[E];
#pragma unroll
  for (int e = 0; e < E; ++e) x[e] = base[(size_t)nz * (t + T * e)];
  auto buf = [xb, bz, l](int idx) -> C & { return xb[idx * bz + l]; };
  auto sync = [] { __syncthreads(); };
  line_fft<C, N, E, S>(x, t, tw, buf, sync);
#pragma unroll
  for (int e = 0; e < E; ++e) base[(size_t)nz * (t + T * e)] = x[e];
}

// ====================================================================
// X pass helpers
// ====================================================================
// Stage the (M+1) x BZ tile of kx rows at (z0.., j) of one field.
template <typename C, int BZ>
__device__ __forceinline__ void x_tile_load(C *tile, const C *src, int M, size_t rowstride, int tid, int nthr) {
  constexpr int CH = BZ * (int)sizeof(C) / 16;  // 16-byte chunks per row
  const int nch = (M + 1) * CH;
  for (int q = tid; q < nch; q += nthr) {
    const int row = q / CH, c = q - row * CH;
    cp_async16(reinterpret_cast<unsigned char *>(tile + row * BZ) + 16 * c,
               reinterpret_cast<const unsigned char *>(src + rowstride * row) + 16 * c);
  }
}

// complex-to-real packing of the half spectrum for the M = nx/2 point
// inverse transform:  Z_k = (X_k + conj X_{M-k}) + i e^{+2 pi i k/nx} (X_k - conj X_{M-k}),
// with only the real parts of X_0 and X_M taken.
template <typename C>
__device__ __forceinline__ C c2r_pack(const C *tile, int bz, int l, int k, int M, const C *tw) {
  C xk = tile[k * bz + l], xm = tile[(M - k) * bz + l];
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
// scale is 1/(nx ny nz)^2; outputs may alias in[0..NOUT-1].
// ====================================================================
template <typename R, int NX, int E, int BZ, int PHYS>
__global__ void __launch_bounds__(BZ *(NX / 2) / E) xpass_nl_kernel(CFields<R> in, Fields<R> out,
                                                                    const cx<R> *__restrict__ twg, int ny,
                                                                    int nz, R scale) {
  using C = cx<R>;
  constexpr int M = NX / 2, T = M / E, NT = BZ * T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);  // NX
  C *tile0 = tw + NX;                       // (M+1)*BZ
  C *tile1 = tile0 + (M + 1) * BZ;
  C *xb = tile1 + (M + 1) * BZ;             // M*BZ
  const int tid = threadIdx.x, l = tid % BZ, t = tid / BZ;
  const int z0 = blockIdx.x * BZ, j = blockIdx.y;
  const size_t rowstride = (size_t)nz * ny;
  const size_t off = (size_t)z0 + (size_t)nz * j;
  for (int e = tid; e < NX; e += NT) tw[e] = twg[e];
  x_tile_load<C, BZ>(tile0, in.p[0] + off, M, rowstride, tid, NT);
  cp_async_commit();
  auto buf = [xb, l](int idx) -> C & { return xb[idx * BZ + l]; };
  auto sync = [] { __syncthreads(); };
  constexpr int NIN = PHYS == 0 ? 6 : 9, NOUT = PHYS == 0 ? 3 : 4;
  C V[3][E], P[NOUT][E];
#pragma unroll 1
  for (int f = 0; f < NIN; ++f) {
    C *tile = (f & 1) ? tile1 : tile0;
    if (f + 1 < NIN) {
      x_tile_load<C, BZ>((f & 1) ? tile0 : tile1, in.p[f + 1] + off, M, rowstride, tid, NT);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    C x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = c2r_pack(tile, BZ, l, t + T * e, M, tw);
    line_fft<C, M, E, +1, 2>(x, t, tw, buf, sync);
    // x[e] = (r_{2m}, r_{2m+1}) at m = t + T*e
    switch (f) {
      case 0:
      case 1:
      case 2:
#pragma unroll
        for (int e = 0; e < E; ++e) V[f][e] = x[e];
        break;
      case 3:  // wx: (w x v)_y = wz vx - vz wx ; (w x v)_z = wx vy - vx wy
#pragma unroll
        for (int e = 0; e < E; ++e) {
          P[1][e] = mk(-(V[2][e].x * x[e].x), -(V[2][e].y * x[e].y));
          P[2][e] = mk(x[e].x * V[1][e].x, x[e].y * V[1][e].y);
        }
        break;
      case 4:  // wy: (w x v)_x = wy vz - vy wz
#pragma unroll
        for (int e = 0; e < E; ++e) {
          P[0][e] = mk(x[e].x * V[2][e].x, x[e].y * V[2][e].y);
          P[2][e] = mk(P[2][e].x - V[0][e].x * x[e].x, P[2][e].y - V[0][e].y * x[e].y);
        }
        break;
      case 5:  // wz
#pragma unroll
        for (int e = 0; e < E; ++e) {
          P[0][e] = mk((P[0][e].x - V[1][e].x * x[e].x) * scale, (P[0][e].y - V[1][e].y * x[e].y) * scale);
          P[1][e] = mk((x[e].x * V[0][e].x + P[1][e].x) * scale, (x[e].y * V[0][e].y + P[1][e].y) * scale);
          P[2][e] = mk(P[2][e].x * scale, P[2][e].y * scale);
        }
        break;
      case 6:  // dtheta/dx: advect3 accumulates vx th_x + vy th_y + vz th_z
        if constexpr (NOUT > 3) {
#pragma unroll
          for (int e = 0; e < E; ++e) P[3][e] = mk(V[0][e].x * x[e].x, V[0][e].y * x[e].y);
        }
        break;
      case 7:
        if constexpr (NOUT > 3) {
#pragma unroll
          for (int e = 0; e < E; ++e) P[3][e] = mk(P[3][e].x + V[1][e].x * x[e].x, P[3][e].y + V[1][e].y * x[e].y);
        }
        break;
      default:  // 8: times -1/(nx ny nz)^2
        if constexpr (NOUT > 3) {
#pragma unroll
          for (int e = 0; e < E; ++e)
            P[3][e] = mk((P[3][e].x + V[2][e].x * x[e].x) * -scale, (P[3][e].y + V[2][e].y * x[e].y) * -scale);
        }
        break;
    }
    __syncthreads();  // every thread is done with this tile before it is refilled
  }
  // forward: real-to-complex lines of the products
#pragma unroll 1
  for (int c = 0; c < NOUT; ++c) {
    C x[E];
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = P[c][e];
    line_fft<C, M, E, -1, 2>(x, t, tw, buf, sync);
#pragma unroll
    for (int e = 0; e < E; ++e) buf(t + T * e) = x[e];
    __syncthreads();
    C *dst = out.p[c] + off + l;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = t + T * e;
      const C zk = buf(k), zm = buf((M - k) & (M - 1));
      dst[rowstride * k] = r2c_unpack(zk, zm, tw[k]);
      if (k == 0) {
        // X_M = F_0 - G_0
        const C x0 = r2c_unpack(zk, zm, mk((R)-1, (R)0));
        dst[rowstride * M] = x0;
      }
    }
    __syncthreads();
  }
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
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  C *tile = tw + NX;
  C *xb = tile + (M + 1) * BZ;
  const int tid = threadIdx.x, l = tid % BZ, t = tid / BZ;
  const int z0 = blockIdx.x * BZ, j = blockIdx.y;
  const size_t rowstride = (size_t)nz * ny;
  for (int e = tid; e < NX; e += NT) tw[e] = twg[e];
  x_tile_load<C, BZ>(tile, in + (size_t)z0 + (size_t)nz * j, M, rowstride, tid, NT);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  auto buf = [xb, l](int idx) -> C & { return xb[idx * BZ + l]; };
  auto sync = [] { __syncthreads(); };
  C x[E];
#pragma unroll
  for (int e = 0; e < E; ++e) x[e] = c2r_pack(tile, BZ, l, t + T * e, M, tw);
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

template <typename R, int NX, int E, int BZ>
__global__ void __launch_bounds__(BZ *(NX / 2) / E) xpass_r2c_kernel(const R *__restrict__ in,
                                                                     cx<R> *__restrict__ out,
                                                                     const cx<R> *__restrict__ twg, int ny,
                                                                     int nz) {
  using C = cx<R>;
  constexpr int M = NX / 2, T = M / E, NT = BZ * T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
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
