// ops.cuh -- pointwise spectral operators and deterministic FP64
// reductions of pseudo/pseudospec3D_hd.f90.
#pragma once
#include "common.cuh"

namespace gb {

// mode index p = k + nz*(j + ny*i)
template <typename R> __device__ __forceinline__ void unflat(const KParams<R> &kp, size_t p, int &i, int &j, int &k) {
  k = (int)(p % kp.nz);
  size_t q = p / kp.nz;
  j = (int)(q % kp.ny);
  i = (int)(q / kp.ny) % kp.nxh;  // batched fields: the run index is folded into kx
}

// i*kd*a as the Fortran expression im*k*a evaluates it
template <typename C, typename R> __device__ __forceinline__ C ik(R kd, C a) { return mk(-(kd * a.y), kd * a.x); }

template <typename R> __device__ __forceinline__ R kdir(const KParams<R> &kp, int dir, int i, int j, int k) {
  return dir == 1 ? kx_of(kp, i) : (dir == 2 ? ky_of(kp, j) : kz_of(kp, k));
}

// curl component dir of (x,y,z) at one mode, rotor3 order (pseudospec3D_hd.f90:155-196)
template <typename C, typename R>
__device__ __forceinline__ C curl_at(const KParams<R> &kp, int dir, int i, int j, int k, C x, C y, C z) {
  const R kx = kx_of(kp, i), ky = ky_of(kp, j), kz = kz_of(kp, k);
  if (dir == 1) return csub(ik(ky, z), ik(kz, y));
  if (dir == 2) return csub(ik(kz, x), ik(kx, z));
  return csub(ik(kx, y), ik(ky, x));
}

template <typename R>
__global__ void derivk3_kernel(KParams<R> kp, const cx<R> *a, cx<R> *b, size_t n, int dir) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    b[p] = ik(kdir(kp, dir, i, j, k), a[p]);
  }
}

template <typename R>
__global__ void laplak3_kernel(KParams<R> kp, const cx<R> *a, cx<R> *b, size_t n) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    const R kk2 = kk2_of(kp, i, j, k);
    const cx<R> v = a[p];
    b[p] = mk(-kk2 * v.x, -kk2 * v.y);
  }
}

// rotor3(a,b,c,dir): the two given components are (a,b) in the order
// GHOST passes them: dir 1 (vy,vz), dir 2 (vx,vz), dir 3 (vx,vy)
template <typename R>
__global__ void rotor3_kernel(KParams<R> kp, const cx<R> *a, const cx<R> *b,
                              cx<R> *c, size_t n, int dir) {
  using C = cx<R>;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    const C va = a[p], vb = b[p];
    const C zero = mk((R)0, (R)0);
    C r;
    if (dir == 1) r = curl_at(kp, 1, i, j, k, zero, va, vb);
    else if (dir == 2) r = curl_at(kp, 2, i, j, k, va, zero, vb);
    else r = curl_at(kp, 3, i, j, k, va, vb, zero);
    c[p] = r;
  }
}

template <typename R>
__global__ void nonlhd3_kernel(KParams<R> kp, const cx<R> *a, const cx<R> *b,
                               const cx<R> *c, cx<R> *g, size_t n, int dir) {
  using C = cx<R>;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    const C va = a[p], vb = b[p], vc = c[p];
    const C self = dir == 1 ? va : (dir == 2 ? vb : vc);
    const int idx = dir == 1 ? i : (dir == 2 ? j : k);
    C r;
    if (idx == 0) {
      r = mk(-self.x, -self.y);
    } else {
      const R kx = kx_of(kp, i), ky = ky_of(kp, j), kz = kz_of(kp, k);
      const R kk2 = kk2_of(kp, i, j, k), kd = kdir(kp, dir, i, j, k);
      const C s = mk(kx * va.x + ky * vb.x + kz * vc.x, kx * va.y + ky * vb.y + kz * vc.y);
      r = mk(-self.x + (kd * s.x) / kk2, -self.y + (kd * s.y) / kk2);
    }
    g[p] = r;
  }
}

template <typename R>
__global__ void sharp_kernel(KParams<R> kp, const cx<R> *a, cx<R> *b, size_t n, R cut) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    b[p] = kn2_of(kp, i, j, k) <= cut ? a[p] : mk((R)0, (R)0);
  }
}

// normalize: f = f*f0/sqrt(tmp) with the division done in FP64 as the
// mixed-kind Fortran expression of module_dns.f90:35-37 does
template <typename R>
__global__ void scale3_kernel(cx<R> *x, cx<R> *y, cx<R> *z, size_t n, R f0, double s) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    cx<R> *f[3] = {x, y, z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cx<R> v = f[c][p];
      f[c][p] = mk((R)((double)(v.x * f0) / s), (R)((double)(v.y * f0) / s));
    }
  }
}

// ---------------------------------------------------------------------
// FP64 reductions over the half spectrum: sum_p w(i) * term(p), w = 1 on
// the kx = 0 plane and 2 elsewhere (the Hermitian weighting of
// pseudospec3D_hd.f90:550-567).  Per-block partials in a fixed grid, then
// one block sums them in a fixed tree: bitwise reproducible.
enum RedKind { RED_ENERGY = 0, RED_ENSTROPHY = 1, RED_LAPLACIAN = 2, RED_HELICITY = 3, RED_CROSS = 4,
               RED_CROSS_K2 = 5, RED_DIVERGENCE = 6, RED_CURL_CROSS = 7, RED_SC_CROSS = 8, RED_SC_VAR = 9,
               RED_SC_VAR_K2 = 10 };

template <typename R> struct RedArgs {
  const cx<R> *a, *b, *c, *d, *e, *f;
};

template <typename R>
__device__ __forceinline__ R red_term(const KParams<R> &kp, const RedArgs<R> &ra, int kind, size_t p, int i, int j, int k) {
  using C = cx<R>;
  const C va = ra.a[p], vb = ra.b[p], vc = ra.c[p];
  switch (kind) {
    case RED_ENERGY:
      return (va.x * va.x + va.y * va.y + vb.x * vb.x + vb.y * vb.y + vc.x * vc.x + vc.y * vc.y) * kp.tmp;
    case RED_ENSTROPHY: {
      const C w1 = curl_at(kp, 1, i, j, k, va, vb, vc), w2 = curl_at(kp, 2, i, j, k, va, vb, vc),
              w3 = curl_at(kp, 3, i, j, k, va, vb, vc);
      return (w1.x * w1.x + w1.y * w1.y + w2.x * w2.x + w2.y * w2.y + w3.x * w3.x + w3.y * w3.y) * kp.tmp;
    }
    case RED_LAPLACIAN: {
      const R kk2 = kk2_of(kp, i, j, k);
      const R s = va.x * va.x + va.y * va.y + vb.x * vb.x + vb.y * vb.y + vc.x * vc.x + vc.y * vc.y;
      return (kk2 * kk2) * s * kp.tmp;
    }
    case RED_HELICITY: {
      const C w1 = curl_at(kp, 1, i, j, k, va, vb, vc), w2 = curl_at(kp, 2, i, j, k, va, vb, vc),
              w3 = curl_at(kp, 3, i, j, k, va, vb, vc);
      return (cmulc(va, w1).x + cmulc(vb, w2).x + cmulc(vc, w3).x) * kp.tmp;
    }
    case RED_CROSS:
    case RED_CROSS_K2: {
      const C vd = ra.d[p], ve = ra.e[p], vf = ra.f[p];
      R s = cmulc(va, vd).x + cmulc(vb, ve).x + cmulc(vc, vf).x;
      if (kind == RED_CROSS_K2) s = s * kk2_of(kp, i, j, k);
      return s * kp.tmp;
    }
    case RED_SC_CROSS: {  // sctrans: Re(a conj(d)) of two scalars
      const C vd = ra.d[p];
      return cmulc(va, vd).x * kp.tmp;
    }
    case RED_SC_VAR:  // variance / spectrscc: |a|^2
      return (va.x * va.x + va.y * va.y) * kp.tmp;
    case RED_SC_VAR_K2:
      return kk2_of(kp, i, j, k) * (va.x * va.x + va.y * va.y) * kp.tmp;
    case RED_CURL_CROSS: {  // heltrans: Re(curl(a,b,c) . conj(d,e,f))
      const C w1 = curl_at(kp, 1, i, j, k, va, vb, vc), w2 = curl_at(kp, 2, i, j, k, va, vb, vc),
              w3 = curl_at(kp, 3, i, j, k, va, vb, vc);
      const C vd = ra.d[p], ve = ra.e[p], vf = ra.f[p];
      return (cmulc(w1, vd).x + cmulc(w2, ve).x + cmulc(w3, vf).x) * kp.tmp;
    }
    default: {  // RED_DIVERGENCE
      const C s = cadd(cadd(ik(kx_of(kp, i), va), ik(ky_of(kp, j), vb)), ik(kz_of(kp, k), vc));
      return (s.x * s.x + s.y * s.y) * kp.tmp;
    }
  }
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[q];
  __syncthreads();
  return s;
}

template <typename R>
__global__ void __launch_bounds__(256) reduce_kernel(KParams<R> kp, RedArgs<R> ra, int kind, size_t n, double *partials) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    const double w = i == 0 ? 1.0 : 2.0;
    acc += w * (double)red_term(kp, ra, kind, p, i, j, k);
  }
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Per-run sums of a batched field: block (x, run) covers run `run`;
// partials laid out [block][run] for finalize_kernel.
template <typename R>
__global__ void __launch_bounds__(256) reduce_runs_kernel(KParams<R> kp, RedArgs<R> ra, int kind, size_t nspec,
                                                          int nruns, double *partials) {
  __shared__ double sh[32];
  const size_t base = (size_t)blockIdx.y * nspec;
  double acc = 0.0;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < nspec; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, base + p, i, j, k);
    const double w = i == 0 ? 1.0 : 2.0;
    acc += w * (double)red_term(kp, ra, kind, base + p, i, j, k);
  }
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[(size_t)blockIdx.x * nruns + blockIdx.y] = s;
}

// f = f*f0/sqrt(e_run) per run of a batched field (normalize, per run)
template <typename R>
__global__ void scale3_runs_kernel(cx<R> *x, cx<R> *y, cx<R> *z, size_t nspec, int nruns, R f0, const double *e) {
  const size_t n = nspec * (size_t)nruns;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const double s = sqrt(e[p / nspec]);
    cx<R> *f[3] = {x, y, z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cx<R> v = f[c][p];
      f[c][p] = mk((R)((double)(v.x * f0) / s), (R)((double)(v.y * f0) / s));
    }
  }
}

// Sums nparts partials in a fixed order (one block).  Also used for the
// per-bin spectrum partials with stride.
__global__ void __launch_bounds__(256) finalize_kernel(const double *partials, int nparts, int nbins, double *out) {
  __shared__ double sh[32];
  for (int b = 0; b < nbins; ++b) {
    double acc = 0.0;
    for (int q = threadIdx.x; q < nparts; q += blockDim.x) acc += partials[(size_t)q * nbins + b];
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) out[b] = s;
  }
}

// Shell spectra (spectrumc, pseudospec3D_hd.f90:1190-1415).  Each warp
// owns a shared histogram; lanes add in lane order, warps are combined in
// warp order, blocks in block order: reproducible bit for bit.
// One warp's contribution to a shared-memory histogram: every lane with
// bin >= 0 adds its NV values to hw[bin + q * stride].  Lanes that share a bin
// are summed in lane order through shuffles and the group's lowest lane adds
// the sum, so distinct lanes never touch one slot and the result does not
// depend on scheduling (the order is fixed: lane order within a chunk, chunk
// order across the loop).
template <int NV>
__device__ __forceinline__ void warp_bin_add(double *hw, int stride, int bin, const double (&v)[NV], int lane) {
  double s[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) s[q] = 0.0;
  for (int src = 0; src < 32; ++src) {
    const int b = __shfl_sync(0xffffffffu, bin, src);
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const double x = __shfl_sync(0xffffffffu, v[q], src);
      if (b == bin) s[q] += x;
    }
  }
  const unsigned peers = __match_any_sync(0xffffffffu, bin);
  if (bin >= 0 && lane == __ffs(peers) - 1) {
#pragma unroll
    for (int q = 0; q < NV; ++q) hw[(size_t)q * stride + bin] += s[q];
  }
  __syncwarp();
}

template <typename R>
__global__ void __launch_bounds__(256) spectrum_kernel(KParams<R> kp, RedArgs<R> ra, int kind, size_t n, int nb,
                                                       R Dkk, R rnd, double *partials) {
  extern __shared__ double hist[];  // (blockDim/32) * nb
  const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = threadIdx.x; q < nw * nb; q += blockDim.x) hist[q] = 0.0;
  __syncthreads();
  double *hw = hist + (size_t)w * nb;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t start = blockIdx.x * (size_t)blockDim.x + (size_t)w * 32;
  for (size_t base = start; base < n; base += stride) {
    const size_t p = base + lane;
    int bin = -1;
    double val = 0.0;
    if (p < n) {
      int i, j, k;
      unflat(kp, p, i, j, k);
      const R kk2 = kk2_of(kp, i, j, k);
      const int kmn = (int)(sqrt(kk2) / Dkk + rnd);  // rnd: .501 rounding of the caller's GHOST routine
      if (kmn > 0 && kmn <= nb) {
        const R wgt = i == 0 ? (R)1 : (R)2;
        bin = kmn - 1;
        val = (double)(wgt * red_term(kp, ra, kind, p, i, j, k));
      }
    }
    const double vals[1] = {val};
    warp_bin_add<1>(hw, nb, bin, vals, lane);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < nw; ++q) s += hist[(size_t)q * nb + b];
    partials[(size_t)blockIdx.x * nb + b] = s;
  }
}

// Anisotropic spectra (pseudospec3D_rot.f90): mode 0 bins by |kz|
// (kmn = int(|kz| Lz + 1): specpara, entpara, heltpara), mode 1 by the
// perpendicular wavenumber (kmn = int(sqrt(kx^2 + ky^2)/Dkk + 1): specperp,
// entperp, heltperp).  Three sums per bin, partials laid out
// [block][3 nb] = total, horizontal, vertical:
//   AN_KIN  (kin 1): horizontal |a|^2 + |b|^2, vertical |c|^2
//   AN_CURL (kin 0): the same of curl(a,b,c)
//   AN_HEL  (hel 1): horizontal Re(a c1*) + Re(b c2*), vertical Re(c c3*),
//                    (c1,c2,c3) = curl(a,b,c)
//   red_term kinds (the transfers): the total only.
// In mode 1 the horizontal and vertical sums take the kz = 0 plane only,
// and the total of the other planes is one three-term sum, as specperp's.
enum AnKind { AN_KIN = 100, AN_CURL = 101, AN_HEL = 102 };

template <typename R>
__device__ __forceinline__ void an_terms(const KParams<R> &kp, const RedArgs<R> &ra, int kind, size_t p, int i, int j,
                                         int k, R &h, R &v) {
  using C = cx<R>;
  const C va = ra.a[p], vb = ra.b[p], vc = ra.c[p];
  if (kind == AN_KIN) {
    h = va.x * va.x + va.y * va.y + (vb.x * vb.x + vb.y * vb.y);
    v = vc.x * vc.x + vc.y * vc.y;
    return;
  }
  const C w1 = curl_at(kp, 1, i, j, k, va, vb, vc), w2 = curl_at(kp, 2, i, j, k, va, vb, vc),
          w3 = curl_at(kp, 3, i, j, k, va, vb, vc);
  if (kind == AN_CURL) {
    h = w1.x * w1.x + w1.y * w1.y + (w2.x * w2.x + w2.y * w2.y);
    v = w3.x * w3.x + w3.y * w3.y;
  } else {
    h = cmulc(va, w1).x + cmulc(vb, w2).x;
    v = cmulc(vc, w3).x;
  }
}

template <typename R>
__global__ void __launch_bounds__(256) aniso_kernel(KParams<R> kp, RedArgs<R> ra, int kind, int mode, size_t n, int nb,
                                                    R Lz, R Dkk, double *partials) {
  extern __shared__ double hist[];  // (blockDim/32) * 3 nb
  const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nb3 = 3 * nb;
  for (int q = threadIdx.x; q < nw * nb3; q += blockDim.x) hist[q] = 0.0;
  __syncthreads();
  double *hw = hist + (size_t)w * nb3;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t start = blockIdx.x * (size_t)blockDim.x + (size_t)w * 32;
  for (size_t base = start; base < n; base += stride) {
    const size_t p = base + lane;
    int bin = -1;
    double t = 0.0, hh = 0.0, vv = 0.0;
    if (p < n) {
      int i, j, k;
      unflat(kp, p, i, j, k);
      int kmn;
      if (mode == 0) {
        kmn = (int)(fabs(kz_of(kp, k)) * Lz + (R)1);
      } else {
        const R a = kx_of(kp, i), b = ky_of(kp, j);
        kmn = (int)(sqrt(a * a + b * b) / Dkk + (R)1);
      }
      if (kmn > 0 && kmn <= nb) {
        const R wgt = i == 0 ? (R)1 : (R)2;
        bin = kmn - 1;
        if (kind >= AN_KIN) {
          R h, v;
          an_terms(kp, ra, kind, p, i, j, k, h, v);
          if (mode == 0 || k == 0) {
            hh = (double)(wgt * h * kp.tmp);
            vv = (double)(wgt * v * kp.tmp);
            t = hh + vv;
          } else {
            t = (double)(wgt * (h + v) * kp.tmp);
          }
        } else {
          t = (double)(wgt * red_term(kp, ra, kind, p, i, j, k));
        }
      }
    }
    const double vals[3] = {t, hh, vv};
    warp_bin_add<3>(hw, nb, bin, vals, lane);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nb3; b += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < nw; ++q) s += hist[(size_t)q * nb3 + b];
    partials[(size_t)blockIdx.x * nb3 + b] = s;
  }
}

// The slowly varying forcing of main3D.fpp:2646-2657 (rand = 2): per mode
// f = (1 - rmp) fold + rmp fnew, products and sum rounded one by one (no
// contraction), as GHOST's Fortran evaluates them.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
template <typename R> struct Blend3 {
  const cx<R> *old[3], *nw[3];
  cx<R> *out[3];
};
template <typename R> __global__ void blend3_kernel(Blend3<R> b, size_t n, R w0, R w1) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const cx<R> u = b.old[a][p], v = b.nw[a][p];
      b.out[a][p] = mk(add_rn(mul_rn(w0, u.x), mul_rn(w1, v.x)), add_rn(mul_rn(w0, u.y), mul_rn(w1, v.y)));
    }
  }
}

// phaseshift (pseudospec3D_hd.f90:2084-2148): a *= c, except on the kx = 0
// plane, where GHOST's loops multiply the modes of one half by c and their
// mirrors by conj(c).  The kz = nz/2 and ky = ny/2 lines of that plane are
// reached by both loops and so take both factors, in the order the loops
// apply them.
template <typename R>
__global__ void phaseshift_kernel(KParams<R> kp, cx<R> *a, size_t n, cx<R> cd) {
  const cx<R> jd = mk(cd.x, -cd.y);
  const int nyh = kp.ny / 2, nzh = kp.nz / 2;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    cx<R> v = a[p];
    if (i > 0) {
      v = cmul(v, cd);
    } else if (k == 0 && j == 0) {
    } else if (k == 0 || j == 0) {  // the ky = 0 row or the kz = 0 row of the plane
      const int q = k == 0 ? j : k, h = k == 0 ? nyh : nzh;
      if (q < h) v = cmul(v, cd);
      else if (q == h) v = cmul(cmul(v, cd), jd);
      else v = cmul(v, jd);
    } else if (k < nzh) {
      v = cmul(v, cd);
    } else if (k > nzh) {
      v = cmul(v, jd);
    } else if (j <= nyh) {  // k = nz/2: reached as the direct mode first
      v = cmul(cmul(v, cd), jd);
    } else {  // reached as a mirror first
      v = cmul(cmul(v, jd), cd);
    }
    a[p] = v;
  }
}

// vector3's real-space cross product (pseudospec3D_mhd.f90:22-105):
// x = (b f - e c) tmp, y = (c d - f a) tmp, z = (a e - d b) tmp for the real
// fields (a, b, c) x (d, e, f), tmp = 1/(nx ny nz)^2
template <typename R>
__global__ void cross_real_kernel(const R *__restrict__ a, const R *__restrict__ b, const R *__restrict__ c,
                                  const R *__restrict__ d, const R *__restrict__ e, const R *__restrict__ f,
                                  R *__restrict__ x, R *__restrict__ y, R *__restrict__ z, size_t n, R tmp) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const R r1 = a[p], r2 = b[p], r3 = c[p], r4 = d[p], r5 = e[p], r6 = f[p];
    x[p] = (r2 * r6 - r5 * r3) * tmp;
    y[p] = (r3 * r4 - r6 * r1) * tmp;
    z[p] = (r1 * r5 - r4 * r2) * tmp;
  }
}

// o = a - d, componentwise over three field pairs (nonlin3's a - d, b - e, c - f)
template <typename R>
__global__ void sub3_kernel(const cx<R> *a, const cx<R> *b, const cx<R> *c, const cx<R> *d, const cx<R> *e,
                            const cx<R> *f, cx<R> *x, cx<R> *y, cx<R> *z, size_t n) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    x[p] = csub(a[p], d[p]);
    y[p] = csub(b[p], e[p]);
    z[p] = csub(c[p], f[p]);
  }
}

template <typename R>
__global__ void neg_kernel(cx<R> *x, size_t n) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
    x[p] = mk(-x[p].x, -x[p].y);
}

// The truncated update of mhd_rkstep2 (include/mhd_rkstep2.f90): with
// laplak3 inline, v = C + dt (nu lap v + g + f)/o and a = C' + dt (mu lap a
// + h + m)/o on tiny <= kn2 <= kmax, everything zero elsewhere.
template <typename R> struct MhdUpd {
  cx<R> *v[3], *a[3];
  const cx<R> *cv[3], *ca[3], *g[3], *h[3], *f[3], *m[3];
};
template <typename R>
__global__ void mhd_update_kernel(KParams<R> kp, MhdUpd<R> u, size_t n, R dt, R nu, R mu, R rmp) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    unflat(kp, p, i, j, k);
    const R kn2 = kn2_of(kp, i, j, k);
    if (kn2 <= kp.kmax && kn2 >= kp.tiny) {
      const R kk2 = kk2_of(kp, i, j, k);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const cx<R> vv = u.v[q][p], aa = u.a[q][p];
        const cx<R> lv = mk(-kk2 * vv.x, -kk2 * vv.y), la = mk(-kk2 * aa.x, -kk2 * aa.y);
        cx<R> sv = mk(nu * lv.x + u.g[q][p].x, nu * lv.y + u.g[q][p].y);
        cx<R> sa = mk(mu * la.x + u.h[q][p].x, mu * la.y + u.h[q][p].y);
        if (u.f[q]) sv = cadd(sv, u.f[q][p]);
        if (u.m[q]) sa = cadd(sa, u.m[q][p]);
        u.v[q][p] = mk(u.cv[q][p].x + dt * sv.x * rmp, u.cv[q][p].y + dt * sv.y * rmp);
        u.a[q][p] = mk(u.ca[q][p].x + dt * sa.x * rmp, u.ca[q][p].y + dt * sa.y * rmp);
      }
    } else {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        u.v[q][p] = mk((R)0, (R)0);
        u.a[q][p] = mk((R)0, (R)0);
      }
    }
  }
}

// Horizontal (x, y) sums of real fields per z-plane (havgcomp,
// pseudospec3D_bouss.f90:19-554): block (k, s) sums a strided part of plane k
// of op(r1, r2, r3) into partials[k * gridDim.y + s].
enum ZProfOp { ZP_SQ2 = 0, ZP_SQ1 = 1, ZP_PROD = 2, ZP_NEGPROD = 3, ZP_CURLTERM = 4, ZP_PV = 5 };
template <typename R> struct ZProfArgs {
  const R *r1, *r2, *r3;
  R fo, bv;
  double tmpn;  // 1/(nx ny nz) for ZP_PV
};
template <typename R>
__global__ void __launch_bounds__(256) zprof_kernel(ZProfArgs<R> za, int op, size_t plane, double *partials) {
  __shared__ double sh[32];
  const int k = blockIdx.x;
  const size_t off = (size_t)k * plane;
  double acc = 0.0;
  for (size_t q = blockIdx.y * (size_t)blockDim.x + threadIdx.x; q < plane; q += (size_t)gridDim.y * blockDim.x) {
    const size_t p = off + q;
    if (op == ZP_SQ2) {
      const R a = za.r1[p], b = za.r2[p];
      acc += (double)(a * a + b * b);
    } else if (op == ZP_SQ1) {
      const R a = za.r1[p];
      acc += (double)(a * a);
    } else if (op == ZP_PROD) {
      acc += (double)(za.r1[p] * za.r2[p]);
    } else if (op == ZP_NEGPROD) {
      acc -= (double)(za.r1[p] * za.r2[p]);
    } else if (op == ZP_CURLTERM) {
      acc += (double)(za.r3[p] * (za.r1[p] - za.r2[p]));
    } else {
      // potential vorticity: fo dtheta/dz - bv w_z + w.grad(theta) - fo bv,
      // each real field carrying the N^3 of the transforms (type 7)
      R pv = (R)((double)za.fo * (double)za.r1[p] * za.tmpn);
      pv = (R)((double)pv - (double)za.bv * (double)za.r2[p] * za.tmpn);
      pv = (R)((double)pv + (double)za.r3[p] * -za.tmpn);
      pv = pv - za.fo * za.bv;
      acc += (double)(pv * pv);
    }
  }
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[(size_t)k * gridDim.y + blockIdx.y] = s;
}

// max over real space of sqrt(r1^2+r2^2+r3^2) (maxabs); non-negative
// floats order like their bit patterns, so an integer max is exact.
template <typename R>
__global__ void maxnorm_kernel(const R *__restrict__ r1, const R *__restrict__ r2, const R *__restrict__ r3, size_t n,
                               unsigned long long *out) {
  R m = 0;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const R s = sqrt(r1[p] * r1[p] + r2[p] * r2[p] + r3[p] * r3[p]);
    m = s > m ? s : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const R q = __shfl_down_sync(0xffffffffu, m, o);
    m = q > m ? q : m;
  }
  if ((threadIdx.x & 31) == 0) {
    const double md = (double)m;
    atomicMax(out, (unsigned long long)__double_as_longlong(md));
  }
}

}  // namespace gb
