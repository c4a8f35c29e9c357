// les.cu -- large-eddy simulation on a coarse grid: sharp-filter data from
// a fine (DNS) grid, the learned subgrid-stress closure (the MLP of
// mlp.cu) and GHOST's EDQNM eddy viscosity as its fallback.
//
// Conventions (GHOST's): spectral fields are unnormalised, a(k,j,i) with z
// fastest; a field on an n^3 grid carries n^3 times its Fourier
// coefficients, so moving a mode from the N^3 grid to the n^3 grid scales
// it by (n/N)^3.  The sharp filter keeps kx^2+ky^2+kz^2 <= kc^2 (GHOST's
// sharp, pseudospec3D_filt.f90:200-241, with Delta = pi/kc).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/ghost_b200.h"
#include "common.cuh"
#include "internal.cuh"

using namespace gb;

namespace les {

constexpr int RED_ENERGY_KIND = 0;
constexpr int RED_HELICITY_KIND = 3;  // the reduction kind of spectrumc's helicity spectrum (ops.cuh RED_HELICITY)

// ---------------------------------------------------------------------
// kernels

// out (coarse n^3 spectrum) = modes of in (fine N^3 spectrum) with
// |k|^2 <= kc2, times scale; the rest zero.  One thread per coarse mode.
template <typename R>
__global__ void truncate_kernel(const cx<R> *__restrict__ in, cx<R> *__restrict__ out, int n, int N, int kc2, R scale) {
  const int nxh = n / 2 + 1;
  const size_t total = (size_t)nxh * n * n;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(p % n), j = (int)((p / n) % n), i = (int)(p / ((size_t)n * n));
    const int kx = i < n / 2 ? i : i - n, ky = j < n / 2 ? j : j - n, kz = k < n / 2 ? k : k - n;
    cx<R> v;
    v.x = 0;
    v.y = 0;
    if (kx >= 0 && kx * kx + ky * ky + kz * kz <= kc2) {
      const int jf = ky >= 0 ? ky : ky + N, kf = kz >= 0 ? kz : kz + N;
      const cx<R> a = in[((size_t)kx * N + jf) * N + kf];
      v.x = a.x * scale;
      v.y = a.y * scale;
    }
    out[p] = v;
  }
}

// p = (a * sa) (b * sb) on a real grid
template <typename R>
__global__ void product_kernel(const R *__restrict__ a, const R *__restrict__ b, R *__restrict__ p, size_t n, R s) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    p[q] = (a[q] * s) * (b[q] * s);
}

// Targets: tau[q][m] = filt(u_a u_b) - ubar_a ubar_b for the pairs m =
// xx, yy, zz, xy, xz, yz; P[m] holds n^3 filt(u_a u_b), U[a] n^3 ubar_a.
template <typename R> struct TauFields {
  const R *P[6];
  const R *U[3];
};
__constant__ int kPairA[6] = {0, 1, 2, 0, 0, 1};
__constant__ int kPairB[6] = {0, 1, 2, 1, 2, 2};
template <typename R>
__global__ void targets_kernel(TauFields<R> tf, float *__restrict__ tau, size_t n, R inv_n3, float ts) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const R u[3] = {tf.U[0][q] * inv_n3, tf.U[1][q] * inv_n3, tf.U[2][q] * inv_n3};
#pragma unroll
    for (int m = 0; m < 6; ++m)
      tau[q * GHOST_MLP_NOUT + m] = (float)(tf.P[m][q] * inv_n3 - u[kPairA[m]] * u[kPairB[m]]) * ts;
  }
}

// tau rows (closure output, scaled by 1/ts) -> six real fields (physical)
template <typename R> struct RealOut6 {
  R *t[6];
};
template <typename R>
__global__ void unpack_tau_kernel(const float *__restrict__ tau, RealOut6<R> o, size_t n, float ts) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int m = 0; m < 6; ++m) o.t[m][q] = (R)(tau[q * GHOST_MLP_NOUT + m] * ts);
  }
}

// o_a = f_a + P(-i k_b T_ab), T the six transformed stresses; P the Leray
// projection; modes outside tiny <= kn2 <= kmax get f only.
template <typename R> struct Spec6 {
  const cx<R> *T[6];
};
template <typename R> struct Spec3 {
  const cx<R> *p[3];
};
template <typename R> struct Spec3w {
  cx<R> *p[3];
};
template <typename R>
__global__ void tau_force_kernel(KParams<R> kp, Spec6<R> T, Spec3<R> f, Spec3w<R> o, size_t total) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(p % kp.nz), j = (int)((p / kp.nz) % kp.ny), i = (int)(p / ((size_t)kp.nz * kp.ny));
    const R kn2 = kn2_of(kp, i, j, k);
    cx<R> F[3] = {{0, 0}, {0, 0}, {0, 0}};
    if (kn2 <= kp.kmax && kn2 >= kp.tiny) {
      const R kv[3] = {kx_of(kp, i), ky_of(kp, j), kz_of(kp, k)};
      // symmetric stress: (a,b) -> slot
      const int slot[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        R re = 0, im = 0;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const cx<R> t = T.T[slot[a][b]][p];
          // -i k_b t = k_b (t.y, -t.x)
          re += kv[b] * t.y;
          im -= kv[b] * t.x;
        }
        F[a].x = re;
        F[a].y = im;
      }
      const R kk2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      const R dre = (kv[0] * F[0].x + kv[1] * F[1].x + kv[2] * F[2].x) / kk2;
      const R dim = (kv[0] * F[0].y + kv[1] * F[1].y + kv[2] * F[2].y) / kk2;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        F[a].x -= kv[a] * dre;
        F[a].y -= kv[a] * dim;
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      cx<R> v = F[a];
      if (f.p[a]) {
        v.x += f.p[a][p].x;
        v.y += f.p[a][p].y;
      }
      o.p[a][p] = v;
    }
  }
}

// EDQNM eddy viscosity as a force: o_a = f_a - tve(ki) kk2 v_a with
// ki = int(sqrt(kk2) + 0.501) (include/edqnmhd_rkstep2.f90:45-56 writes
// (nu + tve(ki)) times the Laplacian); tve 1-based in GHOST, tve[ki-1] here.
// With tvh (heli = 1) the helicity eddy diffusivity adds tvh(ki) w_a, w =
// curl v formed as rotor3 does (:25-27, the C5, C6, C19 of the update).
template <typename R>
__global__ void eddy_force_kernel(KParams<R> kp, Spec3<R> v, Spec3<R> f, Spec3w<R> o, const double *__restrict__ tve,
                                  const double *__restrict__ tvh, int ntve, size_t total) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(p % kp.nz), j = (int)((p / kp.nz) % kp.ny), i = (int)(p / ((size_t)kp.nz * kp.ny));
    const R kn2 = kn2_of(kp, i, j, k);
    R nut = 0, kk2 = 0, nuh = 0;
    if (kn2 <= kp.kmax && kn2 >= kp.tiny) {
      kk2 = kk2_of(kp, i, j, k);
      const int ki = (int)(sqrt(kk2) + (R)0.501f);
      const bool in = ki >= 1 && ki <= ntve;
      nut = in ? (R)tve[ki - 1] : (R)0;
      nuh = (in && tvh) ? (R)tvh[ki - 1] : (R)0;
    }
    const cx<R> vx = v.p[0][p], vy = v.p[1][p], vz = v.p[2][p];
    cx<R> w[3] = {};
    if (nuh != (R)0) {
      const R kx = kx_of(kp, i), ky = ky_of(kp, j), kz = kz_of(kp, k);
      w[0] = mk((-ky * vz.y) - (-kz * vy.y), (ky * vz.x) - (kz * vy.x));
      w[1] = mk((-kz * vx.y) - (-kx * vz.y), (kz * vx.x) - (kx * vz.x));
      w[2] = mk((-kx * vy.y) - (-ky * vx.y), (kx * vy.x) - (ky * vx.x));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const cx<R> u = a == 0 ? vx : (a == 1 ? vy : vz);
      cx<R> r;
      r.x = -(nut * kk2) * u.x;
      r.y = -(nut * kk2) * u.y;
      if (nuh != (R)0) {
        r.x += nuh * w[a].x;
        r.y += nuh * w[a].y;
      }
      if (f.p[a]) {
        r.x += f.p[a][p].x;
        r.y += f.p[a][p].y;
      }
      o.p[a][p] = r;
    }
  }
}

// ---------------------------------------------------------------------
// The spectral network's inputs, one row per resolved shell k = 1..kc (row
// k-1), from the kinetic spectrum E (spectrumc's kin = 1 sums, E[k-1] the
// shell k); non-positive shell energies count as 1e-30 of the resolved sum:
//   x0 = k/kc, x1 = (k/kc)^2, x2 = ln(E(k)/E(kc)) / 8,
//   x3 = d ln E / d ln k at k (centred; one-sided at k = 1 and k = kc) / 4,
//   x4 = the log-slope from kc/2 to kc / 4,
//   x5 = ln(kc E(kc) / sum_{k<=kc} E(k)) / 8,
//   x6 = exp(-(kc - k)/2), x7 = exp(-(kc - k)/8), x8 = x9 = 0.
// Every thread forms the resolved sum itself, in shell order.
__device__ inline double spec_e(const double *E, int k, double floor_) { return fmax(E[k - 1], floor_); }

__global__ void spec_features_kernel(const double *__restrict__ E, int kc, float *__restrict__ x) {
  double tot = 0.0;
  for (int k = 1; k <= kc; ++k) tot += fmax(E[k - 1], 0.0);
  const double fl = 1e-30 * fmax(tot, 1e-300);
  const double ec = spec_e(E, kc, fl);
  const int kh = kc / 2 > 1 ? kc / 2 : 1;
  const double slope_c = kh < kc ? log(ec / spec_e(E, kh, fl)) / log((double)kc / (double)kh) : 0.0;
  const double frac = log((double)kc * ec / fmax(tot, fl));
  for (int k = 1 + (int)threadIdx.x; k <= kc; k += (int)blockDim.x) {
    const double r = (double)k / (double)kc;
    const int ka = k > 1 ? k - 1 : k, kb = k < kc ? k + 1 : k;
    const double sl = ka < kb ? log(spec_e(E, kb, fl) / spec_e(E, ka, fl)) / log((double)kb / (double)ka) : 0.0;
    float *row = x + (size_t)(k - 1) * GHOST_MLP_NIN;
    row[0] = (float)r;
    row[1] = (float)(r * r);
    row[2] = (float)(log(spec_e(E, k, fl) / ec) / 8.0);
    row[3] = (float)(sl / 4.0);
    row[4] = (float)(slope_c / 4.0);
    row[5] = (float)(frac / 8.0);
    row[6] = (float)exp(-(double)(kc - k) / 2.0);
    row[7] = (float)exp(-(double)(kc - k) / 8.0);
    row[8] = 0.f;
    row[9] = 0.f;
  }
}

// tve(k) of the spectral network: the first output of row k-1 times
// out_scale sqrt(E(kc)/kc) (Kraichnan's scaling of a spectral eddy
// viscosity at the cutoff) for k <= kc, zero beyond, and never negative: a
// negative eddy viscosity (backscatter) would feed its shell without
// bound once the molecular viscosity is below it
__global__ void spec_tve_kernel(const float *__restrict__ y, const double *__restrict__ E, int kc, int nb,
                                double out_scale, double *__restrict__ tve) {
  const double s = out_scale * sqrt(fmax(E[kc - 1], 0.0) / (double)kc);
  for (int k = 1 + (int)threadIdx.x; k <= nb; k += (int)blockDim.x)
    tve[k - 1] = k <= kc ? fmax((double)y[(size_t)(k - 1) * GHOST_MLP_NOUT] * s, 0.0) : 0.0;
}

// ---------------------------------------------------------------------
// vcorrect (pseudo/pseudospec3D_edqnm.f90:405-1629) with heli = 0, per mode:
// after the eddy-viscous update each resolved mode is rescaled so that its
// energy becomes E = |v|^2 + 2 tepq(km) dt ef / eold(km) while its helicity
// is kept, by rebuilding the amplitudes and relative phases of the
// components.  The seven Fortran routines are the geometries where some
// wavenumber components vanish; the locals are double precision there and
// here.  v = (vxr,vxi,vyr,vyi,vzr,vzi) already divided by n^3.
__device__ static double vc_sgn(double x) { return copysign(1.0, x); }
__device__ static void vc_phase(double r, double im, double eps, double *c, double *s, double *t) {
  const double pi = 3.14159265358979323846;
  *c = r / (sqrt(r * r + im * im) + eps);
  *s = im / (sqrt(r * r + im * im) + eps);
  *t = *s > 0. ? acos(*c) : 2.0 * pi - acos(*c);
}
/* the common energy ratio of the first branches */
__device__ static double vc_ratio(double E, double H, double v2, double w2, double kk2) {
  return (E * sqrt(1. - H * H / (0.25 * kk2 * (E * E)))) / (v2 * sqrt(1. - w2 * w2 / (0.25 * kk2 * (v2 * v2))));
}
/* the three reconstructions of the three-component geometries */
__device__ static void vc_rebuild3(double *v, double mx, double my, double mz, double cx, double sx, double cy, double sy,
                       double cz, double sz, double cxy, double sxy, double czx, double szx, double cyz, double syz,
                       int bx, int by, int bz) {
  double tmp;
  if (bx) {
    v[0] = mx * cx; v[1] = mx * sx;
    tmp = my / mx; v[2] = tmp * (cxy * v[0] - sxy * v[1]); v[3] = tmp * (sxy * v[0] + cxy * v[1]);
    tmp = mz / mx; v[4] = tmp * (szx * v[1] + czx * v[0]); v[5] = tmp * (czx * v[1] - szx * v[0]);
  }
  if (by) {
    v[2] = my * cy; v[3] = my * sy;
    tmp = mx / my; v[0] = tmp * (cxy * v[2] + sxy * v[3]); v[1] = tmp * (-sxy * v[2] + cxy * v[3]);
    tmp = mz / my; v[4] = tmp * (-syz * v[3] + cyz * v[2]); v[5] = tmp * (cyz * v[3] + syz * v[2]);
  }
  if (bz) {
    v[4] = mz * cz; v[5] = mz * sz;
    tmp = mx / mz; v[0] = tmp * (-szx * v[5] + czx * v[4]); v[1] = tmp * (szx * v[4] + czx * v[5]);
    tmp = my / mz; v[2] = tmp * (cyz * v[4] + syz * v[5]); v[3] = tmp * (-syz * v[4] + cyz * v[5]);
  }
}

__device__ static void vc_vcorr_general(double kx, double ky, double kz, double kk2, double E, double H, double v2, double w2,
                            double cx, double sx, double cy, double sy, double cz, double sz, double txy, double tzx,
                            double tyz, double *v);

/* One mode.  zx/zy/zz: the wavenumber component is zero (index 1 in the
 * Fortran).  kx..kz and kk2 are the GP tables; E and H as above. */
__device__ static void vc_vcorr_mode(int zx, int zy, int zz, double kx, double ky, double kz, double kk2, double E, double dH,
                         double tinyf, double *v) {
  const double kx2 = kx * kx, ky2 = ky * ky, kz2 = kz * kz;
  double cx, sx, tx, cy, sy, ty, cz, sz, tz;
  if (!zx && !zy && !zz) {  /* vcorr_xnynzn: vz from the divergence */
    v[4] = (-kx * v[0] - ky * v[2]) / kz;
    v[5] = (-kx * v[1] - ky * v[3]) / kz;
  } else if (zx && zy) {
    v[4] = v[5] = 0.;        /* vcorr_x0y0zn */
  } else if (zx && zz) {
    v[2] = v[3] = 0.;        /* vcorr_x0ynz0 */
  } else if (zy && zz) {
    v[0] = v[1] = 0.;        /* vcorr_xny0z0 */
  }
  const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3] + v[4] * v[4] + v[5] * v[5];
  const double w2 = kz * (v[0] * v[3] - v[1] * v[2]) + ky * (v[4] * v[1] - v[5] * v[0]) + kx * (v[2] * v[5] - v[3] * v[4]);
  // heli = 1 targets H = w2 + thpq(km) dt hf / hold(km) (:536-540): dH
  const double H = w2 + dH;
  const double eps = (!zx && !zy && zz) ? tinyf : 0.;  /* only vcorr_xnynz0 pads the moduli */
  if (zx && zy) {            /* x, y only; kz != 0 */
    vc_phase(v[0], v[1], 0., &cx, &sx, &tx);
    vc_phase(v[2], v[3], 0., &cy, &sy, &ty);
    const double txy = ty - tx, tmp = vc_ratio(E, H, v2, w2, kk2);
    const double vx2 = tmp * (v[0] * v[0] + v[1] * v[1] - 0.5 * v2) + 0.5 * E;
    const double vy2 = tmp * (v[2] * v[2] + v[3] * v[3] - 0.5 * v2) + 0.5 * E;
    const double mx = sqrt(fabs(vx2)), my = sqrt(fabs(vy2));
    double sxy = H;
    const double dsxy = kz * mx * my;
    if (vc_sgn(vx2) >= 0. && vc_sgn(vy2) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0.) {
      sxy = sxy / dsxy;
      double cxy = sqrt(1. - sxy * sxy);
      if (cos(txy) < 0.) cxy = -cxy;
      if (mx >= my) {
        v[0] = mx * cx; v[1] = mx * sx;
        const double t2 = my / mx;
        v[2] = t2 * (cxy * v[0] - sxy * v[1]); v[3] = t2 * (sxy * v[0] + cxy * v[1]);
      } else {
        v[2] = my * cy; v[3] = my * sy;
        const double t2 = mx / my;
        v[0] = t2 * (cxy * v[2] + sxy * v[3]); v[1] = t2 * (-sxy * v[2] + cxy * v[3]);
      }
    }
  } else if (zx && zz) {     /* x, z only; ky != 0 */
    vc_phase(v[0], v[1], 0., &cx, &sx, &tx);
    vc_phase(v[4], v[5], 0., &cz, &sz, &tz);
    const double tzx = tx - tz, tmp = vc_ratio(E, H, v2, w2, kk2);
    const double vx2 = tmp * (v[0] * v[0] + v[1] * v[1] - 0.5 * v2) + 0.5 * E;
    const double vz2 = tmp * (v[4] * v[4] + v[5] * v[5] - 0.5 * v2) + 0.5 * E;
    const double mx = sqrt(fabs(vx2)), mz = sqrt(fabs(vz2));
    double szx = H;
    const double dszx = ky * mx * mz;
    if (vc_sgn(vx2) >= 0. && vc_sgn(vz2) >= 0. && fabs(szx) <= fabs(dszx) && dszx != 0.) {
      szx = szx / dszx;
      double czx = sqrt(1. - szx * szx);
      if (cos(tzx) < 0.) czx = -czx;
      if (mx >= mz) {
        v[0] = mx * cx; v[1] = mx * sx;
        const double t2 = mz / mx;
        v[4] = t2 * (szx * v[1] + czx * v[0]); v[5] = t2 * (czx * v[1] - szx * v[0]);
      } else {
        v[4] = mz * cz; v[5] = mz * sz;
        const double t2 = mx / mz;
        v[0] = t2 * (-szx * v[5] + czx * v[4]); v[1] = t2 * (szx * v[4] + czx * v[5]);
      }
    }
  } else if (zy && zz) {     /* y, z only; kx != 0 */
    vc_phase(v[2], v[3], 0., &cy, &sy, &ty);
    vc_phase(v[4], v[5], 0., &cz, &sz, &tz);
    const double tyz = tz - ty, tmp = vc_ratio(E, H, v2, w2, kk2);
    const double vy2 = tmp * (v[2] * v[2] + v[3] * v[3] - 0.5 * v2) + 0.5 * E;
    const double vz2 = tmp * (v[4] * v[4] + v[5] * v[5] - 0.5 * v2) + 0.5 * E;
    const double my = sqrt(fabs(vy2)), mz = sqrt(fabs(vz2));
    double syz = H;
    const double dsyz = kx * mz * my;
    if (vc_sgn(vy2) >= 0. && vc_sgn(vz2) >= 0. && fabs(syz) <= fabs(dsyz) && dsyz != 0.) {
      syz = syz / dsyz;
      double cyz = sqrt(1. - syz * syz);
      if (cos(tyz) < 0.) cyz = -cyz;
      if (my >= mz) {
        v[2] = my * cy; v[3] = my * sy;
        const double t2 = mz / my;
        v[4] = t2 * (-syz * v[3] + cyz * v[2]); v[5] = t2 * (cyz * v[3] + syz * v[2]);
      } else {
        v[4] = mz * cz; v[5] = mz * sz;
        const double t2 = my / mz;
        v[2] = t2 * (cyz * v[4] + syz * v[5]); v[3] = t2 * (-syz * v[4] + cyz * v[5]);
      }
    }
  } else {                   /* three components */
    vc_phase(v[0], v[1], eps, &cx, &sx, &tx);
    vc_phase(v[2], v[3], eps, &cy, &sy, &ty);
    vc_phase(v[4], v[5], eps, &cz, &sz, &tz);
    const double txy = ty - tx, tzx = tx - tz, tyz = tz - ty;
    if (zx || zy || zz) {
      /* one vanishing component of k (vcorr_x0ynzn, vcorr_xny0zn, vcorr_xnynz0):
       * the mode along that axis takes its share of E, the other two split
       * the rest in proportion to the other axes' k^2 */
      const double tmp0 = vc_ratio(E, H, v2, w2, kk2);
      double ma, mb, mc, tmp3, t1;
      if (zx) {
        const double vx2 = tmp0 * (v[0] * v[0] + v[1] * v[1] - 0.5 * v2) + 0.5 * E;
        t1 = vc_sgn(vx2); ma = sqrt(fabs(vx2)); tmp3 = E - vx2;
        const double tt = 1. / (ky2 + kz2);
        mb = sqrt(fabs(tmp3) * kz2 * tt); mc = sqrt(fabs(tmp3) * ky2 * tt);  /* my, mz */
        const double mx = ma, my = mb, mz = mc;
        double sxy = kz * H, szx = ky * H;
        const double dsxy = (ky2 + kz2) * mx * my, dszx = (ky2 + kz2) * mx * mz;
        if (t1 >= 0. && vc_sgn(tmp3) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. && fabs(szx) <= fabs(dszx) &&
            dszx != 0.) {
          sxy = sxy / dsxy; szx = szx / dszx;
          double cxy = sqrt(1. - sxy * sxy), czx = sqrt(1. - szx * szx);
          if (cos(txy) < 0.) cxy = -cxy;
          if (cos(tzx) < 0.) czx = -czx;
          const double syz = -szx * cxy - sxy * czx, cyz = czx * cxy - szx * sxy;
          vc_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                     my >= mx && my >= mz, mz >= mx && mz >= my);
        }
      } else if (zy) {
        const double vy2 = tmp0 * (v[2] * v[2] + v[3] * v[3] - 0.5 * v2) + 0.5 * E;
        t1 = vc_sgn(vy2); mb = sqrt(vy2); tmp3 = E - vy2;
        const double tt = 1. / (kx2 + kz2);
        ma = sqrt(fabs(tmp3) * kz2 * tt); mc = sqrt(fabs(tmp3) * kx2 * tt);
        const double mx = ma, my = mb, mz = mc;
        double sxy = kz * H, syz = kx * H;
        const double dsxy = (kx2 + kz2) * mx * my, dsyz = (kx2 + kz2) * my * mz;
        if (t1 >= 0. && vc_sgn(tmp3) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. && fabs(syz) <= fabs(dsyz) &&
            dsyz != 0.) {
          sxy = sxy / dsxy; syz = syz / dsyz;
          double cxy = sqrt(1. - sxy * sxy), cyz = sqrt(1. - syz * syz);
          if (cos(txy) < 0.) cxy = -cxy;
          if (cos(tyz) < 0.) cyz = -cyz;
          const double szx = -sxy * cyz - syz * cxy, czx = cxy * cyz - sxy * syz;
          vc_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                     my >= mx && my >= mz, mz >= mx && mz >= my);
        }
      } else {
        const double vz2 = tmp0 * ((v[4] * v[4] + v[5] * v[5]) - 0.5 * v2) + 0.5 * E;
        t1 = vc_sgn(vz2); mc = sqrt(fabs(vz2)); tmp3 = E - vz2;
        const double tt = 1. / (kx2 + ky2);
        ma = sqrt(fabs(tmp3) * ky2 * tt); mb = sqrt(fabs(tmp3) * kx2 * tt);
        const double mx = ma, my = mb, mz = mc;
        double szx = ky * H, syz = kx * H;
        const double dszx = (kx2 + ky2) * mx * mz, dsyz = (kx2 + ky2) * my * mz;
        if (t1 >= 0. && vc_sgn(tmp3) >= 0. && fabs(szx) <= fabs(dszx) && dszx != 0. && fabs(syz) <= fabs(dsyz) &&
            dsyz != 0.) {
          szx = szx / dszx; syz = syz / dsyz;
          double czx = sqrt(1. - szx * szx), cyz = sqrt(1. - syz * syz);
          if (cos(tzx) < 0.) czx = -czx;
          if (cos(tyz) < 0.) cyz = -cyz;
          const double sxy = -syz * czx - szx * cyz, cxy = cyz * czx - syz * szx;
          vc_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                     my >= mx && my >= mz, mz >= mx && mz >= my);
        }
      }
    } else {
      vc_vcorr_general(kx, ky, kz, kk2, E, H, v2, w2, cx, sx, cy, sy, cz, sz, txy, tzx, tyz, v);
    }
  }
}

// vcorr_xnynzn (:1377-1629): all components of k non-zero
__device__ static void vc_vcorr_general(double kx, double ky, double kz, double kk2, double E, double H, double v2, double w2,
                            double cx, double sx, double cy, double sy, double cz, double sz, double txy, double tzx,
                            double tyz, double *v) {
  const double kx2 = kx * kx, ky2 = ky * ky, kz2 = kz * kz;
  const double fx = 1. - kx2 / kk2, fy = 1. - ky2 / kk2, fz = 1. - kz2 / kk2;
  const double tmq = vc_ratio(E, H, v2, w2, kk2);
  double vx2 = tmq * (v[0] * v[0] + v[1] * v[1] - fx * 0.5 * v2) + fx * 0.5 * E;
  const double vy2 = tmq * (v[2] * v[2] + v[3] * v[3] - fy * 0.5 * v2) + fy * 0.5 * E;
  const double vz2 = tmq * (v[4] * v[4] + v[5] * v[5] - fz * 0.5 * v2) + fz * 0.5 * E;
  double mx = sqrt(fabs(vx2)), my = sqrt(fabs(vy2)), mz = sqrt(fabs(vz2));
  double szx = H * ky, dszx = kk2 * mx * mz, sxy = H * kz, dsxy = kk2 * my * mx, syz = H * kx, dsyz = kk2 * my * mz;
  double czx = (ky2 * E - mx * mx * (kx2 + ky2) - mz * mz * (ky2 + kz2)), dczx = 2. * kx * kz * mx * mz;
  double cxy = (kz2 * E - mx * mx * (kx2 + kz2) - my * my * (ky2 + kz2)), dcxy = 2. * kx * ky * mx * my;
  double cyz = (kx2 * E - my * my * (kx2 + ky2) - mz * mz * (kx2 + kz2)), dcyz = 2. * ky * kz * my * mz;
  if (vc_sgn(vx2) >= 0. && vc_sgn(vy2) >= 0. && vc_sgn(vz2) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. &&
      fabs(szx) <= fabs(dszx) && dszx != 0. && fabs(syz) <= fabs(dsyz) && dsyz != 0. && fabs(cxy) <= fabs(dcxy) &&
      dcxy != 0. && fabs(cyz) <= fabs(dcyz) && dcyz != 0. && fabs(czx) <= fabs(dczx) && dczx != 0.) {
    szx /= dszx; sxy /= dsxy; syz /= dsyz; czx /= dczx; cxy /= dcxy; cyz /= dcyz;
    vc_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
               my > mx && my >= mz, mz > mx && mz > my);
  } else {
    const double hh = sqrt(1. - H * H / (0.25 * (E * E) * kk2));
    const double hi = fx * 0.5 * E * (1. + hh), lo = fx * 0.5 * E * (1. - hh);
    if (vx2 > hi) vx2 = hi;
    if (vx2 < lo) vx2 = lo;
    const double t1 = vc_sgn(vx2);
    mx = sqrt(fabs(vx2));
    const double a2 = 2. * ((ky2 + kz2) * (ky2 + kz2)), iq = 1. / a2;
    double tmp4 = kx2 * ky2 * kz2 *
                  (-((mx * mx) * (mx * mx)) * kk2 + mx * mx * (ky2 + kz2) * E -
                   H * H * ((ky2 + kz2) * (ky2 + kz2)) / (kk2 * kk2));
    const double t0 = vc_sgn(tmp4), delta = 4. * sqrt(fabs(tmp4)) * iq;
    tmp4 = (-vx2 * (2. * (kx2 + kz2) * (ky2 + kz2) - 4. * kx2 * ky2) + 2. * kz2 * E * (ky2 + kz2)) * iq + delta;
    const double t2 = vc_sgn(tmp4);
    my = sqrt(fabs(tmp4));
    tmp4 = (-vx2 * (2. * (kx2 + ky2) * (ky2 + kz2) - 4. * kx2 * kz2) + 2. * ky2 * E * (ky2 + kz2)) * iq - delta;
    const double t3 = vc_sgn(tmp4);
    mz = sqrt(fabs(tmp4));
    szx = H * ky; dszx = kk2 * mx * mz; sxy = H * kz; dsxy = kk2 * my * mx; syz = H * kx; dsyz = kk2 * my * mz;
    czx = (ky2 * E - mx * mx * (kx2 + ky2) - mz * mz * (ky2 + kz2)); dczx = 2. * kx * kz * mx * mz;
    cxy = (kz2 * E - mx * mx * (kx2 + kz2) - my * my * (ky2 + kz2)); dcxy = 2. * kx * ky * mx * my;
    cyz = (kx2 * E - my * my * (kx2 + ky2) - mz * mz * (kx2 + kz2)); dcyz = 2. * ky * kz * my * mz;
    if (t0 >= 0. && t1 >= 0. && t2 >= 0. && t3 >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. &&
        fabs(szx) <= fabs(dszx) && dszx != 0. && fabs(syz) <= fabs(dsyz) && dsyz != 0. && fabs(czx) <= fabs(dczx) &&
        dczx != 0. && fabs(cxy) <= fabs(dcxy) && dcxy != 0. && fabs(cyz) <= fabs(dcyz) && dcyz != 0.) {
      szx /= dszx; sxy /= dsxy; syz /= dsyz; czx /= dczx; cxy /= dcxy; cyz /= dcyz;
      vc_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                 my >= mx && my >= mz, mz >= mx && mz >= my);
    }
  }
  (void)txy; (void)tzx; (void)tyz;
}


// Eden of include/edqnmhd_rkstep2.f90:8-10: (|vx|^2+|vy|^2+|vz|^2)/n^6 per
// mode; with hf (heli = 1) also Hden of :11-17, 2/n^6 times
// kz (Re vx Im vy - Re vy Im vx) + ky (Re vz Im vx - Re vx Im vz)
// + kx (Re vy Im vz - Re vz Im vy)
template <typename R>
__global__ void eden_kernel(KParams<R> kp, Spec3<R> v, R *__restrict__ ef, R *__restrict__ hf, size_t total, R rmp) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const cx<R> a = v.p[0][p], b = v.p[1][p], c = v.p[2][p];
    ef[p] = (a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y + c.x * c.x + c.y * c.y) * rmp;
    if (hf) {
      const int k = (int)(p % kp.nz), j = (int)((p / kp.nz) % kp.ny), i = (int)(p / ((size_t)kp.nz * kp.ny));
      const R t1 = kz_of(kp, k) * (a.x * b.y - b.x * a.y);
      const R t2 = ky_of(kp, j) * (c.x * a.y - a.x * c.y);
      const R t3 = kx_of(kp, i) * (b.x * c.y - c.x * b.y);
      hf[p] = (R)2 * rmp * (t1 + t2 + t3);
    }
  }
}

// vcorrect over every resolved mode but the origin: tepq and eold are the
// shell arrays of the substep's start (1-based shells stored at k-1), ef its
// Eden, dt the substep's dt/o
// heli = 1 also reads hf (Hden of the substep's start), thpq and hold.
template <typename R>
__global__ void vcorrect_kernel(KParams<R> kp, Spec3w<R> v, const R *__restrict__ ef, const double *__restrict__ tepq,
                                const double *__restrict__ eold, const R *__restrict__ hf,
                                const double *__restrict__ thpq, const double *__restrict__ hold, int hel, int nshell,
                                R dt, R tinyf, R norm, size_t total) {
  const double inorm = 1. / (double)norm;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(p % kp.nz), j = (int)((p / kp.nz) % kp.ny), i = (int)(p / ((size_t)kp.nz * kp.ny));
    if (i == 0 && j == 0 && k == 0) continue;
    if (kn2_of(kp, i, j, k) > kp.kmax) continue;
    const R kk2 = kk2_of(kp, i, j, k);
    const int km = (int)(sqrt(kk2) + (R)0.501f);
    if (km < 1 || km > nshell) continue;
    const cx<R> a = v.p[0][p], b = v.p[1][p], c = v.p[2][p];
    double w[6] = {(double)a.x * inorm, (double)a.y * inorm, (double)b.x * inorm,
                   (double)b.y * inorm, (double)c.x * inorm, (double)c.y * inorm};
    const int zx = i == 0, zy = j == 0, zz = k == 0;
    const double kxv = (double)kx_of(kp, i), kyv = (double)ky_of(kp, j), kzv = (double)kz_of(kp, k);
    double u[6] = {w[0], w[1], w[2], w[3], w[4], w[5]};
    if (!zx && !zy && !zz) {
      u[4] = (-kxv * u[0] - kyv * u[2]) / kzv;
      u[5] = (-kxv * u[1] - kyv * u[3]) / kzv;
    } else if (zx && zy) {
      u[4] = u[5] = 0.;
    } else if (zx && zz) {
      u[2] = u[3] = 0.;
    } else if (zy && zz) {
      u[0] = u[1] = 0.;
    }
    const double v2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2] + u[3] * u[3] + u[4] * u[4] + u[5] * u[5];
    const double E = v2 + 2.0 * tepq[km - 1] * (double)dt * (double)ef[p] / eold[km - 1];
    const double dH = hel == 1 ? thpq[km - 1] * (double)dt * (double)hf[p] / hold[km - 1] : 0.0;
    vc_vcorr_mode(zx, zy, zz, kxv, kyv, kzv, (double)kk2, E, dH, (double)tinyf, w);
    cx<R> o;
    o.x = (R)w[0] * norm; o.y = (R)w[1] * norm; v.p[0][p] = o;
    o.x = (R)w[2] * norm; o.y = (R)w[3] * norm; v.p[1][p] = o;
    o.x = (R)w[4] * norm; o.y = (R)w[5] * norm; v.p[2][p] = o;
  }
}

static int blocks(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

// ---------------------------------------------------------------------
// EDQNM eddy viscosity, pseudo/pseudospec3D_edqnm.f90.  R is GHOST's GP
// kind: the spectra are DOUBLE PRECISION, the fit and the quadrature locals
// are REAL(GP), and the literals 0.218 and real(k*k) are default
// (single-precision) reals, as in the Fortran.  The same functions run on
// the host (ghost_evedqnm) and in one device block (the LES closure), so
// the closure needs no host round trip.
__host__ __device__ inline float mlog(float x) { return logf(x); }
__host__ __device__ inline double mlog(double x) { return log(x); }
__host__ __device__ inline float mexp(float x) { return expf(x); }
__host__ __device__ inline double mexp(double x) { return exp(x); }
__host__ __device__ inline float mpow(float x, float y) { return powf(x, y); }
__host__ __device__ inline double mpow(double x, double y) { return pow(x, y); }
__host__ __device__ inline float msqrt(float x) { return sqrtf(x); }
__host__ __device__ inline double msqrt(double x) { return sqrt(x); }

// spec_fit (pseudospec3D_edqnm.f90:278-402): log-linear fit of Ein over
// shells kinf..kc and extrapolation to 3 kc.  Arrays are 0-based copies of
// GHOST's 1-based ones (Efit[k-1] = Efit(k)).
template <typename R>
__host__ __device__ void spec_fit(int n, R kmax, const double *Ein, R delk, double *Efit, R *power_out,
                                  R *ddelta_out) {
  const R tinyf = (R)1e-15 < (R)0.1 / ((R)n * (R)n) ? (R)1e-15 : (R)0.1 / ((R)n * (R)n);
  const int kc = (int)msqrt(kmax);
  const int ktot = 3 * kc, ksup = kc;
  const int kinf = (int)((R)kc - delk);
  const int nfit = 3 * (n / 2 + 1);
  R power = -1, ddelta = -1;
  for (int k = 0; k < nfit; ++k) Efit[k] = 0;
  *power_out = power;
  *ddelta_out = ddelta;
  if (Ein[ksup - 1] <= (double)tinyf) return;
  R x = 0, y = 0, z = 0, v = 0, w = 0, m = 0, nn = 0, o = 0, p = 0, expo = 0;
  for (int i = kinf; i <= ksup; ++i) {
    const R ii = (R)i, li = mlog(ii);
    const R le = (R)mlog(Ein[i - 1] + (double)tinyf);
    x = x + (R)1;
    y = y + li;
    z = z + le;
    v = v + li * le;
    w = w + li * li;
    m = m + ii;
    nn = nn + ii * li;
    o = o + ii * le;
    p = p + ii * ii;
  }
  R pden = (w * p - nn * nn) * (x * nn - y * m) - (y * nn - w * m) * (y * p - m * nn);
  R pnum = ((z * nn - v * m) * (y * p - m * nn) - (v * p - o * nn) * (x * nn - y * m));
  R dden = x * nn - y * m;
  if (pden != 0 && dden != 0) {
    power = pnum / pden;
    expo = ((z * nn - v * m) - power * (w * m - y * nn)) / dden;
    ddelta = expo * x / m - power * y / m - z / m;
  }
  if (power >= 0 && ddelta >= 0) {
    expo = mexp(expo);
    for (int k = 1; k <= ksup; ++k) Efit[k - 1] = Ein[k - 1];
    for (int k = ksup + 1; k <= ktot; ++k) {
      const R kk = (R)k;
      Efit[k - 1] = (double)(expo * mpow(kk, -power) * mexp(-ddelta * kk));
    }
  } else {
    x = y = z = v = w = 0;
    for (int i = kinf; i <= ksup; ++i) {
      const R ii = (R)i, li = mlog(ii);
      const R le = (R)mlog(Ein[i - 1] + (double)tinyf);
      x = x + (R)1;
      y = y + li;
      z = z + le;
      v = v + li * le;
      w = w + li * li;
    }
    pden = y * y - w * x;
    pnum = (v * x - y * z);
    dden = x * y;
    if (pden != 0 && dden != 0) {
      power = pnum / pden;
      expo = mexp((y * z + power * y * y) / dden);
      for (int k = 1; k <= ksup; ++k) Efit[k - 1] = Ein[k - 1];
      for (int k = ksup + 1; k <= ktot; ++k) {
        const R kk = (R)k;
        Efit[k - 1] = (double)(expo * mpow(kk, -power) + tinyf);
      }
    } else {
      for (int k = 1; k <= ksup; ++k) Efit[k - 1] = Ein[k - 1];
    }
  }
  *power_out = power;
  *ddelta_out = ddelta;
}

// cusp (pseudospec3D_edqnm.f90:95-171), split in two: the damping rates
// mu(k) = lambda sqrt(sum_{q<=k} q^2 Ext(q)) for k = 1..3kc (mu[k], 1-based,
// false when Ext(kc+1) = 0 and cusp returns at once), and the quadrature
// over p, q for one k, which gives nut(k) and tepq(k) (arrays zeroed before).
template <typename R>
__host__ __device__ bool cusp_mu(R kmax, R kolmo, const double *Ext, R *mu) {
  const R lambda = (R)0.218f * mpow(kolmo, (R)1.5);
  const int kc = (int)msqrt(kmax);
  const int ktot = 3 * kc;
  if (Ext[kc] == 0.0) return false;  // Ext(kc+1)
  R en = 0;
  mu[0] = 0;
  for (int k = 1; k <= ktot; ++k) {
    const R tmp = (R)(float)(k * k);
    en = (R)((double)en + (double)tmp * Ext[k - 1]);
    mu[k] = lambda * msqrt(en);
  }
  return true;
}

// The quadrature of cusp for one (k, p): the sums over q of the terms that
// GHOST subtracts from nut(k) and adds to tepq(k) (loop body of :139-166).
template <typename R>
__host__ __device__ void cusp_kp(int k, int p, const double *Ext, const R *mu, R nu, R t0, double *dnut,
                                 double *dtepq) {
  const R kk = (R)k, pp = (R)p, ppi = (R)1 / pp;
  double sn = 0.0, st = 0.0;
  for (int q = p - k; q <= p; ++q) {
    if (q == 0) continue;
    const R qq = (R)q, qqi = (R)1 / qq;
    R coeff = (R)0.5;
    if ((qq - (R)0.5) >= (pp - kk) && (qq + (R)0.5) <= pp) coeff = (R)1;
    const R x = (pp * pp + qq * qq - kk * kk) / ((R)2 * pp * qq);
    const R y = (kk * kk + qq * qq - pp * pp) / ((R)2 * kk * qq);
    const R z = (pp * pp + kk * kk - qq * qq) / ((R)2 * pp * kk);
    const R tvvkp = (R)((double)(-qqi * (x * y + z * z * z) * (pp * pp)) * Ext[q - 1] * Ext[k - 1]);
    const R tvvkpsym = (R)((double)(-ppi * (x * z + y * y * y) * (qq * qq)) * Ext[p - 1] * Ext[k - 1]);
    const R tmp = mu[k] + mu[p] + mu[q] + nu * (kk * kk + pp * pp + qq * qq);
    const R frac = (R)1 / tmp;
    const R theta = -mexp(-tmp * t0) / tmp;
    sn += (double)(coeff * (frac + theta)) * (double)(tvvkp + tvvkpsym) / ((double)((R)2 * kk * kk) * Ext[k - 1]);
    st += (double)(coeff * (frac + theta)) * (double)(tvvkp + tvvkpsym);
  }
  *dnut = sn;
  *dtepq = st;
}

// The quadrature of full_cusp (pseudospec3D_edqnm.f90:174-277) for one
// (k, p), on the halved extrapolations: the sums over q of the terms GHOST
// subtracts from nut(k) (out[0]) and adds to tepq(k), tvh(k), thpq(k)
// (out[1..3]).  Every GP product is rounded to GP before it meets a double
// spectrum value, in GHOST's left-to-right order.
template <typename R>
__host__ __device__ void full_cusp_kp(int k, int p, const double *Ext, const double *Hxt, const R *mu, R nu, R t0,
                                      double *out) {
  const R kk = (R)k, pp = (R)p, ppi = (R)1 / pp;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const double Ek = Ext[k - 1], Ep = Ext[p - 1], Hk = Hxt[k - 1], Hp = Hxt[p - 1];
  for (int q = p - k; q <= p; ++q) {
    if (q == 0) continue;
    const R qq = (R)q, qqi = (R)1 / qq;
    R coeff = (R)0.5;
    if ((qq - (R)0.5) >= (pp - kk) && (qq + (R)0.5) <= pp) coeff = (R)1;
    const R x = (pp * pp + qq * qq - kk * kk) / ((R)2 * pp * qq);
    const R y = (kk * kk + qq * qq - pp * pp) / ((R)2 * kk * qq);
    const R z = (pp * pp + kk * kk - qq * qq) / ((R)2 * pp * kk);
    const R xyz = x * y + z * z * z, xzy = x * z + y * y * y;
    const R ym1 = (R)1 - y * y, zm1 = (R)1 - z * z;
    const double Eq = Ext[q - 1], Hq = Hxt[q - 1];
    const R tvvkp = (R)((double)(-(qqi * xyz * (pp * pp))) * Eq * Ek);
    const R tvvpq = (R)((double)(qqi * xyz * (kk * kk)) * Eq * Ep);
    const R tvvkpsym = (R)((double)(-(ppi * xzy * (qq * qq))) * Ep * Ek);
    const R tvvpqsym = (R)((double)(ppi * xzy * (kk * kk)) * Eq * Ep);
    const R twwpq = (R)((double)(-(z * ym1 * kk * kk)) * Hp * Hq / (double)(pp * pp * qq));
    const R twwkp = (R)((double)(z * ym1) * Hk * Hq * (double)qqi);
    const R twwpqsym = (R)((double)(-(y * zm1 * kk * kk)) * Hp * Hq / (double)(pp * qq * qq));
    const R twwkpsym = (R)((double)(y * zm1) * Hk * Hp * (double)ppi);
    const R tvw = (R)((double)(qqi * xyz * kk * kk) * Eq * Hp + (double)(ppi * xzy * kk * kk) * Hq * Ep -
                      (double)(qqi * z * ym1 * kk * kk) * Ep * Hq - (double)(ppi * y * zm1 * kk * kk) * Eq * Hp);
    const R tmp = mu[k] + mu[p] + mu[q] + nu * (kk * kk + pp * pp + qq * qq);
    const R theta = ((R)1 - mexp(-tmp * t0)) / tmp;
    const R ct = coeff * theta;
    s0 += (double)(ct * (tvvkp + tvvkpsym)) / ((double)((R)2 * kk * kk) * Ek);
    s1 += (double)(ct * (tvvpq + tvvpqsym + twwpq + twwpqsym));
    s2 += (double)(ct * (twwkp + twwkpsym)) / (2.0 * Hk);
    s3 += (double)(ct * tvw);
  }
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
  out[3] = s3;
}

// full_cusp's halving of the extrapolated spectra (:212-215) and its mu
// from the halved Ext; false when Ext(kc+1) = 0 (full_cusp returns first).
template <typename R>
__host__ __device__ bool full_cusp_prep(R kmax, R kolmo, double *Ext, double *Hxt, R *mu) {
  const int kc = (int)msqrt(kmax), ktot = 3 * kc;
  if (Ext[kc] == 0.0) return false;
  for (int k = 1; k <= ktot; ++k) {
    Ext[k - 1] = 0.5 * Ext[k - 1];
    Hxt[k - 1] = 0.5 * Hxt[k - 1];
  }
  return cusp_mu<R>(kmax, kolmo, Ext, mu);
}

// evedqnm with hel = 0 (pseudospec3D_edqnm.f90:24-92), host: the partial
// sums of each p are added in p order
template <typename R>
static void evedqnm(int n, R kmax, R kolmo, const double *Eold, R nu, R time, double *tepq, double *tve,
                    double *Ext) {
  const int kc = (int)msqrt(kmax);
  const R delk = (R)3 * (R)kc / (R)4;
  for (int k = 0; k < n / 2 + 1; ++k) tve[k] = tepq[k] = 0;
  R power, ddelta;
  spec_fit<R>(n, kmax, Eold, delk, Ext, &power, &ddelta);
  if (!(power > 0)) return;
  std::vector<R> mu(3 * kc + 1);
  if (!cusp_mu<R>(kmax, kolmo, Ext, mu.data())) return;
  for (int k = 1; k <= kc; ++k) {
    double sn = 0.0, st = 0.0;
    for (int p = kc + 1; p <= 3 * kc; ++p) {
      double dn, dt;
      cusp_kp<R>(k, p, Ext, mu.data(), nu, time, &dn, &dt);
      sn += dn;
      st += dt;
    }
    tve[k - 1] = -sn;
    tepq[k - 1] = st;
  }
}

// evedqnm with hel (pseudospec3D_edqnm.f90:24-92), host.  hel = 1 fits E
// over delk - 2 shells and H over delk; full_cusp when both fits have a
// positive index, cusp when only E's does.  thpq, tvh and Hxt may be null
// for hel = 0.
template <typename R>
static void evedqnm_h(int n, R kmax, R kolmo, const double *Eold, const double *Hold, R nu, R time, int hel,
                      double *tepq, double *thpq, double *tve, double *tvh, double *Ext, double *Hxt) {
  if (hel != 1) {
    evedqnm<R>(n, kmax, kolmo, Eold, nu, time, tepq, tve, Ext);
    for (int k = 0; k < n / 2 + 1; ++k) {
      if (thpq) thpq[k] = 0;
      if (tvh) tvh[k] = 0;
    }
    return;
  }
  const int kc = (int)msqrt(kmax);
  const R delk = (R)3 * (R)kc / (R)4;
  for (int k = 0; k < n / 2 + 1; ++k) tve[k] = tepq[k] = thpq[k] = tvh[k] = 0;
  R power, ddelta, hpower, hddelta;
  spec_fit<R>(n, kmax, Eold, delk - (R)2, Ext, &power, &ddelta);
  spec_fit<R>(n, kmax, Hold, delk, Hxt, &hpower, &hddelta);
  if (!(power > 0)) return;
  std::vector<R> mu(3 * kc + 1);
  if (hpower > 0) {
    if (!full_cusp_prep<R>(kmax, kolmo, Ext, Hxt, mu.data())) return;
    for (int k = 1; k <= kc; ++k) {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int p = kc + 1; p <= 3 * kc; ++p) {
        double d[4];
        full_cusp_kp<R>(k, p, Ext, Hxt, mu.data(), nu, time, d);
        for (int q = 0; q < 4; ++q) acc[q] += d[q];
      }
      tve[k - 1] = -acc[0];
      tepq[k - 1] = acc[1];
      tvh[k - 1] = acc[2];
      thpq[k - 1] = acc[3];
    }
  } else {
    if (!cusp_mu<R>(kmax, kolmo, Ext, mu.data())) return;
    for (int k = 1; k <= kc; ++k) {
      double sn = 0.0, st = 0.0;
      for (int p = kc + 1; p <= 3 * kc; ++p) {
        double dn, dt;
        cusp_kp<R>(k, p, Ext, mu.data(), nu, time, &dn, &dt);
        sn += dn;
        st += dt;
      }
      tve[k - 1] = -sn;
      tepq[k - 1] = st;
    }
  }
}

// Device: one thread fits the spectra and forms mu (go: 0 no closure, 1
// cusp, 2 full_cusp); then one block per shell k, its threads sharing the
// p, partial sums combined in thread order.  Hold, thpq, tvh, Hxt are only
// touched for hel = 1.
template <typename R>
__global__ void __launch_bounds__(128) edqnm_fit_kernel(int n, R kmax, R kolmo, const double *__restrict__ Eold,
                                                        const double *__restrict__ Hold, int hel, double *tepq,
                                                        double *thpq, double *tve, double *tvh, double *Ext,
                                                        double *Hxt, R *mu, int *go) {
  const int nb = n / 2 + 1, kc = (int)msqrt(kmax);
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    tve[k] = tepq[k] = 0;
    if (hel == 1) thpq[k] = tvh[k] = 0;
  }
  if (threadIdx.x == 0) {
    const R delk = (R)3 * (R)kc / (R)4;
    R power, ddelta;
    if (hel == 1) {
      R hpower, hddelta;
      spec_fit<R>(n, kmax, Eold, delk - (R)2, Ext, &power, &ddelta);
      spec_fit<R>(n, kmax, Hold, delk, Hxt, &hpower, &hddelta);
      if (!(power > 0))
        *go = 0;
      else if (hpower > 0)
        *go = full_cusp_prep<R>(kmax, kolmo, Ext, Hxt, mu) ? 2 : 0;
      else
        *go = cusp_mu<R>(kmax, kolmo, Ext, mu) ? 1 : 0;
    } else {
      spec_fit<R>(n, kmax, Eold, delk, Ext, &power, &ddelta);
      *go = (power > 0) && cusp_mu<R>(kmax, kolmo, Ext, mu) ? 1 : 0;
    }
  }
}

template <typename R>
__global__ void __launch_bounds__(128) edqnm_cusp_kernel(R kmax, const double *__restrict__ Ext,
                                                         const double *__restrict__ Hxt, const R *__restrict__ mu,
                                                         R nu, R t0, const int *__restrict__ go, double *tepq,
                                                         double *thpq, double *tve, double *tvh) {
  __shared__ double sh[4][128];
  const int kc = (int)msqrt(kmax), k = blockIdx.x + 1;
  const int g = *go;
  if (k > kc || g == 0) return;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int p = kc + 1 + threadIdx.x; p <= 3 * kc; p += blockDim.x) {
    if (g == 2) {
      double d[4];
      full_cusp_kp<R>(k, p, Ext, Hxt, mu, nu, t0, d);
      for (int q = 0; q < 4; ++q) acc[q] += d[q];
    } else {
      double dn, dt;
      cusp_kp<R>(k, p, Ext, mu, nu, t0, &dn, &dt);
      acc[0] += dn;
      acc[1] += dt;
    }
  }
  for (int q = 0; q < 4; ++q) sh[q][threadIdx.x] = acc[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = 0; t < (int)blockDim.x; ++t)
      for (int q = 0; q < 4; ++q) a[q] += sh[q][t];
    tve[k - 1] = -a[0];
    tepq[k - 1] = a[1];
    if (g == 2) {
      tvh[k - 1] = a[2];
      thpq[k - 1] = a[3];
    }
  }
}

}  // namespace les


using namespace les;

struct ghost_les {
  ghost_ctx *c = nullptr;
  int kc = 0;
  int model = GHOST_LES_NONE;
  ghost_mlp *mlp = nullptr;
  float gs = 1.f, ts = 1.f, delta = 1.f;
  double kolmo = 1.4;
  double t = 0.0;       // time handed to the EDQNM closure (GHOST's (t-1)*dt)
  double nu_cur = 0.0;  // viscosity of the run in progress
  std::vector<void *> bufs;  // owned device buffers
  void *spec[12] = {};       // coarse spectral work fields (9..11: the filtered velocity of samples)
  void *real[9] = {};        // coarse real work fields
  void *rk[3] = {};          // RK copies
  void *force[3] = {};       // closure force + forcing
  float *x = nullptr, *y = nullptr;  // closure inputs / outputs (n^3 rows)
  // EDQNM closure state on the device (n/2+1 shells; Ext 3(n/2+1); mu 3(n/2+1)+1)
  double *tve_dev = nullptr, *tepq_dev = nullptr, *Ek_dev = nullptr, *Ext_dev = nullptr, *mu_dev = nullptr;
  int *go_dev = nullptr;  // 0: no closure; 1: cusp; 2: full_cusp (heli = 1)
  void *ef = nullptr;      // per-mode energy of the substep's start (vcorrect)
  // GHOST's heli flag: the helical closure (full_cusp, tvh, vcorrect's helicity)
  int heli = 0;
  double *thpq_dev = nullptr, *tvh_dev = nullptr, *Hk_dev = nullptr, *Hxt_dev = nullptr;
  void *hf = nullptr;      // per-mode helicity of the substep's start (heli = 1)
  // fallback of the learned closure to EDQNM (ghost_les_set_fallback)
  bool fallback = false;
  double blowup = 10.0;
  long long fell_back_at = -1;  // step of the run at which it happened, or -1
  long long steps_done = 0;
  void *save[3] = {};
  bool edqnm_done = false;
  // fine-grid buffers for ghost_les_samples (size of the last fine grid)
  size_t fine_rbytes = 0, fine_cbytes = 0;
  void *fine_real[4] = {};
  void *fine_spec = nullptr;
};

static int les_alloc(ghost_les *L, size_t bytes, void **out) {
  GB_CHECK(dalloc(out, bytes));
  L->bufs.push_back(*out);
  return GHOST_OK;
}

static int les_fine_buffers(ghost_les *L, ghost_ctx *f) {
  if (L->fine_rbytes == f->rbytes && L->fine_cbytes == f->cbytes) return GHOST_OK;
  for (void *&p : L->fine_real) {
    cudaFree(p);
    p = nullptr;
  }
  cudaFree(L->fine_spec);
  L->fine_spec = nullptr;
  L->fine_rbytes = L->fine_cbytes = 0;
  for (void *&p : L->fine_real) GB_CHECK(dalloc(&p, f->rbytes));
  GB_CHECK(dalloc(&L->fine_spec, f->cbytes));
  L->fine_rbytes = f->rbytes;
  L->fine_cbytes = f->cbytes;
  return GHOST_OK;
}

template <typename R> static int truncate_dev(ghost_les *L, ghost_ctx *f, const void *in, void *out) {
  ghost_ctx *c = L->c;
  const R scale = (R)((double)c->nreal / (double)f->nreal);
  const size_t total = c->nspec;
  truncate_kernel<R><<<blocks(total), 256, 0, c->stream>>>((const cx<R> *)in, (cx<R> *)out, c->nx, f->nx,
                                                           L->kc * L->kc, scale);
  return post_launch(c);
}

template <typename R> static int features_dev(ghost_les *L, const void *const v[3], float gs, float delta) {
  return grad9_features_dev<R>(L->c, v, L->spec, L->x, gs, delta);
}

template <typename R>
static int samples_dev(ghost_les *L, ghost_ctx *f, const void *const v[3], float delta, float *x, float *tau) {
  ghost_ctx *c = L->c;
  GB_CHECK(les_fine_buffers(L, f));
  // filtered velocity on the coarse grid, its gradients and real values
  void *ub[3] = {L->spec[9], L->spec[10], L->spec[11]};
  for (int a = 0; a < 3; ++a) GB_CHECK(truncate_dev<R>(L, f, v[a], ub[a]));
  GB_CHECK(grad9_features_dev<R>(c, ub, L->spec, x, 1.f, delta));
  // real ubar (n^3-scaled) into real[0..2]; the gradient fields are done
  for (int a = 0; a < 3; ++a) GB_CHECK(c2r_dev<R>(c, ub[a], L->real[a]));
  // fine velocity (N^3-scaled) and the six products, filtered to the coarse grid
  for (int a = 0; a < 3; ++a) GB_CHECK(c2r_dev<R>(f, v[a], L->fine_real[a]));
  const R sN = (R)(1.0 / (double)f->nreal);
  for (int m = 0; m < 6; ++m) {
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    product_kernel<R><<<blocks(f->nreal), 256, 0, f->stream>>>((const R *)L->fine_real[pa[m]],
                                                               (const R *)L->fine_real[pb[m]], (R *)L->fine_real[3],
                                                               f->nreal, sN);
    GB_CHECK(post_launch(f));
    GB_CHECK(r2c_dev<R>(f, L->fine_real[3], L->fine_spec));
    GB_CHECK(truncate_dev<R>(L, f, L->fine_spec, L->spec[0]));
    GB_CHECK(c2r_dev<R>(c, L->spec[0], L->real[3 + m]));
  }
  TauFields<R> tf;
  for (int m = 0; m < 6; ++m) tf.P[m] = (const R *)L->real[3 + m];
  for (int a = 0; a < 3; ++a) tf.U[a] = (const R *)L->real[a];
  targets_kernel<R><<<blocks(c->nreal), 256, 0, c->stream>>>(tf, tau, c->nreal, (R)(1.0 / (double)c->nreal), 1.f);
  return post_launch(c);
}

// o = f + P(-div tau), tau rows scaled by 1/ts
template <typename R>
static int tau_force_dev(ghost_les *L, const float *tau, float ts, const void *const f[3], void *const o[3]) {
  ghost_ctx *c = L->c;
  RealOut6<R> ro;
  for (int m = 0; m < 6; ++m) ro.t[m] = (R *)L->real[m];
  unpack_tau_kernel<R><<<blocks(c->nreal), 256, 0, c->stream>>>(tau, ro, c->nreal, ts);
  GB_CHECK(post_launch(c));
  Spec6<R> T;
  GB_CHECK(r2c6_dev<R>(c, L->real, L->spec));
  for (int m = 0; m < 6; ++m) T.T[m] = (const cx<R> *)L->spec[m];
  Spec3<R> fs;
  Spec3w<R> os;
  for (int a = 0; a < 3; ++a) {
    fs.p[a] = f ? (const cx<R> *)f[a] : nullptr;
    os.p[a] = (cx<R> *)o[a];
  }
  tau_force_kernel<R><<<blocks(c->nspec), 256, 0, c->stream>>>(kparams<R>(c), T, fs, os, c->nspec);
  return post_launch(c);
}

// EDQNM closure on the device: kinetic spectrum -> evedqnm (one block) ->
// eddy-viscous force; the host is not involved, so a substep does not wait
template <typename R>
static int eddy_force_dev(ghost_les *L, const void *const v[3], const void *const f[3], void *const o[3]) {
  ghost_ctx *c = L->c;
  const int nb = c->nx / 2 + 1;
  const int hel = L->heli;
  GB_CHECK(spectrum_dev_async<R>(c, RED_ENERGY_KIND, v[0], v[1], v[2], L->Ek_dev));
  if (hel == 1) GB_CHECK(spectrum_dev_async<R>(c, RED_HELICITY_KIND, v[0], v[1], v[2], L->Hk_dev));
  edqnm_fit_kernel<R><<<1, 128, 0, c->stream>>>(c->nx, (R)c->kmax, (R)L->kolmo, L->Ek_dev, L->Hk_dev, hel,
                                                L->tepq_dev, L->thpq_dev, L->tve_dev, L->tvh_dev, L->Ext_dev,
                                                L->Hxt_dev, (R *)L->mu_dev, L->go_dev);
  GB_CHECK(post_launch(c));
  edqnm_cusp_kernel<R><<<nb, 128, 0, c->stream>>>((R)c->kmax, L->Ext_dev, L->Hxt_dev, (const R *)L->mu_dev,
                                                  (R)L->nu_cur, (R)L->t, L->go_dev, L->tepq_dev, L->thpq_dev,
                                                  L->tve_dev, L->tvh_dev);
  GB_CHECK(post_launch(c));
  L->edqnm_done = true;
  Spec3<R> vs, fs;
  Spec3w<R> os;
  for (int a = 0; a < 3; ++a) {
    vs.p[a] = (const cx<R> *)v[a];
    fs.p[a] = f ? (const cx<R> *)f[a] : nullptr;
    os.p[a] = (cx<R> *)o[a];
  }
  eddy_force_kernel<R><<<blocks(c->nspec), 256, 0, c->stream>>>(kparams<R>(c), vs, fs, os, L->tve_dev,
                                                                  hel == 1 ? L->tvh_dev : nullptr, nb, c->nspec);
  return post_launch(c);
}

// The spectral network as a closure: kinetic spectrum -> shell inputs ->
// network (kc rows) -> tve(k) -> the eddy-viscous force, all on the stream
template <typename R>
static int spectral_force_dev(ghost_les *L, const void *const v[3], const void *const f[3], void *const o[3]) {
  ghost_ctx *c = L->c;
  const int nb = c->nx / 2 + 1;
  GB_CHECK(spectrum_dev_async<R>(c, RED_ENERGY_KIND, v[0], v[1], v[2], L->Ek_dev));
  spec_features_kernel<<<1, 64, 0, c->stream>>>(L->Ek_dev, L->kc, L->x);
  GB_CHECK(post_launch(c));
  GB_CHECK(ghost_mlp_set_stream(L->mlp, c->stream));
  GB_CHECK(ghost_mlp_forward(L->mlp, L->x, L->y, L->kc));
  spec_tve_kernel<<<1, 64, 0, c->stream>>>(L->y, L->Ek_dev, L->kc, nb, (double)L->ts, L->tve_dev);
  GB_CHECK(post_launch(c));
  Spec3<R> vs, fs;
  Spec3w<R> os;
  for (int a = 0; a < 3; ++a) {
    vs.p[a] = (const cx<R> *)v[a];
    fs.p[a] = f ? (const cx<R> *)f[a] : nullptr;
    os.p[a] = (cx<R> *)o[a];
  }
  eddy_force_kernel<R><<<blocks(c->nspec), 256, 0, c->stream>>>(kparams<R>(c), vs, fs, os, L->tve_dev, nullptr, nb,
                                                                  c->nspec);
  return post_launch(c);
}

// closure force of the selected model for the velocity v: o = f + F(v)
template <typename R>
static int closure_force_dev(ghost_les *L, const void *const v[3], const void *const f[3], void *const o[3]) {
  ghost_ctx *c = L->c;
  switch (L->model) {
    case GHOST_LES_MLP: {
      GB_CHECK(features_dev<R>(L, v, L->gs, L->delta));
      GB_CHECK(ghost_mlp_set_stream(L->mlp, c->stream));
      GB_CHECK(ghost_mlp_forward(L->mlp, L->x, L->y, (int)c->nreal));
      return tau_force_dev<R>(L, L->y, L->ts, f, o);
    }
    case GHOST_LES_EDQNM:
      return eddy_force_dev<R>(L, v, f, o);
    case GHOST_LES_MLP_SPECTRAL:
      return spectral_force_dev<R>(L, v, f, o);
    default: {
      // no closure: the forcing alone
      const size_t b = c->cbytes;
      for (int a = 0; a < 3; ++a) {
        if (f && f[a])
          GB_CUDA(cudaMemcpyAsync(o[a], f[a], b, cudaMemcpyDeviceToDevice, c->stream));
        else
          GB_CUDA(cudaMemsetAsync(o[a], 0, b, c->stream));
      }
      return GHOST_OK;
    }
  }
}

// nsteps RK steps of the LES: each substep computes the closure force from
// the current velocity, then runs the fused HD substep with it as forcing
template <typename R>
static int les_run_dev(ghost_les *L, int nsteps, int ord, double dt, double nu, void *const v[3],
                       const void *const f[3]) {
  ghost_ctx *c = L->c;
  L->nu_cur = nu;
  bool first = true;
  // GHOST's EDQNM step ends with vcorrect, which needs the per-mode energies
  // of the substep's start (edqnmhd_rkstep2.f90:8-10,63)
  const int nb = c->nx / 2 + 1;
  const R n3 = (R)c->nx * (R)c->ny * (R)c->nz;
  const R rmp = (R)1 / (n3 * n3);
  const R tinyf = (R)1e-15 < (R)0.1 / ((R)c->nmax * (R)c->nmax) ? (R)1e-15 : (R)0.1 / ((R)c->nmax * (R)c->nmax);
  Spec3<R> vr;
  Spec3w<R> vw;
  for (int a = 0; a < 3; ++a) {
    vr.p[a] = (const cx<R> *)v[a];
    vw.p[a] = (cx<R> *)v[a];
  }
  // the learned closure's fallback: each step starts from a saved copy, and a
  // step that ends non-finite or with <|v|^2> above blowup times its value at
  // the start of the call is redone with GHOST's EDQNM closure, which then
  // stays in use
  double e_ref = 0.0;
  auto learned = [L] { return L->model == GHOST_LES_MLP || L->model == GHOST_LES_MLP_SPECTRAL; };
  const bool guard = L->fallback && learned();
  if (guard) GB_CHECK(reduce_dev<R>(c, 0 /* <|v|^2> */, v[0], v[1], v[2], nullptr, nullptr, nullptr, &e_ref));
  for (int s = 0; s < nsteps; ++s) {
    const bool guarded = L->fallback && learned();
    if (guarded)
      for (int a = 0; a < 3; ++a)
        GB_CUDA(cudaMemcpyAsync(L->save[a], v[a], c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
    const bool vcorr_step = L->model == GHOST_LES_EDQNM;
    for (int o = ord; o >= 1; --o) {
      GB_CHECK(closure_force_dev<R>(L, v, f, L->force));
      const int hel = vcorr_step ? L->heli : 0;
      if (vcorr_step) {
        eden_kernel<R><<<blocks(c->nspec), 256, 0, c->stream>>>(kparams<R>(c), vr, (R *)L->ef,
                                                                hel == 1 ? (R *)L->hf : nullptr, c->nspec, rmp);
        GB_CHECK(post_launch(c));
      }
      GB_CHECK(hd_substep_dev<R>(c, o, dt, nu, v, L->rk, L->force, o == ord ? 1 : 0, !first));
      if (vcorr_step) {
        vcorrect_kernel<R><<<blocks(c->nspec), 256, 0, c->stream>>>(
            kparams<R>(c), vw, (const R *)L->ef, L->tepq_dev, L->Ek_dev, (const R *)L->hf, L->thpq_dev, L->Hk_dev, hel,
            nb, (R)dt * ((R)1 / (R)o), tinyf, n3, c->nspec);
        GB_CHECK(post_launch(c));
      }
      first = false;
    }
    if (guarded) {
      double e = 0.0;
      GB_CHECK(reduce_dev<R>(c, 0 /* <|v|^2> */, v[0], v[1], v[2], nullptr, nullptr, nullptr, &e));
      if (!std::isfinite(e) || (e_ref > 0.0 && e > L->blowup * e_ref)) {
        for (int a = 0; a < 3; ++a)
          GB_CUDA(cudaMemcpyAsync(v[a], L->save[a], c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
        L->model = GHOST_LES_EDQNM;
        L->fell_back_at = L->steps_done;
        first = true;  // the restored velocity may carry modes outside the truncation
        --s;           // redo this step
        continue;
      }
    }
    L->t += dt;
    ++L->steps_done;
  }
  return check_status(c);
}

#define LES_CHECK(L)                                                            \
  do {                                                                          \
    if (!(L) || !(L)->c) return fail(GHOST_ERR_ARG, "null LES handle");        \
  } while (0)

static int dev3(const void *a, const void *b, const void *c, const char *what) {
  if (!a || !b || !c) return fail(GHOST_ERR_ARG, "%s: null field", what);
  if (!is_device_ptr(a) || !is_device_ptr(b) || !is_device_ptr(c))
    return fail(GHOST_ERR_ARG, "%s: LES calls take device arrays", what);
  return GHOST_OK;
}

static int fine_compatible(const ghost_les *L, const ghost_ctx *f) {
  const ghost_ctx *c = L->c;
  if (!f) return fail(GHOST_ERR_ARG, "null fine context");
  if (f->precision != c->precision) return fail(GHOST_ERR_ARG, "fine and coarse precisions differ");
  if (f->anis || f->nx != f->ny || f->nx != f->nz) return fail(GHOST_ERR_SIZE, "the fine grid must be cubic");
  if (f->nx < c->nx) return fail(GHOST_ERR_SIZE, "fine grid %d smaller than the LES grid %d", f->nx, c->nx);
  if (2 * L->kc >= f->nx) return fail(GHOST_ERR_SIZE, "kc %d not below the fine Nyquist %d", L->kc, f->nx / 2);
  if (f->nruns != 1) return fail(GHOST_ERR_ARG, "batched fine contexts are not supported");
  return GHOST_OK;
}

extern "C" {

int ghost_les_create(ghost_ctx *c, int kc, ghost_les **out) {
  if (!out) return fail(GHOST_ERR_ARG, "null output");
  *out = nullptr;
  if (!c) return fail(GHOST_ERR_ARG, "null context");
  if (c->anis || c->nx != c->ny || c->nx != c->nz) return fail(GHOST_ERR_SIZE, "the LES grid must be cubic");
  if (c->nruns != 1) return fail(GHOST_ERR_ARG, "batched contexts are not supported");
  if (kc < 1 || 2 * kc >= c->nx) return fail(GHOST_ERR_ARG, "kc %d must be in [1, n/2)", kc);
  ghost_les *L = new ghost_les();
  L->c = c;
  L->kc = kc;
  int st = GHOST_OK;
  for (int q = 0; q < 12 && !st; ++q) st = les_alloc(L, c->cbytes, &L->spec[q]);
  for (int q = 0; q < 9 && !st; ++q) st = les_alloc(L, c->rbytes, &L->real[q]);
  for (int q = 0; q < 3 && !st; ++q) st = les_alloc(L, c->cbytes, &L->rk[q]);
  for (int q = 0; q < 3 && !st; ++q) st = les_alloc(L, c->cbytes, &L->force[q]);
  if (!st) st = les_alloc(L, sizeof(float) * c->nreal * GHOST_MLP_NIN, (void **)&L->x);
  if (!st) st = les_alloc(L, sizeof(float) * c->nreal * GHOST_MLP_NOUT, (void **)&L->y);
  const size_t nb = c->nx / 2 + 1;
  if (!st) st = les_alloc(L, sizeof(double) * nb, (void **)&L->tve_dev);
  if (!st) st = les_alloc(L, sizeof(double) * nb, (void **)&L->tepq_dev);
  if (!st) st = les_alloc(L, sizeof(double) * nb, (void **)&L->Ek_dev);
  if (!st) st = les_alloc(L, sizeof(double) * 3 * nb, (void **)&L->Ext_dev);
  if (!st) st = les_alloc(L, sizeof(double) * (3 * nb + 1), (void **)&L->mu_dev);
  if (!st) st = les_alloc(L, sizeof(int), (void **)&L->go_dev);
  if (!st) st = les_alloc(L, c->cbytes, &L->ef);
  if (!st) st = les_alloc(L, c->cbytes, &L->hf);
  if (!st) st = les_alloc(L, sizeof(double) * nb, (void **)&L->thpq_dev);
  if (!st) st = les_alloc(L, sizeof(double) * nb, (void **)&L->tvh_dev);
  if (!st) st = les_alloc(L, sizeof(double) * nb, (void **)&L->Hk_dev);
  if (!st) st = les_alloc(L, sizeof(double) * 3 * nb, (void **)&L->Hxt_dev);
  for (int q = 0; q < 3 && !st; ++q) st = les_alloc(L, c->cbytes, &L->save[q]);
  if (st) {
    ghost_les_destroy(L);
    return st;
  }
  *out = L;
  return GHOST_OK;
}

int ghost_les_destroy(ghost_les *L) {
  if (!L) return GHOST_OK;
  if (L->c) cudaStreamSynchronize(L->c->stream);
  for (void *p : L->bufs) cudaFree(p);
  for (void *p : L->fine_real) cudaFree(p);
  cudaFree(L->fine_spec);
  delete L;
  return GHOST_OK;
}

int ghost_les_truncate(ghost_les *L, ghost_ctx *f, const void *in, void *out) {
  LES_CHECK(L);
  GB_CHECK(fine_compatible(L, f));
  GB_CHECK(dev3(in, out, out, "ghost_les_truncate"));
  GB_CUDA(cudaStreamSynchronize(f->stream));
  int st = L->c->precision == GHOST_SINGLE ? truncate_dev<float>(L, f, in, out) : truncate_dev<double>(L, f, in, out);
  return st ? st : check_status(L->c);
}

int ghost_les_samples(ghost_les *L, ghost_ctx *f, const void *vx, const void *vy, const void *vz, float delta,
                      float *x, float *tau) {
  LES_CHECK(L);
  GB_CHECK(fine_compatible(L, f));
  GB_CHECK(dev3(vx, vy, vz, "ghost_les_samples"));
  GB_CHECK(dev3(x, tau, tau, "ghost_les_samples"));
  // the fine and coarse contexts may use different streams: order them
  GB_CUDA(cudaStreamSynchronize(f->stream));
  GB_CUDA(cudaStreamSynchronize(L->c->stream));
  const void *v[3] = {vx, vy, vz};
  // the fine-grid passes run on the coarse context's stream, so that every
  // hand-over between the grids is ordered
  cudaStream_t fs = f->stream;
  f->stream = L->c->stream;
  int st = L->c->precision == GHOST_SINGLE ? samples_dev<float>(L, f, v, delta, x, tau)
                                           : samples_dev<double>(L, f, v, delta, x, tau);
  f->stream = fs;
  if (st) return st;
  GB_CUDA(cudaStreamSynchronize(L->c->stream));
  return check_status(L->c);
}

int ghost_les_features(ghost_les *L, const void *vx, const void *vy, const void *vz, float grad_scale, float delta,
                       float *x) {
  LES_CHECK(L);
  GB_CHECK(dev3(vx, vy, vz, "ghost_les_features"));
  GB_CHECK(dev3(x, x, x, "ghost_les_features"));
  const void *v[3] = {vx, vy, vz};
  float *keep = L->x;
  L->x = x;
  int st = L->c->precision == GHOST_SINGLE ? features_dev<float>(L, v, grad_scale, delta)
                                           : features_dev<double>(L, v, grad_scale, delta);
  L->x = keep;
  return st;
}

int ghost_les_spectral_features(ghost_les *L, const double *E, float *x) {
  LES_CHECK(L);
  if (!E || !x || !is_device_ptr(E) || !is_device_ptr(x))
    return fail(GHOST_ERR_ARG, "ghost_les_spectral_features needs device arrays");
  spec_features_kernel<<<1, 64, 0, L->c->stream>>>(E, L->kc, x);
  GB_CHECK(post_launch(L->c));
  GB_CUDA(cudaStreamSynchronize(L->c->stream));
  return check_status(L->c);
}

int ghost_les_tau_force(ghost_les *L, const float *tau, float tau_scale, const void *fx, const void *fy,
                        const void *fz, void *ox, void *oy, void *oz) {
  LES_CHECK(L);
  GB_CHECK(dev3(tau, tau, tau, "ghost_les_tau_force"));
  GB_CHECK(dev3(ox, oy, oz, "ghost_les_tau_force"));
  if ((fx || fy || fz) && (!fx || !fy || !fz)) return fail(GHOST_ERR_ARG, "give all three forcing fields or none");
  if (fx) GB_CHECK(dev3(fx, fy, fz, "ghost_les_tau_force"));
  const void *f[3] = {fx, fy, fz};
  void *o[3] = {ox, oy, oz};
  return L->c->precision == GHOST_SINGLE ? tau_force_dev<float>(L, tau, tau_scale, fx ? f : nullptr, o)
                                         : tau_force_dev<double>(L, tau, tau_scale, fx ? f : nullptr, o);
}

int ghost_les_set_model(ghost_les *L, int model, ghost_mlp *mlp, double grad_scale, double tau_scale, double delta,
                        double kolmo) {
  LES_CHECK(L);
  if (model != GHOST_LES_NONE && model != GHOST_LES_EDQNM && model != GHOST_LES_MLP &&
      model != GHOST_LES_MLP_SPECTRAL)
    return fail(GHOST_ERR_ARG, "unknown closure %d", model);
  if ((model == GHOST_LES_MLP || model == GHOST_LES_MLP_SPECTRAL) && !mlp)
    return fail(GHOST_ERR_ARG, "the MLP closure needs a network");
  if (model == GHOST_LES_MLP_SPECTRAL && L->kc < 4)
    return fail(GHOST_ERR_ARG, "the spectral closure needs a cutoff of at least 4 shells");
  if (model == GHOST_LES_EDQNM && !(kolmo > 0)) return fail(GHOST_ERR_ARG, "kolmo must be positive");
  if (model == GHOST_LES_EDQNM && (int)std::sqrt(L->c->kmax) < 4)
    return fail(GHOST_ERR_ARG, "the EDQNM closure needs a cutoff of at least 4 shells");
  L->model = model;
  L->mlp = mlp;
  L->gs = (float)grad_scale;
  L->ts = (float)tau_scale;
  L->delta = (float)delta;
  L->kolmo = kolmo;
  L->fell_back_at = -1;
  return GHOST_OK;
}

int ghost_les_set_fallback(ghost_les *L, int enable, double blowup) {
  LES_CHECK(L);
  if (enable && !(blowup > 1.0)) return fail(GHOST_ERR_ARG, "blowup factor must exceed 1");
  if (enable && !(L->kolmo > 0)) return fail(GHOST_ERR_ARG, "the fallback needs a positive kolmo (ghost_les_set_model)");
  if (enable && (int)std::sqrt(L->c->kmax) < 4)
    return fail(GHOST_ERR_ARG, "the EDQNM fallback needs a cutoff of at least 4 shells");
  L->fallback = enable != 0;
  L->blowup = blowup;
  return GHOST_OK;
}

int ghost_les_status(const ghost_les *L, int *model, long long *fell_back_at) {
  LES_CHECK(L);
  if (model) *model = L->model;
  if (fell_back_at) *fell_back_at = L->fell_back_at;
  return GHOST_OK;
}

int ghost_les_set_time(ghost_les *L, double t) {
  LES_CHECK(L);
  L->t = t;
  return GHOST_OK;
}

int ghost_les_closure_force(ghost_les *L, double nu, const void *vx, const void *vy, const void *vz, const void *fx,
                            const void *fy, const void *fz, void *ox, void *oy, void *oz) {
  LES_CHECK(L);
  GB_CHECK(dev3(vx, vy, vz, "ghost_les_closure_force"));
  GB_CHECK(dev3(ox, oy, oz, "ghost_les_closure_force"));
  if ((fx || fy || fz) && (!fx || !fy || !fz)) return fail(GHOST_ERR_ARG, "give all three forcing fields or none");
  const void *v[3] = {vx, vy, vz}, *f[3] = {fx, fy, fz};
  void *o[3] = {ox, oy, oz};
  L->nu_cur = nu;
  int st = L->c->precision == GHOST_SINGLE ? closure_force_dev<float>(L, v, fx ? f : nullptr, o)
                                           : closure_force_dev<double>(L, v, fx ? f : nullptr, o);
  return st ? st : check_status(L->c);
}

int ghost_les_run(ghost_les *L, int nsteps, int ord, double dt, double nu, void *vx, void *vy, void *vz,
                  const void *fx, const void *fy, const void *fz) {
  LES_CHECK(L);
  if (nsteps < 0 || ord < 1 || ord > 4) return fail(GHOST_ERR_ARG, "bad nsteps/ord");
  GB_CHECK(dev3(vx, vy, vz, "ghost_les_run"));
  if ((fx || fy || fz) && (!fx || !fy || !fz)) return fail(GHOST_ERR_ARG, "give all three forcing fields or none");
  if (fx) GB_CHECK(dev3(fx, fy, fz, "ghost_les_run"));
  void *v[3] = {vx, vy, vz};
  const void *f[3] = {fx, fy, fz};
  return L->c->precision == GHOST_SINGLE ? les_run_dev<float>(L, nsteps, ord, dt, nu, v, fx ? f : nullptr)
                                         : les_run_dev<double>(L, nsteps, ord, dt, nu, v, fx ? f : nullptr);
}

int ghost_les_edqnm_last(ghost_les *L, double *tve, double *tepq, double *Ek) {
  LES_CHECK(L);
  const int nb = L->c->nx / 2 + 1;
  if (!L->edqnm_done) return fail(GHOST_ERR_STATE, "no EDQNM evaluation yet");
  GB_CUDA(cudaStreamSynchronize(L->c->stream));
  if (tve) GB_CUDA(cudaMemcpy(tve, L->tve_dev, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  if (tepq) GB_CUDA(cudaMemcpy(tepq, L->tepq_dev, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  if (Ek) GB_CUDA(cudaMemcpy(Ek, L->Ek_dev, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  return GHOST_OK;
}

int ghost_les_set_helicity(ghost_les *L, int heli) {
  LES_CHECK(L);
  if (heli != 0 && heli != 1) return fail(GHOST_ERR_ARG, "heli %d not 0 or 1", heli);
  L->heli = heli;
  return GHOST_OK;
}

int ghost_les_edqnm_last_hel(ghost_les *L, double *tvh, double *thpq, double *Hk) {
  LES_CHECK(L);
  const int nb = L->c->nx / 2 + 1;
  if (!L->edqnm_done) return fail(GHOST_ERR_STATE, "no EDQNM evaluation yet");
  if (L->heli != 1) return fail(GHOST_ERR_STATE, "the helical closure is off (ghost_les_set_helicity)");
  GB_CUDA(cudaStreamSynchronize(L->c->stream));
  if (tvh) GB_CUDA(cudaMemcpy(tvh, L->tvh_dev, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  if (thpq) GB_CUDA(cudaMemcpy(thpq, L->thpq_dev, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  if (Hk) GB_CUDA(cudaMemcpy(Hk, L->Hk_dev, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  return GHOST_OK;
}

int ghost_evedqnm_hel(int n, int precision, double kmax, double kolmo, const double *Eold, const double *Hold,
                      double nu, double time, int hel, double *tepq, double *thpq, double *tve, double *tvh,
                      double *Ext, double *Hxt) {
  if (!Eold || !tepq || !tve || !Ext) return fail(GHOST_ERR_ARG, "null argument");
  if (hel != 0 && hel != 1) return fail(GHOST_ERR_ARG, "hel %d not 0 or 1", hel);
  if (hel == 1 && (!Hold || !thpq || !tvh || !Hxt)) return fail(GHOST_ERR_ARG, "null helicity argument");
  if (n < 16 || (n & (n - 1))) return fail(GHOST_ERR_SIZE, "n %d", n);
  const int kc = (int)std::sqrt(kmax);
  // the energy fit of hel = 1 uses shells kc - (3kc/4 - 2) .. kc
  if (kc < 4 || kc > n / 2) return fail(GHOST_ERR_ARG, "kmax %g: EDQNM needs 4 <= sqrt(kmax) <= n/2", kmax);
  if (precision == GHOST_SINGLE)
    evedqnm_h<float>(n, (float)kmax, (float)kolmo, Eold, Hold, (float)nu, (float)time, hel, tepq, thpq, tve, tvh, Ext,
                     Hxt);
  else if (precision == GHOST_DOUBLE)
    evedqnm_h<double>(n, kmax, kolmo, Eold, Hold, nu, time, hel, tepq, thpq, tve, tvh, Ext, Hxt);
  else
    return fail(GHOST_ERR_ARG, "precision %d", precision);
  return GHOST_OK;
}

int ghost_evedqnm(int n, int precision, double kmax, double kolmo, const double *Eold, double nu, double time,
                  double *tepq, double *tve, double *Ext) {
  if (!Eold || !tepq || !tve || !Ext) return fail(GHOST_ERR_ARG, "null argument");
  if (n < 16 || (n & (n - 1))) return fail(GHOST_ERR_SIZE, "n %d", n);
  const int kc = (int)std::sqrt(kmax);
  // the fit uses shells kc - 3kc/4 .. kc, so kc >= 4 keeps them >= 1
  if (kc < 4 || kc > n / 2) return fail(GHOST_ERR_ARG, "kmax %g: EDQNM needs 4 <= sqrt(kmax) <= n/2", kmax);
  if (precision == GHOST_SINGLE)
    evedqnm<float>(n, (float)kmax, (float)kolmo, Eold, (float)nu, (float)time, tepq, tve, Ext);
  else if (precision == GHOST_DOUBLE)
    evedqnm<double>(n, kmax, kolmo, Eold, nu, time, tepq, tve, Ext);
  else
    return fail(GHOST_ERR_ARG, "precision %d", precision);
  return GHOST_OK;
}

}  // extern "C"
