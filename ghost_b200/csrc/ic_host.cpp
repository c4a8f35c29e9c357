// ic_host.cpp -- seeded initial conditions on the host.
//
// GHOST draws its random phases from randu, a Park-Miller generator with an
// XOR mask (pseudo/pseudospec3D_mod.fpp:130-148).  The masked state update
// has no jump-ahead, so the draw order is inherently sequential and stays
// on the host, as in GHOST; the curl and the normalisation that follow run
// on the GPU.
#include <math.h>
#include <stdint.h>
#include <stddef.h>

#include <complex>

#include "ic_host.h"

namespace gb {

template <typename R> R randu(int32_t &idum) {
  const int32_t iq = 127773, ir = 2836, mask = 123459876, ia = 16807, im = 2147483647;
  // am is the default-REAL parameter 1./im: 2^-31 in both precisions
  const R am = (R)(1.0f / (float)im);
  idum ^= mask;
  const int32_t k = idum / iq;
  idum = ia * (idum - k * iq) - ir * k;
  if (idum < 0) idum += im;
  R r = am * (R)idum;
  r = (r - (R)0.5) * (R)2;
  idum ^= mask;
  return r;
}

template <typename R> static R kval(int idx, int n, double dk, int arbsize) {
  R v = (R)(idx < n / 2 ? idx : idx - n);
  return arbsize ? v * (R)dk : v;
}

template <typename R> static R kk2_at(const Grid &g, int i, int j, int k) {
  if (!g.anis) {
    const R a = (R)(i < g.nx / 2 ? i : i - g.nx), b = (R)(j < g.ny / 2 ? j : j - g.ny),
            c = (R)(k < g.nz / 2 ? k : k - g.nz);
    return a * a + b * b + c * c;
  }
  const R a = kval<R>(i, g.nx, g.Dkx, g.arbsize), b = kval<R>(j, g.ny, g.Dky, g.arbsize),
          c = kval<R>(k, g.nz, g.Dkz, g.arbsize);
  return a * a + b * b + c * c;
}

template <typename R> static R amplitude(int shape, R kk2) {
  if (shape == 0) return (R)1.0 / (R)sqrt((double)kk2);
  return (R)exp(-(double)kk2 / 4.0);
}

// Vector potential with random phases on kdn <= |k| <= kup, in the loop
// order of examples/initialfv.f90_random:16-111 (kx = 0 plane made
// Hermitian there, factor 2 on kx > 0).  C1..C3 are host arrays in GHOST's
// (nz,ny,nx/2+1) layout, interleaved re/im.
template <typename R>
int32_t random_vpot(const Grid &g, int32_t seed, double kdn_d, double kup_d, int shape, R *C1, R *C2, R *C3) {
  typedef std::complex<R> cplx;
  cplx *C[3] = {reinterpret_cast<cplx *>(C1), reinterpret_cast<cplx *>(C2), reinterpret_cast<cplx *>(C3)};
  const R kdn = (R)kdn_d, kup = (R)kup_d;
  const R pi = (R)3.14159265358979323846;
  const int ny = g.ny, nz = g.nz;
  auto idx = [&](int k, int j, int i) { return (size_t)k + (size_t)nz * ((size_t)j + (size_t)ny * i); };
  auto inshell = [&](R kk2) { return kk2 <= kup * kup && kk2 >= kdn * kdn; };
  auto draw = [&](R dump) {
    const R phase = (R)2 * pi * randu<R>(seed);
    return cplx((R)cos((double)phase) * dump, (R)sin((double)phase) * dump);
  };
  for (int q = 0; q < 3; ++q) C[q][idx(0, 0, 0)] = cplx(0, 0);
  for (int j = 1; j <= ny / 2; ++j) {
    const size_t p = idx(0, j, 0), pc = idx(0, ny - j, 0);
    const R kk2 = kk2_at<R>(g, 0, j, 0);
    for (int q = 0; q < 3; ++q) {
      if (inshell(kk2)) {
        C[q][p] = draw(amplitude<R>(shape, kk2));
        C[q][pc] = std::conj(C[q][p]);
      } else {
        C[q][p] = cplx(0, 0);
        C[q][pc] = cplx(0, 0);
      }
    }
  }
  for (int k = 1; k <= nz / 2; ++k) {
    const size_t p = idx(k, 0, 0), pc = idx(nz - k, 0, 0);
    const R kk2 = kk2_at<R>(g, 0, 0, k);
    for (int q = 0; q < 3; ++q) {
      if (inshell(kk2)) {
        C[q][p] = draw(amplitude<R>(shape, kk2));
        C[q][pc] = std::conj(C[q][p]);
      } else {
        C[q][p] = cplx(0, 0);
        C[q][pc] = cplx(0, 0);
      }
    }
  }
  for (int j = 1; j < ny; ++j)
    for (int k = 1; k <= nz / 2; ++k) {
      const size_t p = idx(k, j, 0), pc = idx(nz - k, ny - j, 0);
      const R kk2 = kk2_at<R>(g, 0, j, k);
      for (int q = 0; q < 3; ++q) {
        if (inshell(kk2)) {
          C[q][p] = draw(amplitude<R>(shape, kk2));
          C[q][pc] = std::conj(C[q][p]);
        } else {
          C[q][p] = cplx(0, 0);
          C[q][pc] = cplx(0, 0);
        }
      }
    }
  for (int i = 1; i < g.nxh; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const size_t p = idx(k, j, i);
        const R kk2 = kk2_at<R>(g, i, j, k);
        for (int q = 0; q < 3; ++q) {
          if (inshell(kk2)) {
            const cplx v = draw(amplitude<R>(shape, kk2));
            C[q][p] = cplx((R)2 * v.real(), (R)2 * v.imag());
          } else {
            C[q][p] = cplx(0, 0);
          }
        }
      }
  return seed;
}

template float randu<float>(int32_t &);
template double randu<double>(int32_t &);
template int32_t random_vpot<float>(const Grid &, int32_t, double, double, int, float *, float *, float *);
template int32_t random_vpot<double>(const Grid &, int32_t, double, double, int, double *, double *, double *);

}  // namespace gb
