/*
 * ghost_oracle.c -- CPU restatement of GHOST's 3D HD pseudospectral path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library
 * under ghost_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  Nothing in
 * the product links it.
 *
 * Parity status: the reference (Fortran 90 + MPI + FFTW 3.x) cannot be
 * compiled here (no Fortran compiler, no MPI, no FFTW) and ships no test
 * vectors, so no reference-run outputs exist.  The restatement is pinned
 * instead to
 *   - the DFT definition (direct O(N^2) sums and scipy's pocketfft,
 *     tests/test_oracle_fft.py), which is exactly what FFTW computes,
 *   - the reference's own analytic initial conditions (ABC Beltrami flow of
 *     examples/initialv.f90_abc decays as exp(-nu k^2 t) with zero
 *     nonlinear term), the energy budget dE/dt = -2 nu Omega + eps of
 *     3D/src/README:490-502, and div v = 0,
 * and the reference's source is followed statement by statement below
 * (file:line citations are relative to the GHOST tree, 3D/src/).
 *
 * Layouts are GHOST's (Fortran column-major, 0-based here):
 *   spectral a(k,j,i): k = z index (fastest), j = y, i = kx index 0..nx/2
 *                      offset k + nz*(j + ny*i)
 *   real     r(i,j,k): i = x (fastest), j = y, k = z
 *                      offset i + nx*(j + ny*k)
 * Transforms are unnormalised both ways (fftp-3/fftp3D.fpp:204-431).
 *
 * Built twice: -DORACLE_FP32 gives GHOST's PRECISION=SINGLE build
 * (fftp-3/fprecision_mod.fpp:14-16), otherwise PRECISION=DOUBLE.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_FP32
typedef float real;
#else
typedef double real;
#endif

typedef struct { real re, im; } cplx;

static inline cplx cadd(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cplx csub(cplx a, cplx b) { cplx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}
static inline cplx cscal(real s, cplx a) { cplx r = {s * a.re, s * a.im}; return r; }
static inline cplx cconj(cplx a) { cplx r = {a.re, -a.im}; return r; }
/* im*s*a: the Fortran expression im*kx(i)*a(k,j,i) of derivk3 */
static inline cplx cimul(real s, cplx a) {
  cplx ims = {(real)0, s};
  return cmul(ims, a);
}
static inline real cabs2(cplx a) { return a.re * a.re + a.im * a.im; }

/* ------------------------------------------------------------------ */
/* 1D complex FFT: iterative radix-2, twiddles evaluated in FP64 once and
 * rounded to the working precision (the role FFTW plays for GHOST,
 * fftp-3/fftp3D.fpp:92-107). */
typedef struct {
  int n, logn;
  cplx *tw; /* exp(-2 pi i t / n), t < n/2 */
  int *rev;
} fft1_t;

static int ilog2(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }

static int fft1_init(fft1_t *p, int n) {
  p->n = n;
  p->logn = ilog2(n);
  if ((1 << p->logn) != n) return -1;
  p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)(n / 2 + 1));
  p->rev = (int *)malloc(sizeof(int) * (size_t)n);
  for (int t = 0; t <= n / 2; ++t) {
    double a = -2.0 * 3.14159265358979323846 * (double)t / (double)n;
    p->tw[t].re = (real)cos(a);
    p->tw[t].im = (real)sin(a);
  }
  for (int t = 0; t < n; ++t) {
    int r = 0;
    for (int b = 0; b < p->logn; ++b) r |= ((t >> b) & 1) << (p->logn - 1 - b);
    p->rev[t] = r;
  }
  return 0;
}
static void fft1_free(fft1_t *p) { free(p->tw); free(p->rev); }

/* sign = -1 forward (FFTW_FORWARD), +1 backward; unnormalised */
static void fft1(const fft1_t *p, cplx *x, int sign) {
  int n = p->n;
  for (int t = 0; t < n; ++t) {
    int r = p->rev[t];
    if (r > t) { cplx s = x[t]; x[t] = x[r]; x[r] = s; }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1, step = n / len;
    for (int b = 0; b < n; b += len) {
      for (int j = 0; j < half; ++j) {
        cplx w = p->tw[j * step];
        if (sign > 0) w.im = -w.im;
        cplx u = x[b + j], v = cmul(w, x[b + j + half]);
        x[b + j] = cadd(u, v);
        x[b + j + half] = csub(u, v);
      }
    }
  }
}

/* ------------------------------------------------------------------ */
/* Context: the grid, kes, ali and boxsize modules
 * (pseudo/pseudospec3D_mod.fpp:13-21,53-72,112-120) set up as in
 * main3D.fpp:1727-1801. */
typedef struct {
  int nx, ny, nz, nxh;
  int anis, arbsize, nmax, nmaxperp;
  real Lx, Ly, Lz, Dkx, Dky, Dkz, Dkk;
  real kmax, tiny;
  real *kx, *ky, *kz;
  real *kn2, *kk2; /* (nz,ny,nxh) */
  fft1_t fx, fy, fz;
  size_t nspec, nreal;
} octx;

#define SIDX(c, k, j, i) ((size_t)(k) + (size_t)(c)->nz * ((size_t)(j) + (size_t)(c)->ny * (size_t)(i)))

/* edqnm != 0 selects the EDQNM truncation kmax=(n/2-0.5)^2 of main3D.fpp:1732-1734 */
octx *o_ctx_create(int nx, int ny, int nz, double Lx, double Ly, double Lz,
                   int arbsize, int edqnm) {
  octx *c = (octx *)calloc(1, sizeof(octx));
  c->nx = nx; c->ny = ny; c->nz = nz; c->nxh = nx / 2 + 1;
  c->arbsize = arbsize;
  c->nspec = (size_t)nz * ny * c->nxh;
  c->nreal = (size_t)nx * ny * nz;
  /* main3D.fpp:881-909: default box 1,1,1 unless ARBSIZE */
  if (arbsize) {
    c->Lx = (real)Lx; c->Ly = (real)Ly; c->Lz = (real)Lz;
    c->Dkx = (real)1 / c->Lx; c->Dky = (real)1 / c->Ly; c->Dkz = (real)1 / c->Lz;
  } else {
    c->Lx = c->Ly = c->Lz = 1; c->Dkx = c->Dky = c->Dkz = 1;
  }
  c->Dkk = c->Dkx < c->Dky ? c->Dkx : c->Dky;
  if (c->Dkz < c->Dkk) c->Dkk = c->Dkz;
  /* main3D.fpp:740-749 */
  c->anis = arbsize ? 1 : ((nx != ny) || (ny != nz));
  /* main3D.fpp:1727-1737 */
  c->kmax = (real)1.0 / (real)9.0;
  {
    real m = (real)nx * c->Dkx;
    if ((real)ny * c->Dky > m) m = (real)ny * c->Dky;
    if ((real)nz * c->Dkz > m) m = (real)nz * c->Dkz;
    c->nmax = (int)(m / c->Dkk);
    real mp = (real)nx * c->Dkx;
    if ((real)ny * c->Dky > mp) mp = (real)ny * c->Dky;
    c->nmaxperp = (int)(mp / c->Dkk);
  }
  if (!arbsize && c->anis == 0) c->kmax = c->kmax * ((real)nx * (real)nx);
  if (edqnm) c->kmax = ((real)nx / (real)2.0 - (real)0.5) * ((real)nx / (real)2.0 - (real)0.5);
  {
    real t = (real)0.1 / ((real)c->nmax * (real)c->nmax);
    c->tiny = (real)1e-5 < t ? (real)1e-5 : t;
  }
  /* main3D.fpp:1746-1763 */
  c->kx = (real *)malloc(sizeof(real) * nx);
  c->ky = (real *)malloc(sizeof(real) * ny);
  c->kz = (real *)malloc(sizeof(real) * nz);
  for (int i = 0; i < nx / 2; ++i) { c->kx[i] = (real)i; c->kx[i + nx / 2] = (real)(i - nx / 2); }
  for (int j = 0; j < ny / 2; ++j) { c->ky[j] = (real)j; c->ky[j + ny / 2] = (real)(j - ny / 2); }
  for (int k = 0; k < nz / 2; ++k) { c->kz[k] = (real)k; c->kz[k + nz / 2] = (real)(k - nz / 2); }
  if (nx == 1) c->kx[0] = 0;
  if (ny == 1) c->ky[0] = 0;
  if (nz == 1) c->kz[0] = 0;
  real rmp = 1, rmq = 1, rms = 1;
  if (c->anis) {
    rmp = (real)1 / ((real)nx * (real)nx);
    rmq = (real)1 / ((real)ny * (real)ny);
    rms = (real)1 / ((real)nz * (real)nz);
  }
  c->kn2 = (real *)malloc(sizeof(real) * c->nspec);
  for (int i = 0; i < c->nxh; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k)
        c->kn2[SIDX(c, k, j, i)] = rmp * (c->kx[i] * c->kx[i]) + rmq * (c->ky[j] * c->ky[j]) +
                                   rms * (c->kz[k] * c->kz[k]);
  /* main3D.fpp:1785-1800 */
  if (arbsize) {
    for (int i = 0; i < nx; ++i) c->kx[i] *= c->Dkx;
    for (int j = 0; j < ny; ++j) c->ky[j] *= c->Dky;
    for (int k = 0; k < nz; ++k) c->kz[k] *= c->Dkz;
  }
  if (c->anis) {
    c->kk2 = (real *)malloc(sizeof(real) * c->nspec);
    for (int i = 0; i < c->nxh; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
          c->kk2[SIDX(c, k, j, i)] = c->kx[i] * c->kx[i] + c->ky[j] * c->ky[j] + c->kz[k] * c->kz[k];
  } else {
    c->kk2 = c->kn2;
  }
  if (fft1_init(&c->fx, nx) || fft1_init(&c->fy, ny) || fft1_init(&c->fz, nz)) {
    return NULL;
  }
  return c;
}

void o_ctx_destroy(octx *c) {
  if (!c) return;
  if (c->kk2 != c->kn2) free(c->kk2);
  free(c->kn2); free(c->kx); free(c->ky); free(c->kz);
  fft1_free(&c->fx); fft1_free(&c->fy); fft1_free(&c->fz);
  free(c);
}

/* accessors for the Python wrapper */
void o_ctx_info(const octx *c, double *out) {
  out[0] = c->kmax; out[1] = c->tiny; out[2] = c->Dkk; out[3] = c->nmax;
  out[4] = c->anis; out[5] = c->nmaxperp; out[6] = c->Dkx; out[7] = c->Dky; out[8] = c->Dkz;
}
void o_ctx_tables(const octx *c, real *kx, real *ky, real *kz, real *kn2, real *kk2) {
  memcpy(kx, c->kx, sizeof(real) * c->nx);
  memcpy(ky, c->ky, sizeof(real) * c->ny);
  memcpy(kz, c->kz, sizeof(real) * c->nz);
  memcpy(kn2, c->kn2, sizeof(real) * c->nspec);
  memcpy(kk2, c->kk2, sizeof(real) * c->nspec);
}
int o_nthreads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void o_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------ */
/* fftp3d_real_to_complex (fftp-3/fftp3D.fpp:204-315):
 *   2D r2c over (x,y) for each z plane -> carr(nx/2+1,ny,nz)
 *   transpose -> out(nz,ny,nx/2+1)
 *   1D c2c along z, direction -1. */
void o_fftp3d_real_to_complex(const octx *c, const real *in, cplx *out) {
  int nx = c->nx, ny = c->ny, nz = c->nz, nxh = c->nxh;
  cplx *carr = (cplx *)malloc(sizeof(cplx) * c->nspec);
  /* r2c along x: a full complex transform of (x_n + 0i), first nx/2+1 kept */
#pragma omp parallel
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * (size_t)(nx > ny ? nx : ny));
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const real *row = in + (size_t)nx * ((size_t)j + (size_t)ny * k);
        for (int i = 0; i < nx; ++i) { buf[i].re = row[i]; buf[i].im = 0; }
        fft1(&c->fx, buf, -1);
        cplx *dst = carr + (size_t)nxh * ((size_t)j + (size_t)ny * k);
        for (int i = 0; i < nxh; ++i) dst[i] = buf[i];
      }
    /* c2c along y */
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nxh; ++i) {
        cplx *base = carr + (size_t)i + (size_t)nxh * (size_t)ny * k;
        for (int j = 0; j < ny; ++j) buf[j] = base[(size_t)nxh * j];
        fft1(&c->fy, buf, -1);
        for (int j = 0; j < ny; ++j) base[(size_t)nxh * j] = buf[j];
      }
    free(buf);
  }
  /* transpose (fftp3D.fpp:282-298) out(k,j,i) = c1(i,j,k) */
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nxh; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k)
        out[SIDX(c, k, j, i)] = carr[(size_t)i + (size_t)nxh * ((size_t)j + (size_t)ny * k)];
  /* c2c along z (contiguous) */
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nxh; ++i)
    for (int j = 0; j < ny; ++j) fft1(&c->fz, out + SIDX(c, 0, j, i), -1);
  free(carr);
}

/* fftp3d_complex_to_real (fftp-3/fftp3D.fpp:318-431).  The input is left
 * untouched here (GHOST destroys it; callers never rely on its content).
 * The final c2r along x takes only the real parts of the kx=0 and kx=nx/2
 * coefficients, as a complex-to-real transform of a Hermitian line does. */
void o_fftp3d_complex_to_real(const octx *c, const cplx *in, real *out) {
  int nx = c->nx, ny = c->ny, nz = c->nz, nxh = c->nxh;
  cplx *tmp = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *carr = (cplx *)malloc(sizeof(cplx) * c->nspec);
  memcpy(tmp, in, sizeof(cplx) * c->nspec);
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 0; i < nxh; ++i)
    for (int j = 0; j < ny; ++j) fft1(&c->fz, tmp + SIDX(c, 0, j, i), +1);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nxh; ++i)
        carr[(size_t)i + (size_t)nxh * ((size_t)j + (size_t)ny * k)] = tmp[SIDX(c, k, j, i)];
#pragma omp parallel
  {
    cplx *buf = (cplx *)malloc(sizeof(cplx) * (size_t)(nx > ny ? nx : ny));
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nxh; ++i) {
        cplx *base = carr + (size_t)i + (size_t)nxh * (size_t)ny * k;
        for (int j = 0; j < ny; ++j) buf[j] = base[(size_t)nxh * j];
        fft1(&c->fy, buf, +1);
        for (int j = 0; j < ny; ++j) base[(size_t)nxh * j] = buf[j];
      }
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const cplx *src = carr + (size_t)nxh * ((size_t)j + (size_t)ny * k);
        if (nx == 1) {
          out[(size_t)nx * ((size_t)j + (size_t)ny * k)] = src[0].re;
          continue;
        }
        buf[0].re = src[0].re; buf[0].im = 0;
        buf[nx / 2].re = src[nx / 2].re; buf[nx / 2].im = 0;
        for (int i = 1; i < nx / 2; ++i) { buf[i] = src[i]; buf[nx - i] = cconj(src[i]); }
        fft1(&c->fx, buf, +1);
        real *row = out + (size_t)nx * ((size_t)j + (size_t)ny * k);
        for (int i = 0; i < nx; ++i) row[i] = buf[i].re;
      }
    free(buf);
  }
  free(tmp);
  free(carr);
}

/* ------------------------------------------------------------------ */
/* pseudo/pseudospec3D_hd.f90 */

/* derivk3 (pseudospec3D_hd.f90:22-88): b = i k_dir a */
void o_derivk3(const octx *c, const cplx *a, cplx *b, int dir) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < c->nxh; ++i)
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        real kd = dir == 1 ? c->kx[i] : (dir == 2 ? c->ky[j] : c->kz[k]);
        b[p] = cimul(kd, a[p]);
      }
}

/* laplak3 (pseudospec3D_hd.f90:91-121): b = -kk2 a */
void o_laplak3(const octx *c, const cplx *a, cplx *b) {
#pragma omp parallel for schedule(static)
  for (size_t p = 0; p < c->nspec; ++p) b[p] = cscal(-c->kk2[p], a[p]);
}

/* rotor3 (pseudospec3D_hd.f90:124-200) */
void o_rotor3(const octx *c, const cplx *a, const cplx *b, cplx *out, int dir) {
  cplx *c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  if (dir == 1) {
    o_derivk3(c, a, c1, 3); o_derivk3(c, b, c2, 2);
  } else if (dir == 2) {
    o_derivk3(c, a, c1, 3); o_derivk3(c, b, c2, 1);
  } else {
    o_derivk3(c, a, c1, 2); o_derivk3(c, b, c2, 1);
  }
#pragma omp parallel for schedule(static)
  for (size_t p = 0; p < c->nspec; ++p)
    out[p] = (dir == 2) ? csub(c1[p], c2[p]) : csub(c2[p], c1[p]);
  free(c1);
  free(c2);
}

/* prodre3 (pseudospec3D_hd.f90:316-396): [curl(A) x A] in Fourier space */
void o_prodre3(const octx *c, const cplx *a, const cplx *b, const cplx *cc, cplx *d, cplx *e, cplx *f) {
  size_t nr = c->nreal;
  real *r[8];
  for (int q = 1; q <= 7; ++q) r[q] = (real *)malloc(sizeof(real) * nr);
  cplx *t1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  o_rotor3(c, b, cc, t1, 1); o_fftp3d_complex_to_real(c, t1, r[1]);
  o_rotor3(c, a, cc, t1, 2); o_fftp3d_complex_to_real(c, t1, r[2]);
  o_rotor3(c, a, b, t1, 3);  o_fftp3d_complex_to_real(c, t1, r[3]);
  o_fftp3d_complex_to_real(c, a, r[4]);
  o_fftp3d_complex_to_real(c, b, r[5]);
  o_fftp3d_complex_to_real(c, cc, r[6]);
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
#pragma omp parallel for schedule(static)
  for (size_t p = 0; p < nr; ++p) {
    real r1 = r[1][p], r2 = r[2][p], r3 = r[3][p], r4 = r[4][p], r5 = r[5][p], r6 = r[6][p];
    r[7][p] = (r2 * r6 - r5 * r3) * tmp;
    r[3][p] = (r3 * r4 - r6 * r1) * tmp;
    r[1][p] = (r1 * r5 - r4 * r2) * tmp;
  }
  o_fftp3d_real_to_complex(c, r[7], d);
  o_fftp3d_real_to_complex(c, r[3], e);
  o_fftp3d_real_to_complex(c, r[1], f);
  for (int q = 1; q <= 7; ++q) free(r[q]);
  free(t1);
}

/* nonlhd3 (pseudospec3D_hd.f90:399-509): g = -a_dir + k_dir (k.a)/k^2,
 * with the k_dir = 0 plane set to -a_dir.  g may alias a, b or c. */
void o_nonlhd3(const octx *c, const cplx *a, const cplx *b, const cplx *cc, cplx *g, int dir) {
  cplx *tmp = (cplx *)malloc(sizeof(cplx) * c->nspec);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < c->nxh; ++i)
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        cplx self = dir == 1 ? a[p] : (dir == 2 ? b[p] : cc[p]);
        int zero_plane = dir == 1 ? (i == 0) : (dir == 2 ? (j == 0) : (k == 0));
        if (zero_plane) {
          tmp[p].re = -self.re; tmp[p].im = -self.im;
        } else {
          real kd = dir == 1 ? c->kx[i] : (dir == 2 ? c->ky[j] : c->kz[k]);
          cplx s = cadd(cadd(cscal(c->kx[i], a[p]), cscal(c->ky[j], b[p])), cscal(c->kz[k], cc[p]));
          cplx q = cscal(kd, s);
          q.re = q.re / c->kk2[p];
          q.im = q.im / c->kk2[p];
          cplx ms = {-self.re, -self.im};
          tmp[p] = cadd(ms, q);
        }
      }
  memcpy(g, tmp, sizeof(cplx) * c->nspec);
  free(tmp);
}

/* energy (pseudospec3D_hd.f90:512-662); kin: 1 field, 0 curl, 2 Laplacian */
double o_energy(const octx *c, const cplx *a, const cplx *b, const cplx *cc, int kin) {
  const cplx *x = a, *y = b, *z = cc;
  cplx *c1 = NULL, *c2 = NULL, *c3 = NULL;
  if (kin != 1) {
    c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    c3 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    if (kin == 0) {
      o_rotor3(c, b, cc, c1, 1); o_rotor3(c, a, cc, c2, 2); o_rotor3(c, a, b, c3, 3);
    } else {
      o_laplak3(c, a, c1); o_laplak3(c, b, c2); o_laplak3(c, cc, c3);
    }
    x = c1; y = c2; z = c3;
  }
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  double dloc = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    double w = i == 0 ? 1.0 : 2.0;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        real s = (cabs2(x[p]) + cabs2(y[p]) + cabs2(z[p])) * tmp;
        dloc += w * (double)s;
      }
  }
  free(c1); free(c2); free(c3);
  return dloc;
}

/* helicity (pseudospec3D_hd.f90:665-784) */
double o_helicity(const octx *c, const cplx *a, const cplx *b, const cplx *cc) {
  cplx *c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  double dloc = 0.0;
  const cplx *comp[3] = {a, b, cc};
  for (int d = 1; d <= 3; ++d) {
    if (d == 1) o_rotor3(c, b, cc, c1, 1);
    else if (d == 2) o_rotor3(c, a, cc, c1, 2);
    else o_rotor3(c, a, b, c1, 3);
    for (int i = 0; i < c->nxh; ++i) {
      double w = i == 0 ? 1.0 : 2.0;
      for (int j = 0; j < c->ny; ++j)
        for (int k = 0; k < c->nz; ++k) {
          size_t p = SIDX(c, k, j, i);
          real s = cmul(comp[d - 1][p], cconj(c1[p])).re * tmp;
          dloc += w * (double)s;
        }
    }
  }
  free(c1);
  return dloc;
}

/* cross (pseudospec3D_hd.f90:787-907); kin 1: <A.B>, 0: weighted by kk2 */
double o_cross(const octx *c, const cplx *a, const cplx *b, const cplx *cc, const cplx *d,
               const cplx *e, const cplx *f, int kin) {
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  double g = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    double w = i == 0 ? 1.0 : 2.0;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        real s = cadd(cadd(cmul(a[p], cconj(d[p])), cmul(b[p], cconj(e[p]))), cmul(cc[p], cconj(f[p]))).re;
        if (kin == 1) s = s * tmp;
        else s = s * c->kk2[p] * tmp;
        g += w * (double)s;
      }
  }
  return g;
}

/* divergence check of hdcheck (pseudospec3D_hd.f90:1036-1070) */
double o_divergence(const octx *c, const cplx *a, const cplx *b, const cplx *cc) {
  real tmq = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  double t = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    double w = i == 0 ? 1.0 : 2.0;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        cplx s = cadd(cadd(cimul(c->kx[i], a[p]), cimul(c->ky[j], b[p])), cimul(c->kz[k], cc[p]));
        t += w * (double)(cabs2(s) * tmq);
      }
  }
  return t;
}

/* maxabs (pseudospec3D_hd.f90:910-981); kin 0 curl, 1 Laplacian, 2 field */
double o_maxabs(const octx *c, const cplx *a, const cplx *b, const cplx *cc, int kin) {
  cplx *c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *c3 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  if (kin == 0) {
    o_rotor3(c, b, cc, c1, 1); o_rotor3(c, a, cc, c2, 2); o_rotor3(c, a, b, c3, 3);
  } else if (kin == 1) {
    o_laplak3(c, a, c1); o_laplak3(c, b, c2); o_laplak3(c, cc, c3);
  } else {
    memcpy(c1, a, sizeof(cplx) * c->nspec); memcpy(c2, b, sizeof(cplx) * c->nspec);
    memcpy(c3, cc, sizeof(cplx) * c->nspec);
  }
  real *r1 = (real *)malloc(sizeof(real) * c->nreal);
  real *r2 = (real *)malloc(sizeof(real) * c->nreal);
  real *r3 = (real *)malloc(sizeof(real) * c->nreal);
  o_fftp3d_complex_to_real(c, c1, r1);
  o_fftp3d_complex_to_real(c, c2, r2);
  o_fftp3d_complex_to_real(c, c3, r3);
  real d = 0;
  for (size_t p = 0; p < c->nreal; ++p) {
    real s = (real)sqrt(r1[p] * r1[p] + r2[p] * r2[p] + r3[p] * r3[p]);
    if (s > d) d = s;
  }
  d = d / ((real)c->nx * (real)c->ny * (real)c->nz);
  free(c1); free(c2); free(c3); free(r1); free(r2); free(r3);
  return (double)d;
}

/* spectrumc (pseudospec3D_hd.f90:1190-1415).  Ek, Hk have nmax/2+1 bins.
 * kin: 1 kinetic, 0 curl, 2 skip; hel: 1 helicity spectrum. */
void o_spectrumc(const octx *c, const cplx *a, const cplx *b, const cplx *cc, int kin, int hel,
                 double *Ek, double *Hk) {
  int nb = c->nmax / 2 + 1;
  cplx *c1 = NULL, *c2 = NULL, *c3 = NULL;
  if (kin == 0 || hel == 1) {
    c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    c3 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    o_rotor3(c, b, cc, c1, 1); o_rotor3(c, a, cc, c2, 2); o_rotor3(c, a, b, c3, 3);
  }
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  if (kin <= 1) {
    for (int q = 0; q < nb; ++q) Ek[q] = 0.0;
    const cplx *x = kin == 1 ? a : c1, *y = kin == 1 ? b : c2, *z = kin == 1 ? cc : c3;
    for (int i = 0; i < c->nxh; ++i) {
      real w = i == 0 ? (real)1 : (real)2;
      for (int j = 0; j < c->ny; ++j)
        for (int k = 0; k < c->nz; ++k) {
          size_t p = SIDX(c, k, j, i);
          int kmn = (int)((real)sqrt(c->kk2[p]) / c->Dkk + (real)0.501f);
          if (kmn > 0 && kmn <= nb) {
            double tmq = (double)(w * (cabs2(x[p]) + cabs2(y[p]) + cabs2(z[p])) * tmp);
            Ek[kmn - 1] += tmq;
          }
        }
    }
  }
  if (hel == 1) {
    for (int q = 0; q < nb; ++q) Hk[q] = 0.0;
    for (int i = 0; i < c->nxh; ++i) {
      real w = i == 0 ? (real)1 : (real)2;
      for (int j = 0; j < c->ny; ++j)
        for (int k = 0; k < c->nz; ++k) {
          size_t p = SIDX(c, k, j, i);
          int kmn = (int)((real)sqrt(c->kk2[p]) / c->Dkk + (real)0.501f);
          if (kmn > 0 && kmn <= nb) {
            real s = cmul(a[p], cconj(c1[p])).re + cmul(b[p], cconj(c2[p])).re + cmul(cc[p], cconj(c3[p])).re;
            double tmq = (double)(w * s * tmp);
            Hk[kmn - 1] += tmq;
          }
        }
    }
  }
  free(c1); free(c2); free(c3);
}

/* entrans (pseudospec3D_hd.f90:1629-1820): Ektot, the shell sums of
 * w Re(a.conj d + b.conj e + c.conj f) tmp (times kk2 for kin = 0), w = 2 off
 * the kx = 0 plane.  heltrans (:1823-1949) is the same with curl(a,b,c),
 * through rotor3 as there (curl != 0 selects it). */
static void o_transfer(const octx *c, const cplx *x, const cplx *y, const cplx *z, const cplx *d,
                       const cplx *e, const cplx *f, int with_kk2, double *Ek) {
  int nb = c->nmax / 2 + 1;
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  for (int q = 0; q < nb; ++q) Ek[q] = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    real w = i == 0 ? (real)1 : (real)2;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        int kmn = (int)((real)sqrt(c->kk2[p]) / c->Dkk + (real)0.501f);
        if (kmn > 0 && kmn <= nb) {
          real s = cmul(x[p], cconj(d[p])).re + cmul(y[p], cconj(e[p])).re + cmul(z[p], cconj(f[p])).re;
          if (with_kk2) s = c->kk2[p] * s;
          Ek[kmn - 1] += (double)(w * s * tmp);
        }
      }
  }
}

void o_entrans(const octx *c, const cplx *a, const cplx *b, const cplx *cc, const cplx *d, const cplx *e,
               const cplx *f, int kin, double *Ek) {
  o_transfer(c, a, b, cc, d, e, f, kin == 0, Ek);
}

void o_heltrans(const octx *c, const cplx *a, const cplx *b, const cplx *cc, const cplx *d, const cplx *e,
                const cplx *f, double *Hk) {
  cplx *c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *c3 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  o_rotor3(c, b, cc, c1, 1); o_rotor3(c, a, cc, c2, 2); o_rotor3(c, a, b, c3, 3);
  o_transfer(c, c1, c2, c3, d, e, f, 0, Hk);
  free(c1); free(c2); free(c3);
}

/* Anisotropic spectra (pseudospec3D_rot.f90).  mode 0 (specpara, entpara,
 * heltpara, :25-335, 689-875, 1067-1196): kmn = int(|kz| Lz + 1) over
 * nz/2+1 bins; mode 1 (specperp, entperp, heltperp, :338-686, 878-1064,
 * 1199-1328): kmn = int(sqrt(kx^2 + ky^2)/Dkk + 1) over nmaxperp/2+1.
 * The spectra return E[3 nb] = total, horizontal (x, y), vertical (z); in
 * mode 1 the horizontal and vertical sums hold the kz = 0 plane and the
 * other planes enter the total as one three-term sum. */
static int o_an_bin(const octx *c, int mode, int i, int j, int k) {
  if (mode == 0) return (int)(fabs(c->kz[k]) * c->Lz + (real)1);
  return (int)((real)sqrt(c->kx[i] * c->kx[i] + c->ky[j] * c->ky[j]) / c->Dkk + (real)1);
}

/* what: 0 kinetic of (x,y,z), 1 helicity Re(a.conj(x)), x = curl */
static void o_an_spec(const octx *c, int mode, const cplx *a, const cplx *b, const cplx *cc, const cplx *x,
                      const cplx *y, const cplx *z, int what, double *E) {
  int nb = mode == 0 ? c->nz / 2 + 1 : c->nmaxperp / 2 + 1;
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  for (int q = 0; q < 3 * nb; ++q) E[q] = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    real w = i == 0 ? (real)1 : (real)2;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        int kmn = o_an_bin(c, mode, i, j, k);
        if (kmn <= 0 || kmn > nb) continue;
        size_t p = SIDX(c, k, j, i);
        real h, v;
        if (what == 0) {
          h = cabs2(x[p]) + cabs2(y[p]);
          v = cabs2(z[p]);
        } else {
          h = cmul(a[p], cconj(x[p])).re + cmul(b[p], cconj(y[p])).re;
          v = cmul(cc[p], cconj(z[p])).re;
        }
        if (mode == 0 || k == 0) {
          double tq = (double)(w * h * tmp), tr = (double)(w * v * tmp);
          E[kmn - 1] += tq + tr;
          E[nb + kmn - 1] += tq;
          E[2 * nb + kmn - 1] += tr;
        } else {
          E[kmn - 1] += (double)(w * (h + v) * tmp);
        }
      }
  }
}

void o_spec_aniso(const octx *c, int mode, const cplx *a, const cplx *b, const cplx *cc, int kin, int hel,
                  double *Ek, double *Hk) {
  cplx *c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  cplx *c3 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  o_rotor3(c, b, cc, c1, 1); o_rotor3(c, a, cc, c2, 2); o_rotor3(c, a, b, c3, 3);
  if (kin == 1) o_an_spec(c, mode, a, b, cc, a, b, cc, 0, Ek);
  if (kin == 0) o_an_spec(c, mode, a, b, cc, c1, c2, c3, 0, Ek);
  if (hel == 1) o_an_spec(c, mode, a, b, cc, c1, c2, c3, 1, Hk);
  free(c1); free(c2); free(c3);
}

/* the transfers binned the same way: Re(x.conj d + y.conj e + z.conj f) tmp
 * (times kk2 with_kk2), x = (a,b,c) or curl(a,b,c) (curl != 0) */
void o_trans_aniso(const octx *c, int mode, const cplx *a, const cplx *b, const cplx *cc, const cplx *d,
                   const cplx *e, const cplx *f, int with_kk2, int curl, double *E) {
  int nb = mode == 0 ? c->nz / 2 + 1 : c->nmaxperp / 2 + 1;
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  const cplx *x = a, *y = b, *z = cc;
  cplx *c1 = NULL, *c2 = NULL, *c3 = NULL;
  if (curl) {
    c1 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    c3 = (cplx *)malloc(sizeof(cplx) * c->nspec);
    o_rotor3(c, b, cc, c1, 1); o_rotor3(c, a, cc, c2, 2); o_rotor3(c, a, b, c3, 3);
    x = c1; y = c2; z = c3;
  }
  for (int q = 0; q < nb; ++q) E[q] = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    real w = i == 0 ? (real)1 : (real)2;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        int kmn = o_an_bin(c, mode, i, j, k);
        if (kmn <= 0 || kmn > nb) continue;
        size_t p = SIDX(c, k, j, i);
        real s = cmul(x[p], cconj(d[p])).re + cmul(y[p], cconj(e[p])).re + cmul(z[p], cconj(f[p])).re;
        if (with_kk2) s = c->kk2[p] * s;
        E[kmn - 1] += (double)(w * s * tmp);
      }
  }
  free(c1); free(c2); free(c3);
}

/* ------------------------------------------------------------------ */
/* Random numbers: randu of pseudo/pseudospec3D_mod.fpp:130-148.  am is the
 * default-REAL constant 1./im, which is 2^-31 in both precisions. */
real o_randu(int32_t *idum) {
  const int32_t iq = 127773, ir = 2836, mask = 123459876, ia = 16807, im = 2147483647;
  const real am = (real)(1.0f / (float)im);
  int32_t k;
  *idum = *idum ^ mask;
  k = *idum / iq;
  *idum = ia * (*idum - k * iq) - ir * k;
  if (*idum < 0) *idum = *idum + im;
  real r = am * (real)(*idum);
  r = (r - (real)0.5) * (real)2;
  *idum = *idum ^ mask;
  return r;
}

/* radial amplitude of the random vector potential:
 *   shape 0: 1/|k|            (examples/initialfv.f90_random:23)
 *   shape 1: exp(-|k|^2/4)    gives E(k) ~ k^4 exp(-2 (k/2)^2) after the curl */
static real amp_of(int shape, real kk2v) {
  if (shape == 0) return (real)1.0 / (real)sqrt(kk2v);
  return (real)exp(-(double)kk2v / 4.0);
}

static inline cplx phasor(real phase, real dump) {
  cplx r = {(real)cos(phase) * dump, (real)sin(phase) * dump};
  return r;
}

/* Random-phase vector potential on kdn <= |k| <= kup, with the loop order,
 * seeding and Hermitian kx=0 plane of examples/initialfv.f90_random:16-134.
 * Returns the updated seed. */
int32_t o_random_vpot(const octx *c, int32_t seed, double kdn_d, double kup_d, int shape, cplx *C1, cplx *C2,
                      cplx *C3) {
  int ny = c->ny, nz = c->nz;
  real kdn = (real)kdn_d, kup = (real)kup_d;
  const real pi = (real)3.14159265358979323846;
  cplx zero = {0, 0};
  cplx *Cs[3] = {C1, C2, C3};
#define INSHELL(p) ((c->kk2[p] <= kup * kup) && (c->kk2[p] >= kdn * kdn))
  /* kx = 0 plane */
  for (int q = 0; q < 3; ++q) Cs[q][SIDX(c, 0, 0, 0)] = zero;
  for (int j = 1; j <= ny / 2; ++j) {
    size_t p = SIDX(c, 0, j, 0), pc = SIDX(c, 0, ny - j, 0);
    if (INSHELL(p)) {
      real dump = amp_of(shape, c->kk2[p]);
      for (int q = 0; q < 3; ++q) {
        real phase = 2 * pi * o_randu(&seed);
        Cs[q][p] = phasor(phase, dump);
        Cs[q][pc] = cconj(Cs[q][p]);
      }
    } else {
      for (int q = 0; q < 3; ++q) { Cs[q][p] = zero; Cs[q][pc] = zero; }
    }
  }
  for (int k = 1; k <= nz / 2; ++k) {
    size_t p = SIDX(c, k, 0, 0), pc = SIDX(c, nz - k, 0, 0);
    if (INSHELL(p)) {
      real dump = amp_of(shape, c->kk2[p]);
      for (int q = 0; q < 3; ++q) {
        real phase = 2 * pi * o_randu(&seed);
        Cs[q][p] = phasor(phase, dump);
        Cs[q][pc] = cconj(Cs[q][p]);
      }
    } else {
      for (int q = 0; q < 3; ++q) { Cs[q][p] = zero; Cs[q][pc] = zero; }
    }
  }
  for (int j = 1; j < ny; ++j)
    for (int k = 1; k <= nz / 2; ++k) {
      size_t p = SIDX(c, k, j, 0), pc = SIDX(c, nz - k, ny - j, 0);
      if (INSHELL(p)) {
        real dump = amp_of(shape, c->kk2[p]);
        for (int q = 0; q < 3; ++q) {
          real phase = 2 * pi * o_randu(&seed);
          Cs[q][p] = phasor(phase, dump);
          Cs[q][pc] = cconj(Cs[q][p]);
        }
      } else {
        for (int q = 0; q < 3; ++q) { Cs[q][p] = zero; Cs[q][pc] = zero; }
      }
    }
  for (int i = 1; i < c->nxh; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        if (INSHELL(p)) {
          real dump = amp_of(shape, c->kk2[p]);
          for (int q = 0; q < 3; ++q) {
            real phase = 2 * pi * o_randu(&seed);
            cplx v = phasor(phase, dump);
            Cs[q][p] = cscal((real)2, v);
          }
        } else {
          for (int q = 0; q < 3; ++q) Cs[q][p] = zero;
        }
      }
#undef INSHELL
  return seed;
}

/* normalize (pseudo/module_dns.f90:13-41) */
void o_normalize(const octx *c, cplx *fx, cplx *fy, cplx *fz, double f0, int kin) {
  double tmp = o_energy(c, fx, fy, fz, kin);
  double s = sqrt(tmp);
  for (size_t p = 0; p < c->nspec; ++p) {
    fx[p].re = (real)((double)(fx[p].re * (real)f0) / s); fx[p].im = (real)((double)(fx[p].im * (real)f0) / s);
    fy[p].re = (real)((double)(fy[p].re * (real)f0) / s); fy[p].im = (real)((double)(fy[p].im * (real)f0) / s);
    fz[p].re = (real)((double)(fz[p].re * (real)f0) / s); fz[p].im = (real)((double)(fz[p].im * (real)f0) / s);
  }
}

/* A solenoidal field = curl of the random vector potential, normalised
 * so that <|v|^2> = amp^2 (examples/initialfv.f90_random:136-139). */
int32_t o_random_solenoidal(const octx *c, int32_t seed, double kdn, double kup, int shape, double amp, cplx *vx,
                            cplx *vy, cplx *vz) {
  size_t n = c->nspec;
  cplx *C1 = (cplx *)malloc(sizeof(cplx) * n), *C2 = (cplx *)malloc(sizeof(cplx) * n),
       *C3 = (cplx *)malloc(sizeof(cplx) * n);
  seed = o_random_vpot(c, seed, kdn, kup, shape, C1, C2, C3);
  o_rotor3(c, C2, C3, vx, 1);
  o_rotor3(c, C1, C3, vy, 2);
  o_rotor3(c, C1, C2, vz, 3);
  o_normalize(c, vx, vy, vz, amp, 1);
  free(C1); free(C2); free(C3);
  return seed;
}

/* ABC flow of examples/initialv.f90_abc:25-54 (before normalize) */
void o_abc(const octx *c, double kdn, double kup, double A, double B, double C, real *R1, real *R2, real *R3) {
  const real pi = (real)3.14159265358979323846;
  int nx = c->nx, ny = c->ny, nz = c->nz;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        size_t p = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
        real r1 = 0, r2 = 0, r3 = 0;
        for (int ki = (int)kdn; ki <= (int)kup; ++ki) {
          real kk = (real)(ki * ki);
          r1 += ((real)B * (real)cos(2 * pi * ki * (real)j / (real)ny) +
                 (real)C * (real)sin(2 * pi * ki * (real)k / (real)nz)) / kk;
          r2 += ((real)A * (real)sin(2 * pi * ki * (real)i / (real)nx) +
                 (real)C * (real)cos(2 * pi * ki * (real)k / (real)nz)) / kk;
          r3 += ((real)A * (real)cos(2 * pi * ki * (real)i / (real)nx) +
                 (real)B * (real)sin(2 * pi * ki * (real)j / (real)ny)) / kk;
        }
        R1[p] = r1; R2[p] = r2; R3[p] = r3;
      }
}

/* ------------------------------------------------------------------ */
/* RK: hd_rkstep1 (include/hd_rkstep1.f90:4-6) and hd_rkstep2
 * (include/hd_rkstep2.f90:3-32) under the DO o = ord,1,-1 loop of
 * main3D.fpp:3229-3231. */
void o_hd_rkstep1(const octx *c, const cplx *vx, const cplx *vy, const cplx *vz, cplx *C1, cplx *C2, cplx *C3) {
  memcpy(C1, vx, sizeof(cplx) * c->nspec);
  memcpy(C2, vy, sizeof(cplx) * c->nspec);
  memcpy(C3, vz, sizeof(cplx) * c->nspec);
}

void o_hd_rkstep2(const octx *c, int o, double dt_d, double nu_d, cplx *vx, cplx *vy, cplx *vz, const cplx *C1,
                  const cplx *C2, const cplx *C3, const cplx *fx, const cplx *fy, const cplx *fz) {
  size_t n = c->nspec;
  real dt = (real)dt_d, nu = (real)nu_d;
  cplx *C4 = (cplx *)malloc(sizeof(cplx) * n), *C5 = (cplx *)malloc(sizeof(cplx) * n),
       *C6 = (cplx *)malloc(sizeof(cplx) * n), *C7 = (cplx *)malloc(sizeof(cplx) * n),
       *C8 = (cplx *)malloc(sizeof(cplx) * n);
  o_prodre3(c, vx, vy, vz, C4, C5, C6);
  o_nonlhd3(c, C4, C5, C6, C7, 1);
  o_nonlhd3(c, C4, C5, C6, C8, 2);
  o_nonlhd3(c, C4, C5, C6, C4, 3);
  o_laplak3(c, vx, vx);
  o_laplak3(c, vy, vy);
  o_laplak3(c, vz, vz);
  real rmp = (real)1 / (real)o;
#pragma omp parallel for schedule(static)
  for (size_t p = 0; p < n; ++p) {
    if (c->kn2[p] <= c->kmax && c->kn2[p] >= c->tiny) {
      vx[p] = cadd(C1[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vx[p]), C7[p]), fx[p]))));
      vy[p] = cadd(C2[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vy[p]), C8[p]), fy[p]))));
      vz[p] = cadd(C3[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vz[p]), C4[p]), fz[p]))));
    } else {
      cplx z = {0, 0};
      vx[p] = z; vy[p] = z; vz[p] = z;
    }
  }
  free(C4); free(C5); free(C6); free(C7); free(C8);
}

/* The rand = 2 forcing update of main3D.fpp:2646-2657: f = (1-rmp) fold +
 * rmp fnew with rmp = FLOAT(timef+1)/float(fstep) in default REAL. */
void o_forcing_slow(const octx *c, int timef, int fstep, const cplx *const fold[3], const cplx *const fnew[3],
                    cplx *const f[3]) {
  const real rmp = (real)((float)(timef + 1) / (float)fstep);
  const real w0 = (real)1 - rmp;
  for (int a = 0; a < 3; ++a)
    for (size_t p = 0; p < c->nspec; ++p) {
      cplx o = fold[a][p], nw = fnew[a][p];
      f[a][p].re = w0 * o.re + rmp * nw.re;
      f[a][p].im = w0 * o.im + rmp * nw.im;
    }
}

/* nsteps full RK steps of the HD solver (f may be NULL: no forcing) */
void o_hd_run(const octx *c, int nsteps, int ord, double dt, double nu, cplx *vx, cplx *vy, cplx *vz,
              const cplx *fx, const cplx *fy, const cplx *fz) {
  size_t n = c->nspec;
  cplx *C1 = (cplx *)malloc(sizeof(cplx) * n), *C2 = (cplx *)malloc(sizeof(cplx) * n),
       *C3 = (cplx *)malloc(sizeof(cplx) * n);
  cplx *zf = NULL;
  if (!fx) {
    zf = (cplx *)calloc(n, sizeof(cplx));
    fx = fy = fz = zf;
  }
  for (int t = 0; t < nsteps; ++t) {
    o_hd_rkstep1(c, vx, vy, vz, C1, C2, C3);
    for (int o = ord; o >= 1; --o) o_hd_rkstep2(c, o, dt, nu, vx, vy, vz, C1, C2, C3, fx, fy, fz);
  }
  free(C1); free(C2); free(C3); free(zf);
}

/* ------------------------------------------------------------------ */
/* Boussinesq: advect3 (pseudo/pseudospec3D_phd.f90:23-114) gives
 * e = -(A.grad)B in Fourier space. */
void o_advect3(const octx *c, const cplx *a, const cplx *b, const cplx *cc, const cplx *d, cplx *e) {
  size_t nr = c->nreal;
  real *r1 = (real *)malloc(sizeof(real) * nr), *r2 = (real *)malloc(sizeof(real) * nr),
       *r3 = (real *)malloc(sizeof(real) * nr);
  cplx *c2 = (cplx *)malloc(sizeof(cplx) * c->nspec);
  const cplx *comp[3] = {a, b, cc};
  for (int dir = 1; dir <= 3; ++dir) {
    o_derivk3(c, d, c2, dir);
    o_fftp3d_complex_to_real(c, comp[dir - 1], r1);
    o_fftp3d_complex_to_real(c, c2, r2);
    if (dir == 1) {
      for (size_t p = 0; p < nr; ++p) r3[p] = r1[p] * r2[p];
    } else if (dir == 2) {
      for (size_t p = 0; p < nr; ++p) r3[p] = r3[p] + r1[p] * r2[p];
    } else {
      real tmp = -(real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
      for (size_t p = 0; p < nr; ++p) r3[p] = (r3[p] + r1[p] * r2[p]) * tmp;
    }
  }
  o_fftp3d_real_to_complex(c, r3, e);
  free(r1); free(r2); free(r3); free(c2);
}

/* rotbouss_rkstep2 (include/rotbouss_rkstep2.f90:12-83); xmom and xtemp
 * are already multiplied by bvfreq (main3D.fpp:973-974). */
void o_bouss_rkstep2(const octx *c, int o, double dt_d, double nu_d, double kappa_d, double omegaz_d,
                     double xmom_d, double xtemp_d, cplx *vx, cplx *vy, cplx *vz, cplx *th, const cplx *C1,
                     const cplx *C2, const cplx *C3, const cplx *C20, const cplx *fx, const cplx *fy,
                     const cplx *fz, const cplx *fs) {
  size_t n = c->nspec;
  real dt = (real)dt_d, nu = (real)nu_d, kappa = (real)kappa_d, omegaz = (real)omegaz_d;
  real xmom = (real)xmom_d, xtemp = (real)xtemp_d;
  cplx *C4 = (cplx *)malloc(sizeof(cplx) * n), *C5 = (cplx *)malloc(sizeof(cplx) * n),
       *C6 = (cplx *)malloc(sizeof(cplx) * n), *C7 = (cplx *)malloc(sizeof(cplx) * n),
       *C8 = (cplx *)malloc(sizeof(cplx) * n);
  o_prodre3(c, vx, vy, vz, C4, C5, C6);
  for (size_t p = 0; p < n; ++p) {
    C4[p] = csub(C4[p], cscal(2 * omegaz, vy[p]));
    C5[p] = cadd(C5[p], cscal(2 * omegaz, vx[p]));
    C6[p] = cadd(C6[p], cscal(xmom, th[p]));
  }
  o_nonlhd3(c, C4, C5, C6, C7, 1);
  o_nonlhd3(c, C4, C5, C6, C8, 2);
  o_nonlhd3(c, C4, C5, C6, C4, 3);
  o_advect3(c, vx, vy, vz, th, C5);
  for (size_t p = 0; p < n; ++p) C5[p] = cadd(C5[p], cscal(xtemp, vz[p]));
  o_laplak3(c, vx, vx);
  o_laplak3(c, vy, vy);
  o_laplak3(c, vz, vz);
  o_laplak3(c, th, th);
  real rmp = (real)1 / (real)o;
  cplx z = {0, 0};
  for (size_t p = 0; p < n; ++p) {
    if (c->kn2[p] <= c->kmax && c->kn2[p] >= c->tiny) {
      vx[p] = cadd(C1[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vx[p]), C7[p]), fx[p]))));
      vy[p] = cadd(C2[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vy[p]), C8[p]), fy[p]))));
      vz[p] = cadd(C3[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vz[p]), C4[p]), fz[p]))));
      th[p] = cadd(C20[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(kappa, th[p]), C5[p]), fs[p]))));
    } else if (c->kn2[p] > c->kmax) {
      vx[p] = z; vy[p] = z; vz[p] = z; th[p] = z;
    } else if (c->kn2[p] < c->tiny) {
      vx[p] = z; vy[p] = z; vz[p] = z; th[p] = C20[p];
    }
  }
  free(C4); free(C5); free(C6); free(C7); free(C8);
}

void o_bouss_run(const octx *c, int nsteps, int ord, double dt, double nu, double kappa, double omegaz,
                 double xmom, double xtemp, cplx *vx, cplx *vy, cplx *vz, cplx *th, const cplx *fx,
                 const cplx *fy, const cplx *fz, const cplx *fs) {
  size_t n = c->nspec;
  cplx *C1 = (cplx *)malloc(sizeof(cplx) * n), *C2 = (cplx *)malloc(sizeof(cplx) * n),
       *C3 = (cplx *)malloc(sizeof(cplx) * n), *C20 = (cplx *)malloc(sizeof(cplx) * n);
  cplx *zf = (cplx *)calloc(n, sizeof(cplx));
  if (!fx) fx = fy = fz = zf;
  if (!fs) fs = zf;
  for (int t = 0; t < nsteps; ++t) {
    memcpy(C1, vx, sizeof(cplx) * n); memcpy(C2, vy, sizeof(cplx) * n);
    memcpy(C3, vz, sizeof(cplx) * n); memcpy(C20, th, sizeof(cplx) * n);
    for (int o = ord; o >= 1; --o)
      o_bouss_rkstep2(c, o, dt, nu, kappa, omegaz, xmom, xtemp, vx, vy, vz, th, C1, C2, C3, C20, fx, fy, fz, fs);
  }
  free(C1); free(C2); free(C3); free(C20); free(zf);
}

/* sharp (pseudo/pseudospec3D_filt.f90:200-241): keep kn2 <= (pi/delta)^2 */
void o_sharp(const octx *c, const cplx *a, cplx *b, double delta) {
  const real pi = (real)3.14159265358979323846;
  real tmp = (pi / (real)delta) * (pi / (real)delta);
  cplx z = {0, 0};
  for (size_t p = 0; p < c->nspec; ++p) b[p] = c->kn2[p] <= tmp ? a[p] : z;
}

/* ------------------------------------------------------------------ */
/* EDQNM eddy viscosity (pseudo/pseudospec3D_edqnm.f90), heli = 0.
 * Spectra are DOUBLE PRECISION as in the Fortran; the fit and quadrature
 * locals are REAL(GP) = real; 0.218 and real(k*k) are default (single)
 * reals.  Arrays are 0-based copies of the 1-based Fortran ones. */

/* spec_fit (:278-402) */
static void o_spec_fit(const octx *c, const double *Ein, real delk, double *Efit, real *power_o, real *ddelta_o) {
  int n = c->nx;
  real tinyf = (real)1e-15 < (real)0.1 / ((real)c->nmax * (real)c->nmax) ? (real)1e-15
                                                                             : (real)0.1 / ((real)c->nmax * (real)c->nmax);
  int kc = (int)sqrt(c->kmax);
  int ktot = 3 * kc, ksup = kc, kinf = (int)((real)kc - delk);
  real power = -1, ddelta = -1, expo = 0;
  for (int k = 0; k < 3 * (n / 2 + 1); ++k) Efit[k] = 0;
  *power_o = power;
  *ddelta_o = ddelta;
  if (Ein[ksup - 1] <= (double)tinyf) return;
  real x = 0, y = 0, z = 0, v = 0, w = 0, m = 0, nn = 0, o = 0, p = 0;
  for (int i = kinf; i <= ksup; ++i) {
    real ii = (real)i;
    real lg = (real)log(Ein[i - 1] + (double)tinyf);
    x = x + (real)1.;
    y = y + (real)log(ii);
    z = z + lg;
    v = v + (real)log(ii) * lg;
    w = w + (real)log(ii) * (real)log(ii);
    m = m + ii;
    nn = nn + ii * (real)log(ii);
    o = o + ii * lg;
    p = p + ii * ii;
  }
  real pden = (w * p - nn * nn) * (x * nn - y * m) - (y * nn - w * m) * (y * p - m * nn);
  real pnum = ((z * nn - v * m) * (y * p - m * nn) - (v * p - o * nn) * (x * nn - y * m));
  real dden = x * nn - y * m;
  if (pden != 0 && dden != 0) {
    power = pnum / pden;
    expo = ((z * nn - v * m) - power * (w * m - y * nn)) / dden;
    ddelta = expo * x / m - power * y / m - z / m;
  }
  if (power >= 0 && ddelta >= 0) {
    expo = (real)exp(expo);
    for (int k = 1; k <= ksup; ++k) Efit[k - 1] = Ein[k - 1];
    for (int k = ksup + 1; k <= ktot; ++k) {
      real kk = (real)k;
      Efit[k - 1] = (double)(expo * (real)pow(kk, -power) * (real)exp(-ddelta * kk));
    }
  } else {
    x = 0; y = 0; z = 0; v = 0; w = 0;
    for (int i = kinf; i <= ksup; ++i) {
      real ii = (real)i;
      real lg = (real)log(Ein[i - 1] + (double)tinyf);
      x = x + (real)1.;
      y = y + (real)log(ii);
      z = z + lg;
      v = v + (real)log(ii) * lg;
      w = w + (real)log(ii) * (real)log(ii);
    }
    pden = y * y - w * x;
    pnum = (v * x - y * z);
    dden = x * y;
    if (pden != 0 && dden != 0) {
      power = pnum / pden;
      expo = (real)exp((y * z + power * y * y) / dden);
      for (int k = 1; k <= ksup; ++k) Efit[k - 1] = Ein[k - 1];
      for (int k = ksup + 1; k <= ktot; ++k) {
        real kk = (real)k;
        Efit[k - 1] = (double)(expo * (real)pow(kk, -power) + tinyf);
      }
    } else {
      for (int k = 1; k <= ksup; ++k) Efit[k - 1] = Ein[k - 1];
    }
  }
  *power_o = power;
  *ddelta_o = ddelta;
}

/* cusp (:95-171) */
static void o_cusp(const octx *c, real kolmo, const double *Ext, real nu, real t0, double *tepq, double *nut) {
  real lambda = (real)0.218f * (real)pow(kolmo, (real)1.5);
  int kc = (int)sqrt(c->kmax), ktot = 3 * kc;
  if (Ext[kc] == 0.) return;
  real *mu = (real *)calloc((size_t)ktot + 1, sizeof(real));
  real en = 0;
  for (int k = 1; k <= ktot; ++k) {
    real tmp = (real)(float)(k * k);
    en = (real)((double)en + (double)tmp * Ext[k - 1]);
    mu[k] = lambda * (real)sqrt(en);
  }
  for (int k = 1; k <= kc; ++k) {
    real kk = (real)k;
    for (int p = kc + 1; p <= ktot; ++p) {
      real pp = (real)p, ppi = (real)1.0 / pp;
      for (int q = p - k; q <= p; ++q) {
        real qq = (real)q, qqi;
        if (q == 0) continue;
        qqi = (real)1.0 / qq;
        real coeff = (real)0.5;
        if ((qq - (real)0.5) >= (pp - kk) && (qq + (real)0.5) <= pp) coeff = (real)1.0;
        real x = (pp * pp + qq * qq - kk * kk) / ((real)2.0 * pp * qq);
        real y = (kk * kk + qq * qq - pp * pp) / ((real)2.0 * kk * qq);
        real z = (pp * pp + kk * kk - qq * qq) / ((real)2.0 * pp * kk);
        real tvvkp = (real)((double)(-qqi * (x * y + z * z * z) * (pp * pp)) * Ext[q - 1] * Ext[k - 1]);
        real tvvkpsym = (real)((double)(-ppi * (x * z + y * y * y) * (qq * qq)) * Ext[p - 1] * Ext[k - 1]);
        real tmp = mu[k] + mu[p] + mu[q] + nu * (kk * kk + pp * pp + qq * qq);
        real frac = (real)1.0 / tmp;
        real theta = -(real)exp(-tmp * t0) / tmp;
        nut[k - 1] = nut[k - 1] - (double)(coeff * (frac + theta)) * (double)(tvvkp + tvvkpsym) /
                                      ((double)((real)2. * kk * kk) * Ext[k - 1]);
        tepq[k - 1] = tepq[k - 1] + (double)(coeff * (frac + theta)) * (double)(tvvkp + tvvkpsym);
      }
    }
  }
  free(mu);
}

/* full_cusp (:174-277): cusp with helicity.  Ext and Hxt are halved in
 * place first, as GHOST does.  Every GP product is rounded to GP before it
 * meets a double spectrum value, in GHOST's left-to-right order. */
static void o_full_cusp(const octx *c, real kolmo, double *Ext, double *Hxt, real nu, real t0, double *tepq,
                        double *thpq, double *nut, double *tvh) {
  real lambda = (real)0.218f * (real)pow(kolmo, (real)1.5);
  int kc = (int)sqrt(c->kmax), ktot = 3 * kc;
  if (Ext[kc] == 0.) return;
  for (int k = 1; k <= ktot; ++k) {
    Ext[k - 1] = 0.5 * Ext[k - 1];
    Hxt[k - 1] = 0.5 * Hxt[k - 1];
  }
  real *mu = (real *)calloc((size_t)ktot + 1, sizeof(real));
  real en = 0;
  for (int k = 1; k <= ktot; ++k) {
    real tmp = (real)(float)(k * k);
    en = (real)((double)en + (double)tmp * Ext[k - 1]);
    mu[k] = lambda * (real)sqrt(en);
  }
  for (int k = 1; k <= kc; ++k) {
    real kk = (real)k;
    for (int p = kc + 1; p <= ktot; ++p) {
      real pp = (real)p, ppi = (real)1.0 / pp;
      for (int q = p - k; q <= p; ++q) {
        if (q == 0) continue;
        real qq = (real)q, qqi = (real)1.0 / qq;
        real coeff = (real)0.5;
        if ((qq - (real)0.5) >= (pp - kk) && (qq + (real)0.5) <= pp) coeff = (real)1.0;
        real x = (pp * pp + qq * qq - kk * kk) / ((real)2.0 * pp * qq);
        real y = (kk * kk + qq * qq - pp * pp) / ((real)2.0 * kk * qq);
        real z = (pp * pp + kk * kk - qq * qq) / ((real)2.0 * pp * kk);
        real xyz = x * y + z * z * z, xzy = x * z + y * y * y;
        real ym1 = (real)1. - y * y, zm1 = (real)1. - z * z;
        double Eq = Ext[q - 1], Ek = Ext[k - 1], Ep = Ext[p - 1];
        double Hq = Hxt[q - 1], Hk = Hxt[k - 1], Hp = Hxt[p - 1];
        real tvvkp = (real)((double)(-(qqi * xyz * (pp * pp))) * Eq * Ek);
        real tvvpq = (real)((double)(qqi * xyz * (kk * kk)) * Eq * Ep);
        real tvvkpsym = (real)((double)(-(ppi * xzy * (qq * qq))) * Ep * Ek);
        real tvvpqsym = (real)((double)(ppi * xzy * (kk * kk)) * Eq * Ep);
        real twwpq = (real)((double)(-(z * ym1 * kk * kk)) * Hp * Hq / (double)(pp * pp * qq));
        real twwkp = (real)((double)(z * ym1) * Hk * Hq * (double)qqi);
        real twwpqsym = (real)((double)(-(y * zm1 * kk * kk)) * Hp * Hq / (double)(pp * qq * qq));
        real twwkpsym = (real)((double)(y * zm1) * Hk * Hp * (double)ppi);
        real tvw = (real)((double)(qqi * xyz * kk * kk) * Eq * Hp + (double)(ppi * xzy * kk * kk) * Hq * Ep -
                          (double)(qqi * z * ym1 * kk * kk) * Ep * Hq - (double)(ppi * y * zm1 * kk * kk) * Eq * Hp);
        real tmp = mu[k] + mu[p] + mu[q] + nu * (kk * kk + pp * pp + qq * qq);
        real theta = ((real)1.0 - (real)exp(-tmp * t0)) / tmp;
        real ct = coeff * theta;
        nut[k - 1] = nut[k - 1] - (double)(ct * (tvvkp + tvvkpsym)) / ((double)((real)2. * kk * kk) * Ek);
        tepq[k - 1] = tepq[k - 1] + (double)(ct * (tvvpq + tvvpqsym + twwpq + twwpqsym));
        tvh[k - 1] = tvh[k - 1] + (double)(ct * (twwkp + twwkpsym)) / (2. * Hk);
        thpq[k - 1] = thpq[k - 1] + (double)(ct * tvw);
      }
    }
  }
  free(mu);
}

/* evedqnm (:24-92): Eold, Hold[n/2+1] -> tepq, thpq, tve, tvh[n/2+1] and
 * Ext, Hxt[3(n/2+1)].  hel = 1 fits E over delk - 2 shells and H over delk,
 * then full_cusp when both fits have positive index, else cusp. */
void o_evedqnm_h(const octx *c, double kolmo, const double *Eold, const double *Hold, double nu, double time, int hel,
                 double *tepq, double *thpq, double *tve, double *tvh, double *Ext, double *Hxt) {
  int n = c->nx, kc = (int)sqrt(c->kmax);
  real delk = (real)3. * (real)kc / (real)4.;
  for (int k = 0; k < n / 2 + 1; ++k) tve[k] = tvh[k] = tepq[k] = thpq[k] = 0.;
  real power, ddelta, hpower, hddelta;
  if (hel == 1) {
    o_spec_fit(c, Eold, delk - (real)2, Ext, &power, &ddelta);
    o_spec_fit(c, Hold, delk, Hxt, &hpower, &hddelta);
    if (power > 0) {
      if (hpower > 0)
        o_full_cusp(c, (real)kolmo, Ext, Hxt, (real)nu, (real)time, tepq, thpq, tve, tvh);
      else
        o_cusp(c, (real)kolmo, Ext, (real)nu, (real)time, tepq, tve);
    }
  } else {
    o_spec_fit(c, Eold, delk, Ext, &power, &ddelta);
    if (power > 0) o_cusp(c, (real)kolmo, Ext, (real)nu, (real)time, tepq, tve);
  }
}

/* evedqnm (:24-92) with hel = 0: Eold[n/2+1] -> tepq, tve[n/2+1], Ext[3(n/2+1)] */
void o_evedqnm(const octx *c, double kolmo, const double *Eold, double nu, double time, double *tepq, double *tve,
               double *Ext) {
  int n = c->nx, kc = (int)sqrt(c->kmax);
  real delk = (real)3. * (real)kc / (real)4.;
  for (int k = 0; k < n / 2 + 1; ++k) tve[k] = tepq[k] = 0.;
  real power, ddelta;
  o_spec_fit(c, Eold, delk, Ext, &power, &ddelta);
  if (power > 0) o_cusp(c, (real)kolmo, Ext, (real)nu, (real)time, tepq, tve);
}

/* include/edqnmhd_rkstep2.f90 with heli = 0, without the closing vcorrect:
 * the update of :41-58 with (nu + tve(ki)) times the Laplacian */
void o_vcorrect(const octx *c, cplx *vx, cplx *vy, cplx *vz, const real *ef, const double *tepq, const double *eold,
                double dt_d);
void o_vcorrect_h(const octx *c, cplx *vx, cplx *vy, cplx *vz, const real *ef, const real *hf, const double *tepq,
                  const double *thpq, const double *eold, const double *hold, double dt_d, int hel);

void o_edqnm_rkstep2(const octx *c, int o, double dt_d, double nu_d, const double *tve, const double *tepq,
                     const double *eold, int vcorr, cplx *vx, cplx *vy, cplx *vz, const cplx *C1, const cplx *C2,
                     const cplx *C3, const cplx *fx, const cplx *fy, const cplx *fz) {
  size_t n = c->nspec;
  real dt = (real)dt_d, nu = (real)nu_d;
  /* Eden of edqnmhd_rkstep2.f90:8-10, from the velocity before the update */
  real *ef = NULL;
  if (vcorr) {
    const real rmp = (real)1 / ((real)c->nx * (real)c->nx * (real)c->nx * (real)c->nx * (real)c->nx * (real)c->nx);
    ef = (real *)malloc(sizeof(real) * n);
    for (size_t p = 0; p < n; ++p) ef[p] = (cabs2(vx[p]) + cabs2(vy[p]) + cabs2(vz[p])) * rmp;
  }
  cplx *C4 = (cplx *)malloc(sizeof(cplx) * n), *C5 = (cplx *)malloc(sizeof(cplx) * n),
       *C6 = (cplx *)malloc(sizeof(cplx) * n), *C7 = (cplx *)malloc(sizeof(cplx) * n),
       *C8 = (cplx *)malloc(sizeof(cplx) * n);
  o_prodre3(c, vx, vy, vz, C4, C5, C6);
  o_nonlhd3(c, C4, C5, C6, C7, 1);
  o_nonlhd3(c, C4, C5, C6, C8, 2);
  o_nonlhd3(c, C4, C5, C6, C4, 3);
  o_laplak3(c, vx, vx);
  o_laplak3(c, vy, vy);
  o_laplak3(c, vz, vz);
  real rmp = (real)1. / (real)o;
#pragma omp parallel for schedule(static)
  for (size_t p = 0; p < n; ++p) {
    if (c->kn2[p] <= c->kmax && c->kn2[p] >= c->tiny) {
      int ki = (int)((real)sqrt(c->kk2[p]) + (real)0.501f);
      double nt = (double)nu + tve[ki - 1];
      cplx *v[3] = {&vx[p], &vy[p], &vz[p]};
      const cplx *C[3] = {&C1[p], &C2[p], &C3[p]}, *N[3] = {&C7[p], &C8[p], &C4[p]}, *F[3] = {&fx[p], &fy[p], &fz[p]};
      for (int a = 0; a < 3; ++a) {
        double re = (double)C[a]->re + (double)dt * (nt * v[a]->re + N[a]->re + F[a]->re) * (double)rmp;
        double im = (double)C[a]->im + (double)dt * (nt * v[a]->im + N[a]->im + F[a]->im) * (double)rmp;
        v[a]->re = (real)re;
        v[a]->im = (real)im;
      }
    } else {
      cplx z = {0, 0};
      vx[p] = z; vy[p] = z; vz[p] = z;
    }
  }
  free(C4); free(C5); free(C6); free(C7); free(C8);
  if (vcorr) {
    o_vcorrect(c, vx, vy, vz, ef, tepq, eold, (double)(dt * rmp));
    free(ef);
  }
}

/* include/edqnmhd_rkstep2.f90 with heli (:1-63): Eden and Hden of the
 * velocity before the update, prodre3 and nonlhd3, w = curl v (rotor3), the
 * update C + dt ((nu + tve(ki)) lap v + NL + tvh(ki) w + f) / o on the kept
 * modes, then vcorrect with hel (when vcorr).  tvh and thpq are zero arrays
 * for heli = 0, which leaves the update of o_edqnm_rkstep2 bit for bit. */
void o_edqnm_rkstep2_h(const octx *c, int o, double dt_d, double nu_d, int hel, const double *tve, const double *tvh,
                       const double *tepq, const double *thpq, const double *eold, const double *hold, int vcorr,
                       cplx *vx, cplx *vy, cplx *vz, const cplx *C1, const cplx *C2, const cplx *C3, const cplx *fx,
                       const cplx *fy, const cplx *fz) {
  size_t n = c->nspec;
  real dt = (real)dt_d, nu = (real)nu_d;
  real *ef = NULL, *hf = NULL;
  if (vcorr) {
    const real rmp = (real)1 / ((real)c->nx * (real)c->nx * (real)c->nx * (real)c->nx * (real)c->nx * (real)c->nx);
    ef = (real *)malloc(sizeof(real) * n);
    hf = (real *)malloc(sizeof(real) * n);
    for (int i = 0; i < c->nxh; ++i)
      for (int j = 0; j < c->ny; ++j)
        for (int k = 0; k < c->nz; ++k) {
          const size_t p = SIDX(c, k, j, i);
          ef[p] = (cabs2(vx[p]) + cabs2(vy[p]) + cabs2(vz[p])) * rmp;
          real a = c->kz[k] * (vx[p].re * vy[p].im - vy[p].re * vx[p].im);
          real b = c->ky[j] * (vz[p].re * vx[p].im - vx[p].re * vz[p].im);
          real d = c->kx[i] * (vy[p].re * vz[p].im - vz[p].re * vy[p].im);
          hf[p] = (real)2 * rmp * (a + b + d);
        }
  }
  cplx *C4 = (cplx *)malloc(sizeof(cplx) * n), *C5 = (cplx *)malloc(sizeof(cplx) * n),
       *C6 = (cplx *)malloc(sizeof(cplx) * n), *C7 = (cplx *)malloc(sizeof(cplx) * n),
       *C8 = (cplx *)malloc(sizeof(cplx) * n), *C19 = (cplx *)malloc(sizeof(cplx) * n);
  o_prodre3(c, vx, vy, vz, C4, C5, C6);
  o_nonlhd3(c, C4, C5, C6, C7, 1);
  o_nonlhd3(c, C4, C5, C6, C8, 2);
  o_nonlhd3(c, C4, C5, C6, C4, 3);
  o_rotor3(c, vy, vz, C5, 1);
  o_rotor3(c, vx, vz, C6, 2);
  o_rotor3(c, vx, vy, C19, 3);
  o_laplak3(c, vx, vx);
  o_laplak3(c, vy, vy);
  o_laplak3(c, vz, vz);
  real rmp = (real)1. / (real)o;
#pragma omp parallel for schedule(static)
  for (size_t p = 0; p < n; ++p) {
    if (c->kn2[p] <= c->kmax && c->kn2[p] >= c->tiny) {
      int ki = (int)((real)sqrt(c->kk2[p]) + (real)0.501f);
      double nt = (double)nu + tve[ki - 1], th = tvh[ki - 1];
      cplx *v[3] = {&vx[p], &vy[p], &vz[p]};
      const cplx *C[3] = {&C1[p], &C2[p], &C3[p]}, *N[3] = {&C7[p], &C8[p], &C4[p]}, *F[3] = {&fx[p], &fy[p], &fz[p]};
      const cplx *W[3] = {&C5[p], &C6[p], &C19[p]};
      for (int a = 0; a < 3; ++a) {
        double re = (double)C[a]->re + (double)dt * (nt * v[a]->re + N[a]->re + th * W[a]->re + F[a]->re) * (double)rmp;
        double im = (double)C[a]->im + (double)dt * (nt * v[a]->im + N[a]->im + th * W[a]->im + F[a]->im) * (double)rmp;
        v[a]->re = (real)re;
        v[a]->im = (real)im;
      }
    } else {
      cplx z = {0, 0};
      vx[p] = z; vy[p] = z; vz[p] = z;
    }
  }
  free(C4); free(C5); free(C6); free(C7); free(C8); free(C19);
  if (vcorr) {
    o_vcorrect_h(c, vx, vy, vz, ef, hf, tepq, thpq, eold, hold, (double)(dt * rmp), hel);
    free(ef);
    free(hf);
  }
}

/* nsteps RK steps of the EDQNM LES with heli: per substep spectrumc (E and,
 * for hel = 1, H) -> evedqnm at t0 + (step index) dt -> edqnm_rkstep2 */
void o_edqnm_run_h(const octx *c, int nsteps, int ord, double dt, double nu, double kolmo, double t0, int vcorr,
                   int hel, cplx *vx, cplx *vy, cplx *vz, const cplx *fx, const cplx *fy, const cplx *fz) {
  size_t n = c->nspec;
  int nb = c->nx / 2 + 1;
  cplx *C1 = (cplx *)malloc(sizeof(cplx) * n), *C2 = (cplx *)malloc(sizeof(cplx) * n),
       *C3 = (cplx *)malloc(sizeof(cplx) * n), *zf = NULL;
  double *Ek = (double *)calloc(nb, sizeof(double)), *Hk = (double *)calloc(nb, sizeof(double)),
         *tepq = (double *)calloc(nb, sizeof(double)), *thpq = (double *)calloc(nb, sizeof(double)),
         *tve = (double *)calloc(nb, sizeof(double)), *tvh = (double *)calloc(nb, sizeof(double)),
         *Ext = (double *)calloc(3 * nb, sizeof(double)), *Hxt = (double *)calloc(3 * nb, sizeof(double));
  if (!fx) {
    zf = (cplx *)calloc(n, sizeof(cplx));
    fx = fy = fz = zf;
  }
  for (int t = 0; t < nsteps; ++t) {
    o_hd_rkstep1(c, vx, vy, vz, C1, C2, C3);
    for (int o = ord; o >= 1; --o) {
      o_spectrumc(c, vx, vy, vz, 1, hel, Ek, Hk);
      o_evedqnm_h(c, kolmo, Ek, Hk, nu, t0 + t * dt, hel, tepq, thpq, tve, tvh, Ext, Hxt);
      o_edqnm_rkstep2_h(c, o, dt, nu, hel, tve, tvh, tepq, thpq, Ek, Hk, vcorr, vx, vy, vz, C1, C2, C3, fx, fy, fz);
    }
  }
  free(C1); free(C2); free(C3); free(zf); free(Ek); free(Hk); free(tepq); free(thpq); free(tve); free(tvh);
  free(Ext); free(Hxt);
}

/* nsteps RK steps of the EDQNM LES: per substep spectrumc -> evedqnm at
 * time t0 + (step index) dt -> edqnm_rkstep2 (f may be NULL) */
void o_edqnm_run(const octx *c, int nsteps, int ord, double dt, double nu, double kolmo, double t0, int vcorr,
                 cplx *vx, cplx *vy, cplx *vz, const cplx *fx, const cplx *fy, const cplx *fz) {
  size_t n = c->nspec;
  int nb = c->nx / 2 + 1;
  cplx *C1 = (cplx *)malloc(sizeof(cplx) * n), *C2 = (cplx *)malloc(sizeof(cplx) * n),
       *C3 = (cplx *)malloc(sizeof(cplx) * n), *zf = NULL;
  double *Ek = (double *)calloc(nb, sizeof(double)), *tepq = (double *)calloc(nb, sizeof(double)),
         *tve = (double *)calloc(nb, sizeof(double)), *Ext = (double *)calloc(3 * nb, sizeof(double));
  if (!fx) {
    zf = (cplx *)calloc(n, sizeof(cplx));
    fx = fy = fz = zf;
  }
  for (int t = 0; t < nsteps; ++t) {
    o_hd_rkstep1(c, vx, vy, vz, C1, C2, C3);
    for (int o = ord; o >= 1; --o) {
      o_spectrumc(c, vx, vy, vz, 1, 0, Ek, NULL);
      o_evedqnm(c, kolmo, Ek, nu, t0 + t * dt, tepq, tve, Ext);
      o_edqnm_rkstep2(c, o, dt, nu, tve, tepq, Ek, vcorr, vx, vy, vz, C1, C2, C3, fx, fy, fz);
    }
  }
  free(C1); free(C2); free(C3); free(zf); free(Ek); free(tepq); free(tve); free(Ext);
}

/* Modes |k|^2 <= kc^2 of the fine spectrum (ctx f) on the coarse grid (ctx
 * c), times (n/N)^3 (analysis/trunc3D.fpp with GHOST's sharp cutoff). */
void o_les_truncate(const octx *f, const octx *c, const cplx *in, cplx *out, int kc) {
  int n = c->nx, N = f->nx;
  real scale = (real)((double)c->nreal / (double)f->nreal);
  for (int i = 0; i < c->nxh; ++i)
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < n; ++k) {
        int kx = i < n / 2 ? i : i - n, ky = j < n / 2 ? j : j - n, kz = k < n / 2 ? k : k - n;
        cplx v = {0, 0};
        if (kx >= 0 && kx * kx + ky * ky + kz * kz <= kc * kc) {
          int jf = ky >= 0 ? ky : ky + N, kf = kz >= 0 ? kz : kz + N;
          v = cscal(scale, in[SIDX(f, kf, jf, kx)]);
        }
        out[SIDX(c, k, j, i)] = v;
      }
}

/* kmax override (main3D.fpp sets kmax once; LES runs set it to kc^2) */
void o_ctx_set_kmax(octx *c, double kmax) { c->kmax = (real)kmax; }

/* ------------------------------------------------------------------ */
/* vcorrect (pseudo/pseudospec3D_edqnm.f90:405-1629), heli = 0: after the
 * eddy-viscous update, every resolved mode is rescaled so that its energy
 * becomes E = |v|^2 + 2 tepq(km) dt ef / eold(km) while its helicity H
 * (hel = 0: the mode's own w2) is kept, by rebuilding the amplitudes and
 * relative phases of the components.  The seven routines of the Fortran
 * handle the geometries where some wavenumber components vanish; the
 * locals are DOUBLE PRECISION there and here.  v6 = (vxr,vxi,vyr,vyi,vzr,vzi)
 * already divided by n^3. */
static double o_sgn(double x) { return copysign(1.0, x); }
static void o_phase(double r, double im, double eps, double *c, double *s, double *t) {
  const double pi = 3.14159265358979323846;
  *c = r / (sqrt(r * r + im * im) + eps);
  *s = im / (sqrt(r * r + im * im) + eps);
  *t = *s > 0. ? acos(*c) : 2.0 * pi - acos(*c);
}
/* the common energy ratio of the first branches */
static double o_ratio(double E, double H, double v2, double w2, double kk2) {
  return (E * sqrt(1. - H * H / (0.25 * kk2 * (E * E)))) / (v2 * sqrt(1. - w2 * w2 / (0.25 * kk2 * (v2 * v2))));
}
/* the three reconstructions of the three-component geometries */
static void o_rebuild3(double *v, double mx, double my, double mz, double cx, double sx, double cy, double sy,
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

static void o_vcorr_general(double kx, double ky, double kz, double kk2, double E, double H, double v2, double w2,
                            double cx, double sx, double cy, double sy, double cz, double sz, double txy, double tzx,
                            double tyz, double *v);

/* One mode.  zx/zy/zz: the wavenumber component is zero (index 1 in the
 * Fortran).  kx..kz and kk2 are the GP tables; E and H as above. */
static void o_vcorr_mode(int zx, int zy, int zz, double kx, double ky, double kz, double kk2, double E, double dH,
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
  /* heli = 1: H = w2 + thpq(km) dt hf / hold(km), the caller's dH (:536-540) */
  const double H = w2 + dH;
  const double eps = (!zx && !zy && zz) ? tinyf : 0.;  /* only vcorr_xnynz0 pads the moduli */
  if (zx && zy) {            /* x, y only; kz != 0 */
    o_phase(v[0], v[1], 0., &cx, &sx, &tx);
    o_phase(v[2], v[3], 0., &cy, &sy, &ty);
    const double txy = ty - tx, tmp = o_ratio(E, H, v2, w2, kk2);
    const double vx2 = tmp * (v[0] * v[0] + v[1] * v[1] - 0.5 * v2) + 0.5 * E;
    const double vy2 = tmp * (v[2] * v[2] + v[3] * v[3] - 0.5 * v2) + 0.5 * E;
    const double mx = sqrt(fabs(vx2)), my = sqrt(fabs(vy2));
    double sxy = H;
    const double dsxy = kz * mx * my;
    if (o_sgn(vx2) >= 0. && o_sgn(vy2) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0.) {
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
    o_phase(v[0], v[1], 0., &cx, &sx, &tx);
    o_phase(v[4], v[5], 0., &cz, &sz, &tz);
    const double tzx = tx - tz, tmp = o_ratio(E, H, v2, w2, kk2);
    const double vx2 = tmp * (v[0] * v[0] + v[1] * v[1] - 0.5 * v2) + 0.5 * E;
    const double vz2 = tmp * (v[4] * v[4] + v[5] * v[5] - 0.5 * v2) + 0.5 * E;
    const double mx = sqrt(fabs(vx2)), mz = sqrt(fabs(vz2));
    double szx = H;
    const double dszx = ky * mx * mz;
    if (o_sgn(vx2) >= 0. && o_sgn(vz2) >= 0. && fabs(szx) <= fabs(dszx) && dszx != 0.) {
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
    o_phase(v[2], v[3], 0., &cy, &sy, &ty);
    o_phase(v[4], v[5], 0., &cz, &sz, &tz);
    const double tyz = tz - ty, tmp = o_ratio(E, H, v2, w2, kk2);
    const double vy2 = tmp * (v[2] * v[2] + v[3] * v[3] - 0.5 * v2) + 0.5 * E;
    const double vz2 = tmp * (v[4] * v[4] + v[5] * v[5] - 0.5 * v2) + 0.5 * E;
    const double my = sqrt(fabs(vy2)), mz = sqrt(fabs(vz2));
    double syz = H;
    const double dsyz = kx * mz * my;
    if (o_sgn(vy2) >= 0. && o_sgn(vz2) >= 0. && fabs(syz) <= fabs(dsyz) && dsyz != 0.) {
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
    o_phase(v[0], v[1], eps, &cx, &sx, &tx);
    o_phase(v[2], v[3], eps, &cy, &sy, &ty);
    o_phase(v[4], v[5], eps, &cz, &sz, &tz);
    const double txy = ty - tx, tzx = tx - tz, tyz = tz - ty;
    if (zx || zy || zz) {
      /* one vanishing component of k (vcorr_x0ynzn, vcorr_xny0zn, vcorr_xnynz0):
       * the mode along that axis takes its share of E, the other two split
       * the rest in proportion to the other axes' k^2 */
      const double tmp0 = o_ratio(E, H, v2, w2, kk2);
      double ma, mb, mc, tmp3, t1;
      if (zx) {
        const double vx2 = tmp0 * (v[0] * v[0] + v[1] * v[1] - 0.5 * v2) + 0.5 * E;
        t1 = o_sgn(vx2); ma = sqrt(fabs(vx2)); tmp3 = E - vx2;
        const double tt = 1. / (ky2 + kz2);
        mb = sqrt(fabs(tmp3) * kz2 * tt); mc = sqrt(fabs(tmp3) * ky2 * tt);  /* my, mz */
        const double mx = ma, my = mb, mz = mc;
        double sxy = kz * H, szx = ky * H;
        const double dsxy = (ky2 + kz2) * mx * my, dszx = (ky2 + kz2) * mx * mz;
        if (t1 >= 0. && o_sgn(tmp3) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. && fabs(szx) <= fabs(dszx) &&
            dszx != 0.) {
          sxy = sxy / dsxy; szx = szx / dszx;
          double cxy = sqrt(1. - sxy * sxy), czx = sqrt(1. - szx * szx);
          if (cos(txy) < 0.) cxy = -cxy;
          if (cos(tzx) < 0.) czx = -czx;
          const double syz = -szx * cxy - sxy * czx, cyz = czx * cxy - szx * sxy;
          o_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                     my >= mx && my >= mz, mz >= mx && mz >= my);
        }
      } else if (zy) {
        const double vy2 = tmp0 * (v[2] * v[2] + v[3] * v[3] - 0.5 * v2) + 0.5 * E;
        t1 = o_sgn(vy2); mb = sqrt(vy2); tmp3 = E - vy2;
        const double tt = 1. / (kx2 + kz2);
        ma = sqrt(fabs(tmp3) * kz2 * tt); mc = sqrt(fabs(tmp3) * kx2 * tt);
        const double mx = ma, my = mb, mz = mc;
        double sxy = kz * H, syz = kx * H;
        const double dsxy = (kx2 + kz2) * mx * my, dsyz = (kx2 + kz2) * my * mz;
        if (t1 >= 0. && o_sgn(tmp3) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. && fabs(syz) <= fabs(dsyz) &&
            dsyz != 0.) {
          sxy = sxy / dsxy; syz = syz / dsyz;
          double cxy = sqrt(1. - sxy * sxy), cyz = sqrt(1. - syz * syz);
          if (cos(txy) < 0.) cxy = -cxy;
          if (cos(tyz) < 0.) cyz = -cyz;
          const double szx = -sxy * cyz - syz * cxy, czx = cxy * cyz - sxy * syz;
          o_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                     my >= mx && my >= mz, mz >= mx && mz >= my);
        }
      } else {
        const double vz2 = tmp0 * ((v[4] * v[4] + v[5] * v[5]) - 0.5 * v2) + 0.5 * E;
        t1 = o_sgn(vz2); mc = sqrt(fabs(vz2)); tmp3 = E - vz2;
        const double tt = 1. / (kx2 + ky2);
        ma = sqrt(fabs(tmp3) * ky2 * tt); mb = sqrt(fabs(tmp3) * kx2 * tt);
        const double mx = ma, my = mb, mz = mc;
        double szx = ky * H, syz = kx * H;
        const double dszx = (kx2 + ky2) * mx * mz, dsyz = (kx2 + ky2) * my * mz;
        if (t1 >= 0. && o_sgn(tmp3) >= 0. && fabs(szx) <= fabs(dszx) && dszx != 0. && fabs(syz) <= fabs(dsyz) &&
            dsyz != 0.) {
          szx = szx / dszx; syz = syz / dsyz;
          double czx = sqrt(1. - szx * szx), cyz = sqrt(1. - syz * syz);
          if (cos(tzx) < 0.) czx = -czx;
          if (cos(tyz) < 0.) cyz = -cyz;
          const double sxy = -syz * czx - szx * cyz, cxy = cyz * czx - syz * szx;
          o_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                     my >= mx && my >= mz, mz >= mx && mz >= my);
        }
      }
    } else {
      o_vcorr_general(kx, ky, kz, kk2, E, H, v2, w2, cx, sx, cy, sy, cz, sz, txy, tzx, tyz, v);
    }
  }
}

/* vcorr_xnynzn (:1377-1629): all components of k non-zero */
static void o_vcorr_general(double kx, double ky, double kz, double kk2, double E, double H, double v2, double w2,
                            double cx, double sx, double cy, double sy, double cz, double sz, double txy, double tzx,
                            double tyz, double *v) {
  const double kx2 = kx * kx, ky2 = ky * ky, kz2 = kz * kz;
  const double fx = 1. - kx2 / kk2, fy = 1. - ky2 / kk2, fz = 1. - kz2 / kk2;
  const double tmq = o_ratio(E, H, v2, w2, kk2);
  double vx2 = tmq * (v[0] * v[0] + v[1] * v[1] - fx * 0.5 * v2) + fx * 0.5 * E;
  const double vy2 = tmq * (v[2] * v[2] + v[3] * v[3] - fy * 0.5 * v2) + fy * 0.5 * E;
  const double vz2 = tmq * (v[4] * v[4] + v[5] * v[5] - fz * 0.5 * v2) + fz * 0.5 * E;
  double mx = sqrt(fabs(vx2)), my = sqrt(fabs(vy2)), mz = sqrt(fabs(vz2));
  double szx = H * ky, dszx = kk2 * mx * mz, sxy = H * kz, dsxy = kk2 * my * mx, syz = H * kx, dsyz = kk2 * my * mz;
  double czx = (ky2 * E - mx * mx * (kx2 + ky2) - mz * mz * (ky2 + kz2)), dczx = 2. * kx * kz * mx * mz;
  double cxy = (kz2 * E - mx * mx * (kx2 + kz2) - my * my * (ky2 + kz2)), dcxy = 2. * kx * ky * mx * my;
  double cyz = (kx2 * E - my * my * (kx2 + ky2) - mz * mz * (kx2 + kz2)), dcyz = 2. * ky * kz * my * mz;
  if (o_sgn(vx2) >= 0. && o_sgn(vy2) >= 0. && o_sgn(vz2) >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. &&
      fabs(szx) <= fabs(dszx) && dszx != 0. && fabs(syz) <= fabs(dsyz) && dsyz != 0. && fabs(cxy) <= fabs(dcxy) &&
      dcxy != 0. && fabs(cyz) <= fabs(dcyz) && dcyz != 0. && fabs(czx) <= fabs(dczx) && dczx != 0.) {
    szx /= dszx; sxy /= dsxy; syz /= dsyz; czx /= dczx; cxy /= dcxy; cyz /= dcyz;
    o_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
               my > mx && my >= mz, mz > mx && mz > my);
  } else {
    const double hh = sqrt(1. - H * H / (0.25 * (E * E) * kk2));
    const double hi = fx * 0.5 * E * (1. + hh), lo = fx * 0.5 * E * (1. - hh);
    if (vx2 > hi) vx2 = hi;
    if (vx2 < lo) vx2 = lo;
    const double t1 = o_sgn(vx2);
    mx = sqrt(fabs(vx2));
    const double a2 = 2. * ((ky2 + kz2) * (ky2 + kz2)), iq = 1. / a2;
    double tmp4 = kx2 * ky2 * kz2 *
                  (-((mx * mx) * (mx * mx)) * kk2 + mx * mx * (ky2 + kz2) * E -
                   H * H * ((ky2 + kz2) * (ky2 + kz2)) / (kk2 * kk2));
    const double t0 = o_sgn(tmp4), delta = 4. * sqrt(fabs(tmp4)) * iq;
    tmp4 = (-vx2 * (2. * (kx2 + kz2) * (ky2 + kz2) - 4. * kx2 * ky2) + 2. * kz2 * E * (ky2 + kz2)) * iq + delta;
    const double t2 = o_sgn(tmp4);
    my = sqrt(fabs(tmp4));
    tmp4 = (-vx2 * (2. * (kx2 + ky2) * (ky2 + kz2) - 4. * kx2 * kz2) + 2. * ky2 * E * (ky2 + kz2)) * iq - delta;
    const double t3 = o_sgn(tmp4);
    mz = sqrt(fabs(tmp4));
    szx = H * ky; dszx = kk2 * mx * mz; sxy = H * kz; dsxy = kk2 * my * mx; syz = H * kx; dsyz = kk2 * my * mz;
    czx = (ky2 * E - mx * mx * (kx2 + ky2) - mz * mz * (ky2 + kz2)); dczx = 2. * kx * kz * mx * mz;
    cxy = (kz2 * E - mx * mx * (kx2 + kz2) - my * my * (ky2 + kz2)); dcxy = 2. * kx * ky * mx * my;
    cyz = (kx2 * E - my * my * (kx2 + ky2) - mz * mz * (kx2 + kz2)); dcyz = 2. * ky * kz * my * mz;
    if (t0 >= 0. && t1 >= 0. && t2 >= 0. && t3 >= 0. && fabs(sxy) <= fabs(dsxy) && dsxy != 0. &&
        fabs(szx) <= fabs(dszx) && dszx != 0. && fabs(syz) <= fabs(dsyz) && dsyz != 0. && fabs(czx) <= fabs(dczx) &&
        dczx != 0. && fabs(cxy) <= fabs(dcxy) && dcxy != 0. && fabs(cyz) <= fabs(dcyz) && dcyz != 0.) {
      szx /= dszx; sxy /= dsxy; syz /= dsyz; czx /= dczx; cxy /= dcxy; cyz /= dcyz;
      o_rebuild3(v, mx, my, mz, cx, sx, cy, sy, cz, sz, cxy, sxy, czx, szx, cyz, syz, mx >= my && mx >= mz,
                 my >= mx && my >= mz, mz >= mx && mz >= my);
    }
  }
  (void)txy; (void)tzx; (void)tyz;
}

/* vcorrect over every resolved mode but the origin; ef: Eden of the
 * substep's start, (|vx|^2+|vy|^2+|vz|^2)/n^6 per mode (edqnmhd_rkstep2.f90:
 * 8-10); tepq, eold: 0-based copies of the shell arrays; dt: dt/o. */
void o_vcorrect_h(const octx *c, cplx *vx, cplx *vy, cplx *vz, const real *ef, const real *hf, const double *tepq,
                  const double *thpq, const double *eold, const double *hold, double dt_d, int hel);
void o_vcorrect(const octx *c, cplx *vx, cplx *vy, cplx *vz, const real *ef, const double *tepq, const double *eold,
                double dt_d) {
  o_vcorrect_h(c, vx, vy, vz, ef, NULL, tepq, NULL, eold, NULL, dt_d, 0);
}

/* vcorrect (:405-470) with hel: hf is Hden of the substep's start, thpq and
 * hold the helicity transfer and spectrum (hel = 1 only) */
void o_vcorrect_h(const octx *c, cplx *vx, cplx *vy, cplx *vz, const real *ef, const real *hf, const double *tepq,
                  const double *thpq, const double *eold, const double *hold, double dt_d, int hel) {
  const real dt = (real)dt_d;
  const real norm = (real)c->nx * (real)c->nx * (real)c->nx;
  const double inorm = 1. / (double)norm;
  const real tinyf = (real)1e-15 < (real)0.1 / ((real)c->nmax * (real)c->nmax) ? (real)1e-15
                                                                             : (real)0.1 / ((real)c->nmax * (real)c->nmax);
  for (int i = 0; i < c->nxh; ++i)
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        if (i == 0 && j == 0 && k == 0) continue;
        const size_t p = SIDX(c, k, j, i);
        if (c->kn2[p] > c->kmax) continue;
        const int km = (int)((real)sqrt(c->kk2[p]) + (real)0.501f);
        double v[6] = {(double)vx[p].re * inorm, (double)vx[p].im * inorm, (double)vy[p].re * inorm,
                       (double)vy[p].im * inorm, (double)vz[p].re * inorm, (double)vz[p].im * inorm};
        /* E needs v2 of the geometry's components: the mode routine sets them
         * first, so E is formed there from the corrected v2 */
        double vv[6];
        memcpy(vv, v, sizeof vv);
        const int zx = i == 0, zy = j == 0, zz = k == 0;
        const double kxv = c->kx[i], kyv = c->ky[j], kzv = c->kz[k];
        if (!zx && !zy && !zz) {
          vv[4] = (-kxv * vv[0] - kyv * vv[2]) / kzv;
          vv[5] = (-kxv * vv[1] - kyv * vv[3]) / kzv;
        } else if (zx && zy) {
          vv[4] = vv[5] = 0.;
        } else if (zx && zz) {
          vv[2] = vv[3] = 0.;
        } else if (zy && zz) {
          vv[0] = vv[1] = 0.;
        }
        const double v2 = vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2] + vv[3] * vv[3] + vv[4] * vv[4] + vv[5] * vv[5];
        const double E = v2 + 2.0 * tepq[km - 1] * (double)dt * (double)ef[p] / eold[km - 1];
        const double dH = hel == 1 ? thpq[km - 1] * (double)dt * (double)hf[p] / hold[km - 1] : 0.0;
        o_vcorr_mode(zx, zy, zz, kxv, kyv, kzv, (double)c->kk2[p], E, dH, (double)tinyf, v);
        vx[p].re = (real)v[0] * norm; vx[p].im = (real)v[1] * norm;
        vy[p].re = (real)v[2] * norm; vy[p].im = (real)v[3] * norm;
        vz[p].re = (real)v[4] * norm; vz[p].im = (real)v[5] * norm;
      }
}

/* ------------------------------------------------------------------ */
/* havgcomp (pseudospec3D_bouss.f90:19-554): the horizontal sums per z
 * plane of the real fields of itype's quantity.  itype 9 enters GHOST's
 * type-0 branch and returns from it; type 2 uses dtheta/dz for the factor
 * its code leaves unset (the profile its comment names). */
static void o_zsum(const octx *c, int op, const real *r1, const real *r2, const real *r3, real fo, real bv,
                   double *sh) {
  size_t plane = (size_t)c->nx * c->ny;
  double tmpn = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
  for (int k = 0; k < c->nz; ++k)
    for (size_t q = 0; q < plane; ++q) {
      size_t p = (size_t)k * plane + q;
      if (op == 0) sh[k] += (double)(r1[p] * r1[p] + r2[p] * r2[p]);
      else if (op == 1) sh[k] += (double)(r1[p] * r1[p]);
      else if (op == 2) sh[k] += (double)(r1[p] * r2[p]);
      else if (op == 3) sh[k] -= (double)(r1[p] * r2[p]);
      else if (op == 4) sh[k] += (double)(r3[p] * (r1[p] - r2[p]));
      else {
        real pv = 0;
        pv = (real)((double)pv + (double)fo * (double)r1[p] * tmpn);
        pv = (real)((double)pv - (double)bv * (double)r2[p] * tmpn);
        pv = (real)((double)pv + (double)r3[p] * -tmpn);
        pv = pv - fo * bv;
        sh[k] += (double)(pv * pv);
      }
    }
}

void o_havgcomp(const octx *c, const cplx *u, const cplx *v, const cplx *w, const cplx *s, double fo_d,
                double bv_d, int itype, double *gsh) {
  real fo = (real)fo_d, bv = (real)bv_d;
  size_t ns = c->nspec, nr = c->nreal;
  cplx *c1 = (cplx *)malloc(sizeof(cplx) * ns), *c2 = (cplx *)malloc(sizeof(cplx) * ns);
  cplx *c3 = (cplx *)malloc(sizeof(cplx) * ns), *c4 = (cplx *)malloc(sizeof(cplx) * ns);
  real *r1 = (real *)malloc(sizeof(real) * nr), *r2 = (real *)malloc(sizeof(real) * nr);
  real *r3 = (real *)malloc(sizeof(real) * nr);
  double tmp0 = 1.0 / (pow((double)c->nx, 3) * pow((double)c->ny, 3) * pow((double)c->nz, 2)), scale = tmp0;
  for (int k = 0; k < c->nz; ++k) gsh[k] = 0.0;
  switch (itype == 9 ? 0 : itype) {
    case 0:
      o_derivk3(c, u, c1, 3); o_fftp3d_complex_to_real(c, c1, r1);
      o_derivk3(c, v, c1, 3); o_fftp3d_complex_to_real(c, c1, r2);
      o_zsum(c, 0, r1, r2, NULL, fo, bv, gsh);
      break;
    case 1:
      o_derivk3(c, s, c1, 3); o_fftp3d_complex_to_real(c, c1, r3);
      o_zsum(c, 1, r3, NULL, NULL, fo, bv, gsh);
      break;
    case 2:
      o_derivk3(c, s, c1, 3); o_fftp3d_complex_to_real(c, c1, r3);
      o_fftp3d_complex_to_real(c, w, r2);
      o_zsum(c, 2, r3, r2, NULL, fo, bv, gsh);
      break;
    case 3:
      o_fftp3d_complex_to_real(c, u, r1); o_fftp3d_complex_to_real(c, v, r2);
      o_zsum(c, 0, r1, r2, NULL, fo, bv, gsh);
      break;
    case 4:
      o_fftp3d_complex_to_real(c, w, r1);
      o_zsum(c, 1, r1, NULL, NULL, fo, bv, gsh);
      break;
    case 5:
      o_derivk3(c, v, c1, 3); o_fftp3d_complex_to_real(c, c1, r2); o_fftp3d_complex_to_real(c, u, r1);
      o_zsum(c, 3, r1, r2, NULL, fo, bv, gsh);
      o_derivk3(c, u, c1, 3); o_fftp3d_complex_to_real(c, c1, r2); o_fftp3d_complex_to_real(c, v, r1);
      o_zsum(c, 2, r1, r2, NULL, fo, bv, gsh);
      break;
    case 6:
      o_rotor3(c, u, v, c1, 3); o_fftp3d_complex_to_real(c, c1, r1);
      o_fftp3d_complex_to_real(c, s, r2);
      o_zsum(c, 2, r1, r2, NULL, fo, bv, gsh);
      break;
    case 7:
      o_derivk3(c, s, c1, 3); o_fftp3d_complex_to_real(c, c1, r1);
      o_rotor3(c, u, v, c1, 3); o_fftp3d_complex_to_real(c, c1, r2);
      o_rotor3(c, v, w, c1, 1); o_rotor3(c, u, w, c2, 2); o_rotor3(c, u, v, c3, 3);
      o_advect3(c, c1, c2, c3, s, c4);
      o_fftp3d_complex_to_real(c, c4, r3);
      o_zsum(c, 5, r1, r2, r3, fo, bv, gsh);
      scale = 1.0 / ((double)c->nx * (double)c->ny);
      break;
    case 8:
      o_rotor3(c, u, v, c1, 3); o_derivk3(c, c1, c2, 2); o_fftp3d_complex_to_real(c, c2, r1);
      o_rotor3(c, u, w, c1, 2); o_derivk3(c, c1, c2, 3); o_fftp3d_complex_to_real(c, c2, r2);
      o_rotor3(c, v, w, c1, 1); o_fftp3d_complex_to_real(c, c1, r3);
      o_zsum(c, 4, r1, r2, r3, fo, bv, gsh);
      o_rotor3(c, v, w, c1, 1); o_derivk3(c, c1, c2, 3); o_fftp3d_complex_to_real(c, c2, r1);
      o_rotor3(c, u, v, c1, 3); o_derivk3(c, c1, c2, 1); o_fftp3d_complex_to_real(c, c2, r2);
      o_rotor3(c, u, w, c1, 2); o_fftp3d_complex_to_real(c, c1, r3);
      o_zsum(c, 4, r1, r2, r3, fo, bv, gsh);
      o_rotor3(c, u, w, c1, 2); o_derivk3(c, c1, c2, 1); o_fftp3d_complex_to_real(c, c2, r1);
      o_rotor3(c, v, w, c1, 1); o_derivk3(c, c1, c2, 2); o_fftp3d_complex_to_real(c, c2, r2);
      o_rotor3(c, u, v, c1, 3); o_fftp3d_complex_to_real(c, c1, r3);
      o_zsum(c, 4, r1, r2, r3, fo, bv, gsh);
      break;
    default:  /* 10 */
      o_fftp3d_complex_to_real(c, w, r1); o_fftp3d_complex_to_real(c, s, r2);
      o_zsum(c, 2, r1, r2, NULL, fo, bv, gsh);
      break;
  }
  for (int k = 0; k < c->nz; ++k) gsh[k] *= scale;
  free(c1); free(c2); free(c3); free(c4); free(r1); free(r2); free(r3);
}

/* ------------------------------------------------------------------ */
/* Passive scalar (PHD_SOL).  phd_rkstep2 (include/phd_rkstep2.f90):
 * prodre3, three nonlhd3, advect3, four laplak3, the three-way truncated
 * update in which th keeps its mean. */
void o_phd_rkstep2(const octx *c, int o, double dt_d, double nu_d, double kappa_d, cplx *vx, cplx *vy, cplx *vz,
                   cplx *th, const cplx *C1, const cplx *C2, const cplx *C3, const cplx *C20, const cplx *fx,
                   const cplx *fy, const cplx *fz, const cplx *fs) {
  size_t n = c->nspec;
  real dt = (real)dt_d, nu = (real)nu_d, kappa = (real)kappa_d;
  cplx *C4 = (cplx *)malloc(sizeof(cplx) * n), *C5 = (cplx *)malloc(sizeof(cplx) * n),
       *C6 = (cplx *)malloc(sizeof(cplx) * n), *C7 = (cplx *)malloc(sizeof(cplx) * n),
       *C8 = (cplx *)malloc(sizeof(cplx) * n);
  o_prodre3(c, vx, vy, vz, C4, C5, C6);
  o_nonlhd3(c, C4, C5, C6, C7, 1);
  o_nonlhd3(c, C4, C5, C6, C8, 2);
  o_nonlhd3(c, C4, C5, C6, C4, 3);
  o_advect3(c, vx, vy, vz, th, C5);
  o_laplak3(c, vx, vx);
  o_laplak3(c, vy, vy);
  o_laplak3(c, vz, vz);
  o_laplak3(c, th, th);
  real rmp = (real)1 / (real)o;
  cplx z = {0, 0};
  for (size_t p = 0; p < n; ++p) {
    if (c->kn2[p] <= c->kmax && c->kn2[p] >= c->tiny) {
      vx[p] = cadd(C1[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vx[p]), C7[p]), fx[p]))));
      vy[p] = cadd(C2[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vy[p]), C8[p]), fy[p]))));
      vz[p] = cadd(C3[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(nu, vz[p]), C4[p]), fz[p]))));
      th[p] = cadd(C20[p], cscal(rmp, cscal(dt, cadd(cadd(cscal(kappa, th[p]), C5[p]), fs[p]))));
    } else if (c->kn2[p] > c->kmax) {
      vx[p] = z; vy[p] = z; vz[p] = z; th[p] = z;
    } else {
      vx[p] = z; vy[p] = z; vz[p] = z; th[p] = C20[p];
    }
  }
  free(C4); free(C5); free(C6); free(C7); free(C8);
}

void o_phd_run(const octx *c, int nsteps, int ord, double dt, double nu, double kappa, cplx *vx, cplx *vy,
               cplx *vz, cplx *th, const cplx *fx, const cplx *fy, const cplx *fz, const cplx *fs) {
  size_t n = c->nspec;
  cplx *C1 = (cplx *)malloc(sizeof(cplx) * n), *C2 = (cplx *)malloc(sizeof(cplx) * n),
       *C3 = (cplx *)malloc(sizeof(cplx) * n), *C20 = (cplx *)malloc(sizeof(cplx) * n);
  cplx *zf = (cplx *)calloc(n, sizeof(cplx));
  if (!fx) fx = fy = fz = zf;
  if (!fs) fs = zf;
  for (int t = 0; t < nsteps; ++t) {
    memcpy(C1, vx, sizeof(cplx) * n); memcpy(C2, vy, sizeof(cplx) * n);
    memcpy(C3, vz, sizeof(cplx) * n); memcpy(C20, th, sizeof(cplx) * n);
    for (int o = ord; o >= 1; --o) o_phd_rkstep2(c, o, dt, nu, kappa, vx, vy, vz, th, C1, C2, C3, C20, fx, fy, fz, fs);
  }
  free(C1); free(C2); free(C3); free(C20); free(zf);
}

/* variance (pseudospec3D_phd.f90:116-216): sum of w tmp |a|^2 (times kk2 for kin 0) */
double o_variance(const octx *c, const cplx *a, int kin) {
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  double b = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    real w = i == 0 ? (real)1 : (real)2;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        real t = w * tmp;
        if (kin == 0) t = t * c->kk2[p];
        b += (double)(t * cabs2(a[p]));
      }
  }
  return b;
}

/* spectrscc (:516-609, bins int(|k|/Dkk + shift + .501_GP)) and sctrans
 * (:612-726, Re(a conj b)) */
void o_spectrscc(const octx *c, const cplx *a, double shift, double *Ek) {
  int nb = c->nmax / 2 + 1;
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  real rnd = (real)shift + (real)0.501;
  for (int q = 0; q < nb; ++q) Ek[q] = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    real w = i == 0 ? (real)1 : (real)2;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        int kmn = (int)((real)sqrt(c->kk2[p]) / c->Dkk + rnd);
        if (kmn > 0 && kmn <= nb) Ek[kmn - 1] += (double)(w * tmp * cabs2(a[p]));
      }
  }
}

void o_sctrans(const octx *c, const cplx *a, const cplx *b, double *Ek) {
  int nb = c->nmax / 2 + 1;
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  for (int q = 0; q < nb; ++q) Ek[q] = 0.0;
  for (int i = 0; i < c->nxh; ++i) {
    real w = i == 0 ? (real)1 : (real)2;
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        int kmn = (int)((real)sqrt(c->kk2[p]) / c->Dkk + (real)0.501f);
        if (kmn > 0 && kmn <= nb) Ek[kmn - 1] += (double)(w * tmp * cmul(a[p], cconj(b[p])).re);
      }
  }
}

/* ------------------------------------------------------------------ */
/* MHD (pseudospec3D_mhd.f90, include/mhd_rkstep2.f90). */
/* vector3 (:22-105): the real fields of (a,b,c) and (d,e,f), their cross
 * product times 1/(nx ny nz)^2, back to Fourier space */
void o_vector3(const octx *c, const cplx *a, const cplx *b, const cplx *cc, const cplx *d, const cplx *e,
               const cplx *f, cplx *x, cplx *y, cplx *z) {
  size_t nr = c->nreal;
  real *r[7];
  for (int q = 0; q < 7; ++q) r[q] = (real *)malloc(sizeof(real) * nr);
  o_fftp3d_complex_to_real(c, a, r[0]); o_fftp3d_complex_to_real(c, b, r[1]);
  o_fftp3d_complex_to_real(c, cc, r[2]); o_fftp3d_complex_to_real(c, d, r[3]);
  o_fftp3d_complex_to_real(c, e, r[4]); o_fftp3d_complex_to_real(c, f, r[5]);
  real tmp = (real)1 / (((real)c->nx * (real)c->ny * (real)c->nz) * ((real)c->nx * (real)c->ny * (real)c->nz));
  for (size_t p = 0; p < nr; ++p) {
    real r1 = r[0][p], r2 = r[1][p], r3 = r[2][p], r4 = r[3][p], r5 = r[4][p], r6 = r[5][p];
    r[6][p] = (r2 * r6 - r5 * r3) * tmp;
    r[2][p] = (r3 * r4 - r6 * r1) * tmp;
    r[0][p] = (r1 * r5 - r4 * r2) * tmp;
  }
  o_fftp3d_real_to_complex(c, r[6], x);
  o_fftp3d_real_to_complex(c, r[2], y);
  o_fftp3d_real_to_complex(c, r[0], z);
  for (int q = 0; q < 7; ++q) free(r[q]);
}

/* nonlin3 (:108-227) and gauge3 (:230-336), statement by statement */
void o_nonlin3(const octx *c, const cplx *a, const cplx *b, const cplx *cc, const cplx *d, const cplx *e,
               const cplx *f, cplx *g, int dir) {
  cplx *out = (cplx *)malloc(sizeof(cplx) * c->nspec);
  for (int i = 0; i < c->nxh; ++i)
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        cplx s = dir == 1 ? a[p] : (dir == 2 ? b[p] : cc[p]);
        cplx t = dir == 1 ? d[p] : (dir == 2 ? e[p] : f[p]);
        cplx base = cadd(cscal(-1, s), t);
        int zero_plane = dir == 1 ? (i == 0) : (dir == 2 ? (j == 0) : (k == 0));
        if (zero_plane) {
          out[p] = base;
        } else {
          real kd = dir == 1 ? c->kx[i] : (dir == 2 ? c->ky[j] : c->kz[k]);
          cplx q = cadd(cadd(cscal(c->kx[i], csub(a[p], d[p])), cscal(c->ky[j], csub(b[p], e[p]))),
                        cscal(c->kz[k], csub(cc[p], f[p])));
          q = cscal(kd, q);
          q.re = q.re / c->kk2[p];
          q.im = q.im / c->kk2[p];
          out[p] = cadd(base, q);
        }
      }
  memcpy(g, out, sizeof(cplx) * c->nspec);
  free(out);
}

void o_gauge3(const octx *c, const cplx *a, const cplx *b, const cplx *cc, cplx *g, int dir) {
  cplx *out = (cplx *)malloc(sizeof(cplx) * c->nspec);
  for (int i = 0; i < c->nxh; ++i)
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k) {
        size_t p = SIDX(c, k, j, i);
        cplx s = dir == 1 ? a[p] : (dir == 2 ? b[p] : cc[p]);
        int zero_plane = dir == 1 ? (i == 0) : (dir == 2 ? (j == 0) : (k == 0));
        if (zero_plane) {
          out[p] = s;
        } else {
          real kd = dir == 1 ? c->kx[i] : (dir == 2 ? c->ky[j] : c->kz[k]);
          cplx q = cadd(cadd(cscal(c->kx[i], a[p]), cscal(c->ky[j], b[p])), cscal(c->kz[k], cc[p]));
          q = cscal(kd, q);
          q.re = q.re / c->kk2[p];
          q.im = q.im / c->kk2[p];
          out[p] = csub(s, q);
        }
      }
  memcpy(g, out, sizeof(cplx) * c->nspec);
  free(out);
}

/* mhd_rkstep2 (include/mhd_rkstep2.f90) */
void o_mhd_rkstep2(const octx *c, int o, double dt_d, double nu_d, double mu_d, cplx *vx, cplx *vy, cplx *vz,
                   cplx *ax, cplx *ay, cplx *az, const cplx *const C[6], const cplx *const fv[3],
                   const cplx *const fm[3]) {
  size_t n = c->nspec;
  real dt = (real)dt_d, nu = (real)nu_d, mu = (real)mu_d;
  cplx *W[11];
  for (int q = 0; q < 11; ++q) W[q] = (cplx *)malloc(sizeof(cplx) * n);
  cplx *C7 = W[0], *C8 = W[1], *C9 = W[2], *C10 = W[3], *C11 = W[4], *C12 = W[5], *C13 = W[6], *C14 = W[7],
       *C15 = W[8], *C16 = W[9], *C17 = W[10];
  o_rotor3(c, ay, az, C7, 1);
  o_rotor3(c, ax, az, C8, 2);
  o_rotor3(c, ax, ay, C9, 3);
  o_prodre3(c, vx, vy, vz, C10, C11, C12);
  o_prodre3(c, C7, C8, C9, C13, C14, C15);
  o_nonlin3(c, C10, C11, C12, C13, C14, C15, C16, 1);
  o_nonlin3(c, C10, C11, C12, C13, C14, C15, C17, 2);
  o_nonlin3(c, C10, C11, C12, C13, C14, C15, C10, 3);
  o_vector3(c, vx, vy, vz, C7, C8, C9, C11, C12, C13);
  o_gauge3(c, C11, C12, C13, C7, 1);
  o_gauge3(c, C11, C12, C13, C8, 2);
  o_gauge3(c, C11, C12, C13, C9, 3);
  o_laplak3(c, vx, vx); o_laplak3(c, vy, vy); o_laplak3(c, vz, vz);
  o_laplak3(c, ax, ax); o_laplak3(c, ay, ay); o_laplak3(c, az, az);
  real rmp = (real)1 / (real)o;
  cplx zc = {0, 0};
  cplx *vv[3] = {vx, vy, vz}, *aa[3] = {ax, ay, az};
  const cplx *gv[3] = {C16, C17, C10}, *ga[3] = {C7, C8, C9};
  for (size_t p = 0; p < n; ++p) {
    int keep = c->kn2[p] <= c->kmax && c->kn2[p] >= c->tiny;
    for (int q = 0; q < 3; ++q) {
      if (keep) {
        cplx sv = cadd(cscal(nu, vv[q][p]), gv[q][p]);
        if (fv) sv = cadd(sv, fv[q][p]);
        cplx sa = cadd(cscal(mu, aa[q][p]), ga[q][p]);
        if (fm) sa = cadd(sa, fm[q][p]);
        vv[q][p] = cadd(C[q][p], cscal(rmp, cscal(dt, sv)));
        aa[q][p] = cadd(C[3 + q][p], cscal(rmp, cscal(dt, sa)));
      } else {
        vv[q][p] = zc;
        aa[q][p] = zc;
      }
    }
  }
  for (int q = 0; q < 11; ++q) free(W[q]);
}

void o_mhd_run(const octx *c, int nsteps, int ord, double dt, double nu, double mu, cplx *vx, cplx *vy, cplx *vz,
               cplx *ax, cplx *ay, cplx *az, const cplx *fx, const cplx *fy, const cplx *fz, const cplx *mx,
               const cplx *my, const cplx *mz) {
  size_t n = c->nspec;
  cplx *Cs[6];
  for (int q = 0; q < 6; ++q) Cs[q] = (cplx *)malloc(sizeof(cplx) * n);
  const cplx *C[6] = {Cs[0], Cs[1], Cs[2], Cs[3], Cs[4], Cs[5]};
  const cplx *fv[3] = {fx, fy, fz}, *fm[3] = {mx, my, mz};
  cplx *src[6] = {vx, vy, vz, ax, ay, az};
  for (int t = 0; t < nsteps; ++t) {
    for (int q = 0; q < 6; ++q) memcpy(Cs[q], src[q], sizeof(cplx) * n);
    for (int o = ord; o >= 1; --o)
      o_mhd_rkstep2(c, o, dt, nu, mu, vx, vy, vz, ax, ay, az, C, fx ? fv : NULL, mx ? fm : NULL);
  }
  for (int q = 0; q < 6; ++q) free(Cs[q]);
}

/* phaseshift (pseudospec3D_hd.f90:2084-2148), its loops as written (1-based
 * j, k of the Fortran shifted to 0-based storage) */
void o_phaseshift(const octx *c, cplx *a, double cre, double cim) {
  cplx cd = {(real)cre, (real)cim}, jd = {(real)cre, -(real)cim};
  int ny = c->ny, nz = c->nz;
  for (int j = 2; j <= ny / 2 + 1; ++j) {
    a[SIDX(c, 0, j - 1, 0)] = cmul(a[SIDX(c, 0, j - 1, 0)], cd);
    a[SIDX(c, 0, ny - j + 1, 0)] = cmul(a[SIDX(c, 0, ny - j + 1, 0)], jd);
  }
  for (int k = 2; k <= nz / 2 + 1; ++k) {
    a[SIDX(c, k - 1, 0, 0)] = cmul(a[SIDX(c, k - 1, 0, 0)], cd);
    a[SIDX(c, nz - k + 1, 0, 0)] = cmul(a[SIDX(c, nz - k + 1, 0, 0)], jd);
  }
  for (int j = 2; j <= ny; ++j)
    for (int k = 2; k <= nz / 2 + 1; ++k) {
      a[SIDX(c, k - 1, j - 1, 0)] = cmul(a[SIDX(c, k - 1, j - 1, 0)], cd);
      a[SIDX(c, nz - k + 1, ny - j + 1, 0)] = cmul(a[SIDX(c, nz - k + 1, ny - j + 1, 0)], jd);
    }
  for (int i = 1; i < c->nxh; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) a[SIDX(c, k, j, i)] = cmul(a[SIDX(c, k, j, i)], cd);
}
