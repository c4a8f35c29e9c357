/*
 * ghost_b200.h -- C ABI of the B200 (sm_100a) pseudospectral HD library.
 *
 * Drop-in boundary for GHOST's 3D HD hot path.  Every entry point names the
 * GHOST routine it replaces (paths relative to the GHOST tree, 3D/src/).
 * The Fortran side binds these with ISO_C_BINDING (ghost_b200/fortran/
 * ghost_gpu.f90); C and Python (ctypes) callers use them directly.
 *
 * Conventions
 *  - Every function returns an int status (GHOST_OK == 0) and never exits
 *    the process; ghost_last_error_string() describes the last failure on
 *    the calling thread.
 *  - Precision is fixed per context: GHOST_SINGLE (4) or GHOST_DOUBLE (8),
 *    the KIND values of GHOST's GP (fftp-3/fprecision_mod.fpp:14-16).
 *    "real" below means float or double accordingly; "complex" means two
 *    interleaved reals (Fortran COMPLEX(KIND=GP) layout).
 *  - Layouts are GHOST's, column-major:
 *      spectral a(nz,ny,nx/2+1): offset k + nz*(j + ny*i), z fastest,
 *               i = kx index 0..nx/2 (the Nyquist index carries kx=-nx/2
 *               as in main3D.fpp:1746-1749);
 *      real     r(nx,ny,nz):     offset i + nx*(j + ny*k), x fastest.
 *  - Field pointers may be device memory (the fast path: no copies) or host
 *    memory (pageable or pinned).  Host arrays are staged through the
 *    context's device buffers and the call returns after the results are
 *    back on the host, as GHOST's fftp-cu path does with every array
 *    (fftp-cu/fftp3D.fpp:364-402).  Device-pointer calls are asynchronous
 *    on the context's stream unless they return host scalars.
 *  - Transforms are unnormalised both ways (c2r(r2c(x)) = nx*ny*nz * x).
 *  - One context per host thread; calls on one context are not re-entrant.
 */
#ifndef GHOST_B200_H
#define GHOST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define GHOST_OK 0
#define GHOST_ERR_ARG 1     /* bad argument: null pointer, dir/kin/o out of range */
#define GHOST_ERR_SIZE 2    /* unsupported grid: each n must be a power of two in [16,1024] */
#define GHOST_ERR_ALLOC 3   /* device allocation failed */
#define GHOST_ERR_CUDA 4    /* CUDA runtime error (launch or execution) */
#define GHOST_ERR_TIMEOUT 5 /* a bounded device-side wait gave up */
#define GHOST_ERR_NAN 6     /* non-finite value detected by a checked call */
#define GHOST_ERR_STATE 7   /* call not valid in the current state */
#define GHOST_ERR_NODEV 8   /* no usable CUDA device */
#define GHOST_ERR_IO 9      /* a field file could not be opened, read or written */

/* precision (GHOST's GP kind values) */
#define GHOST_SINGLE 4
#define GHOST_DOUBLE 8

/* FFT directions, FFTW's values as used by fftp3d_create_plan
 * (fftp-3/fftp3D.fpp:64-66) */
#define GHOST_REAL_TO_COMPLEX (-1)
#define GHOST_COMPLEX_TO_REAL (+1)

typedef struct ghost_ctx ghost_ctx;
typedef struct ghost_fftplan ghost_fftplan;

/* Scalars of the grid, kes, ali and boxsize modules
 * (pseudo/pseudospec3D_mod.fpp:13-21,53-72,112-120). */
typedef struct {
  int nx, ny, nz;
  int precision;
  int anis;      /* 1: anisotropic wavenumber normalisation (main3D.fpp:740-749) */
  int nmax, nmaxperp;
  double kmax, tiny;
  double Lx, Ly, Lz, Dkx, Dky, Dkz, Dkk;
  size_t spectral_elems; /* nz*ny*(nx/2+1) complex values per field */
  size_t real_elems;     /* nx*ny*nz reals per field */
} ghost_info;

/* ---------------------------------------------------------------- */
/* Context: replaces the module state set up in main3D.fpp:1721-1801
 * (kmax, tiny, nmax, kx/ky/kz, kn2, kk2) and holds the device scratch,
 * twiddle tables and stream.  arbsize != 0 is GHOST's ARBSIZE build
 * (box Lx,Ly,Lz in units of 2*pi, main3D.fpp:881-909); arbsize == 0
 * ignores Lx,Ly,Lz and uses the 2*pi-periodic cube. */
int ghost_ctx_create(int nx, int ny, int nz, double Lx, double Ly, double Lz, int arbsize,
                     int precision, ghost_ctx **ctx);
int ghost_ctx_destroy(ghost_ctx *ctx);
int ghost_ctx_get_info(const ghost_ctx *ctx, ghost_info *info);
/* Run all further work on this cudaStream_t (NULL: the legacy stream). */
int ghost_ctx_set_stream(ghost_ctx *ctx, void *cuda_stream);
/* Override the truncation wavenumber kmax, e.g. the EDQNM choice
 * kmax = (n/2-0.5)^2 of main3D.fpp:1732-1734. */
int ghost_ctx_set_kmax(ghost_ctx *ctx, double kmax);
/* Tile variant of the FFT passes (no GHOST counterpart; FFTW's planner
 * plays this role in fftp-3/fftp3D.fpp:92-107): bit 0 y tiles 16 z-lines
 * wide instead of 8; bit 1 z-pass CTAs of 128 threads instead of 256; bits
 * 1 and 2 together a two-stage z ring with three CTAs per SM; bit 3 a
 * two-stage y ring with a second exchange buffer; bit 4 (FP32, y lines of
 * 256 points or more) y passes with 16 values per thread; bits 1, 2 and 5
 * (z lines of 256 points or more) a one-stage z ring with four CTAs per SM;
 * bits 3, 4 and 6 the FP32 y inverse in tiles of 4 z-lines (four CTAs per
 * SM).  Results do not depend on the variant (0..127). */
int ghost_ctx_set_tile_cfg(ghost_ctx *ctx, int cfg);
int ghost_ctx_get_tile_cfg(const ghost_ctx *ctx, int *cfg);
/* Times one RK step of every tile variant on a copy of v (device arrays;
 * v does not advance) and keeps the fastest; cfg_out may be NULL. */
int ghost_hd_autotune(ghost_ctx *ctx, int ord, double dt, double nu, const void *vx, const void *vy,
                      const void *vz, const void *fx, const void *fy, const void *fz, int *cfg_out);
/* Block until the context's stream is idle; reports asynchronous errors. */
int ghost_ctx_synchronize(ghost_ctx *ctx);
/* Bound on the polls of every device-side wait (tile arrivals in the
 * pipelined passes).  A wait that runs out makes its kernel give up
 * cleanly and records GHOST_ERR_TIMEOUT, which the next synchronising call
 * on the context returns.  Default 2^22 polls; 0 restores the default. */
int ghost_ctx_set_wait_cap(ghost_ctx *ctx, unsigned int cap);
/* Fault injection for testing failure detection: with enable != 0 every
 * pipelined pass additionally waits on a barrier that nothing completes,
 * so its bounded wait runs out and the next synchronising call returns
 * GHOST_ERR_TIMEOUT.  Nothing faults or hangs; results are not computed. */
int ghost_ctx_inject_stall(ghost_ctx *ctx, int enable);
/* Number of this library's kernels launched on the context so far. */
int ghost_ctx_launch_count(const ghost_ctx *ctx, long long *count);
const char *ghost_last_error_string(void);

/* Per-kernel device timers, the role of FFTP's ffttime/tratime/comtime
 * accumulators (fftp-cu/fftp_mod.fpp:39-45): when enabled, CUDA events are
 * recorded on the context's stream around every launch, grouped by kernel
 * kind (GHOST_TIMER_*).  Reading synchronises the stream, returns the
 * accumulated milliseconds and launch counts per kind, and resets them. */
#define GHOST_TIMER_Z_INV 0     /* fused inverse z pass (curl / gradient prologue) */
#define GHOST_TIMER_Y_INV 1     /* inverse y pass */
#define GHOST_TIMER_X_NL 2      /* fused x pass: c2r, real-space products, r2c */
#define GHOST_TIMER_Y_FWD 3     /* forward y pass */
#define GHOST_TIMER_Z_FWD 4     /* fused forward z pass (projection + RK update) */
#define GHOST_TIMER_Z_C2C 5     /* plain z pass */
#define GHOST_TIMER_X_C2R 6     /* plain complex-to-real x pass */
#define GHOST_TIMER_X_R2C 7     /* plain real-to-complex x pass */
#define GHOST_TIMER_POINTWISE 8 /* pointwise spectral operators */
#define GHOST_TIMER_REDUCE 9    /* reductions and spectra */
#define GHOST_TIMER_KINDS 10
int ghost_ctx_enable_timers(ghost_ctx *ctx, int enable);
int ghost_ctx_read_timers(ghost_ctx *ctx, double ms[GHOST_TIMER_KINDS], long long launches[GHOST_TIMER_KINDS]);

/* ---------------------------------------------------------------- */
/* FFTP: fftp-3/fftp3D.fpp and fftp-cu/fftp3D.fpp */

/* fftp3d_create_plan(plan,n,fftdir,flags) (fftp-3/fftp3D.fpp:56-123).
 * n must equal the context grid; flags is accepted and ignored. */
int ghost_fftp3d_create_plan(ghost_ctx *ctx, const int n[3], int fftdir, int flags,
                             ghost_fftplan **plan);
/* fftp3d_destroy_plan(plan) (fftp-3/fftp3D.fpp:126-155) */
int ghost_fftp3d_destroy_plan(ghost_fftplan *plan);
/* fftp3d_real_to_complex(plan,in,out,comm) (fftp-3/fftp3D.fpp:204-315):
 * in real(nx,ny,nz) -> out complex(nz,ny,nx/2+1), sign -1. */
int ghost_fftp3d_real_to_complex(ghost_fftplan *plan, const void *in, void *out);
/* fftp3d_complex_to_real(plan,in,out,comm) (fftp-3/fftp3D.fpp:318-431):
 * in complex(nz,ny,nx/2+1) -> out real(nx,ny,nz), sign +1.  The input is
 * left unmodified (GHOST overwrites it; callers rely on neither).  The
 * imaginary parts of the kx=0 and kx=nx/2 planes are ignored after the z
 * and y transforms, as a complex-to-real transform of Hermitian data does. */
int ghost_fftp3d_complex_to_real(ghost_fftplan *plan, const void *in, void *out);

/* ---------------------------------------------------------------- */
/* Spectral operators: pseudo/pseudospec3D_hd.f90.  All fields complex
 * (nz,ny,nx/2+1).  Outputs may alias inputs. */

/* derivk3(a,b,dir) (:22-88): b = i k_dir a */
int ghost_derivk3(ghost_ctx *ctx, const void *a, void *b, int dir);
/* laplak3(a,b) (:91-121): b = -kk2 a */
int ghost_laplak3(ghost_ctx *ctx, const void *a, void *b);
/* rotor3(a,b,c,dir) (:124-200): c = curl component dir of the field whose
 * other two components are a,b in right-hand order */
int ghost_rotor3(ghost_ctx *ctx, const void *a, const void *b, void *c, int dir);
/* prodre3(a,b,c,d,e,f) (:316-396): (d,e,f) = [curl(A) x A] in Fourier space
 * (normalised by 1/(nx ny nz)^2 in real space, as GHOST does) */
int ghost_prodre3(ghost_ctx *ctx, const void *a, const void *b, const void *c, void *d, void *e,
                  void *f);
/* nonlhd3(a,b,c,g,dir) (:399-509): g = -a_dir + k_dir (k.a)/kk2, the
 * k_dir = 0 plane gets -a_dir */
int ghost_nonlhd3(ghost_ctx *ctx, const void *a, const void *b, const void *c, void *g, int dir);
/* energy(a,b,c,d,kin) (:512-662): kin 1 <|A|^2>, 0 <|curl A|^2>,
 * 2 <|lap A|^2>; FP64 accumulation, deterministic */
int ghost_energy(ghost_ctx *ctx, const void *a, const void *b, const void *c, double *d, int kin);
/* helicity(a,b,c,d) (:665-784): <A . curl A> */
int ghost_helicity(ghost_ctx *ctx, const void *a, const void *b, const void *c, double *d);
/* cross(a,b,c,d,e,f,g,kin) (:787-907): kin 1 <A.B>, 0 <kk2 A.B> */
int ghost_cross(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d,
                const void *e, const void *f, double *g, int kin);
/* divergence term of hdcheck(...,chk=1) (:1036-1070): <(div A)^2> */
int ghost_divergence(ghost_ctx *ctx, const void *a, const void *b, const void *c, double *d);
/* maxabs(a,b,c,d,kin) (:910-981): kin 0 max|curl A|, 1 max|lap A|,
 * 2 max|A| in real space, divided by nx ny nz */
int ghost_maxabs(ghost_ctx *ctx, const void *a, const void *b, const void *c, double *d, int kin);
/* spectrumc(a,b,c,kin,hel,Ek,Hk) (:1190-1415): shell spectra on
 * nmax/2+1 bins (host arrays); Ek skipped when kin == 2, Hk computed only
 * when hel == 1 (Hk may then be NULL otherwise) */
int ghost_spectrumc(ghost_ctx *ctx, const void *a, const void *b, const void *c, int kin, int hel,
                    double *Ek, double *Hk);
/* entrans(a,b,c,d,e,f,nmb,kin) (pseudospec3D_hd.f90:1629-1820): the shell
 * sums Ek[nmax/2+1] of Re(a.conj(d) + b.conj(e) + c.conj(f))/(nx ny nz)^2,
 * times kk2 for kin = 0, doubled off the kx = 0 plane: GHOST's Ektot.  Its
 * file (ktransfer.NNNN.txt for kin = 1 and the others by kin) holds
 * (Dkk*k, Ek[k-1]/Dkk).  Ek is a host array. */
int ghost_entrans(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                  const void *f, int kin, double *Ek);
/* heltrans(a,b,c,d,e,f,nmb,kin) (pseudospec3D_hd.f90:1823-1949): the same
 * with curl(a,b,c) in place of (a,b,c); kin only names GHOST's file
 * (hmtransfer / hktransfer). */
int ghost_heltrans(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                   const void *f, int kin, double *Hk);
/* phaseshift(a,cdump) (pseudospec3D_hd.f90:2084-2148): a *= cdump in place,
 * with conj(cdump) on the mirror half of the kx = 0 plane (GHOST's loop
 * order, including its Nyquist lines that take both factors) */
int ghost_phaseshift(ghost_ctx *ctx, void *a, double cdump_re, double cdump_im);
/* The rand = 2 (slowly varying) forcing update of main3D.fpp:2581-2657,
 * which GHOST inlines in its time loop: f = (1-rmp) fold + rmp fnew with
 * rmp = FLOAT(timef+1)/float(fstep) (default REAL), timef in 0..fstep-1
 * the steps since the last regeneration.  Every fstep steps the caller
 * copies f to fold and draws a new random forcing into fnew (initialfv:
 * ghost_init_random_solenoidal continuing the seed), as GHOST does.  The
 * outputs may alias either input. */
int ghost_forcing_slow(ghost_ctx *ctx, int timef, int fstep, const void *fxold, const void *fyold, const void *fzold,
                       const void *fxnew, const void *fynew, const void *fznew, void *fx, void *fy, void *fz);

/* ------------------------------------------------------------------
 * MHD (MHD_SOL, pseudospec3D_mhd.f90, include/mhd_rkstep1/2.f90): velocity
 * v and magnetic vector potential a (b = curl a).
 * ------------------------------------------------------------------ */
/* vector3(a,b,c,d,e,f,x,y,z) (:22-105): (a,b,c) x (d,e,f) through real
 * space, times 1/(nx ny nz)^2 */
int ghost_vector3(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                  const void *f, void *x, void *y, void *z);
/* nonlin3(a,b,c,d,e,f,g,dir) (:108-227): g = -(a-d)_dir + k_dir k.(a-d)/k^2,
 * the projected difference of the two nonlinear terms (w x v and j x b) */
int ghost_nonlin3(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                  const void *f, void *g, int dir);
/* gauge3(a,b,c,g,dir) (:230-336): g = a_dir - k_dir k.a/k^2 (Coulomb gauge) */
int ghost_gauge3(ghost_ctx *ctx, const void *a, const void *b, const void *c, void *g, int dir);
/* nsteps RK steps of GHOST's MHD solver: per substep b = curl a, the
 * projected (w x v - j x b), the gauged v x b, and the truncated update of
 * v (viscosity nu, forcing f) and a (diffusivity mu, forcing m); f and m
 * may be NULL */
int ghost_mhd_run(ghost_ctx *ctx, int nsteps, int ord, double dt, double nu, double mu, void *vx, void *vy, void *vz,
                  void *ax, void *ay, void *az, const void *fx, const void *fy, const void *fz, const void *mx,
                  const void *my, const void *mz);

/* ------------------------------------------------------------------
 * Passive scalar (PHD_SOL, pseudospec3D_phd.f90).
 * ------------------------------------------------------------------ */
/* nsteps RK steps of GHOST's PHD solver (include/phd_rkstep2.f90): the HD
 * step plus th advanced by -v.grad(th) + kappa lap(th) + fs, with the
 * three-way truncation (th keeps its mean).  Equal to ghost_bouss_run with
 * omegaz = xmom = xtemp = 0. */
int ghost_phd_run(ghost_ctx *ctx, int nsteps, int ord, double dt, double nu, double kappa, void *vx, void *vy,
                  void *vz, void *th, const void *fx, const void *fy, const void *fz, const void *fs);
/* variance(a,b,kin) (:116-216): b = <|a|^2> (kin 1) or <k^2 |a|^2> (kin 0) */
int ghost_variance(ghost_ctx *ctx, const void *a, int kin, double *b);
/* spectrscc(a,Ektot,shift) (:516-609): the scalar's shell sums with bins
 * int(|k|/Dkk + shift + .501); Ek[nmax/2+1] */
int ghost_spectrscc(ghost_ctx *ctx, const void *a, double shift, double *Ek);
/* sctrans(a,b,nmb,isc) (:612-726): shell sums of Re(a conj(b))/(nx ny nz)^2
 * (GHOST's Ektot; isc only names its file) */
int ghost_sctrans(ghost_ctx *ctx, const void *a, const void *b, int isc, double *Ek);
/* havgcomp(gsh,u,v,w,s,fo,bv,itype) (pseudospec3D_bouss.f90:19-554): the
 * horizontally averaged profile gsh[nz] of quantity itype of the
 * Boussinesq fields (velocity u, v, w; temperature s; fo the Coriolis and
 * bv the Brunt-Vaisala frequency): 0 <(du_perp/dz)^2>, 1 <(ds/dz)^2>,
 * 2 <w ds/dz>, 3 <u^2+v^2>, 4 <w^2>, 5 <v du/dz - u dv/dz>, 6 <w_z s>,
 * 7 <PV^2>, 8 the vorticity-gradient term, 9 as GHOST computes it (its type-0
 * branch also takes itype 9), 10 <w s>.  Type 2 follows the profile GHOST's
 * comment names; its code reads an array it has not set. */
int ghost_havgcomp(ghost_ctx *ctx, const void *u, const void *v, const void *w, const void *s, double fo, double bv,
                   int itype, double *gsh);
/* tbouss (pseudospec3D_bouss.f90:611-711): per itype 0..10 the z-average,
 * the maximum and the minimum of the havgcomp profile (host arrays of 11);
 * GHOST appends them to tboussavg/max/min.txt */
int ghost_tbouss(ghost_ctx *ctx, const void *u, const void *v, const void *w, const void *s, double fo, double bv,
                 double *avg, double *mx, double *mn);
/* Anisotropic spectra of rotating flows (pseudospec3D_rot.f90).  specpara
 * bins by |kz| (kmn = int(|kz| Lz + 1), nb = nz/2+1 bins), specperp by the
 * perpendicular wavenumber (kmn = int(sqrt(kx^2+ky^2)/Dkk + 1),
 * nb = nmaxperp/2+1).  Ek and Hk are host arrays of 3 nb doubles: GHOST's
 * Ektot, then the horizontal (x, y components) and vertical (z component)
 * sums (specperp: of the kz = 0 plane, as GHOST's Eptot / Eztot).  kin 1
 * kinetic, 0 of curl(a,b,c), 2 none; hel 1 the helicity Re(v . conj(curl v)).
 * GHOST's files hold (Dkz (k-1), .5 E Lz) resp. (Dkk (k-1), .5 E/Dkk). */
int ghost_specpara(ghost_ctx *ctx, const void *a, const void *b, const void *c, int kin, int hel, double *Ek,
                   double *Hk);
int ghost_specperp(ghost_ctx *ctx, const void *a, const void *b, const void *c, int kin, int hel, double *Ek,
                   double *Hk);
/* entpara/entperp, heltpara/heltperp (pseudospec3D_rot.f90:689-1328): the
 * entrans / heltrans sums binned as specpara / specperp (nb doubles). */
int ghost_entpara(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                  const void *f, int kin, double *Ek);
int ghost_entperp(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                  const void *f, int kin, double *Ek);
int ghost_heltpara(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                   const void *f, int kin, double *Hk);
int ghost_heltperp(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, const void *e,
                   const void *f, int kin, double *Hk);
/* ghost_spectrumc_noalloc: the same shell spectra as ghost_spectrumc,
 * computed without allocating any memory.  It has no counterpart in the
 * reference; it exists for callers that cannot let the library allocate:
 * runs that hand the device memory to their own fields at start-up (a GHOST
 * grid sized to fill HBM, or an application under a fixed memory budget),
 * where the lazy cudaMalloc of ghost_spectrumc's partial-sum buffer would
 * fail at the first spectrum output step, and time loops that cannot
 * afford the device-wide synchronisation an allocation brings.
 * The partial sums live in a static device array of
 * GHOST_SPECTRUM_NOALLOC_DOUBLES doubles (512 KiB, held by every GPU that
 * loads the library until the process exits); a grid with more than
 * GHOST_SPECTRUM_NOALLOC_MAX_BINS shells (nmax/2+1 <= 1008, i.e.
 * nmax <= 2015) is rejected with GHOST_ERR_SIZE.  On a batched context
 * (ghost_ctx_create_batch) the spectra sum every run, as ghost_spectrumc
 * does.  a, b, c must be device arrays (host arrays would need staging
 * buffers: GHOST_ERR_ARG); Ek, Hk are host arrays as above.
 * The array is committed when the library's device code is loaded on a
 * device, which with CUDA's default lazy module loading happens at the
 * first library call that launches a kernel there (this one included):
 * make some library call on each device before filling its memory.  The
 * first call on a device also looks up the array's device address with
 * that device current; make that first call before any stream capture.
 * The address stays valid for the process unless the device is reset
 * (cudaDeviceReset), after which this entry point must not be used on it.
 * All calls share the one array and it keeps the last call's contents:
 * calls that overlap on the GPU (other streams, other contexts on the
 * device) race and must be serialised by the caller. */
#define GHOST_SPECTRUM_NOALLOC_DOUBLES 65536
#define GHOST_SPECTRUM_NOALLOC_MAX_BINS 1008
int ghost_spectrumc_noalloc(ghost_ctx *ctx, const void *a, const void *b, const void *c, int kin, int hel,
                            double *Ek, double *Hk);
/* hdcheck(a,b,c,d,e,f,t,dt,hel,chk) (:984-1105) without the file output:
 * out[0]=<|v|^2>, out[1]=<|w|^2>, out[2]=helicity (hel==1), out[3]=<v.f>,
 * out[4]=<(div v)^2> (chk==1) */
int ghost_hdcheck(ghost_ctx *ctx, const void *vx, const void *vy, const void *vz, const void *fx,
                  const void *fy, const void *fz, int hel, int chk, double out[5]);
/* normalize(fx,fy,fz,f0,kin) (pseudo/module_dns.f90:13-41) */
int ghost_normalize(ghost_ctx *ctx, void *fx, void *fy, void *fz, double f0, int kin);
/* sharp(a,b,delta) (pseudo/pseudospec3D_filt.f90:200-241) */
int ghost_sharp(ghost_ctx *ctx, const void *a, void *b, double delta);

/* ---------------------------------------------------------------- */
/* Runge-Kutta fragments of the HD solver */

/* hd_rkstep1 (include/hd_rkstep1.f90:4-6): C1..C3 = vx..vz */
int ghost_hd_rkstep1(ghost_ctx *ctx, const void *vx, const void *vy, const void *vz, void *C1, void *C2,
                     void *C3);
/* hd_rkstep2 (include/hd_rkstep2.f90:3-32) for substep o:
 * v = C + dt*(nu*lap v - P(w x v) + f)/o on tiny <= kn2 <= kmax, else 0.
 * f may be NULL (no forcing). */
int ghost_hd_rkstep2(ghost_ctx *ctx, int o, double dt, double nu, void *vx, void *vy, void *vz,
                     const void *C1, const void *C2, const void *C3, const void *fx, const void *fy,
                     const void *fz);
/* nsteps steps of the loop main3D.fpp:3195-3231 (RK1 then DO o=ord,1,-1
 * RK2), the copy of RK1 fused into the first substep.  C1..C3 are the
 * RK storage (device, or NULL: context-owned).  f may be NULL.  With host
 * arrays, only the live box of f and v crosses the bus (the kx rows, y-lines
 * and kz values that can hold a mode of the truncation), as long as v holds only zero
 * bits outside it, on the way in (scanned by up to 16 host threads during
 * the copy) and in the result (checked on the device); otherwise the whole
 * of v moves.  The results are the same bits either way. */
int ghost_hd_run(ghost_ctx *ctx, int nsteps, int ord, double dt, double nu, void *vx, void *vy, void *vz,
                 void *C1, void *C2, void *C3, const void *fx, const void *fy, const void *fz);

/* ---------------------------------------------------------------- */
/* Rotating stratified Boussinesq (ROTBOUSS solver) */

/* advect3(a,b,c,d,e) (pseudo/pseudospec3D_phd.f90:23-114): e = -(A.grad)d */
int ghost_advect3(ghost_ctx *ctx, const void *a, const void *b, const void *c, const void *d, void *e);
/* rotbouss_rkstep2 (include/rotbouss_rkstep2.f90:12-83); xmom and xtemp
 * already multiplied by bvfreq (main3D.fpp:973-974).  f, fs may be NULL. */
int ghost_bouss_rkstep2(ghost_ctx *ctx, int o, double dt, double nu, double kappa, double omegaz,
                        double xmom, double xtemp, void *vx, void *vy, void *vz, void *th,
                        const void *C1, const void *C2, const void *C3, const void *C20,
                        const void *fx, const void *fy, const void *fz, const void *fs);
/* nsteps steps of rotbouss_rkstep1 (include/rotbouss_rkstep1.f90) + RK2 */
int ghost_bouss_run(ghost_ctx *ctx, int nsteps, int ord, double dt, double nu, double kappa,
                    double omegaz, double xmom, double xtemp, void *vx, void *vy, void *vz, void *th,
                    const void *fx, const void *fy, const void *fz, const void *fs);

/* ---------------------------------------------------------------- */
/* Batches and ensembles of independent runs (no counterpart in GHOST,
 * whose runs are separate MPI jobs).  A batched context holds nruns runs of
 * one grid; its fields are nruns spectral fields one after the other
 * (nruns*(nx/2+1)*ny*nz complex), so every pass covers the whole batch in
 * one launch.  ghost_hd_run, the operators and the sums of ghost_energy
 * act on the whole batch; ghost_batch_* give per-run results. */
int ghost_ctx_create_batch(int nx, int ny, int nz, int nruns, int precision, ghost_ctx **ctx);
/* per-run viscosity (host array of nruns); ghost_hd_run then ignores its nu */
int ghost_batch_set_nu(ghost_ctx *ctx, const double *nu);
/* per-run energy(kin) into out[nruns] */
int ghost_batch_energy(ghost_ctx *ctx, const void *a, const void *b, const void *c, int kin, double *out);
/* per-run ghost_init_random_solenoidal with seeds[nruns] (updated in place) */
int ghost_batch_init_random_solenoidal(ghost_ctx *ctx, int32_t *seeds, double kdn, double kup, int shape,
                                       double amp, void *ox, void *oy, void *oz);

/* An ensemble: batches of cubic runs of several sizes advanced together.
 * Each class (size n[c], nruns[c] runs) is a batched context on its own
 * stream; one RK step of every class is captured in a CUDA graph and
 * replayed.  Runs are numbered class by class. */
typedef struct ghost_ensemble ghost_ensemble;
int ghost_ensemble_create(int nclasses, const int *n, const int *nruns, int precision, ghost_ensemble **ens);
int ghost_ensemble_destroy(ghost_ensemble *ens);
/* device pointers of class c's batched velocity.  The replayed steps of
 * ghost_ensemble_run take every mode outside the kept set (kn2 > kmax, and
 * k = 0) to be zero, as every step leaves it, and do not rewrite it: values
 * written through these pointers between runs must keep those modes zero. */
int ghost_ensemble_fields(ghost_ensemble *ens, int c, void **vx, void **vy, void **vz);
/* the batched context of class c (for operators and diagnostics) */
int ghost_ensemble_class(ghost_ensemble *ens, int c, ghost_ctx **ctx);
/* seeded initial velocities (the recipe of ghost_init_random_solenoidal
 * with kdn, kup = kup_frac*n, shape, amp) and per-run viscosities */
int ghost_ensemble_init(ghost_ensemble *ens, const int32_t *seeds, double kdn, double kup_frac, int shape,
                        double amp, const double *nu);
/* Times each tile variant of every class on a copy of its state and keeps
 * the fastest; cfg_out[c] receives the choice (may be NULL).  Then, where
 * one launch per pass is allowed (ghost_ensemble_set_mode), times a step in
 * each mode and keeps the faster (ghost_ensemble_get_mode reports it). */
int ghost_ensemble_autotune(ghost_ensemble *ens, int ord, double dt, int *cfg_out);
/* nsteps RK steps of every run; after one uncaptured step the step is a
 * replayed CUDA graph */
int ghost_ensemble_run(ghost_ensemble *ens, int nsteps, int ord, double dt);
/* How the ensemble runs its passes: multi = 1 (allowed for at most 4
 * classes of 16..128 points per side) makes each of the five passes of a
 * substep one kernel launch over every class, each CTA working for one
 * class (a tile table splits the persistent CTAs in proportion to the
 * classes' tiles); multi = 0 (the default) runs every class's own launches
 * on its own stream, with the per-class tile variants of
 * ghost_ensemble_autotune.  Both give the same bits.  Where multi = 1 is
 * allowed, ghost_ensemble_autotune times both modes and keeps the faster. */
int ghost_ensemble_set_mode(ghost_ensemble *ens, int multi);
int ghost_ensemble_get_mode(const ghost_ensemble *ens, int *multi);
/* per-run energy(kin), runs in class order */
int ghost_ensemble_energy(ghost_ensemble *ens, int kin, double *out);

/* ---------------------------------------------------------------- */
/* Seeded initial conditions (host RNG, GHOST's randu of
 * pseudo/pseudospec3D_mod.fpp:130-148) */

/* Random-phase vector potential on kdn <= |k| <= kup with the loop order,
 * seeding and Hermitian kx=0 plane of examples/initialfv.f90_random:16-134;
 * shape 0: amplitude 1/|k| (GHOST's forcing); shape 1: exp(-|k|^2/4)
 * (velocity with E(k) ~ k^4 exp(-2(k/2)^2)).  Then (out) = curl of it,
 * normalised to <|out|^2> = amp^2 (initialfv.f90_random:136-139).
 * *seed is updated as GHOST's seed variable is. */
int ghost_init_random_solenoidal(ghost_ctx *ctx, int32_t *seed, double kdn, double kup, int shape,
                                 double amp, void *ox, void *oy, void *oz);

/* ---------------------------------------------------------------- */
/* Learned subgrid-stress closure for LES (no counterpart in GHOST; GHOST's
 * own LES closure is the EDQNM closure of pseudo/pseudospec3D_edqnm.f90).
 * A 10 -> 64 -> 64 -> 6 MLP with GELU activations (tanh form:
 * z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))), BF16 tensor-core
 * products with FP32 accumulation, FP32 master weights and Adam.
 * Inputs per grid point: the 9 resolved velocity gradients du_i/dx_j
 * (row-major i, j) and the filter width; outputs: the 6 independent
 * components of the subgrid stress (xx, yy, zz, xy, xz, yz).
 * Parameters (FP32, GHOST_MLP_NPARAM): W1[64][10], b1[64], W2[64][64],
 * b2[64], W3[6][64], b3[6] (y = W x + b). */
#define GHOST_MLP_NIN 10
#define GHOST_MLP_NHID 64
#define GHOST_MLP_NOUT 6
#define GHOST_MLP_NPARAM 5254
typedef struct ghost_mlp ghost_mlp;
/* Glorot-uniform weights from a seeded host RNG, zero biases; the MLP lives
 * on the current device */
int ghost_mlp_create(int seed, ghost_mlp **mlp);
int ghost_mlp_destroy(ghost_mlp *mlp);
int ghost_mlp_set_stream(ghost_mlp *mlp, void *stream);
/* host copies of the FP32 parameters (set resets Adam's moments) */
int ghost_mlp_get_params(ghost_mlp *mlp, float *params);
int ghost_mlp_set_params(ghost_mlp *mlp, const float *params);
/* y[B][6] = mlp(x[B][10]); device arrays */
int ghost_mlp_forward(ghost_mlp *mlp, const float *x, float *y, int B);
/* gradient of the mean squared error mean((mlp(x) - t)^2) over B*6 values
 * (grad and loss on the host, either may be NULL); no update */
int ghost_mlp_gradients(ghost_mlp *mlp, const float *x, const float *t, int B, float *grad, double *loss);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on that loss; loss may
 * be NULL (then the call does not synchronise) */
int ghost_mlp_train_step(ghost_mlp *mlp, const float *x, const float *t, int B, float lr, double *loss);

/* ---------------------------------------------------------------- */
/* Large-eddy simulation on a cubic coarse grid n^3 with a sharp spectral
 * cutoff kc (modes kx^2+ky^2+kz^2 <= kc^2 are resolved; GHOST's sharp,
 * pseudo/pseudospec3D_filt.f90:200-241, with Delta = pi/kc).  Set the
 * coarse context's kmax to kc^2 (ghost_ctx_set_kmax) so that the LES
 * resolves exactly the filtered modes.  All field arguments are device
 * arrays of the coarse context unless named fine.  Closures:
 *   GHOST_LES_NONE   no subgrid term;
 *   GHOST_LES_EDQNM  GHOST's EDQNM closure, include/edqnmhd_rkstep2.f90
 *                    (heli = 0 unless ghost_les_set_helicity): the kinetic spectrum of the current
 *                    velocity gives tve(k) and tepq(k) (evedqnm: spec_fit +
 *                    cusp, pseudo/pseudospec3D_edqnm.f90:24-402), the update
 *                    uses nu + tve(k), and vcorrect (:405-1629) then sets
 *                    every mode's energy from tepq, keeping its helicity;
 *   GHOST_LES_MLP    the learned subgrid stress: tau = mlp(inputs) gives
 *                    the force -P div tau (P the Leray projection);
 *   GHOST_LES_MLP_SPECTRAL  a learned spectral eddy viscosity: the network
 *                    maps each resolved shell's inputs (ghost_les_spectral_features,
 *                    from the current kinetic spectrum) to tve(k) =
 *                    max(y0 tau_scale sqrt(E(kc)/kc), 0), applied as
 *                    EDQNM's tve is (the update uses nu + tve(k)), without
 *                    vcorrect. */
#define GHOST_LES_NONE 0
#define GHOST_LES_EDQNM 1
#define GHOST_LES_MLP 2
#define GHOST_LES_MLP_SPECTRAL 3
typedef struct ghost_les ghost_les;
int ghost_les_create(ghost_ctx *coarse, int kc, ghost_les **les);
int ghost_les_destroy(ghost_les *les);
/* out = the modes |k| <= kc of the fine spectrum in, on the coarse grid
 * (scaled by (n/N)^3, GHOST's unnormalised convention; analysis/trunc3D.fpp) */
int ghost_les_truncate(ghost_les *les, ghost_ctx *fine, const void *in, void *out);
/* Training samples from a fine (DNS) velocity, one per coarse grid point
 * (real layout, x fastest): x[q][0..8] = d ubar_a / dx_b (a-major),
 * x[q][9] = delta; tau[q][0..5] = filt(u_a u_b) - ubar_a ubar_b for xx, yy,
 * zz, xy, xz, yz, ubar = sharp-filtered u, filt(u_a u_b) from the fine
 * products.  x and tau are float device arrays of n^3 rows. */
int ghost_les_samples(ghost_les *les, ghost_ctx *fine, const void *vx, const void *vy, const void *vz, float delta,
                      float *x, float *tau);
/* the closure inputs of a coarse velocity: gradients times grad_scale, delta */
int ghost_les_features(ghost_les *les, const void *vx, const void *vy, const void *vz, float grad_scale, float delta,
                       float *x);
/* the spectral network's inputs: E a device array of the n/2+1 shell sums
 * of ghost_spectrumc (kin = 1; shell k at k-1), x a device float array of kc
 * rows of GHOST_MLP_NIN, row k-1 for shell k: k/kc, (k/kc)^2,
 * ln(E(k)/E(kc))/8, the local log-slope d ln E/d ln k /4 (centred, one-sided
 * at k = 1 and kc), the log-slope from kc/2 to kc /4, ln(kc E(kc)/sum E)/8,
 * exp(-(kc-k)/2), exp(-(kc-k)/8), 0, 0 (shell energies floored at 1e-30 of
 * the resolved sum) */
int ghost_les_spectral_features(ghost_les *les, const double *E, float *x);
/* o = f + P(-div tau), tau[q][6] rows scaled by tau_scale (f may be NULL) */
int ghost_les_tau_force(ghost_les *les, const float *tau, float tau_scale, const void *fx, const void *fy,
                        const void *fz, void *ox, void *oy, void *oz);
/* closure selection; the MLP maps inputs scaled by grad_scale (and delta)
 * to stresses scaled by 1/tau_scale; kolmo is EDQNM's Kolmogorov constant
 * (GHOST's default 1.4, main3D.fpp:1579).  The MLP is moved to the
 * context's stream. */
int ghost_les_set_model(ghost_les *les, int model, ghost_mlp *mlp, double grad_scale, double tau_scale, double delta,
                        double kolmo);
/* fallback of the MLP closure to EDQNM in ghost_les_run: every step then
 * starts from a saved copy of v, and a step that ends with a non-finite
 * <|v|^2>, or one above blowup (> 1) times its value when the call started,
 * is redone with the EDQNM closure (kolmo from ghost_les_set_model), which
 * stays selected.  Costs one energy reduction and a host sync per step. */
int ghost_les_set_fallback(ghost_les *les, int enable, double blowup);
/* the selected closure (GHOST_LES_*) and the step count of the LES's runs
 * at which the fallback switched to EDQNM (-1: it has not) */
int ghost_les_status(const ghost_les *les, int *model, long long *fell_back_at);
/* time handed to the EDQNM closure (GHOST's (t-1)*dt); ghost_les_run
 * advances it by dt per step */
int ghost_les_set_time(ghost_les *les, double t);
/* o = f + the selected closure's force for velocity v (f may be NULL) */
int ghost_les_closure_force(ghost_les *les, double nu, const void *vx, const void *vy, const void *vz, const void *fx,
                            const void *fy, const void *fz, void *ox, void *oy, void *oz);
/* nsteps RK steps (order ord) of the LES; each substep evaluates the
 * closure on the current velocity and runs the fused HD substep with
 * f + closure force as its forcing (f may be NULL) */
int ghost_les_run(ghost_les *les, int nsteps, int ord, double dt, double nu, void *vx, void *vy, void *vz,
                  const void *fx, const void *fy, const void *fz);
/* the last EDQNM evaluation (host arrays of n/2+1, GHOST's 1-based index
 * k stored at k-1); any pointer may be NULL */
int ghost_les_edqnm_last(ghost_les *les, double *tve, double *tepq, double *Ek);
/* GHOST's heli flag for the EDQNM closure (include/edqnmhd_rkstep2.f90;
 * default 0): with heli = 1 the closure also takes the helicity spectrum,
 * fits E over 3kc/4 - 2 shells and H over 3kc/4, and (when both fits have a
 * positive index) runs full_cusp (pseudo/pseudospec3D_edqnm.f90:174-277),
 * which gives the helicity eddy diffusivity tvh(k) and transfer thpq(k);
 * the update adds tvh(k) curl v and vcorrect sets every mode's helicity to
 * w2 + thpq(km) dt hf / hold(km) (:536-540) as well as its energy. */
int ghost_les_set_helicity(ghost_les *les, int heli);
/* the last helical EDQNM evaluation (host arrays of n/2+1): tvh, thpq and
 * the helicity spectrum Hk; any pointer may be NULL */
int ghost_les_edqnm_last_hel(ghost_les *les, double *tvh, double *thpq, double *Hk);
/* evedqnm(Eold,Hold,nu,time,hel,tepq,thpq,tve,tvh,Ext,Hxt)
 * (pseudo/pseudospec3D_edqnm.f90:24-92) on the host, GHOST's full
 * signature: Eold, Hold[n/2+1] -> tepq, thpq, tve, tvh[n/2+1] and the
 * extrapolations Ext, Hxt[3(n/2+1)] (halved by full_cusp when it runs);
 * with hel = 0, Hold, thpq, tvh and Hxt may be NULL. */
int ghost_evedqnm_hel(int n, int precision, double kmax, double kolmo, const double *Eold, const double *Hold,
                      double nu, double time, int hel, double *tepq, double *thpq, double *tve, double *tvh,
                      double *Ext, double *Hxt);
/* evedqnm with heli = 0 on the host: Eold[n/2+1] -> tepq, tve[n/2+1] and
 * the extrapolated spectrum Ext[3(n/2+1)]; precision selects GHOST's GP
 * kind for the fit and quadrature (GHOST_SINGLE or GHOST_DOUBLE) */
int ghost_evedqnm(int n, int precision, double kmax, double kolmo, const double *Eold, double nu, double time,
                  double *tepq, double *tve, double *Ext);

/* ------------------------------------------------------------------
 * GHOST's binary field files (mpiio/binary_io.f90:13-186): one raw file
 * per field holding r(nx,ny,nz) in Fortran order (x fastest), GP precision
 * (the context's), native byte order, no header.  swap != 0 reverses the
 * bytes of every value (GHOST's iswap / oswap).  Fields may be device or
 * host arrays.  Batched contexts: GHOST_ERR_STATE (one file per run).
 * ------------------------------------------------------------------ */
/* "<dir>/<name>.<index>.out", index zero-padded to width digits (GHOST's
 * fmtext '(i4.4)' is width 4; a wider index prints as width asterisks) */
int ghost_io_filename(const char *dir, const char *name, int index, int width, char *buf, size_t len);
/* io_write(unit,dir,fname,nmb,plan,var): a real field to path */
int ghost_io_write(ghost_ctx *ctx, const void *real, const char *path, int swap);
/* io_read(unit,dir,fname,nmb,plan,var): path (exactly nx*ny*nz values,
 * else GHOST_ERR_SIZE) into a real field */
int ghost_io_read(ghost_ctx *ctx, const char *path, int swap, void *real);
/* one field of GHOST's output step (main3D.fpp:2678-2709): the real field
 * of spec/(nx ny nz) (fftp3d_complex_to_real), written as io_write does;
 * spec is left unmodified */
int ghost_io_output(ghost_ctx *ctx, const void *spec, const char *path, int swap);
/* one field of GHOST's restart (main3D.fpp:2155-2161): io_read, then
 * fftp3d_real_to_complex into spec (so output then restart gives spec back) */
int ghost_io_restart(ghost_ctx *ctx, const char *path, int swap, void *spec);

/* ---------------------------------------------------------------- */
/* Slab decomposition of one run over ranks (GHOST's MPI layout).
 * Rank r holds the kx-slab of the spectral fields, kx rows ista_r..,
 * as (nxh_loc, ny, nz) arrays (Fortran (nz,ny,ista:iend)), and works on
 * the z-slab (nxh, ny, nz_loc) (Fortran (nz_loc planes, ny, nx/2+1)) in the
 * x pass; the slabs follow range() (fftp-3/fftp.f90, main3D.fpp:634-635).
 * One HD substep (include/hd_rkstep2.f90, with hd_rkstep1 when copy) is
 *   ghost_slab_hd_front -> ghost_slab_pack(0) -> all-to-all ->
 *   ghost_slab_unpack(0) -> ghost_slab_hd_xpass -> ghost_slab_pack(1) ->
 *   all-to-all -> ghost_slab_unpack(1) -> ghost_slab_hd_back,
 * the all-to-alls taking the place of the transposes of
 * fftp-3/fftp3D.fpp:158-201,255-278 (the caller runs them: NCCL, or copies
 * between ranks that one process holds).  Send and receive buffers are
 * peer-major; in direction 0 the chunk for peer p holds nf blocks of
 * nxh_loc[me] x ny x nz_loc[p] complex values and the chunk from p nf
 * blocks of nxh_loc[p] x ny x nz_loc[me]; direction 1 is the reverse.
 * Every z-slab must hold a multiple of 8 planes (GHOST_ERR_SIZE).  All
 * arrays are device arrays; the calls are asynchronous on the slab's
 * stream.  prune: a substep whose v is zero outside the truncation (every
 * substep after the first of a run, as ghost_hd_run does) runs pruned
 * passes, and its exchanges move only the kx rows below ghost_slab_rows
 * (a rank's live rows are a prefix of its slab: min(rows - ista_r,
 * nxh_loc_r) rows, clamped at 0, take the place of nxh_loc_r above). */
typedef struct ghost_slab ghost_slab;
/* range(n1,n2,nprocs,irank,ista,iend) of GHOST (1-based, inclusive) */
int ghost_slab_range(int n1, int n2, int nprocs, int irank, int *ista, int *iend);
int ghost_slab_create(int nx, int ny, int nz, double Lx, double Ly, double Lz, int arbsize, int precision, int rank,
                      int nranks, ghost_slab **out);
int ghost_slab_destroy(ghost_slab *s);
/* per-rank 0-based kx-row starts, kx-row counts, z-plane starts, z-plane
 * counts (arrays of nranks ints; any may be NULL) */
int ghost_slab_layout(const ghost_slab *s, int *ista, int *nxh_loc, int *ksta, int *nz_loc);
/* the kx rows 0..rows-1 that hold every mode with kn2 <= kmax */
int ghost_slab_rows(const ghost_slab *s, int *rows);
/* kernels this rank's slab contexts have launched (ghost_ctx_launch_count) */
int ghost_slab_launch_count(const ghost_slab *s, long long *count);
int ghost_slab_set_stream(ghost_slab *s, void *stream);
int ghost_slab_synchronize(ghost_slab *s);
/* Z inverse and Y inverse of the substep on the kx-slab: v -> w[0..2] = v,
 * w[3..5] = curl v (rotor3), inverse-transformed along z and y; C = v when
 * copy (hd_rkstep1) */
int ghost_slab_hd_front(ghost_slab *s, const void *const v[3], void *const C[3], int copy, int prune,
                        void *const w[6]);
/* the x pass (prodre3's real-space product and the x transforms) on the
 * z-slab: in[0..5] -> out[0..2] = omega x v / (nx ny nz)^2, x transformed
 * back (out may alias in[0..2]) */
int ghost_slab_hd_xpass(ghost_slab *s, int prune, const void *const in[6], void *const out[3]);
/* Y forward, Z forward and the truncated update of substep o on the
 * kx-slab: w[0..2] (from the x pass) -> v = C + dt (nu lap v + NL + f)/o
 * (f NULL, or f[0] NULL: no forcing) */
int ghost_slab_hd_back(ghost_slab *s, int o, double dt, double nu, int prune, void *const w[3], void *const v[3],
                       const void *const C[3], const void *const f[3]);
/* the blocks of nf fields for every peer into send (dir 0: from kx-slab
 * fields; dir 1: from z-slab fields) */
int ghost_slab_pack(ghost_slab *s, int dir, int nf, int prune, const void *const *fields, void *send);
/* the blocks from every peer out of recv into nf fields (dir 0: z-slab
 * fields; dir 1: kx-slab fields) */
int ghost_slab_unpack(ghost_slab *s, int dir, int nf, int prune, const void *recv, void *const *fields);
/* on = 1: ghost_slab_pack and ghost_slab_unpack skip the rank's own block
 * (its chunk in the send and receive buffers has size 0), and
 * ghost_slab_exchange_self moves it from the source fields straight into
 * the destination fields; the all-to-all then carries only the peers'
 * blocks.  Default 0 (the own block travels through the buffers). */
int ghost_slab_set_self_direct(ghost_slab *s, int on);
/* the rank's own block of an exchange of nf fields, field to field: dir 0
 * from kx-slab fields (in) into z-slab fields (out), dir 1 the reverse
 * (the transposes' local part, fftp-3/fftp3D.fpp:158-201) */
int ghost_slab_exchange_self(ghost_slab *s, int dir, int nf, int prune, const void *const *in, void *const *out);
/* The front and back phases split around their Y passes, so that the
 * exchange of some fields can run while the others are transformed:
 * ghost_slab_hd_front = ghost_slab_hd_front_z, then ghost_slab_ypass(+1)
 * of the six fields (in any grouping); ghost_slab_hd_back =
 * ghost_slab_ypass(-1) of the three fields (in any grouping), then
 * ghost_slab_hd_back_z.  A line's arithmetic does not depend on the
 * grouping: the results are the same bits. */
int ghost_slab_hd_front_z(ghost_slab *s, const void *const v[3], void *const C[3], int copy, int prune,
                          void *const w[6]);
/* the Y pass (sign +1 inverse, -1 forward) of nf <= 9 kx-slab fields */
int ghost_slab_ypass(ghost_slab *s, int sign, int nf, int prune, void *const *fields);
int ghost_slab_hd_back_z(ghost_slab *s, int o, double dt, double nu, int prune, void *const w[3], void *const v[3],
                         const void *const C[3], const void *const f[3]);

#ifdef __cplusplus
}
#endif
#endif /* GHOST_B200_H */
