// common.cuh -- context state, wavenumber parameters and error plumbing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "../../include/ghost_b200.h"
#include "fft_core.cuh"

namespace gb {

// Thread-local last error, reported by ghost_last_error_string().
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);

#define GB_CUDA(call)                                                                     \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return ::gb::fail(GHOST_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,        \
                        cudaGetErrorString(e_));                                          \
  } while (0)

#define GB_CHECK(expr)          \
  do {                          \
    int s_ = (expr);            \
    if (s_ != GHOST_OK) return s_; \
  } while (0)

// Wavenumber state passed by value to kernels (the kes/ali modules).
// Wavenumbers are rebuilt from indices with the operation order of
// main3D.fpp:1746-1800, so they match the host tables bit for bit.
template <typename R> struct KParams {
  int nx, ny, nz, nxh;
  int anis, arbsize;
  R Dkx, Dky, Dkz;
  R rmp, rmq, rms;  // per-axis normalisation of kn2 when anis
  R kmax, tiny;
  R tmp;            // 1/(nx ny nz)^2
  // batches of independent runs of one grid: fields hold nruns runs one
  // after the other, i.e. the kx index runs over nxh*nruns
  int nruns;
  const R *nu_run;  // per-run viscosity (batched RK), or null
  // global index of the first local kx row (a kx-slab of a decomposed
  // grid; 0 otherwise): the passes' row i of a field is kx row i + i0
  int i0;
};

template <typename R> __device__ __forceinline__ R kx_of(const KParams<R> &p, int i) {
  R v = (R)(i < p.nx / 2 ? i : i - p.nx);
  return p.arbsize ? v * p.Dkx : v;
}
template <typename R> __device__ __forceinline__ R ky_of(const KParams<R> &p, int j) {
  R v = (R)(j < p.ny / 2 ? j : j - p.ny);
  return p.arbsize ? v * p.Dky : v;
}
template <typename R> __device__ __forceinline__ R kz_of(const KParams<R> &p, int k) {
  R v = (R)(k < p.nz / 2 ? k : k - p.nz);
  return p.arbsize ? v * p.Dkz : v;
}
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }

// kn2 (dealias measure) with the unfused operation order of main3D.fpp:1778
template <typename R> __device__ __forceinline__ R kn2_of(const KParams<R> &p, int i, int j, int k) {
  R a = (R)(i < p.nx / 2 ? i : i - p.nx), b = (R)(j < p.ny / 2 ? j : j - p.ny),
    c = (R)(k < p.nz / 2 ? k : k - p.nz);
  if (p.anis)
    return radd(radd(rmul(p.rmp, rmul(a, a)), rmul(p.rmq, rmul(b, b))), rmul(p.rms, rmul(c, c)));
  return radd(radd(rmul(a, a), rmul(b, b)), rmul(c, c));
}
// kk2 (physical |k|^2), main3D.fpp:1790-1800
template <typename R> __device__ __forceinline__ R kk2_of(const KParams<R> &p, int i, int j, int k) {
  if (!p.anis) return kn2_of(p, i, j, k);
  R a = kx_of(p, i), b = ky_of(p, j), c = kz_of(p, k);
  return radd(radd(rmul(a, a), rmul(b, b)), rmul(c, c));
}

struct DeviceBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace gb

// The opaque context of the C ABI.
struct ghost_ctx {
  int nx, ny, nz, nxh;
  int precision;     // GHOST_SINGLE or GHOST_DOUBLE
  int arbsize, anis;
  int nmax, nmaxperp;
  double Lx, Ly, Lz, Dkx, Dky, Dkz, Dkk;
  double kmax, tiny;
  size_t nspec, nreal;   // elements per spectral / real field
  size_t cbytes, rbytes; // bytes per spectral / real field
  int device;
  cudaStream_t stream;
  long long launches;
  // device twiddle tables exp(-2 pi i e/n) for n = nx, ny, nz (precision of ctx)
  void *tw_x, *tw_y, *tw_z;
  // scratch spectral fields (allocated on demand, grow only)
  std::vector<void *> scratch;
  // FP64 partial sums for deterministic reductions
  double *partials;
  size_t partials_elems;
  // staging buffers for host-array calls
  std::vector<void *> stage;
  // RK storage owned by the context when the caller passes none
  void *rk[4];
  gb::KParams<float> kp32;
  gb::KParams<double> kp64;
  int nruns;          // runs in a batched context (1 otherwise)
  size_t ntot;        // nspec * nruns
  // slab decomposition: the first kx row of a kx-slab context (0 otherwise),
  // and the global nz (the normalisation of a z-slab context's x pass)
  int i0, nz_glob;
  void *nu_run;       // per-run viscosity on the device (precision of ctx), or null
  int tile_cfg;       // tile variant (bit 0: y tile 16 wide, bit 1: z CTAs of 128 threads, bits 1+2: two-stage z ring,
                      // bit 3: two-stage y ring with a second exchange buffer)
  int num_sms;
  // device status word written by kernels whose bounded waits ran out
  int *status;
  uint32_t wait_cap;
  int inject_stall;  // fault injection (ghost_ctx_inject_stall)
  // zero-pruning tables of the 2/3 truncation (built on first use):
  // active (j,i) z-lines padded with -1 to a multiple of 256, the
  // contiguous live y-wavenumber counts per kx index, and the last live kx
  bool prune_valid, prune_ok;
  int *prune_lines, *prune_jpos, *prune_jneg;
  int prune_nlines, prune_imax;
  int prune_jtop, prune_jbot;  // largest live y-line counts from the top and the bottom over the kx rows
  int prune_ktop, prune_kbot;  // live kz counts from the top and the bottom of a z-line
  // host-array calls: a device flag and its pinned host copy (nonzero values
  // beyond the live kx rows of a staged field), allocated on first use
  int *dead_flag, *dead_flag_host;
  // host-array calls: a second stream for inputs needed late in a substep
  // (the forcing), the event after the early inputs, the event the next
  // forcing read waits on (f_pending), all created on first use
  cudaStream_t side;
  cudaEvent_t ev_early, ev_late;
  bool late_pending;
  // per-kernel timers (ghost_ctx_enable_timers)
  bool timers_on;
  std::vector<cudaEvent_t> ev_free;
  struct Pending {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Pending> ev_pending;
  double t_ms[GHOST_TIMER_KINDS];
  long long t_n[GHOST_TIMER_KINDS];
};

struct ghost_fftplan {
  ghost_ctx *ctx;
  int fftdir;
};
