// api.cu -- the C ABI of include/ghost_b200.h: context, FFT plans,
// spectral operators, reductions and the fused RK substeps.
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <thread>
#include <vector>

#include <cudaTypedefs.h>

#include "common.cuh"
#include "ic_host.h"
#include "internal.cuh"
#include "ops.cuh"
#include "passes.cuh"
#include "xwarp.cuh"
#include "ensemble.cuh"

namespace gb {

// ---------------------------------------------------------------------
// errors
static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}


static bool pow2_ok(int n) { return n >= 16 && n <= 1024 && (n & (n - 1)) == 0; }

// ---------------------------------------------------------------------
// device memory helpers
int dalloc(void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(GHOST_ERR_ALLOC, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  }
  return GHOST_OK;
}

// scratch spectral fields 0..n-1 (each cbytes), grown on demand
int scratch(ghost_ctx *c, int n, void **out) {
  while ((int)c->scratch.size() < n) {
    void *p;
    GB_CHECK(dalloc(&p, c->cbytes));
    c->scratch.push_back(p);
  }
  for (int q = 0; q < n; ++q) out[q] = c->scratch[q];
  return GHOST_OK;
}

static int partials(ghost_ctx *c, size_t n, double **out) {
  if (c->partials_elems < n) {
    if (c->partials) cudaFree(c->partials);
    c->partials = nullptr;
    c->partials_elems = 0;
    void *p;
    GB_CHECK(dalloc(&p, n * sizeof(double)));
    c->partials = (double *)p;
    c->partials_elems = n;
  }
  *out = c->partials;
  return GHOST_OK;
}

// ---------------------------------------------------------------------
// host-array staging: pointers that are not device memory are copied
// through context buffers, and the call syncs before returning.
bool is_device_ptr(const void *p) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int check_status(ghost_ctx *c);

// The live box of a spectral field: kx rows [0, live), in each the y-lines
// [0, jt) and [ny - jb, ny), and in each of those the 16-byte words
// [0, kt) and [line - kb, line) of the z-line (a field of nruns runs of
// `rows` kx rows of ny lines of line_u4 16-byte words; the z bounds are
// rounded out to whole words).  flag |= 1 when any word outside the box is
// nonzero.
struct LiveBox {
  int rows, live, ny, jt, jb;
  size_t line_u4, kt, kb;
};
__global__ void dead_box_kernel(const uint4 *__restrict__ p, int nruns, LiveBox b, int *__restrict__ flag) {
  const int mid = b.ny - b.jt - b.jb;                // lines between the two live blocks of a live row
  const size_t midz = b.line_u4 - b.kt - b.kb;       // words between the two live z-blocks of a box line
  const size_t part_a = (size_t)(b.rows - b.live) * b.ny * b.line_u4;  // the rows beyond the live ones
  const size_t part_b = (size_t)b.live * mid * b.line_u4;               // the middle lines of the live rows
  const size_t part_c = (size_t)b.live * (b.jt + b.jb) * midz;         // the middle words of the box lines
  const size_t per_run = part_a + part_b + part_c, total = per_run * nruns;
  bool any = false;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const size_t r = q / per_run;
    size_t o = q - r * per_run, idx;
    if (o < part_a) {
      idx = ((size_t)r * b.rows + b.live) * b.ny * b.line_u4 + o;
    } else if (o < part_a + part_b) {
      o -= part_a;
      const size_t per_row = (size_t)mid * b.line_u4, row = o / per_row, rem = o - row * per_row;
      const size_t line = b.jt + rem / b.line_u4, w = rem % b.line_u4;
      idx = (((size_t)r * b.rows + row) * b.ny + line) * b.line_u4 + w;
    } else {
      o -= part_a + part_b;
      const size_t per_row = (size_t)(b.jt + b.jb) * midz, row = o / per_row, rem = o - row * per_row;
      const size_t lb = rem / midz, w = rem % midz;
      const size_t line = lb < (size_t)b.jt ? lb : (size_t)(b.ny - b.jb) + (lb - b.jt);
      idx = (((size_t)r * b.rows + row) * b.ny + line) * b.line_u4 + b.kt + w;
    }
    const uint4 v = p[idx];
    any |= (v.x | v.y | v.z | v.w) != 0u;
  }
  if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// the context stream waits for late inputs still in flight (ghost_ctx::late_pending)
static int late_wait(ghost_ctx *c) {
  if (c->late_pending) {
    GB_CUDA(cudaStreamWaitEvent(c->stream, c->ev_late, 0));
    c->late_pending = false;
  }
  return GHOST_OK;
}

// Staging of host arrays for a call on device fields.  Two kinds of field
// move only their live box (LiveBox: the kx rows that hold a mode of the
// truncation and, in them, the two blocks of y-lines that do):
//   IN_LIVE:  an input read only at kept modes and only late in a substep
//             (the forcing): the box goes in on a side stream after the
//             early inputs, while the work starts, and the read waits for it
//             (late_wait); the rest of the staging buffer is never read;
//   OUT_LIVE: an in/out field that the call leaves zero outside the kept
//             modes (the velocity).  The box goes in while host threads scan
//             the rest of the host array: if it holds only zero bits, the
//             device copy is zeroed there, else the whole field goes in.  The
//             box comes back when the result also holds zero bits outside it
//             (a device check; then the host array already holds them), else
//             the whole field comes back.
struct Staging {
  static constexpr int IN = 1, OUT = 2, IN_LIVE = 4, OUT_LIVE = 8;
  ghost_ctx *c;
  int used = 0;
  bool any_host = false;
  struct Back {
    void *host;
    const void *dev;
    size_t bytes;
    bool live;   // the box comes back unless the result check finds bits outside it
    bool whole;  // the input held nonzero bits outside the box: the whole field comes back
  };
  std::vector<Back> back;
  // the live box (live = 0: unknown, whole fields move)
  LiveBox box{0, 0, 0, 0, 0, 0, 0, 0};
  size_t line_bytes = 0;
  bool flag_armed = false;
  explicit Staging(ghost_ctx *ctx) : c(ctx) {}
  // kt, kb: live values from the top and the bottom of a z-line of `elem`
  // bytes each (rounded out to 16-byte words)
  void set_live(int live_rows, int run_rows, int ny, int jt, int jb, int nz, int kt, int kb, size_t elem) {
    const size_t line_u4 = (size_t)nz * elem / 16;
    const size_t kt_u4 = std::min(line_u4, ((size_t)kt * elem + 15) / 16);
    const size_t kb_u4 = std::min(line_u4 - kt_u4, ((size_t)kb * elem + 15) / 16);
    box = LiveBox{run_rows, live_rows, ny, jt, jb, line_u4, kt_u4, kb_u4};
    line_bytes = (size_t)nz * elem;
  }
  bool live_ok(size_t bytes) const {
    return box.live > 0 && line_bytes % 16 == 0 && box.jt + box.jb <= box.ny &&
           box.kt + box.kb <= box.line_u4 &&
           (size_t)box.rows * box.ny * line_bytes * c->nruns == bytes;
  }
  // nonzero bits in a host array outside the box (up to 16 host threads,
  // rows dealt round robin; an array not 8-byte aligned counts as nonzero)
  bool host_outside_nonzero(const void *host) const {
    if (((uintptr_t)host & 7u) != 0) return true;
    const size_t row_b = (size_t)box.ny * line_bytes, nrows = (size_t)box.rows * c->nruns;
    const size_t z_lo = box.kt * 16, z_hi = line_bytes - box.kb * 16;  // the middle bytes of a box line
    std::atomic<bool> found(false);
    auto any_bits = [](const unsigned char *p, size_t n) {
      const uint64_t *w = (const uint64_t *)p;
      uint64_t acc = 0;
      for (size_t k = 0; k < n / 8; ++k) acc |= w[k];
      return acc != 0;
    };
    auto scan = [&](int tid, int nth) {
      for (size_t q = tid; q < nrows && !found.load(std::memory_order_relaxed); q += nth) {
        const size_t row = q % box.rows;
        const unsigned char *base = (const unsigned char *)host + q * row_b;
        bool hit = false;
        if (row >= (size_t)box.live) {
          hit = any_bits(base, row_b);
        } else {
          for (int j = 0; j < box.ny && !hit; ++j) {
            const unsigned char *line = base + (size_t)j * line_bytes;
            hit = (j >= box.jt && j < box.ny - box.jb) ? any_bits(line, line_bytes)
                                                        : (z_hi > z_lo && any_bits(line + z_lo, z_hi - z_lo));
          }
        }
        if (hit) found.store(true, std::memory_order_relaxed);
      }
    };
    const int nth = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 1; t < nth; ++t) pool.emplace_back(scan, t, nth);
    scan(0, nth);
    for (auto &th : pool) th.join();
    return found.load();
  }
  // zero a device field outside the box
  int zero_outside(void *dev) {
    const size_t pitch = (size_t)box.ny * line_bytes, run_b = (size_t)box.rows * pitch;
    const size_t midz = (box.line_u4 - box.kt - box.kb) * 16;
    for (int r = 0; r < c->nruns; ++r) {
      unsigned char *base = (unsigned char *)dev + (size_t)r * run_b;
      if (box.rows > box.live)
        GB_CUDA(cudaMemsetAsync(base + (size_t)box.live * pitch, 0, (size_t)(box.rows - box.live) * pitch, c->stream));
      const int mid = box.ny - box.jt - box.jb;
      if (mid > 0)
        GB_CUDA(cudaMemset2DAsync(base + (size_t)box.jt * line_bytes, pitch, 0, (size_t)mid * line_bytes, box.live,
                                  c->stream));
      // the middle of the box lines: a 3D block (z bytes, lines, rows) per line block
      const int j0[2] = {0, box.ny - box.jb}, nj[2] = {box.jt, box.jb};
      for (int q = 0; q < 2 && midz > 0; ++q) {
        if (nj[q] == 0) continue;
        cudaPitchedPtr pp = make_cudaPitchedPtr(base, line_bytes, line_bytes, box.ny);
        pp.ptr = base + (size_t)j0[q] * line_bytes + box.kt * 16;
        GB_CUDA(cudaMemset3DAsync(pp, 0, make_cudaExtent(midz, nj[q], box.live), c->stream));
      }
    }
    return GHOST_OK;
  }
  // the four blocks of the box of every run (two line blocks times two z
  // blocks, each a 3D copy of z bytes x lines x rows), host <-> device
  int copy_box(void *dst, const void *src, cudaMemcpyKind kind, cudaStream_t stream = nullptr) {
    if (!stream) stream = c->stream;
    const size_t pitch = (size_t)box.ny * line_bytes, run_b = (size_t)box.rows * pitch;
    const int j0[2] = {0, box.ny - box.jb}, nj[2] = {box.jt, box.jb};
    const size_t z0[2] = {0, line_bytes - box.kb * 16}, nz[2] = {box.kt * 16, box.kb * 16};
    for (int r = 0; r < c->nruns; ++r)
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
          if (nj[a] == 0 || nz[b] == 0) continue;
          cudaMemcpy3DParms prm = {};
          prm.srcPtr = make_cudaPitchedPtr(const_cast<void *>(src), line_bytes, line_bytes, box.ny);
          prm.dstPtr = make_cudaPitchedPtr(dst, line_bytes, line_bytes, box.ny);
          prm.srcPos = prm.dstPos = make_cudaPos(z0[b], (size_t)j0[a], (size_t)r * box.rows);
          prm.extent = make_cudaExtent(nz[b], nj[a], box.live);
          prm.kind = kind;
          GB_CUDA(cudaMemcpy3DAsync(&prm, stream));
        }
    (void)run_b;
    return GHOST_OK;
  }
  int check_dead(const void *dev) {
    if (!c->dead_flag) {
      GB_CHECK(dalloc((void **)&c->dead_flag, sizeof(int)));
      GB_CUDA(cudaMallocHost((void **)&c->dead_flag_host, sizeof(int)));
    }
    if (!flag_armed) {
      GB_CUDA(cudaMemsetAsync(c->dead_flag, 0, sizeof(int), c->stream));
      flag_armed = true;
    }
    const size_t total = (((size_t)(box.rows - box.live) * box.ny + (size_t)box.live * (box.ny - box.jt - box.jb)) *
                              box.line_u4 +
                          (size_t)box.live * (box.jt + box.jb) * (box.line_u4 - box.kt - box.kb)) *
                         c->nruns;
    const int grid = (int)std::max<size_t>(1, std::min<size_t>((total + 255) / 256, 148 * 8));
    dead_box_kernel<<<grid, 256, 0, c->stream>>>((const uint4 *)dev, c->nruns, box, c->dead_flag);
    GB_CUDA(cudaGetLastError());
    return GHOST_OK;
  }
  int buffer(void **out) {
    while ((int)c->stage.size() <= used) {
      void *p;
      GB_CHECK(dalloc(&p, c->cbytes));
      c->stage.push_back(p);
    }
    *out = c->stage[used++];
    return GHOST_OK;
  }
  // dir: 1 in, 2 out, 3 in/out
  template <typename T> int map(T *user, size_t bytes, int dir, T **dev) {
    if (user == nullptr) {
      *dev = nullptr;
      return GHOST_OK;
    }
    if (is_device_ptr(user)) {
      // the passes move tiles with TMA bulk copies: 16-byte alignment
      if (((uintptr_t)(const void *)user & 15u) != 0)
        return fail(GHOST_ERR_ARG, "device array %p is not 16-byte aligned", (const void *)user);
      *dev = user;
      return GHOST_OK;
    }
    any_host = true;
    void *d;
    GB_CHECK(buffer(&d));
    const bool lv = (dir & (IN_LIVE | OUT_LIVE)) && live_ok(bytes);
    if ((dir & IN_LIVE) && lv) {
      late.push_back({(const void *)user, d});  // copied by resolve() on the side stream
    } else if ((dir & IN) && (dir & OUT_LIVE) && lv) {
      GB_CHECK(copy_box(d, (const void *)user, cudaMemcpyHostToDevice));  // in flight while resolve() scans
      pending.push_back({(const void *)user, d, bytes, back.size()});
    } else if (dir & IN) {
      GB_CUDA(cudaMemcpyAsync(d, (const void *)user, bytes, cudaMemcpyHostToDevice, c->stream));
    }
    if (dir & OUT) back.push_back({(void *)user, d, bytes, (dir & OUT_LIVE) && lv, false});
    *dev = (T *)d;
    return GHOST_OK;
  }
  // OUT_LIVE inputs whose boxes are in flight: the host scans the rest of
  // each while the copies run, then zeroes the device copy there or sends
  // the whole field (call after the last map, before the work)
  struct Pending {
    const void *host;
    void *dev;
    size_t bytes;
    size_t back_index;  // the field's entry in back, or back.size() for an input only
  };
  std::vector<Pending> pending;
  // IN_LIVE inputs (read late in a substep): their boxes go on the side
  // stream after the early inputs, while the work starts; the first read
  // waits on ev_late (late_wait)
  struct Late {
    const void *host;
    void *dev;
  };
  std::vector<Late> late;
  int resolve() {
    // the late boxes first, on the side stream after the early boxes (and
    // after the last call's reads of these buffers), so that the copies run
    // back to back while the host scans
    if (!late.empty()) {
      if (!c->side) {
        GB_CUDA(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
        GB_CUDA(cudaEventCreateWithFlags(&c->ev_early, cudaEventDisableTiming));
        GB_CUDA(cudaEventCreateWithFlags(&c->ev_late, cudaEventDisableTiming));
      }
      GB_CUDA(cudaEventRecord(c->ev_early, c->stream));
      GB_CUDA(cudaStreamWaitEvent(c->side, c->ev_early, 0));
      for (auto &l : late) GB_CHECK(copy_box(l.dev, l.host, cudaMemcpyHostToDevice, c->side));
      GB_CUDA(cudaEventRecord(c->ev_late, c->side));
      c->late_pending = true;
      late.clear();
    }
    for (auto &p : pending) {
      const bool whole = host_outside_nonzero(p.host);
      if (whole) {
        GB_CUDA(cudaMemcpyAsync(p.dev, p.host, p.bytes, cudaMemcpyHostToDevice, c->stream));
        if (p.back_index < back.size()) {
          back[p.back_index].live = false;
          back[p.back_index].whole = true;
        }
      } else {
        GB_CHECK(zero_outside(p.dev));
      }
    }
    pending.clear();
    return GHOST_OK;
  }
  int finish();
};

int Staging::finish() {
  if (!pending.empty() || !late.empty()) return fail(GHOST_ERR_STATE, "staged inputs left unresolved");
  GB_CHECK(late_wait(c));  // a call with no step still orders the late copies before returning
  bool any_live = false;
  for (auto &b : back)
    if (b.live) {
      GB_CHECK(check_dead(b.dev));  // the result outside the live box
      any_live = true;
    }
  if (any_live) GB_CUDA(cudaMemcpyAsync(c->dead_flag_host, c->dead_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  for (auto &b : back) {
    if (b.live)
      GB_CHECK(copy_box(b.host, b.dev, cudaMemcpyDeviceToHost));
    else
      GB_CUDA(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, c->stream));  // whole field
  }
  if (!any_host) return GHOST_OK;
  GB_CUDA(cudaStreamSynchronize(c->stream));
  if (any_live && *c->dead_flag_host != 0) {
    // nonzero bits outside the live box in a result: the whole field comes back
    for (auto &b : back)
      if (b.live) GB_CUDA(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, c->stream));
    GB_CUDA(cudaStreamSynchronize(c->stream));
  }
  return check_status(c);
}

template <typename R> const KParams<R> &kparams(const ghost_ctx *c);
template <> const KParams<float> &kparams<float>(const ghost_ctx *c) { return c->kp32; }
template <> const KParams<double> &kparams<double>(const ghost_ctx *c) { return c->kp64; }

int post_launch(ghost_ctx *c) {
  c->launches++;
  GB_CUDA(cudaGetLastError());
  return GHOST_OK;
}

// Reads and clears the device status word (caller has synchronised).
int check_status(ghost_ctx *c) {
  if (!c->status) return GHOST_OK;
  int st = 0;
  GB_CUDA(cudaMemcpy(&st, c->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != 0) {
    GB_CUDA(cudaMemset(c->status, 0, sizeof(int)));
    return fail(GHOST_ERR_TIMEOUT, "a device-side wait gave up (status %d); results of the affected calls are invalid",
                st);
  }
  return GHOST_OK;
}

// ---------------------------------------------------------------------
// per-kernel timers
static cudaEvent_t take_event(ghost_ctx *c) {
  if (!c->ev_free.empty()) {
    cudaEvent_t e = c->ev_free.back();
    c->ev_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records the start event of a launch; returns the pending slot or -1.
static int timer_begin(ghost_ctx *c, int kind) {
  if (!c->timers_on) return -1;
  ghost_ctx::Pending p{kind, take_event(c), take_event(c)};
  cudaEventRecord(p.a, c->stream);
  c->ev_pending.push_back(p);
  return (int)c->ev_pending.size() - 1;
}
static void timer_end(ghost_ctx *c, int slot) {
  if (slot >= 0) cudaEventRecord(c->ev_pending[slot].b, c->stream);
}
static int timers_collect(ghost_ctx *c) {
  if (c->ev_pending.empty()) return GHOST_OK;
  GB_CUDA(cudaStreamSynchronize(c->stream));
  for (auto &p : c->ev_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      c->t_ms[p.kind] += ms;
      c->t_n[p.kind] += 1;
    } else {
      cudaGetLastError();
    }
    c->ev_free.push_back(p.a);
    c->ev_free.push_back(p.b);
  }
  c->ev_pending.clear();
  return GHOST_OK;
}

template <class Op> struct ZKind;
template <typename R, int S, int NF> struct ZKind<ZC2C<R, S, NF>> { static constexpr int value = GHOST_TIMER_Z_C2C; };
template <typename R, int P> struct ZKind<ZInv<R, P>> { static constexpr int value = GHOST_TIMER_Z_INV; };
template <typename R> struct ZKind<ZGrad<R>> { static constexpr int value = GHOST_TIMER_Z_INV; };
template <typename R> struct ZKind<ZFwdHD<R>> { static constexpr int value = GHOST_TIMER_Z_FWD; };
template <typename R> struct ZKind<ZFwdBouss<R>> { static constexpr int value = GHOST_TIMER_Z_FWD; };

int grid1d(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)std::min<size_t>(b, 148 * 16);
}

// ---------------------------------------------------------------------
// pass launchers
template <typename R> constexpr int xE() { return sizeof(R) == 4 ? 8 : 4; }
template <typename R> constexpr int xBZ() { return sizeof(R) == 4 ? 8 : 4; }

// Pruning state for one substep: null tables = every line.
struct Prune {
  const int *lines = nullptr;
  int nlines = 0;
  const int *jpos = nullptr, *jneg = nullptr;
  int ni = 0;    // kx indices processed by the y passes
  int rows = 0;  // kx rows present in / written by the x pass
};

template <typename R> constexpr int zE() { return sizeof(R) == 4 ? 8 : 4; }

static int sm_count(ghost_ctx *c) {
  if (c->num_sms <= 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, c->device);
    c->num_sms = n > 0 ? n : 148;
  }
  return c->num_sms;
}

// Persistent grid: as many CTAs as fit on the device at once, or fewer
// when there are fewer tiles.
template <class K> static int persistent_grid(ghost_ctx *c, K kern, int threads, size_t smem, long ntiles) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (per_sm < 1) per_sm = 1;
  const long g = (long)per_sm * sm_count(c);
  return (int)std::max<long>(1, std::min<long>(g, ntiles));
}

// ---------------------------------------------------------------------
// TMA tensor maps of spectral fields: a 3D tensor (z in 8-byte units, y,
// kx) over one field, with the box the pass loads.
static PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;
static std::mutex g_encode_mu;

static int encode_fn(PFN_cuTensorMapEncodeTiled_v12000 *fn) {
  std::lock_guard<std::mutex> lock(g_encode_mu);
  if (!g_encode_tiled) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || p == nullptr || q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return fail(GHOST_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    }
    g_encode_tiled = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  *fn = g_encode_tiled;
  return GHOST_OK;
}

static int field_map(ghost_ctx *c, const void *base, unsigned box0, unsigned box1, unsigned box2, CUtensorMap *out,
                     CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_NONE) {
  PFN_cuTensorMapEncodeTiled_v12000 enc;
  GB_CHECK(encode_fn(&enc));
  const cuuint64_t U = c->precision == GHOST_SINGLE ? 1 : 2;
  const cuuint64_t dims[3] = {(cuuint64_t)c->nz * U, (cuuint64_t)c->ny, (cuuint64_t)c->nxh * c->nruns};
  const cuuint64_t strides[2] = {(cuuint64_t)c->nz * U * 8, (cuuint64_t)c->nz * c->ny * U * 8};
  const cuuint32_t box[3] = {box0, box1, box2};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<void *>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(GHOST_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return GHOST_OK;
}

static PipeCtl pipe_ctl(ghost_ctx *c) { return PipeCtl{c->status, c->wait_cap, c->inject_stall}; }

template <typename R, int N, int LPB, int STAGES0, int MINB, class Op>
int launch_z_cfg(ghost_ctx *c, const Op &op, const Prune &pr) {
  constexpr int E = zE<R>() < N ? zE<R>() : N, T = N / E;
  using G = ZGeom<R, N, E, LPB, Op::NLOAD>;
  constexpr int STAGES = G::smem_bytes(STAGES0) <= 200 * 1024 ? STAGES0 : 2;
  const size_t smem = G::smem_bytes(STAGES);
  const int nlines = pr.lines ? pr.nlines : c->ny * c->nxh * c->nruns;
  auto kern = zpipe_kernel<R, N, E, LPB, STAGES, MINB, Op>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = persistent_grid(c, kern, LPB * T, smem, (nlines + LPB - 1) / LPB);
  const int ts = timer_begin(c, ZKind<Op>::value);
  kern<<<grid, LPB * T, smem, c->stream>>>(op, (const cx<R> *)c->tw_z, pr.lines, nlines, pipe_ctl(c));
  timer_end(c, ts);
  return post_launch(c);
}

// CTAs of 256 threads; with tile variant bit 1 of 128 threads; with bits 1
// and 2 of 128 threads with a two-stage ring and at most 170 registers, so
// that three CTAs share an SM (lines of 256 points or more)
// lines per CTA, halved from want until a two-stage ring of NL fields fits
template <typename R, int N, int NL> constexpr int fit_lines(int want) {
  int lpb = want;
  while (lpb > 1 && ((size_t)2 * NL * lpb * N + N + (size_t)2 * lpb * (N + N / 8)) * sizeof(cx<R>) + 24 > 220 * 1024)
    lpb /= 2;
  return lpb;
}

template <typename R, int N, class Op> int launch_z_n(ghost_ctx *c, const Op &op, const Prune &pr) {
  constexpr int E = zE<R>() < N ? zE<R>() : N, T = N / E;
  constexpr int L256 = fit_lines<R, N, Op::NLOAD>(256 / T > 0 ? 256 / T : 1);
  constexpr int L128 = fit_lines<R, N, Op::NLOAD>(128 / T > 0 ? 128 / T : 1);
  if constexpr (N >= 256 && L128 != L256) {
    if ((c->tile_cfg & 38) == 38) return launch_z_cfg<R, N, L128, 1, 4>(c, op, pr);
    if ((c->tile_cfg & 6) == 6) return launch_z_cfg<R, N, L128, 2, 3>(c, op, pr);
  }
  if ((c->tile_cfg & 2) && L128 != L256) return launch_z_cfg<R, N, L128, 3, 1>(c, op, pr);
  return launch_z_cfg<R, N, L256, 3, 1>(c, op, pr);
}

template <typename R, class Op> int launch_z(ghost_ctx *c, const Op &op, const Prune &pr = Prune()) {
  switch (c->nz) {
    case 16: return launch_z_n<R, 16>(c, op, pr);
    case 32: return launch_z_n<R, 32>(c, op, pr);
    case 64: return launch_z_n<R, 64>(c, op, pr);
    case 128: return launch_z_n<R, 128>(c, op, pr);
    case 256: return launch_z_n<R, 256>(c, op, pr);
    case 512: return launch_z_n<R, 512>(c, op, pr);
    case 1024: return launch_z_n<R, 1024>(c, op, pr);
  }
  return fail(GHOST_ERR_SIZE, "nz=%d unsupported", c->nz);
}

// y tile width: BZ0 z-lines, at most 1024 threads, narrowed until a
// two-stage ring fits in shared memory (FP64 with 1024-point lines)
template <typename R, int N, int BZ0> constexpr int y_tile_width() {
  constexpr int E = N < 8 ? N : 8, T = N / E;
  int bz = BZ0 * T <= 1024 ? BZ0 : 1024 / T;
  while (bz > 1 && ((size_t)3 * bz * N + N) * sizeof(cx<R>) + 24 > 220 * 1024) bz /= 2;
  return bz;
}

// kx indices per y tile: short lines put several kx in one tile so that a
// CTA has at least 128 threads (not with the second exchange buffer)
template <int N, int E, int BZ, bool DUAL> constexpr int y_kb() {
  return (DUAL || BZ * (N / E) >= 128) ? 1 : 128 / (BZ * (N / E));
}

template <typename R, int N, int S, int BZ0, bool DUAL = false, int E0 = 8>
int launch_y_cfg(ghost_ctx *c, const Fields<R> &f, int nf, const Prune &pr) {
  constexpr int E = N < E0 ? N : E0, T = N / E;
  constexpr int BZ = y_tile_width<R, N, BZ0>();
  constexpr int KB = y_kb<N, E, BZ, DUAL>();
  using G = YGeom<R, N, E, BZ, DUAL, KB>;
  constexpr int STAGES = DUAL ? 2 : (G::smem_bytes(3) <= 200 * 1024 ? 3 : 2);
  if (c->nz < BZ) return fail(GHOST_ERR_SIZE, "nz=%d below the y-pass tile width %d", c->nz, BZ);
  const size_t smem = G::smem_bytes(STAGES);
  auto kern = ypipe_kernel<R, N, E, BZ, STAGES, S, DUAL, KB>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int ni = pr.jpos ? pr.ni : c->nxh;
  const long ntiles = (long)(c->nz / BZ) * ((ni + KB - 1) / KB) * c->nruns * nf;
  const int grid = persistent_grid(c, kern, KB * BZ * T, smem, ntiles);
  // box rows: 32 (or N/2) for the pruned inverse, whole halves otherwise
  const int rb = (pr.jpos && S > 0) ? std::min(32, N / 2) : std::min(N, 256);
  // store boxes of the dual-buffer variant (TMA stores): whole halves for the
  // inverse, 32 rows for the forward pass, whose pruned tiles store the live
  // rows only; both divide N
  const int rbo = S > 0 ? std::min(N, 256) : std::min(N, 32);
  const unsigned U = sizeof(R) == 4 ? 1 : 2;
  FieldMaps maps, omaps;
  for (int q = 0; q < nf; ++q) GB_CHECK(field_map(c, f.p[q], BZ * U, rb, 1, &maps.m[q]));
  if (DUAL)
    for (int q = 0; q < nf; ++q) GB_CHECK(field_map(c, f.p[q], BZ * U, rbo, 1, &omaps.m[q]));
  const int ts = timer_begin(c, S > 0 ? GHOST_TIMER_Y_INV : GHOST_TIMER_Y_FWD);
  kern<<<grid, KB * BZ * T, smem, c->stream>>>(maps, DUAL ? omaps : maps, f, (const cx<R> *)c->tw_y, c->nz, ni, nf,
                                          c->nruns, c->nxh, pr.jpos, pr.jneg, rb, rbo, pipe_ctl(c));
  timer_end(c, ts);
  return post_launch(c);
}

// tiles 8 z-lines wide, or 16 with tile variant bit 0
template <typename R, int N, int S> int launch_y_n(ghost_ctx *c, const Fields<R> &f, int nf, const Prune &pr) {
  // the 16-wide tile needs two stages of 16 lines in shared memory; where
  // that does not fit (FP64, long lines) the variant falls back to 8
  constexpr int E = N < 8 ? N : 8, T = N / E;
  constexpr int BZ16 = 16 * T <= 1024 ? 16 : 1024 / T;
  constexpr bool fits16 = YGeom<R, N, E, BZ16>::smem_bytes(2) <= 227 * 1024;
  if constexpr (fits16) {
    if ((c->tile_cfg & 1) && c->nz >= 16) return launch_y_cfg<R, N, S, 16>(c, f, nf, pr);
  }
  // bit 4 (FP32, lines of 256 points or more): 16 values per thread, two
  // radix-8 butterflies per stage, half the threads per line
  if constexpr (sizeof(R) == 4 && N >= 256) {
    if (c->tile_cfg & 16) {
      // bit 6 with bit 3: the inverse pass in tiles of 4 z-lines, four CTAs per SM
      if constexpr (S > 0)
        if ((c->tile_cfg & 72) == 72) return launch_y_cfg<R, N, S, 4, true, 16>(c, f, nf, pr);
      if (c->tile_cfg & 8) return launch_y_cfg<R, N, S, 8, true, 16>(c, f, nf, pr);
      return launch_y_cfg<R, N, S, 8, false, 16>(c, f, nf, pr);
    }
  }
  // bit 3: two stages and a second exchange buffer (one barrier per exchange)
  constexpr bool fits_dual = YGeom<R, N, E, 8, true>::smem_bytes(2) <= 113 * 1024;
  if constexpr (N >= 256 && fits_dual) {
    if (c->tile_cfg & 8) return launch_y_cfg<R, N, S, 8, true>(c, f, nf, pr);
  }
  return launch_y_cfg<R, N, S, 8>(c, f, nf, pr);
}

template <typename R, int S> int launch_y(ghost_ctx *c, const Fields<R> &f, int nf, const Prune &pr = Prune()) {
  switch (c->ny) {
    case 16: return launch_y_n<R, 16, S>(c, f, nf, pr);
    case 32: return launch_y_n<R, 32, S>(c, f, nf, pr);
    case 64: return launch_y_n<R, 64, S>(c, f, nf, pr);
    case 128: return launch_y_n<R, 128, S>(c, f, nf, pr);
    case 256: return launch_y_n<R, 256, S>(c, f, nf, pr);
    case 512: return launch_y_n<R, 512, S>(c, f, nf, pr);
    case 1024: return launch_y_n<R, 1024, S>(c, f, nf, pr);
  }
  return fail(GHOST_ERR_SIZE, "ny=%d unsupported", c->ny);
}

// X pass kinds
enum XKind { X_HD = 0, X_C2R = 1, X_R2C = 2, X_BOUSS = 3 };

// y rows per x tile: short lines put several y rows in one tile so that a
// CTA has at least 128 threads
template <typename R, int NX, int BZ> constexpr int x_yb() {
  constexpr int E = xE<R>() < NX / 2 ? xE<R>() : NX / 2;
  return BZ * (NX / 2 / E) >= 128 ? 1 : 128 / (BZ * (NX / 2 / E));
}

// The fused X pass with tiles of BZ z-values (MINB CTAs per SM).
template <typename R, int NX, int KIND, int BZ, int MINB>
int launch_x_fused(ghost_ctx *c, const void *const *ins, void *const *outs, int rows) {
  constexpr int E = xE<R>() < NX / 2 ? xE<R>() : NX / 2;
  constexpr int YB = x_yb<R, NX, BZ>();
  if (c->ny % YB != 0) return fail(GHOST_ERR_SIZE, "ny=%d not a multiple of the x tile's %d rows", c->ny, YB);
  constexpr int M = NX / 2, T = M / E, NT = YB * BZ * T;
  typedef cx<R> C;
  constexpr int PHYS = KIND == X_HD ? 0 : 1;
  constexpr int NIN = PHYS == 0 ? 6 : 9, NOUT = PHYS == 0 ? 3 : 4;
  using G = XGeom<R, NX, BZ, YB>;
  constexpr size_t cap = 220 * 1024 / MINB;  // four stages while MINB CTAs fit an SM
  constexpr int STAGES = G::smem_bytes(4) <= cap ? 4 : (G::smem_bytes(3) <= 200 * 1024 ? 3 : 2);
  const size_t smem = G::smem_bytes(STAGES);
  auto kern = xpipe_nl_kernel<R, NX, E, BZ, PHYS, STAGES, MINB, YB>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  Fields<R> fo{};
  for (int q = 0; q < NOUT; ++q) fo.p[q] = (C *)outs[q];
  const R nn = (R)c->nx * (R)c->ny * (R)c->nz_glob;
  const int nrows = rows > 0 ? rows : M + 1;
  // tensor boxes: nbox boxes of rb kx-rows; rb keeps every box 128-byte aligned in shared memory
  const int nbox = (nrows + 255) / 256;
  const int align = std::max(1, 128 / (YB * BZ * (int)sizeof(C)));
  const int rb = ((nrows + nbox - 1) / nbox + align - 1) / align * align;
  if (nbox * rb > M + 8 || rb > 256) return fail(GHOST_ERR_STATE, "x-pass box plan %d x %d exceeds the tile", nbox, rb);
  const unsigned U = sizeof(R) == 4 ? 1 : 2;
  FieldMaps maps;
  for (int q = 0; q < NIN; ++q) GB_CHECK(field_map(c, ins[q], BZ * U, YB, rb, &maps.m[q]));
  const int pgrid = persistent_grid(c, kern, NT, smem, (long)(c->nz / BZ) * (c->ny / YB) * c->nruns);
  kern<<<pgrid, NT, smem, c->stream>>>(maps, fo, (const C *)c->tw_x, c->ny, c->nz, (R)1 / (nn * nn), nrows, nbox, rb,
                                       c->nruns, c->nxh, pipe_ctl(c));
  return GHOST_OK;
}

// TMA map of a real FP32 field (x fastest) as 8-byte pairs: a box of
// nx/2 pairs x 1 y-row x 8 z-values, the tiles of the plain x transforms.
static int real_map(ghost_ctx *c, const void *base, CUtensorMap *out) {
  PFN_cuTensorMapEncodeTiled_v12000 enc;
  GB_CHECK(encode_fn(&enc));
  const cuuint64_t dims[3] = {(cuuint64_t)c->nx / 2, (cuuint64_t)c->ny, (cuuint64_t)c->nz};
  const cuuint64_t strides[2] = {(cuuint64_t)c->nx * 4, (cuuint64_t)c->nx * c->ny * 4};
  const cuuint32_t box[3] = {(cuuint32_t)c->nx / 2, 1, 8};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<void *>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(GHOST_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return GHOST_OK;
}

// The plain x transforms with one warp per line (FP32, nx = 512, one run).
static bool xw_plain_ok(const ghost_ctx *c) {
  return c->precision == GHOST_SINGLE && c->nx == 512 && c->nruns == 1 && c->nz % 8 == 0;
}
static int launch_xw_r2c(ghost_ctx *c, const void *in, void *out) {
  constexpr int NX = 512, M = NX / 2, STAGES = 3;
  using G = XWPlainGeom<NX, STAGES>;
  auto kern = xwarp_r2c_kernel<NX, STAGES>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::r2c_bytes));
  const int rb = ((M + 1 + 1) / 2 + 15) / 16 * 16;  // 2 x 144 rows cover the M+1 kx rows
  static_assert(2 * (((M + 2) / 2 + 15) / 16 * 16) <= G::OROWS, "r2c store boxes exceed the output tile");
  CUtensorMap rm, cm;
  GB_CHECK(real_map(c, in, &rm));
  GB_CHECK(field_map(c, out, 8, 1, rb, &cm, CU_TENSOR_MAP_SWIZZLE_64B));
  const int grid = persistent_grid(c, kern, 256, G::r2c_bytes, (long)(c->nz / 8) * c->ny);
  kern<<<grid, 256, G::r2c_bytes, c->stream>>>(rm, cm, (const float2 *)c->tw_x, c->ny, c->nz, rb, pipe_ctl(c));
  return GHOST_OK;
}
static int launch_xw_c2r(ghost_ctx *c, const void *in, void *out) {
  constexpr int NX = 512, M = NX / 2, STAGES = 4;
  using G = XWPlainGeom<NX, STAGES>;
  auto kern = xwarp_c2r_kernel<NX, STAGES>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::c2r_bytes));
  const int nbox = 2, rb = ((M + 1 + 1) / 2 + 15) / 16 * 16;  // 2 x 144 rows cover the M+1 kx rows
  static_assert(2 * (((M + 2) / 2 + 15) / 16 * 16) <= G::SROWS, "c2r box plan exceeds the slot");
  CUtensorMap m;
  GB_CHECK(field_map(c, in, 8, 1, rb, &m, CU_TENSOR_MAP_SWIZZLE_64B));
  const int grid = persistent_grid(c, kern, 256, G::c2r_bytes, (long)(c->nz / 8) * c->ny);
  kern<<<grid, 256, G::c2r_bytes, c->stream>>>(m, (float *)out, (const float2 *)c->tw_x, c->ny, c->nz, nbox, rb,
                                               pipe_ctl(c));
  return GHOST_OK;
}

template <typename R, int NX, int KIND> int launch_x_n(ghost_ctx *c, const void *in, void *out, const void *const *ins,
                                                       void *const *outs, int rows) {
  constexpr int E = xE<R>() < NX / 2 ? xE<R>() : NX / 2;
  constexpr int M = NX / 2, T = M / E;
  // rows of BZ z values; at most 256 threads so the register-resident
  // real fields of the fused pass fit the register file
  constexpr int BZ = xBZ<R>() * T <= 256 ? xBZ<R>() : (256 / T > 0 ? 256 / T : 1);
  constexpr int NT = BZ * T;
  typedef cx<R> C;
  dim3 grid(c->nz / BZ, c->ny);
  const C *tw = (const C *)c->tw_x;
  const int ts = timer_begin(c, KIND == X_C2R ? GHOST_TIMER_X_C2R : (KIND == X_R2C ? GHOST_TIMER_X_R2C : GHOST_TIMER_X_NL));
  if (KIND == X_HD || KIND == X_BOUSS) {
    // FP32 512-point lines: tiles of 16 z-values (128-byte rows, one CTA of
    // 512 threads per SM) where nz allows, else BZ
    if constexpr (sizeof(R) == 4 && NX == 512 && BZ == 8) {
      if (c->nz % 16 == 0) {
        GB_CHECK((launch_x_fused<R, NX, KIND, 16, 1>(c, ins, outs, rows)));
        timer_end(c, ts);
        return post_launch(c);
      }
    }
    // FP32 1024-point lines: tiles of 8 z-values (64-byte rows instead of
    // 32, one CTA of 512 threads per SM) where nz allows (bit 8 of the tile
    // variant asks for the 4-value tiles)
    if constexpr (sizeof(R) == 4 && NX == 1024 && BZ == 4) {
      if (c->nz % 8 == 0 && !(c->tile_cfg & 256)) {
        GB_CHECK((launch_x_fused<R, NX, KIND, 8, 1>(c, ins, outs, rows)));
        timer_end(c, ts);
        return post_launch(c);
      }
    }
    GB_CHECK((launch_x_fused<R, NX, KIND, BZ, 2>(c, ins, outs, rows)));
  } else if (KIND == X_C2R && xw_plain_ok(c)) {
    GB_CHECK(launch_xw_c2r(c, in, out));
  } else if (KIND == X_R2C && xw_plain_ok(c)) {
    GB_CHECK(launch_xw_r2c(c, in, out));
  } else if (KIND == X_C2R) {
    const size_t smem = (size_t)(NX + (M + 1) * BZ + M * BZ) * sizeof(C);
    auto kern = xpass_c2r_kernel<R, NX, E, BZ>;
    GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, NT, smem, c->stream>>>((const C *)in, (R *)out, tw, c->ny, c->nz);
  } else {
    const size_t smem = (size_t)(NX + M * BZ) * sizeof(C);
    auto kern = xpass_r2c_kernel<R, NX, E, BZ>;
    GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, NT, smem, c->stream>>>((const R *)in, (C *)out, tw, c->ny, c->nz);
  }
  timer_end(c, ts);
  return post_launch(c);
}

template <typename R, int KIND>
int launch_x(ghost_ctx *c, const void *in, void *out, const void *const *ins = nullptr, void *const *outs = nullptr,
             int rows = 0) {
  switch (c->nx) {
    case 16: return launch_x_n<R, 16, KIND>(c, in, out, ins, outs, rows);
    case 32: return launch_x_n<R, 32, KIND>(c, in, out, ins, outs, rows);
    case 64: return launch_x_n<R, 64, KIND>(c, in, out, ins, outs, rows);
    case 128: return launch_x_n<R, 128, KIND>(c, in, out, ins, outs, rows);
    case 256: return launch_x_n<R, 256, KIND>(c, in, out, ins, outs, rows);
    case 512: return launch_x_n<R, 512, KIND>(c, in, out, ins, outs, rows);
    case 1024: return launch_x_n<R, 1024, KIND>(c, in, out, ins, outs, rows);
  }
  return fail(GHOST_ERR_SIZE, "nx=%d unsupported", c->nx);
}

// ---------------------------------------------------------------------
// zero-pruning tables.  After a substep, v is exactly zero outside
// tiny <= kn2 <= kmax.  kn2 grows with |kz|, so a z-line (j,i) holds live
// modes iff its kz = 0 entry has kn2 <= kmax; at fixed kx the live ky form
// a run from j = 0 up and a run from j = ny-1 down.  The tables are built
// with kn2 evaluated exactly as the kernels evaluate it; if the live set
// does not have that shape (an unusual kmax), pruning is disabled.
template <typename R> int build_prune(ghost_ctx *c) {
  const KParams<R> &kp = kparams<R>(c);
  // local kx row i is global row i + i0 (a kx-slab; 0 otherwise)
  auto kn2h = [&](int il, int j) -> R {
    const int i = il + kp.i0;
    const R a = (R)(i < kp.nx / 2 ? i : i - kp.nx), b = (R)(j < kp.ny / 2 ? j : j - kp.ny);
    volatile R aa = a * a, bb = b * b;  // no contraction: same rounding as the kernels
    if (kp.anis) {
      volatile R x = kp.rmp * aa, y = kp.rmq * bb;
      volatile R s = x + y;
      return s + (R)0;
    }
    volatile R s = aa + bb;
    return s + (R)0;
  };
  const int nxh = c->nxh, ny = c->ny;
  std::vector<int> jpos(nxh, 0), jneg(nxh, 0), lines;
  bool ok = true;
  int imax = -1;
  for (int i = 0; i < nxh; ++i) {
    int p = 0;
    while (p < ny / 2 && kn2h(i, p) <= kp.kmax) ++p;
    int q = 0;
    while (q < ny - ny / 2 && kn2h(i, ny - 1 - q) <= kp.kmax) ++q;
    jpos[i] = p;
    jneg[i] = q;
    for (int j = 0; j < ny; ++j) {
      const bool live = kn2h(i, j) <= kp.kmax;
      const bool said = j < p || j >= ny - q;
      if (live != said) ok = false;
      if (live) lines.push_back(j + ny * i);
    }
    if (p + q > 0) {
      if (imax != i - 1) ok = false;  // live kx indices must be 0..imax
      imax = i;
    }
  }
  c->prune_ok = ok && imax >= 0;
  c->prune_valid = true;
  if (!c->prune_ok) return GHOST_OK;
  const int nrun = (int)lines.size();
  for (int r = 1; r < c->nruns; ++r)
    for (int q = 0; q < nrun; ++q) lines.push_back(lines[q] + r * ny * nxh);
  const int n = (int)lines.size();
  const int padded = (n + 255) / 256 * 256;
  lines.resize(padded, -1);
  if (c->prune_lines) cudaFree(c->prune_lines);
  if (c->prune_jpos) cudaFree(c->prune_jpos);
  if (c->prune_jneg) cudaFree(c->prune_jneg);
  c->prune_lines = c->prune_jpos = c->prune_jneg = nullptr;
  GB_CHECK(dalloc((void **)&c->prune_lines, sizeof(int) * padded));
  GB_CHECK(dalloc((void **)&c->prune_jpos, sizeof(int) * nxh));
  GB_CHECK(dalloc((void **)&c->prune_jneg, sizeof(int) * nxh));
  GB_CUDA(cudaMemcpy(c->prune_lines, lines.data(), sizeof(int) * padded, cudaMemcpyHostToDevice));
  GB_CUDA(cudaMemcpy(c->prune_jpos, jpos.data(), sizeof(int) * nxh, cudaMemcpyHostToDevice));
  GB_CUDA(cudaMemcpy(c->prune_jneg, jneg.data(), sizeof(int) * nxh, cudaMemcpyHostToDevice));
  c->prune_nlines = n;
  c->prune_imax = imax;
  c->prune_jtop = *std::max_element(jpos.begin(), jpos.end());
  c->prune_jbot = *std::max_element(jneg.begin(), jneg.end());
  // kz values that can be kept: kn2 >= its kz term (every term is >= 0 and
  // the sums round monotonically), so |kz| beyond those is never kept
  auto kz_term = [&](int k) -> R {
    const R cz = (R)(k < kp.nz / 2 ? k : k - kp.nz);
    volatile R cc = cz * cz;
    if (kp.anis) {
      volatile R z = kp.rms * cc;
      return z + (R)0;
    }
    return cc + (R)0;
  };
  int kt = 0, kb = 0;
  while (kt < kp.nz / 2 && kz_term(kt) <= kp.kmax) ++kt;
  while (kb < kp.nz - kp.nz / 2 && kz_term(kp.nz - 1 - kb) <= kp.kmax) ++kb;
  c->prune_ktop = kt;
  c->prune_kbot = kb;
  return GHOST_OK;
}

// Pruning plan for a substep whose input fields are zero outside the
// truncation; an empty plan (full passes) when want == false.
template <typename R> int prune_plan(ghost_ctx *c, bool want, Prune *pr) {
  *pr = Prune();
  if (!want) return GHOST_OK;
  if (!c->prune_valid) GB_CHECK(build_prune<R>(c));
  if (!c->prune_ok) return GHOST_OK;
  pr->lines = c->prune_lines;
  pr->nlines = c->prune_nlines;
  pr->jpos = c->prune_jpos;
  pr->jneg = c->prune_jneg;
  pr->ni = c->prune_imax + 1;
  pr->rows = c->prune_imax + 1;
  return GHOST_OK;
}

// ---------------------------------------------------------------------
// 3D transforms on device pointers
template <typename R> int r2c_dev(ghost_ctx *c, const void *in, void *out) {
  GB_CHECK((launch_x<R, X_R2C>(c, in, out)));
  Fields<R> f{};
  f.p[0] = (cx<R> *)out;
  GB_CHECK((launch_y<R, -1>(c, f, 1)));
  ZC2C<R, -1, 1> op{};
  op.in.p[0] = (const cx<R> *)out;
  op.out.p[0] = (cx<R> *)out;
  return launch_z<R>(c, op);
}

template <typename R> int c2r_dev(ghost_ctx *c, const void *in, void *out) {
  void *w[1];
  GB_CHECK(scratch(c, 1, w));
  ZC2C<R, +1, 1> op{};
  op.in.p[0] = (const cx<R> *)in;
  op.out.p[0] = (cx<R> *)w[0];
  GB_CHECK(launch_z<R>(c, op));
  Fields<R> f{};
  f.p[0] = (cx<R> *)w[0];
  GB_CHECK((launch_y<R, +1>(c, f, 1)));
  return launch_x<R, X_C2R>(c, w[0], out);
}

// The LES closure's input rows from a spectral velocity: the nine gradients
// through z and y passes over all nine, then one x pass that writes
// x[q][3a+b] = (d v_a / d x_b) * gs and x[q][9] = delta directly.
template <typename R, int NX>
int grad9_features_n(ghost_ctx *c, void *const spec[9], float *x, float gs, float delta) {
  constexpr int E = xE<R>() < NX / 2 ? xE<R>() : NX / 2;
  constexpr int M = NX / 2, T = M / E;
  constexpr int BZ = xBZ<R>() * T <= 256 ? xBZ<R>() : (256 / T > 0 ? 256 / T : 1);
  typedef cx<R> C;
  const size_t smem = (size_t)(NX + (M + 1) * BZ + M * BZ) * sizeof(C);
  auto kern = xpass_c2r_features_kernel<R, NX, E, BZ>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  Fields<R> in{};
  for (int q = 0; q < 9; ++q) in.p[q] = (C *)spec[q];
  const int ts = timer_begin(c, GHOST_TIMER_X_C2R);
  kern<<<dim3(c->nz / BZ, c->ny), BZ * T, smem, c->stream>>>(in, x, (const C *)c->tw_x, c->ny, c->nz,
                                                              (R)(1.0 / (double)c->nreal), gs, delta);
  timer_end(c, ts);
  return post_launch(c);
}

template <typename R>
int grad9_features_dev(ghost_ctx *c, const void *const v[3], void *const spec[9], float *x, float gs, float delta) {
  ZGrad<R> zg{};
  for (int a = 0; a < 3; ++a) zg.v.p[a] = (const cx<R> *)v[a];
  for (int q = 0; q < 9; ++q) zg.w.p[q] = (cx<R> *)spec[q];
  zg.kp = kparams<R>(c);
  GB_CHECK(launch_z<R>(c, zg));
  Fields<R> fy{};
  for (int q = 0; q < 9; ++q) fy.p[q] = (cx<R> *)spec[q];
  GB_CHECK((launch_y<R, +1>(c, fy, 9)));
  switch (c->nx) {
    case 16: return grad9_features_n<R, 16>(c, spec, x, gs, delta);
    case 32: return grad9_features_n<R, 32>(c, spec, x, gs, delta);
    case 64: return grad9_features_n<R, 64>(c, spec, x, gs, delta);
    case 128: return grad9_features_n<R, 128>(c, spec, x, gs, delta);
    case 256: return grad9_features_n<R, 256>(c, spec, x, gs, delta);
    case 512: return grad9_features_n<R, 512>(c, spec, x, gs, delta);
    case 1024: return grad9_features_n<R, 1024>(c, spec, x, gs, delta);
  }
  return fail(GHOST_ERR_SIZE, "nx=%d unsupported", c->nx);
}

// Six real fields to spectra at once (the stresses of the LES closure):
// x r2c per field, then one y and one z pass over all six.
template <typename R> int r2c6_dev(ghost_ctx *c, const void *const in[6], void *const out[6]) {
  for (int q = 0; q < 6; ++q) GB_CHECK((launch_x<R, X_R2C>(c, in[q], out[q])));
  Fields<R> f{};
  for (int q = 0; q < 6; ++q) f.p[q] = (cx<R> *)out[q];
  GB_CHECK((launch_y<R, -1>(c, f, 6)));
  ZC2C<R, -1, 6> op{};
  for (int q = 0; q < 6; ++q) {
    op.in.p[q] = (const cx<R> *)out[q];
    op.out.p[q] = (cx<R> *)out[q];
  }
  return launch_z<R>(c, op);
}

// prodre3 on device pointers (outputs may alias inputs)
template <typename R> int prodre3_dev(ghost_ctx *c, const void *a, const void *b, const void *cc, void *d, void *e, void *f) {
  void *w[6];
  GB_CHECK(scratch(c, 6, w));
  ZInv<R, 0> zi{};
  zi.v.p[0] = (const cx<R> *)a;
  zi.v.p[1] = (const cx<R> *)b;
  zi.v.p[2] = (const cx<R> *)cc;
  for (int q = 0; q < 6; ++q) zi.w.p[q] = (cx<R> *)w[q];
  zi.kp = kparams<R>(c);
  zi.copy = 0;
  GB_CHECK(launch_z<R>(c, zi));
  Fields<R> fy{};
  for (int q = 0; q < 6; ++q) fy.p[q] = (cx<R> *)w[q];
  GB_CHECK((launch_y<R, +1>(c, fy, 6)));
  GB_CHECK((launch_x<R, X_HD>(c, nullptr, nullptr, (const void *const *)w, (void *const *)w)));
  GB_CHECK((launch_y<R, -1>(c, fy, 3)));
  ZC2C<R, -1, 3> zf{};
  void *outs[3] = {d, e, f};
  for (int q = 0; q < 3; ++q) {
    zf.in.p[q] = (const cx<R> *)w[q];
    zf.out.p[q] = (cx<R> *)outs[q];
  }
  return launch_z<R>(c, zf);
}

// One HD substep on device pointers: include/hd_rkstep2.f90 with
// hd_rkstep1 folded in when copy != 0.
template <typename R>
int hd_substep_dev(ghost_ctx *c, int o, double dt, double nu, void *const v[3], void *const C[3], const void *const f[3],
                   int copy, bool prune) {
  void *w[6];
  GB_CHECK(scratch(c, 6, w));
  Prune pr;
  GB_CHECK(prune_plan<R>(c, prune, &pr));
  ZInv<R, 0> zi{};
  for (int q = 0; q < 3; ++q) {
    zi.v.p[q] = (const cx<R> *)v[q];
    zi.cpy.p[q] = (cx<R> *)C[q];
  }
  for (int q = 0; q < 6; ++q) zi.w.p[q] = (cx<R> *)w[q];
  zi.kp = kparams<R>(c);
  zi.copy = copy;
  GB_CHECK(launch_z<R>(c, zi, pr));
  Fields<R> fy{};
  for (int q = 0; q < 6; ++q) fy.p[q] = (cx<R> *)w[q];
  GB_CHECK((launch_y<R, +1>(c, fy, 6, pr)));
  GB_CHECK((launch_x<R, X_HD>(c, nullptr, nullptr, (const void *const *)w, (void *const *)w, pr.rows)));
  GB_CHECK((launch_y<R, -1>(c, fy, 3, pr)));
  GB_CHECK(late_wait(c));  // a staged forcing may still be on its way
  ZFwdHD<R> zf{};
  for (int q = 0; q < 3; ++q) {
    zf.nl.p[q] = (const cx<R> *)w[q];
    zf.v.p[q] = (cx<R> *)v[q];
    zf.c0.p[q] = (const cx<R> *)C[q];
    zf.f.p[q] = f ? (const cx<R> *)f[q] : nullptr;
  }
  zf.kp = kparams<R>(c);
  zf.dt = (R)dt;
  zf.nu = (R)nu;
  zf.rmp = (R)1 / (R)o;
  return launch_z<R>(c, zf, pr);
}

// One Boussinesq substep (include/rotbouss_rkstep2.f90) on device
// pointers: v[0..2] velocity, v[3] theta; C[0..3] the RK1 copies (C20 last).
template <typename R>
int bouss_substep_dev(ghost_ctx *c, int o, double dt, double nu, double kappa, double omegaz, double xmom,
                      double xtemp, void *const v[4], void *const C[4], const void *const f[4], int copy,
                      bool prune = false) {
  void *w[9];
  GB_CHECK(scratch(c, 9, w));
  Prune pr;
  GB_CHECK(prune_plan<R>(c, prune, &pr));
  ZInv<R, 1> zi{};
  for (int q = 0; q < 4; ++q) {
    zi.v.p[q] = (const cx<R> *)v[q];
    zi.cpy.p[q] = (cx<R> *)C[q];
  }
  for (int q = 0; q < 9; ++q) zi.w.p[q] = (cx<R> *)w[q];
  zi.kp = kparams<R>(c);
  zi.copy = copy;
  GB_CHECK(launch_z<R>(c, zi, pr));
  Fields<R> fy{};
  for (int q = 0; q < 9; ++q) fy.p[q] = (cx<R> *)w[q];
  GB_CHECK((launch_y<R, +1>(c, fy, 9, pr)));
  GB_CHECK((launch_x<R, X_BOUSS>(c, nullptr, nullptr, (const void *const *)w, (void *const *)w, pr.rows)));
  GB_CHECK((launch_y<R, -1>(c, fy, 4, pr)));
  ZFwdBouss<R> zf{};
  for (int q = 0; q < 4; ++q) {
    zf.nl.p[q] = (const cx<R> *)w[q];
    zf.v.p[q] = (cx<R> *)v[q];
    zf.c0.p[q] = (const cx<R> *)C[q];
    zf.f.p[q] = f ? (const cx<R> *)f[q] : nullptr;
  }
  zf.kp = kparams<R>(c);
  zf.dt = (R)dt;
  zf.nu = (R)nu;
  zf.kappa = (R)kappa;
  zf.omegaz = (R)omegaz;
  zf.xmom = (R)xmom;
  zf.xtemp = (R)xtemp;
  zf.rmp = (R)1 / (R)o;
  return launch_z<R>(c, zf, pr);
}

// advect3 on device pointers: e = -(A.grad)d via the fused Boussinesq
// passes with zero vorticity work discarded (the three omega x v outputs
// are computed and dropped)
template <typename R>
int advect3_dev(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, void *e) {
  void *w[9];
  GB_CHECK(scratch(c, 9, w));
  ZInv<R, 1> zi{};
  zi.v.p[0] = (const cx<R> *)a;
  zi.v.p[1] = (const cx<R> *)b;
  zi.v.p[2] = (const cx<R> *)cc;
  zi.v.p[3] = (const cx<R> *)d;
  for (int q = 0; q < 9; ++q) zi.w.p[q] = (cx<R> *)w[q];
  zi.kp = kparams<R>(c);
  zi.copy = 0;
  GB_CHECK(launch_z<R>(c, zi));
  Fields<R> fy{};
  for (int q = 0; q < 9; ++q) fy.p[q] = (cx<R> *)w[q];
  GB_CHECK((launch_y<R, +1>(c, fy, 9)));
  GB_CHECK((launch_x<R, X_BOUSS>(c, nullptr, nullptr, (const void *const *)w, (void *const *)w)));
  Fields<R> f1{};
  f1.p[0] = (cx<R> *)w[3];
  GB_CHECK((launch_y<R, -1>(c, f1, 1)));
  ZC2C<R, -1, 1> zf{};
  zf.in.p[0] = (const cx<R> *)w[3];
  zf.out.p[0] = (cx<R> *)e;
  return launch_z<R>(c, zf);
}

// ---------------------------------------------------------------------
// reductions
template <typename R>
int reduce_dev(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, const void *d, const void *e,
               const void *f, double *out_host) {
  const size_t n = c->ntot;
  const int nb = grid1d(n);
  double *part;
  GB_CHECK(partials(c, (size_t)nb + 1, &part));
  RedArgs<R> ra{(const cx<R> *)a, (const cx<R> *)b, (const cx<R> *)cc, (const cx<R> *)d, (const cx<R> *)e,
                (const cx<R> *)f};
  const int ts = timer_begin(c, GHOST_TIMER_REDUCE);
  reduce_kernel<R><<<nb, 256, 0, c->stream>>>(kparams<R>(c), ra, kind, n, part);
  GB_CHECK(post_launch(c));
  finalize_kernel<<<1, 256, 0, c->stream>>>(part, nb, 1, part + nb);
  timer_end(c, ts);
  GB_CHECK(post_launch(c));
  GB_CUDA(cudaMemcpyAsync(out_host, part + nb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

// Shell-binned sums of a reduction term over two field triplets (the
// transfer spectra of entrans / heltrans); spectrum_dev is its one-triplet form.
// rnd is the shell rounding: GHOST's spectra add the default-REAL literal
// .501 (0.501f), spectrscc adds shift + .501 in GP
template <typename R>
int spectrum6_dev(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, const void *d, const void *e,
                  const void *f, double *out_host, R rnd = (R)0.501f) {
  const size_t n = c->ntot;
  const int nbins = c->nmax / 2 + 1;
  const int nblk = std::min(grid1d(n), 148 * 4);
  double *part;
  GB_CHECK(partials(c, (size_t)(nblk + 1) * nbins, &part));
  RedArgs<R> ra{(const cx<R> *)a, (const cx<R> *)b, (const cx<R> *)cc, (const cx<R> *)d, (const cx<R> *)e,
                (const cx<R> *)f};
  const size_t smem = (size_t)(256 / 32) * nbins * sizeof(double);
  GB_CUDA(cudaFuncSetAttribute(spectrum_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int ts = timer_begin(c, GHOST_TIMER_REDUCE);
  spectrum_kernel<R><<<nblk, 256, smem, c->stream>>>(kparams<R>(c), ra, kind, n, nbins, (R)c->Dkk, rnd, part);
  GB_CHECK(post_launch(c));
  double *fin = part + (size_t)nblk * nbins;
  finalize_kernel<<<1, 256, 0, c->stream>>>(part, nblk, nbins, fin);
  timer_end(c, ts);
  GB_CHECK(post_launch(c));
  GB_CUDA(cudaMemcpyAsync(out_host, fin, sizeof(double) * nbins, cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return GHOST_OK;
}

template <typename R>
int spectrum_dev(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, double *out_host) {
  return spectrum6_dev<R>(c, kind, a, b, cc, nullptr, nullptr, nullptr, out_host);
}

// Anisotropic sums (aniso_kernel): out_host[3 nb] = total, horizontal, vertical.
template <typename R>
int aniso_dev(ghost_ctx *c, int kind, int mode, int nb, const void *a, const void *b, const void *cc, const void *d,
              const void *e, const void *f, double *out_host) {
  const size_t n = c->ntot;
  const int nb3 = 3 * nb;
  const int nblk = std::min(grid1d(n), 148 * 2);
  double *part;
  GB_CHECK(partials(c, (size_t)(nblk + 1) * nb3, &part));
  RedArgs<R> ra{(const cx<R> *)a, (const cx<R> *)b, (const cx<R> *)cc, (const cx<R> *)d, (const cx<R> *)e,
                (const cx<R> *)f};
  const size_t smem = (size_t)(256 / 32) * nb3 * sizeof(double);
  if (smem > 227 * 1024) return fail(GHOST_ERR_SIZE, "%d bins exceed the shared-memory histogram", nb);
  GB_CUDA(cudaFuncSetAttribute(aniso_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int ts = timer_begin(c, GHOST_TIMER_REDUCE);
  aniso_kernel<R><<<nblk, 256, smem, c->stream>>>(kparams<R>(c), ra, kind, mode, n, nb, (R)c->Lz, (R)c->Dkk, part);
  GB_CHECK(post_launch(c));
  double *fin = part + (size_t)nblk * nb3;
  finalize_kernel<<<1, 256, 0, c->stream>>>(part, nblk, nb3, fin);
  timer_end(c, ts);
  GB_CHECK(post_launch(c));
  GB_CUDA(cudaMemcpyAsync(out_host, fin, sizeof(double) * nb3, cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

// The same shell spectrum left on the device (out_dev[nmax/2+1]); no
// synchronisation, for closures that consume it in later kernels.
template <typename R>
int spectrum_dev_async(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, double *out_dev) {
  const size_t n = c->ntot;
  const int nbins = c->nmax / 2 + 1;
  const int nblk = std::min(grid1d(n), 148 * 4);
  double *part;
  GB_CHECK(partials(c, (size_t)nblk * nbins, &part));
  RedArgs<R> ra{(const cx<R> *)a, (const cx<R> *)b, (const cx<R> *)cc, nullptr, nullptr, nullptr};
  const size_t smem = (size_t)(256 / 32) * nbins * sizeof(double);
  GB_CUDA(cudaFuncSetAttribute(spectrum_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int ts = timer_begin(c, GHOST_TIMER_REDUCE);
  spectrum_kernel<R><<<nblk, 256, smem, c->stream>>>(kparams<R>(c), ra, kind, n, nbins, (R)c->Dkk, (R)0.501f, part);
  GB_CHECK(post_launch(c));
  finalize_kernel<<<1, 256, 0, c->stream>>>(part, nblk, nbins, out_dev);
  timer_end(c, ts);
  return post_launch(c);
}

// twiddles exp(-2 pi i e/n), e < n, evaluated in extended precision and
// rounded once to the working precision
template <typename R> int make_twiddles(int n, void **out) {
  std::vector<R> h(2 * (size_t)n);
  const long double tau = 6.283185307179586476925286766559005768L;
  for (int e = 0; e < n; ++e) {
    // exact values at multiples of pi/4 (avoid last-bit noise at the axes)
    long double re, im;
    if ((8 * e) % n == 0) {
      const int o = (8 * e) / n;  // multiple of pi/4
      const long double s = 0.707106781186547524400844362104849039L;
      const long double tab_re[8] = {1, s, 0, -s, -1, -s, 0, s};
      const long double tab_im[8] = {0, -s, -1, -s, 0, s, 1, s};
      re = tab_re[o];
      im = tab_im[o];
    } else {
      const long double a = tau * (long double)e / (long double)n;
      re = cosl(a);
      im = -sinl(a);
    }
    h[2 * e] = (R)re;
    h[2 * e + 1] = (R)im;
  }
  GB_CHECK(dalloc(out, sizeof(R) * 2 * n));
  GB_CUDA(cudaMemcpy(*out, h.data(), sizeof(R) * 2 * n, cudaMemcpyHostToDevice));
  return GHOST_OK;
}

template <typename R> void fill_kparams(ghost_ctx *c, KParams<R> &kp) {
  kp.nx = c->nx;
  kp.ny = c->ny;
  kp.nz = c->nz;
  kp.nxh = c->nxh;
  kp.anis = c->anis;
  kp.arbsize = c->arbsize;
  kp.Dkx = (R)c->Dkx;
  kp.Dky = (R)c->Dky;
  kp.Dkz = (R)c->Dkz;
  kp.rmp = kp.rmq = kp.rms = (R)1;
  if (c->anis) {
    kp.rmp = (R)1 / ((R)c->nx * (R)c->nx);
    kp.rmq = (R)1 / ((R)c->ny * (R)c->ny);
    kp.rms = (R)1 / ((R)c->nz * (R)c->nz);
  }
  kp.kmax = (R)c->kmax;
  kp.tiny = (R)c->tiny;
  const R nn = (R)c->nx * (R)c->ny * (R)c->nz;
  kp.tmp = (R)1 / (nn * nn);
  kp.nruns = c->nruns;
  kp.nu_run = (sizeof(R) == (c->precision == GHOST_SINGLE ? 4 : 8)) ? (const R *)c->nu_run : nullptr;
  kp.i0 = c->i0;
}

// kmax, tiny, nmax, Dk of main3D.fpp:881-909,1727-1737 in precision R
template <typename R> void setup_scalars(ghost_ctx *c, double Lx, double Ly, double Lz) {
  R lx = 1, ly = 1, lz = 1, dkx = 1, dky = 1, dkz = 1;
  if (c->arbsize) {
    lx = (R)Lx;
    ly = (R)Ly;
    lz = (R)Lz;
    dkx = (R)1 / lx;
    dky = (R)1 / ly;
    dkz = (R)1 / lz;
  }
  R dkk = std::min(dkx, std::min(dky, dkz));
  R m = std::max((R)c->nx * dkx, std::max((R)c->ny * dky, (R)c->nz * dkz));
  R mp = std::max((R)c->nx * dkx, (R)c->ny * dky);
  c->nmax = (int)(m / dkk);
  c->nmaxperp = (int)(mp / dkk);
  R kmax = (R)1.0 / (R)9.0;
  if (!c->arbsize && c->anis == 0) kmax = kmax * ((R)c->nx * (R)c->nx);
  R t = (R)0.1 / ((R)c->nmax * (R)c->nmax);
  R tiny = (R)1e-5 < t ? (R)1e-5 : t;
  c->Lx = lx;
  c->Ly = ly;
  c->Lz = lz;
  c->Dkx = dkx;
  c->Dky = dky;
  c->Dkz = dkz;
  c->Dkk = dkk;
  c->kmax = kmax;
  c->tiny = tiny;
}

template <typename R> int ctx_init_prec(ghost_ctx *c, double Lx, double Ly, double Lz) {
  setup_scalars<R>(c, Lx, Ly, Lz);
  GB_CHECK(make_twiddles<R>(c->nx, &c->tw_x));
  GB_CHECK(make_twiddles<R>(c->ny, &c->tw_y));
  GB_CHECK(make_twiddles<R>(c->nz, &c->tw_z));
  return GHOST_OK;
}

static void refresh_kparams(ghost_ctx *c) {
  fill_kparams<float>(c, c->kp32);
  fill_kparams<double>(c, c->kp64);
}

// ---------------------------------------------------------------------
// generic dispatch on the context precision
#define GB_DISPATCH(c, CALL)                           \
  ((c)->precision == GHOST_SINGLE ? CALL##_impl<float> : CALL##_impl<double>)

template <typename R> int derivk3_impl(ghost_ctx *c, const void *a, void *b, int dir) {
  const int ts = timer_begin(c, GHOST_TIMER_POINTWISE);
  derivk3_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<R>(c), (const cx<R> *)a, (cx<R> *)b, c->ntot, dir);
  timer_end(c, ts);
  return post_launch(c);
}
template <typename R> int laplak3_impl(ghost_ctx *c, const void *a, void *b) {
  const int ts = timer_begin(c, GHOST_TIMER_POINTWISE);
  laplak3_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<R>(c), (const cx<R> *)a, (cx<R> *)b, c->ntot);
  timer_end(c, ts);
  return post_launch(c);
}
template <typename R> int rotor3_impl(ghost_ctx *c, const void *a, const void *b, void *o, int dir) {
  const int ts = timer_begin(c, GHOST_TIMER_POINTWISE);
  rotor3_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<R>(c), (const cx<R> *)a, (const cx<R> *)b,
                                                             (cx<R> *)o, c->ntot, dir);
  timer_end(c, ts);
  return post_launch(c);
}
template <typename R> int nonlhd3_impl(ghost_ctx *c, const void *a, const void *b, const void *cc, void *g, int dir) {
  const int ts = timer_begin(c, GHOST_TIMER_POINTWISE);
  nonlhd3_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<R>(c), (const cx<R> *)a, (const cx<R> *)b,
                                                              (const cx<R> *)cc, (cx<R> *)g, c->ntot, dir);
  timer_end(c, ts);
  return post_launch(c);
}
template <typename R> int sharp_impl(ghost_ctx *c, const void *a, void *b, double delta) {
  const R pi = (R)3.14159265358979323846;
  const R cut = (pi / (R)delta) * (pi / (R)delta);
  const int ts = timer_begin(c, GHOST_TIMER_POINTWISE);
  sharp_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<R>(c), (const cx<R> *)a, (cx<R> *)b, c->ntot, cut);
  timer_end(c, ts);
  return post_launch(c);
}
template <typename R> int scale3_impl(ghost_ctx *c, void *x, void *y, void *z, double f0, double s) {
  const int ts = timer_begin(c, GHOST_TIMER_POINTWISE);
  scale3_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>((cx<R> *)x, (cx<R> *)y, (cx<R> *)z, c->ntot, (R)f0, s);
  timer_end(c, ts);
  return post_launch(c);
}

template <typename R> int maxabs_impl(ghost_ctx *c, const void *a, const void *b, const void *cc, double *d, int kin) {
  // scratch 0: the complex-to-real intermediate; 1..3: spectral fields
  // whose real-space norm is wanted; 4..6: their real-space values
  void *w[7];
  GB_CHECK(scratch(c, 7, w));
  if (kin == 0) {
    GB_CHECK(rotor3_impl<R>(c, b, cc, w[1], 1));
    GB_CHECK(rotor3_impl<R>(c, a, cc, w[2], 2));
    GB_CHECK(rotor3_impl<R>(c, a, b, w[3], 3));
  } else if (kin == 1) {
    GB_CHECK(laplak3_impl<R>(c, a, w[1]));
    GB_CHECK(laplak3_impl<R>(c, b, w[2]));
    GB_CHECK(laplak3_impl<R>(c, cc, w[3]));
  } else {
    GB_CUDA(cudaMemcpyAsync(w[1], a, c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
    GB_CUDA(cudaMemcpyAsync(w[2], b, c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
    GB_CUDA(cudaMemcpyAsync(w[3], cc, c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  for (int q = 0; q < 3; ++q) GB_CHECK(c2r_dev<R>(c, w[1 + q], w[4 + q]));
  double *part;
  GB_CHECK(partials(c, 1, &part));
  GB_CUDA(cudaMemsetAsync(part, 0, sizeof(double), c->stream));
  maxnorm_kernel<R><<<grid1d(c->nreal), 256, 0, c->stream>>>((const R *)w[4], (const R *)w[5], (const R *)w[6], c->nreal,
                                                               (unsigned long long *)part);
  GB_CHECK(post_launch(c));
  double m;
  GB_CUDA(cudaMemcpyAsync(&m, part, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  const R nn = (R)c->nx * (R)c->ny * (R)c->nz;
  *d = (double)((R)m / nn);
  return GHOST_OK;
}

template <typename R> int init_random_impl(ghost_ctx *c, int32_t *seed, double kdn, double kup, int shape, double amp,
                                           void *ox, void *oy, void *oz) {
  Grid g{c->nx, c->ny, c->nz, c->nxh, c->anis, c->arbsize, c->Dkx, c->Dky, c->Dkz};
  std::vector<R> h1(2 * c->nspec), h2(2 * c->nspec), h3(2 * c->nspec);
  *seed = random_vpot<R>(g, *seed, kdn, kup, shape, h1.data(), h2.data(), h3.data());
  void *w[3];
  GB_CHECK(scratch(c, 3, w));
  GB_CUDA(cudaMemcpyAsync(w[0], h1.data(), c->cbytes, cudaMemcpyHostToDevice, c->stream));
  GB_CUDA(cudaMemcpyAsync(w[1], h2.data(), c->cbytes, cudaMemcpyHostToDevice, c->stream));
  GB_CUDA(cudaMemcpyAsync(w[2], h3.data(), c->cbytes, cudaMemcpyHostToDevice, c->stream));
  GB_CHECK(rotor3_impl<R>(c, w[1], w[2], ox, 1));
  GB_CHECK(rotor3_impl<R>(c, w[0], w[2], oy, 2));
  GB_CHECK(rotor3_impl<R>(c, w[0], w[1], oz, 3));
  double e;
  GB_CHECK(reduce_dev<R>(c, RED_ENERGY, ox, oy, oz, nullptr, nullptr, nullptr, &e));
  return scale3_impl<R>(c, ox, oy, oz, amp, sqrt(e));
}


// ---------------------------------------------------------------------
// batches of runs
template <typename R>
int batch_reduce_dev(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, double *out_host) {
  const int nb = std::max(1, std::min(grid1d(c->nspec), 4096 / std::max(1, c->nruns)));
  double *part;
  GB_CHECK(partials(c, (size_t)(nb + 1) * c->nruns, &part));
  RedArgs<R> ra{(const cx<R> *)a, (const cx<R> *)b, (const cx<R> *)cc, nullptr, nullptr, nullptr};
  const int ts = timer_begin(c, GHOST_TIMER_REDUCE);
  reduce_runs_kernel<R><<<dim3(nb, c->nruns), 256, 0, c->stream>>>(kparams<R>(c), ra, kind, c->nspec, c->nruns, part);
  GB_CHECK(post_launch(c));
  double *fin = part + (size_t)nb * c->nruns;
  finalize_kernel<<<1, 256, 0, c->stream>>>(part, nb, c->nruns, fin);
  timer_end(c, ts);
  GB_CHECK(post_launch(c));
  GB_CUDA(cudaMemcpyAsync(out_host, fin, sizeof(double) * c->nruns, cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

template <typename R>
int batch_init_random_dev(ghost_ctx *c, const int32_t *seeds, int32_t *seeds_out, double kdn, double kup, int shape,
                          double amp, void *ox, void *oy, void *oz) {
  Grid g{c->nx, c->ny, c->nz, c->nxh, c->anis, c->arbsize, c->Dkx, c->Dky, c->Dkz};
  const size_t ns = c->nspec;
  std::vector<R> h1(2 * c->ntot), h2(2 * c->ntot), h3(2 * c->ntot);
  for (int r = 0; r < c->nruns; ++r) {
    const int32_t s = random_vpot<R>(g, seeds[r], kdn, kup, shape, h1.data() + 2 * ns * r, h2.data() + 2 * ns * r,
                                     h3.data() + 2 * ns * r);
    if (seeds_out) seeds_out[r] = s;
  }
  void *w[3];
  GB_CHECK(scratch(c, 3, w));
  GB_CUDA(cudaMemcpyAsync(w[0], h1.data(), c->cbytes, cudaMemcpyHostToDevice, c->stream));
  GB_CUDA(cudaMemcpyAsync(w[1], h2.data(), c->cbytes, cudaMemcpyHostToDevice, c->stream));
  GB_CUDA(cudaMemcpyAsync(w[2], h3.data(), c->cbytes, cudaMemcpyHostToDevice, c->stream));
  GB_CHECK(rotor3_impl<R>(c, w[1], w[2], ox, 1));
  GB_CHECK(rotor3_impl<R>(c, w[0], w[2], oy, 2));
  GB_CHECK(rotor3_impl<R>(c, w[0], w[1], oz, 3));
  std::vector<double> e(c->nruns);
  GB_CHECK(batch_reduce_dev<R>(c, RED_ENERGY, ox, oy, oz, e.data()));
  double *part;
  GB_CHECK(partials(c, (size_t)c->nruns, &part));
  GB_CUDA(cudaMemcpyAsync(part, e.data(), sizeof(double) * c->nruns, cudaMemcpyHostToDevice, c->stream));
  const int ts = timer_begin(c, GHOST_TIMER_POINTWISE);
  scale3_runs_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>((cx<R> *)ox, (cx<R> *)oy, (cx<R> *)oz, c->nspec,
                                                                  c->nruns, (R)amp, part);
  timer_end(c, ts);
  GB_CHECK(post_launch(c));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return GHOST_OK;
}

// instantiations used by the other translation units (internal.cuh)
#define GB_INST(R)                                                                                             \
  template int r2c_dev<R>(ghost_ctx *, const void *, void *);                                                  \
  template int c2r_dev<R>(ghost_ctx *, const void *, void *);                                                  \
  template int r2c6_dev<R>(ghost_ctx *, const void *const[6], void *const[6]);                                 \
  template int grad9_features_dev<R>(ghost_ctx *, const void *const[3], void *const[9], float *, float, float);     \
  template int hd_substep_dev<R>(ghost_ctx *, int, double, double, void *const[3], void *const[3],             \
                                 const void *const[3], int, bool);                                             \
  template int spectrum_dev<R>(ghost_ctx *, int, const void *, const void *, const void *, double *);          \
  template int reduce_dev<R>(ghost_ctx *, int, const void *, const void *, const void *, const void *,         \
                             const void *, const void *, double *);                                            \
  template int spectrum_dev_async<R>(ghost_ctx *, int, const void *, const void *, const void *, double *);
GB_INST(float)
GB_INST(double)
#undef GB_INST

}  // namespace gb

using namespace gb;

// =====================================================================
// C ABI
// =====================================================================
#define CTX_CHECK(c) \
  if (!(c)) return fail(GHOST_ERR_ARG, "null context")

extern "C" {

const char *ghost_last_error_string(void) { return g_err; }

int ghost_ctx_create(int nx, int ny, int nz, double Lx, double Ly, double Lz, int arbsize, int precision,
                     ghost_ctx **out) {
  if (!out) return fail(GHOST_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (!pow2_ok(nx) || !pow2_ok(ny) || !pow2_ok(nz))
    return fail(GHOST_ERR_SIZE, "grid %dx%dx%d: each n must be a power of two in [16,1024]", nx, ny, nz);
  if (precision != GHOST_SINGLE && precision != GHOST_DOUBLE)
    return fail(GHOST_ERR_ARG, "precision %d: use GHOST_SINGLE (4) or GHOST_DOUBLE (8)", precision);
  if (arbsize && !(Lx > 0 && Ly > 0 && Lz > 0)) return fail(GHOST_ERR_ARG, "box lengths must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(GHOST_ERR_NODEV, "no CUDA device");
  }
  ghost_ctx *c = new ghost_ctx();
  c->nx = nx;
  c->ny = ny;
  c->nz = nz;
  c->nxh = nx / 2 + 1;
  c->precision = precision;
  c->arbsize = arbsize ? 1 : 0;
  c->anis = c->arbsize ? 1 : ((nx != ny) || (ny != nz));
  c->nspec = (size_t)nz * ny * c->nxh;
  c->nreal = (size_t)nx * ny * nz;
  c->nruns = 1;
  c->ntot = c->nspec;
  c->nu_run = nullptr;
  c->i0 = 0;
  c->nz_glob = nz;
  // the fastest variants measured for 512-point lines (ghost_hd_autotune
  // re-measures): two-stage z ring with three CTAs per SM, two-stage y ring
  // with a second exchange buffer, and for FP32 y passes with 16 values per
  // thread
  c->tile_cfg = (nz >= 256 ? 6 : 0) | (ny >= 256 ? (precision == GHOST_SINGLE ? 24 : 8) : 0);
  const size_t rs = precision == GHOST_SINGLE ? 4 : 8;
  c->cbytes = c->nspec * 2 * rs;
  c->rbytes = c->nreal * rs;
  cudaGetDevice(&c->device);
  c->stream = nullptr;
  c->launches = 0;
  c->tw_x = c->tw_y = c->tw_z = nullptr;
  c->partials = nullptr;
  c->partials_elems = 0;
  for (int q = 0; q < 4; ++q) c->rk[q] = nullptr;
  c->timers_on = false;
  c->num_sms = 0;
  c->status = nullptr;
  c->wait_cap = 1u << 22;
  c->inject_stall = 0;
  c->prune_valid = c->prune_ok = false;
  c->prune_lines = c->prune_jpos = c->prune_jneg = nullptr;
  c->prune_nlines = c->prune_imax = 0;
  c->prune_jtop = c->prune_jbot = 0;
  c->prune_ktop = c->prune_kbot = 0;
  c->dead_flag = c->dead_flag_host = nullptr;
  c->side = nullptr;
  c->ev_early = c->ev_late = nullptr;
  c->late_pending = false;
  for (int k = 0; k < GHOST_TIMER_KINDS; ++k) {
    c->t_ms[k] = 0.0;
    c->t_n[k] = 0;
  }
  int s = precision == GHOST_SINGLE ? ctx_init_prec<float>(c, Lx, Ly, Lz) : ctx_init_prec<double>(c, Lx, Ly, Lz);
  if (s != GHOST_OK) {
    ghost_ctx_destroy(c);
    return s;
  }
  refresh_kparams(c);
  if (dalloc((void **)&c->status, sizeof(int)) != GHOST_OK || cudaMemset(c->status, 0, sizeof(int)) != cudaSuccess) {
    ghost_ctx_destroy(c);
    return fail(GHOST_ERR_ALLOC, "status word allocation failed");
  }
  *out = c;
  return GHOST_OK;
}

int ghost_ctx_destroy(ghost_ctx *c) {
  if (!c) return GHOST_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  for (void *p : c->scratch) cudaFree(p);
  for (void *p : c->stage) cudaFree(p);
  for (int q = 0; q < 4; ++q)
    if (c->rk[q]) cudaFree(c->rk[q]);
  cudaFree(c->tw_x);
  cudaFree(c->tw_y);
  cudaFree(c->tw_z);
  cudaFree(c->partials);
  cudaFree(c->status);
  cudaFree(c->nu_run);
  cudaFree(c->prune_lines);
  cudaFree(c->prune_jpos);
  cudaFree(c->prune_jneg);
  cudaFree(c->dead_flag);
  if (c->dead_flag_host) cudaFreeHost(c->dead_flag_host);
  if (c->side) {
    cudaStreamSynchronize(c->side);
    cudaStreamDestroy(c->side);
  }
  if (c->ev_early) cudaEventDestroy(c->ev_early);
  if (c->ev_late) cudaEventDestroy(c->ev_late);
  for (auto &p : c->ev_pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (cudaEvent_t e : c->ev_free) cudaEventDestroy(e);
  delete c;
  return GHOST_OK;
}

int ghost_ctx_get_info(const ghost_ctx *c, ghost_info *info) {
  CTX_CHECK(c);
  if (!info) return fail(GHOST_ERR_ARG, "null info");
  info->nx = c->nx;
  info->ny = c->ny;
  info->nz = c->nz;
  info->precision = c->precision;
  info->anis = c->anis;
  info->nmax = c->nmax;
  info->nmaxperp = c->nmaxperp;
  info->kmax = c->kmax;
  info->tiny = c->tiny;
  info->Lx = c->Lx;
  info->Ly = c->Ly;
  info->Lz = c->Lz;
  info->Dkx = c->Dkx;
  info->Dky = c->Dky;
  info->Dkz = c->Dkz;
  info->Dkk = c->Dkk;
  info->spectral_elems = c->nspec;
  info->real_elems = c->nreal;
  return GHOST_OK;
}

int ghost_ctx_set_stream(ghost_ctx *c, void *stream) {
  CTX_CHECK(c);
  c->stream = (cudaStream_t)stream;
  return GHOST_OK;
}

int ghost_ctx_set_kmax(ghost_ctx *c, double kmax) {
  CTX_CHECK(c);
  c->kmax = c->precision == GHOST_SINGLE ? (double)(float)kmax : kmax;
  refresh_kparams(c);
  c->prune_valid = false;
  return GHOST_OK;
}

int ghost_ctx_synchronize(ghost_ctx *c) {
  CTX_CHECK(c);
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

int ghost_ctx_inject_stall(ghost_ctx *c, int enable) {
  CTX_CHECK(c);
  c->inject_stall = enable != 0;
  return GHOST_OK;
}

int ghost_ctx_set_wait_cap(ghost_ctx *c, unsigned int cap) {
  CTX_CHECK(c);
  c->wait_cap = cap ? cap : (1u << 22);
  return GHOST_OK;
}

int ghost_ctx_enable_timers(ghost_ctx *c, int enable) {
  CTX_CHECK(c);
  GB_CHECK(timers_collect(c));
  c->timers_on = enable != 0;
  return GHOST_OK;
}

int ghost_ctx_read_timers(ghost_ctx *c, double ms[GHOST_TIMER_KINDS], long long launches[GHOST_TIMER_KINDS]) {
  CTX_CHECK(c);
  if (!ms || !launches) return fail(GHOST_ERR_ARG, "null output");
  GB_CHECK(timers_collect(c));
  for (int k = 0; k < GHOST_TIMER_KINDS; ++k) {
    ms[k] = c->t_ms[k];
    launches[k] = c->t_n[k];
    c->t_ms[k] = 0.0;
    c->t_n[k] = 0;
  }
  return GHOST_OK;
}

int ghost_ctx_launch_count(const ghost_ctx *c, long long *count) {
  CTX_CHECK(c);
  if (!count) return fail(GHOST_ERR_ARG, "null count");
  *count = c->launches;
  return GHOST_OK;
}

// ------------------------------------------------------------------ FFT
int ghost_fftp3d_create_plan(ghost_ctx *c, const int n[3], int fftdir, int flags, ghost_fftplan **plan) {
  (void)flags;
  CTX_CHECK(c);
  if (!n || !plan) return fail(GHOST_ERR_ARG, "null argument");
  if (fftdir != GHOST_REAL_TO_COMPLEX && fftdir != GHOST_COMPLEX_TO_REAL)
    return fail(GHOST_ERR_ARG, "fftdir %d: use -1 (real to complex) or +1 (complex to real)", fftdir);
  if (n[0] != c->nx || n[1] != c->ny || n[2] != c->nz)
    return fail(GHOST_ERR_SIZE, "plan size %dx%dx%d differs from the context grid", n[0], n[1], n[2]);
  ghost_fftplan *p = new ghost_fftplan();
  p->ctx = c;
  p->fftdir = fftdir;
  *plan = p;
  return GHOST_OK;
}

int ghost_fftp3d_destroy_plan(ghost_fftplan *plan) {
  delete plan;
  return GHOST_OK;
}

int ghost_fftp3d_real_to_complex(ghost_fftplan *plan, const void *in, void *out) {
  if (!plan || !in || !out) return fail(GHOST_ERR_ARG, "null argument");
  ghost_ctx *c = plan->ctx;
  if (plan->fftdir != GHOST_REAL_TO_COMPLEX) return fail(GHOST_ERR_STATE, "plan is not a real-to-complex plan");
  Staging st(c);
  const void *din;
  void *dout;
  GB_CHECK(st.map(in, c->rbytes, 1, &din));
  GB_CHECK(st.map(out, c->cbytes, 2, &dout));
  GB_CHECK(c->precision == GHOST_SINGLE ? r2c_dev<float>(c, din, dout) : r2c_dev<double>(c, din, dout));
  return st.finish();
}

int ghost_fftp3d_complex_to_real(ghost_fftplan *plan, const void *in, void *out) {
  if (!plan || !in || !out) return fail(GHOST_ERR_ARG, "null argument");
  ghost_ctx *c = plan->ctx;
  if (plan->fftdir != GHOST_COMPLEX_TO_REAL) return fail(GHOST_ERR_STATE, "plan is not a complex-to-real plan");
  Staging st(c);
  const void *din;
  void *dout;
  GB_CHECK(st.map(in, c->cbytes, 1, &din));
  GB_CHECK(st.map(out, c->rbytes, 2, &dout));
  GB_CHECK(c->precision == GHOST_SINGLE ? c2r_dev<float>(c, din, dout) : c2r_dev<double>(c, din, dout));
  return st.finish();
}

// ------------------------------------------------------------ operators
static int dir_ok(int dir) { return dir >= 1 && dir <= 3; }

int ghost_derivk3(ghost_ctx *c, const void *a, void *b, int dir) {
  CTX_CHECK(c);
  if (!a || !b) return fail(GHOST_ERR_ARG, "null field");
  if (!dir_ok(dir)) return fail(GHOST_ERR_ARG, "dir %d not in 1..3", dir);
  Staging st(c);
  const void *da;
  void *db;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 2, &db));
  GB_CHECK(GB_DISPATCH(c, derivk3)(c, da, db, dir));
  return st.finish();
}

int ghost_laplak3(ghost_ctx *c, const void *a, void *b) {
  CTX_CHECK(c);
  if (!a || !b) return fail(GHOST_ERR_ARG, "null field");
  Staging st(c);
  const void *da;
  void *db;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 2, &db));
  GB_CHECK(GB_DISPATCH(c, laplak3)(c, da, db));
  return st.finish();
}

int ghost_rotor3(ghost_ctx *c, const void *a, const void *b, void *o, int dir) {
  CTX_CHECK(c);
  if (!a || !b || !o) return fail(GHOST_ERR_ARG, "null field");
  if (!dir_ok(dir)) return fail(GHOST_ERR_ARG, "dir %d not in 1..3", dir);
  Staging st(c);
  const void *da, *db;
  void *dc;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(o, c->cbytes, 2, &dc));
  GB_CHECK(GB_DISPATCH(c, rotor3)(c, da, db, dc, dir));
  return st.finish();
}

int ghost_prodre3(ghost_ctx *c, const void *a, const void *b, const void *cc, void *d, void *e, void *f) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !d || !e || !f) return fail(GHOST_ERR_ARG, "null field");
  Staging st(c);
  const void *da, *db, *dc;
  void *dd, *de, *df;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  GB_CHECK(st.map(d, c->cbytes, 2, &dd));
  GB_CHECK(st.map(e, c->cbytes, 2, &de));
  GB_CHECK(st.map(f, c->cbytes, 2, &df));
  GB_CHECK(c->precision == GHOST_SINGLE ? prodre3_dev<float>(c, da, db, dc, dd, de, df)
                                        : prodre3_dev<double>(c, da, db, dc, dd, de, df));
  return st.finish();
}

int ghost_nonlhd3(ghost_ctx *c, const void *a, const void *b, const void *cc, void *g, int dir) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !g) return fail(GHOST_ERR_ARG, "null field");
  if (!dir_ok(dir)) return fail(GHOST_ERR_ARG, "dir %d not in 1..3", dir);
  Staging st(c);
  const void *da, *db, *dc;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  // g may alias an input; the kernel reads all three inputs of a mode
  // before writing g at that mode, so aliasing is safe element-wise
  void *dg;
  GB_CHECK(st.map(g, c->cbytes, 2, &dg));
  GB_CHECK(GB_DISPATCH(c, nonlhd3)(c, da, db, dc, dg, dir));
  return st.finish();
}

static int reduce_api(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, const void *d,
                      const void *e, const void *f, double *out) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !out) return fail(GHOST_ERR_ARG, "null argument");
  Staging st(c);
  const void *da, *db, *dc, *dd = nullptr, *de = nullptr, *df = nullptr;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  if (d) {
    GB_CHECK(st.map(d, c->cbytes, 1, &dd));
    GB_CHECK(st.map(e, c->cbytes, 1, &de));
    GB_CHECK(st.map(f, c->cbytes, 1, &df));
  }
  GB_CHECK(c->precision == GHOST_SINGLE ? reduce_dev<float>(c, kind, da, db, dc, dd, de, df, out)
                                        : reduce_dev<double>(c, kind, da, db, dc, dd, de, df, out));
  return st.finish();
}

int ghost_energy(ghost_ctx *c, const void *a, const void *b, const void *cc, double *d, int kin) {
  if (kin < 0 || kin > 2) return fail(GHOST_ERR_ARG, "kin %d not in 0..2", kin);
  const int kind = kin == 1 ? RED_ENERGY : (kin == 0 ? RED_ENSTROPHY : RED_LAPLACIAN);
  return reduce_api(c, kind, a, b, cc, nullptr, nullptr, nullptr, d);
}

int ghost_helicity(ghost_ctx *c, const void *a, const void *b, const void *cc, double *d) {
  return reduce_api(c, RED_HELICITY, a, b, cc, nullptr, nullptr, nullptr, d);
}

int ghost_cross(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                const void *f, double *g, int kin) {
  if (kin != 0 && kin != 1) return fail(GHOST_ERR_ARG, "kin %d not in 0..1", kin);
  if (!d || !e || !f) return fail(GHOST_ERR_ARG, "null field");
  return reduce_api(c, kin == 1 ? RED_CROSS : RED_CROSS_K2, a, b, cc, d, e, f, g);
}

int ghost_divergence(ghost_ctx *c, const void *a, const void *b, const void *cc, double *d) {
  return reduce_api(c, RED_DIVERGENCE, a, b, cc, nullptr, nullptr, nullptr, d);
}

int ghost_maxabs(ghost_ctx *c, const void *a, const void *b, const void *cc, double *d, int kin) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !d) return fail(GHOST_ERR_ARG, "null argument");
  if (kin < 0 || kin > 2) return fail(GHOST_ERR_ARG, "kin %d not in 0..2", kin);
  Staging st(c);
  const void *da, *db, *dc;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  GB_CHECK(GB_DISPATCH(c, maxabs)(c, da, db, dc, d, kin));
  return st.finish();
}

int ghost_spectrumc(ghost_ctx *c, const void *a, const void *b, const void *cc, int kin, int hel, double *Ek,
                    double *Hk) {
  CTX_CHECK(c);
  if (!a || !b || !cc) return fail(GHOST_ERR_ARG, "null field");
  if (kin < 0 || kin > 2) return fail(GHOST_ERR_ARG, "kin %d not in 0..2", kin);
  if (kin <= 1 && !Ek) return fail(GHOST_ERR_ARG, "null Ek");
  if (hel == 1 && !Hk) return fail(GHOST_ERR_ARG, "null Hk");
  Staging st(c);
  const void *da, *db, *dc;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  const bool sp = c->precision == GHOST_SINGLE;
  if (kin <= 1) {
    const int kind = kin == 1 ? RED_ENERGY : RED_ENSTROPHY;
    GB_CHECK(sp ? spectrum_dev<float>(c, kind, da, db, dc, Ek) : spectrum_dev<double>(c, kind, da, db, dc, Ek));
  }
  if (hel == 1)
    GB_CHECK(sp ? spectrum_dev<float>(c, RED_HELICITY, da, db, dc, Hk)
                : spectrum_dev<double>(c, RED_HELICITY, da, db, dc, Hk));
  return st.finish();
}

// entrans / heltrans (pseudospec3D_hd.f90:1629-1949): the shell-binned
// transfer Re(x . conj(d,e,f))/(nx ny nz)^2, x = (a,b,c) (times kk2 when
// entrans' kin is 0) or curl(a,b,c) for heltrans; GHOST's Ektot / Hktot.
static int transfer(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, const void *d,
                    const void *e, const void *f, double *out) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !d || !e || !f || !out) return fail(GHOST_ERR_ARG, "null argument");
  Staging st(c);
  const void *da, *db, *dc, *dd, *de, *df;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  GB_CHECK(st.map(d, c->cbytes, 1, &dd));
  GB_CHECK(st.map(e, c->cbytes, 1, &de));
  GB_CHECK(st.map(f, c->cbytes, 1, &df));
  GB_CHECK(c->precision == GHOST_SINGLE ? spectrum6_dev<float>(c, kind, da, db, dc, dd, de, df, out)
                                        : spectrum6_dev<double>(c, kind, da, db, dc, dd, de, df, out));
  return st.finish();
}

int ghost_entrans(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                  const void *f, int kin, double *Ek) {
  if (kin < 0 || kin > 4) return fail(GHOST_ERR_ARG, "kin %d not in 0..4", kin);
  return transfer(c, kin == 0 ? RED_CROSS_K2 : RED_CROSS, a, b, cc, d, e, f, Ek);
}

int ghost_heltrans(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                   const void *f, int kin, double *Hk) {
  if (kin < 0 || kin > 1) return fail(GHOST_ERR_ARG, "kin %d not in 0..1", kin);
  return transfer(c, RED_CURL_CROSS, a, b, cc, d, e, f, Hk);
}

int ghost_phaseshift(ghost_ctx *c, void *a, double cre, double cim) {
  CTX_CHECK(c);
  if (!a) return fail(GHOST_ERR_ARG, "null field");
  if (c->nruns != 1) return fail(GHOST_ERR_STATE, "batched contexts are not supported here");
  Staging st(c);
  void *da;
  GB_CHECK(st.map(a, c->cbytes, 3, &da));
  if (c->precision == GHOST_SINGLE)
    phaseshift_kernel<float><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<float>(c), (cx<float> *)da, c->ntot,
                                                                      make_float2((float)cre, (float)cim));
  else
    phaseshift_kernel<double><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<double>(c), (cx<double> *)da, c->ntot,
                                                                       make_double2(cre, cim));
  GB_CHECK(post_launch(c));
  return st.finish();
}

// The rand = 2 forcing of main3D.fpp:2581-2657: between two random
// forcings (regenerated every fstep steps by initialfv), each step uses
// f = (1 - rmp) fold + rmp fnew with rmp = FLOAT(timef+1)/float(fstep),
// evaluated in default (single-precision) REAL as GHOST does.
int ghost_forcing_slow(ghost_ctx *c, int timef, int fstep, const void *fxold, const void *fyold, const void *fzold,
                       const void *fxnew, const void *fynew, const void *fznew, void *fx, void *fy, void *fz) {
  CTX_CHECK(c);
  if (fstep < 1) return fail(GHOST_ERR_ARG, "fstep %d must be positive", fstep);
  if (timef < 0 || timef >= fstep) return fail(GHOST_ERR_ARG, "timef %d not in 0..fstep-1", timef);
  const void *in[6] = {fxold, fyold, fzold, fxnew, fynew, fznew};
  void *out[3] = {fx, fy, fz};
  for (const void *p : in)
    if (!p) return fail(GHOST_ERR_ARG, "null field");
  for (void *p : out)
    if (!p) return fail(GHOST_ERR_ARG, "null field");
  Staging st(c);
  const void *din[6];
  void *dout[3];
  for (int q = 0; q < 6; ++q) GB_CHECK(st.map(in[q], c->cbytes, 1, &din[q]));
  for (int q = 0; q < 3; ++q) GB_CHECK(st.map(out[q], c->cbytes, 2, &dout[q]));
  const float rmpf = (float)(timef + 1) / (float)fstep;
  if (c->precision == GHOST_SINGLE) {
    Blend3<float> b;
    for (int q = 0; q < 3; ++q) {
      b.old[q] = (const cx<float> *)din[q];
      b.nw[q] = (const cx<float> *)din[3 + q];
      b.out[q] = (cx<float> *)dout[q];
    }
    blend3_kernel<float><<<grid1d(c->ntot), 256, 0, c->stream>>>(b, c->ntot, 1.0f - rmpf, rmpf);
  } else {
    Blend3<double> b;
    for (int q = 0; q < 3; ++q) {
      b.old[q] = (const cx<double> *)din[q];
      b.nw[q] = (const cx<double> *)din[3 + q];
      b.out[q] = (cx<double> *)dout[q];
    }
    const double rmp = (double)rmpf;
    blend3_kernel<double><<<grid1d(c->ntot), 256, 0, c->stream>>>(b, c->ntot, 1.0 - rmp, rmp);
  }
  GB_CHECK(post_launch(c));
  return st.finish();
}

// ---------------------------------------------------------------------
// MHD (MHD_SOL, pseudospec3D_mhd.f90 and include/mhd_rkstep1/2.f90)
extern "C++" {
// vector3(a,b,c,d,e,f,x,y,z) (pseudospec3D_mhd.f90:22-105): (a,b,c) x (d,e,f)
// through real space, times 1/(nx ny nz)^2.  Uses scratch 37..45.
template <typename R>
static int vector3_dev(ghost_ctx *c, const void *const in[6], void *const out[3]) {
  void *sc[46];
  GB_CHECK(scratch(c, 46, sc));
  void **r = sc + 37;  // six real inputs, three real products
  for (int q = 0; q < 6; ++q) GB_CHECK(c2r_dev<R>(c, in[q], r[q]));
  const R tmp = (R)1 / (((R)c->nx * (R)c->ny * (R)c->nz) * ((R)c->nx * (R)c->ny * (R)c->nz));
  cross_real_kernel<R><<<grid1d(c->nreal), 256, 0, c->stream>>>((const R *)r[0], (const R *)r[1], (const R *)r[2],
                                                                 (const R *)r[3], (const R *)r[4], (const R *)r[5],
                                                                 (R *)r[6], (R *)r[7], (R *)r[8], c->nreal, tmp);
  GB_CHECK(post_launch(c));
  for (int q = 0; q < 3; ++q) GB_CHECK(r2c_dev<R>(c, r[6 + q], out[q]));
  return GHOST_OK;
}

// nonlin3(a,b,c,d,e,f,g,dir) (:108-227) = nonlhd3 of (a-d, b-e, c-f);
// gauge3(a,b,c,g,dir) (:230-336) = -nonlhd3(a,b,c,g,dir).  Scratch 34..36.
template <typename R>
static int nonlin3_dev(ghost_ctx *c, const void *const in[6], void *g, int dir) {
  void *sc[46];
  GB_CHECK(scratch(c, 46, sc));
  sub3_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>(
      (const cx<R> *)in[0], (const cx<R> *)in[1], (const cx<R> *)in[2], (const cx<R> *)in[3], (const cx<R> *)in[4],
      (const cx<R> *)in[5], (cx<R> *)sc[34], (cx<R> *)sc[35], (cx<R> *)sc[36], c->ntot);
  GB_CHECK(post_launch(c));
  return nonlhd3_impl<R>(c, sc[34], sc[35], sc[36], g, dir);
}
template <typename R> static int gauge3_dev(ghost_ctx *c, const void *a, const void *b, const void *cc, void *g, int dir) {
  GB_CHECK(nonlhd3_impl<R>(c, a, b, cc, g, dir));
  neg_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>((cx<R> *)g, c->ntot);
  return post_launch(c);
}

// One MHD substep (include/mhd_rkstep2.f90); Cv, Ca the RK copies of v, a
template <typename R>
static int mhd_substep_dev(ghost_ctx *c, int o, double dt, double nu, double mu, void *const v[3], void *const a[3],
                           void *const Cv[3], void *const Ca[3], const void *const f[3], const void *const m[3]) {
  void *sc[46];
  GB_CHECK(scratch(c, 46, sc));
  void *B[3] = {sc[22], sc[23], sc[24]}, *N1[3] = {sc[25], sc[26], sc[27]}, *N2[3] = {sc[28], sc[29], sc[30]};
  void *G[3] = {sc[31], sc[32], sc[33]};
  // b = curl a (rotor3(ay,az,C7,1), rotor3(ax,az,C8,2), rotor3(ax,ay,C9,3))
  GB_CHECK(rotor3_impl<R>(c, a[1], a[2], B[0], 1));
  GB_CHECK(rotor3_impl<R>(c, a[0], a[2], B[1], 2));
  GB_CHECK(rotor3_impl<R>(c, a[0], a[1], B[2], 3));
  GB_CHECK(prodre3_dev<R>(c, v[0], v[1], v[2], N1[0], N1[1], N1[2]));  // w x v
  GB_CHECK(prodre3_dev<R>(c, B[0], B[1], B[2], N2[0], N2[1], N2[2]));  // j x b
  const void *nl[6] = {N1[0], N1[1], N1[2], N2[0], N2[1], N2[2]};
  for (int d = 0; d < 3; ++d) GB_CHECK(nonlin3_dev<R>(c, nl, G[d], d + 1));
  // v x b into N1, its Coulomb-gauge projection into N2
  const void *vb[6] = {v[0], v[1], v[2], B[0], B[1], B[2]};
  GB_CHECK(vector3_dev<R>(c, vb, N1));
  for (int d = 0; d < 3; ++d) GB_CHECK(gauge3_dev<R>(c, N1[0], N1[1], N1[2], N2[d], d + 1));
  MhdUpd<R> u{};
  for (int q = 0; q < 3; ++q) {
    u.v[q] = (cx<R> *)v[q];
    u.a[q] = (cx<R> *)a[q];
    u.cv[q] = (const cx<R> *)Cv[q];
    u.ca[q] = (const cx<R> *)Ca[q];
    u.g[q] = (const cx<R> *)G[q];
    u.h[q] = (const cx<R> *)N2[q];
    u.f[q] = f ? (const cx<R> *)f[q] : nullptr;
    u.m[q] = m ? (const cx<R> *)m[q] : nullptr;
  }
  mhd_update_kernel<R><<<grid1d(c->ntot), 256, 0, c->stream>>>(kparams<R>(c), u, c->ntot, (R)dt, (R)nu, (R)mu,
                                                                (R)1 / (R)o);
  return post_launch(c);
}

template <typename R>
static int mhd_run_dev(ghost_ctx *c, int nsteps, int ord, double dt, double nu, double mu, void *const v[3],
                       void *const a[3], const void *const f[3], const void *const m[3]) {
  void *sc[46];
  GB_CHECK(scratch(c, 46, sc));
  void *Cv[3] = {sc[16], sc[17], sc[18]}, *Ca[3] = {sc[19], sc[20], sc[21]};
  for (int s = 0; s < nsteps; ++s) {
    // mhd_rkstep1: C1..C6 = v, a
    for (int q = 0; q < 3; ++q) {
      GB_CUDA(cudaMemcpyAsync(Cv[q], v[q], c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
      GB_CUDA(cudaMemcpyAsync(Ca[q], a[q], c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
    }
    for (int o = ord; o >= 1; --o) GB_CHECK(mhd_substep_dev<R>(c, o, dt, nu, mu, v, a, Cv, Ca, f, m));
  }
  return check_status(c);
}
}  // extern "C++"

int ghost_vector3(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                  const void *f, void *x, void *y, void *z) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !d || !e || !f || !x || !y || !z) return fail(GHOST_ERR_ARG, "null field");
  if (c->nruns != 1) return fail(GHOST_ERR_STATE, "batched contexts are not supported here");
  Staging st(c);
  const void *in[6];
  void *out[3];
  const void *src[6] = {a, b, cc, d, e, f};
  void *dst[3] = {x, y, z};
  for (int q = 0; q < 6; ++q) GB_CHECK(st.map(src[q], c->cbytes, 1, &in[q]));
  for (int q = 0; q < 3; ++q) GB_CHECK(st.map(dst[q], c->cbytes, 2, &out[q]));
  GB_CHECK(c->precision == GHOST_SINGLE ? vector3_dev<float>(c, in, out) : vector3_dev<double>(c, in, out));
  return st.finish();
}

int ghost_nonlin3(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                  const void *f, void *g, int dir) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !d || !e || !f || !g) return fail(GHOST_ERR_ARG, "null field");
  if (!dir_ok(dir)) return fail(GHOST_ERR_ARG, "dir %d not in 1..3", dir);
  Staging st(c);
  const void *in[6];
  void *dg;
  const void *src[6] = {a, b, cc, d, e, f};
  for (int q = 0; q < 6; ++q) GB_CHECK(st.map(src[q], c->cbytes, 1, &in[q]));
  GB_CHECK(st.map(g, c->cbytes, 2, &dg));
  GB_CHECK(c->precision == GHOST_SINGLE ? nonlin3_dev<float>(c, in, dg, dir) : nonlin3_dev<double>(c, in, dg, dir));
  return st.finish();
}

int ghost_gauge3(ghost_ctx *c, const void *a, const void *b, const void *cc, void *g, int dir) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !g) return fail(GHOST_ERR_ARG, "null field");
  if (!dir_ok(dir)) return fail(GHOST_ERR_ARG, "dir %d not in 1..3", dir);
  Staging st(c);
  const void *da, *db, *dc;
  void *dg;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  GB_CHECK(st.map(g, c->cbytes, 2, &dg));
  GB_CHECK(c->precision == GHOST_SINGLE ? gauge3_dev<float>(c, da, db, dc, dg, dir)
                                        : gauge3_dev<double>(c, da, db, dc, dg, dir));
  return st.finish();
}

int ghost_mhd_run(ghost_ctx *c, int nsteps, int ord, double dt, double nu, double mu, void *vx, void *vy, void *vz,
                  void *ax, void *ay, void *az, const void *fx, const void *fy, const void *fz, const void *mx,
                  const void *my, const void *mz) {
  CTX_CHECK(c);
  if (!vx || !vy || !vz || !ax || !ay || !az) return fail(GHOST_ERR_ARG, "null field");
  if (nsteps < 0 || ord < 1) return fail(GHOST_ERR_ARG, "nsteps %d, ord %d", nsteps, ord);
  if ((!fx) != (!fy) || (!fx) != (!fz) || (!mx) != (!my) || (!mx) != (!mz))
    return fail(GHOST_ERR_ARG, "forcing components must all be given or all be null");
  if (c->nruns != 1) return fail(GHOST_ERR_STATE, "batched contexts are not supported here");
  Staging st(c);
  void *v[3], *a[3];
  const void *f[3] = {nullptr, nullptr, nullptr}, *m[3] = {nullptr, nullptr, nullptr};
  void *vs[3] = {vx, vy, vz}, *as[3] = {ax, ay, az};
  const void *fs[3] = {fx, fy, fz}, *ms[3] = {mx, my, mz};
  for (int q = 0; q < 3; ++q) {
    GB_CHECK(st.map(vs[q], c->cbytes, 3, &v[q]));
    GB_CHECK(st.map(as[q], c->cbytes, 3, &a[q]));
    if (fx) GB_CHECK(st.map(fs[q], c->cbytes, 1, &f[q]));
    if (mx) GB_CHECK(st.map(ms[q], c->cbytes, 1, &m[q]));
  }
  GB_CHECK(c->precision == GHOST_SINGLE ? mhd_run_dev<float>(c, nsteps, ord, dt, nu, mu, v, a, fx ? f : nullptr,
                                                             mx ? m : nullptr)
                                        : mhd_run_dev<double>(c, nsteps, ord, dt, nu, mu, v, a, fx ? f : nullptr,
                                                              mx ? m : nullptr));
  return st.finish();
}

// Passive scalar (pseudospec3D_phd.f90): variance (:116-216), spectrscc
// (:516-609), sctrans (:612-726) of a scalar spectral field.
int ghost_variance(ghost_ctx *c, const void *a, int kin, double *out) {
  CTX_CHECK(c);
  if (!a || !out) return fail(GHOST_ERR_ARG, "null argument");
  if (kin < 0 || kin > 1) return fail(GHOST_ERR_ARG, "kin %d not in 0..1", kin);
  Staging st(c);
  const void *da;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  const int kind = kin == 1 ? RED_SC_VAR : RED_SC_VAR_K2;
  GB_CHECK(c->precision == GHOST_SINGLE ? reduce_dev<float>(c, kind, da, da, da, nullptr, nullptr, nullptr, out)
                                        : reduce_dev<double>(c, kind, da, da, da, nullptr, nullptr, nullptr, out));
  return st.finish();
}

int ghost_spectrscc(ghost_ctx *c, const void *a, double shift, double *Ek) {
  CTX_CHECK(c);
  if (!a || !Ek) return fail(GHOST_ERR_ARG, "null argument");
  Staging st(c);
  const void *da;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  // round = shift + .501_GP (a GP literal here, unlike spectrumc's default REAL)
  GB_CHECK(c->precision == GHOST_SINGLE
               ? spectrum6_dev<float>(c, RED_SC_VAR, da, da, da, da, da, da, Ek, (float)shift + 0.501f)
               : spectrum6_dev<double>(c, RED_SC_VAR, da, da, da, da, da, da, Ek, shift + 0.501));
  return st.finish();
}

int ghost_sctrans(ghost_ctx *c, const void *a, const void *b, int isc, double *Ek) {
  CTX_CHECK(c);
  if (!a || !b || !Ek) return fail(GHOST_ERR_ARG, "null argument");
  if (isc < 0) return fail(GHOST_ERR_ARG, "isc %d", isc);
  Staging st(c);
  const void *da, *db;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(c->precision == GHOST_SINGLE ? spectrum6_dev<float>(c, RED_SC_CROSS, da, da, da, db, db, db, Ek)
                                        : spectrum6_dev<double>(c, RED_SC_CROSS, da, da, da, db, db, db, Ek));
  return st.finish();
}

// havgcomp (pseudospec3D_bouss.f90:19-554): the horizontally averaged
// profile gsh[nz] of quantity itype (0..10) of the Boussinesq fields u, v,
// w (velocity) and s (temperature).  Scratch fields 0..8 belong to the
// transforms and advect3_dev; this uses 9..15.
extern "C++" {
template <typename R>
static int zsum(ghost_ctx *c, int op, const void *r1, const void *r2, const void *r3, R fo, R bv,
                std::vector<double> &sh) {
  const size_t plane = (size_t)c->nx * c->ny;
  const int nsplit = (int)std::max<size_t>(1, std::min<size_t>(64, plane / 4096));
  double *part;
  GB_CHECK(partials(c, (size_t)c->nz * nsplit, &part));
  ZProfArgs<R> za{(const R *)r1, (const R *)r2, (const R *)r3, fo, bv,
                  1.0 / ((double)c->nx * (double)c->ny * (double)c->nz)};
  zprof_kernel<R><<<dim3(c->nz, nsplit), 256, 0, c->stream>>>(za, op, plane, part);
  GB_CHECK(post_launch(c));
  std::vector<double> host((size_t)c->nz * nsplit);
  GB_CUDA(cudaMemcpyAsync(host.data(), part, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < c->nz; ++k)
    for (int q = 0; q < nsplit; ++q) sh[k] += host[(size_t)k * nsplit + q];
  return GHOST_OK;
}

template <typename R>
static int havg_dev(ghost_ctx *c, const void *u, const void *v, const void *w, const void *s, R fo, R bv, int itype,
                    double *gsh) {
  void *sc[16];
  GB_CHECK(scratch(c, 16, sc));
  void *c1 = sc[9], *c2 = sc[10], *c3 = sc[11], *c4 = sc[12], *r1 = sc[13], *r2 = sc[14], *r3 = sc[15];
  const int nz = c->nz;
  std::vector<double> sh(nz, 0.0);
  // 1/(nx^3 ny^3 nz^2): the transforms' N^3 per factor, over nx ny points
  const double tmp0 = 1.0 / (std::pow((double)c->nx, 3) * std::pow((double)c->ny, 3) * std::pow((double)c->nz, 2));
  double scale = tmp0;
  auto c2r = [&](const void *in, void *out) { return c2r_dev<R>(c, in, out); };
  auto dz = [&](const void *in, void *out) { return derivk3_impl<R>(c, in, out, 3); };
  auto zs = [&](int op, const void *a, const void *b, const void *cc) {
    return zsum<R>(c, op, a, b, cc, fo, bv, sh);
  };
  // GHOST enters the type-0 branch for itype 9 too and returns from it, so
  // its column 10 repeats column 1 (the Richardson-number block is not reached)
  switch (itype == 9 ? 0 : itype) {
    case 0:  // <(du_perp/dz)^2>_perp
      GB_CHECK(dz(u, c1)); GB_CHECK(c2r(c1, r1));
      GB_CHECK(dz(v, c1)); GB_CHECK(c2r(c1, r2));
      GB_CHECK(zs(ZP_SQ2, r1, r2, nullptr));
      break;
    case 1:  // <(dtheta/dz)^2>_perp
      GB_CHECK(dz(s, c1)); GB_CHECK(c2r(c1, r3));
      GB_CHECK(zs(ZP_SQ1, r3, nullptr, nullptr));
      break;
    case 2:  // <u_z dtheta/dz>_perp (the profile GHOST's comment names)
      GB_CHECK(dz(s, c1)); GB_CHECK(c2r(c1, r3));
      GB_CHECK(c2r(w, r2));
      GB_CHECK(zs(ZP_PROD, r3, r2, nullptr));
      break;
    case 3:  // <u^2 + v^2>_perp
      GB_CHECK(c2r(u, r1)); GB_CHECK(c2r(v, r2));
      GB_CHECK(zs(ZP_SQ2, r1, r2, nullptr));
      break;
    case 4:  // <w^2>_perp
      GB_CHECK(c2r(w, r1));
      GB_CHECK(zs(ZP_SQ1, r1, nullptr, nullptr));
      break;
    case 5:  // <v du/dz - u dv/dz>_perp
      GB_CHECK(dz(v, c1)); GB_CHECK(c2r(c1, r2)); GB_CHECK(c2r(u, r1));
      GB_CHECK(zs(ZP_NEGPROD, r1, r2, nullptr));
      GB_CHECK(dz(u, c1)); GB_CHECK(c2r(c1, r2)); GB_CHECK(c2r(v, r1));
      GB_CHECK(zs(ZP_PROD, r1, r2, nullptr));
      break;
    case 6:  // <omega_z theta>_perp
      GB_CHECK(rotor3_impl<R>(c, u, v, c1, 3)); GB_CHECK(c2r(c1, r1));
      GB_CHECK(c2r(s, r2));
      GB_CHECK(zs(ZP_PROD, r1, r2, nullptr));
      break;
    case 7: {  // <PV^2>_perp
      GB_CHECK(dz(s, c1)); GB_CHECK(c2r(c1, r1));
      GB_CHECK(rotor3_impl<R>(c, u, v, c1, 3)); GB_CHECK(c2r(c1, r2));
      GB_CHECK(rotor3_impl<R>(c, v, w, c1, 1));
      GB_CHECK(rotor3_impl<R>(c, u, w, c2, 2));
      GB_CHECK(rotor3_impl<R>(c, u, v, c3, 3));
      GB_CHECK(advect3_dev<R>(c, c1, c2, c3, s, c4));
      GB_CHECK(c2r(c4, r3));
      GB_CHECK(zs(ZP_PV, r1, r2, r3));
      scale = 1.0 / ((double)c->nx * (double)c->ny);
      break;
    }
    case 8:  // <omega . curl(omega) parts>_perp, three terms r3 (r1 - r2)
      GB_CHECK(rotor3_impl<R>(c, u, v, c1, 3)); GB_CHECK(derivk3_impl<R>(c, c1, c2, 2)); GB_CHECK(c2r(c2, r1));
      GB_CHECK(rotor3_impl<R>(c, u, w, c1, 2)); GB_CHECK(derivk3_impl<R>(c, c1, c2, 3)); GB_CHECK(c2r(c2, r2));
      GB_CHECK(rotor3_impl<R>(c, v, w, c1, 1)); GB_CHECK(c2r(c1, r3));
      GB_CHECK(zs(ZP_CURLTERM, r1, r2, r3));
      GB_CHECK(rotor3_impl<R>(c, v, w, c1, 1)); GB_CHECK(derivk3_impl<R>(c, c1, c2, 3)); GB_CHECK(c2r(c2, r1));
      GB_CHECK(rotor3_impl<R>(c, u, v, c1, 3)); GB_CHECK(derivk3_impl<R>(c, c1, c2, 1)); GB_CHECK(c2r(c2, r2));
      GB_CHECK(rotor3_impl<R>(c, u, w, c1, 2)); GB_CHECK(c2r(c1, r3));
      GB_CHECK(zs(ZP_CURLTERM, r1, r2, r3));
      GB_CHECK(rotor3_impl<R>(c, u, w, c1, 2)); GB_CHECK(derivk3_impl<R>(c, c1, c2, 1)); GB_CHECK(c2r(c2, r1));
      GB_CHECK(rotor3_impl<R>(c, v, w, c1, 1)); GB_CHECK(derivk3_impl<R>(c, c1, c2, 2)); GB_CHECK(c2r(c2, r2));
      GB_CHECK(rotor3_impl<R>(c, u, v, c1, 3)); GB_CHECK(c2r(c1, r3));
      GB_CHECK(zs(ZP_CURLTERM, r1, r2, r3));
      break;
    case 10:  // <w theta>_perp
      GB_CHECK(c2r(w, r1)); GB_CHECK(c2r(s, r2));
      GB_CHECK(zs(ZP_PROD, r1, r2, nullptr));
      break;
    default:
      return fail(GHOST_ERR_ARG, "itype %d not in 0..10", itype);
  }
  for (int k = 0; k < nz; ++k) gsh[k] = sh[k] * scale;
  return check_status(c);
}
}  // extern "C++"

static int havg(ghost_ctx *c, const void *u, const void *v, const void *w, const void *s, double fo, double bv,
                int itype, double *gsh) {
  if (c->nruns != 1) return fail(GHOST_ERR_STATE, "batched contexts: one profile per run");
  Staging st(c);
  const void *du, *dv, *dw, *ds;
  GB_CHECK(st.map(u, c->cbytes, 1, &du));
  GB_CHECK(st.map(v, c->cbytes, 1, &dv));
  GB_CHECK(st.map(w, c->cbytes, 1, &dw));
  GB_CHECK(st.map(s, c->cbytes, 1, &ds));
  GB_CHECK(c->precision == GHOST_SINGLE ? havg_dev<float>(c, du, dv, dw, ds, (float)fo, (float)bv, itype, gsh)
                                        : havg_dev<double>(c, du, dv, dw, ds, fo, bv, itype, gsh));
  return st.finish();
}

int ghost_havgcomp(ghost_ctx *c, const void *u, const void *v, const void *w, const void *s, double fo, double bv,
                   int itype, double *gsh) {
  CTX_CHECK(c);
  if (!u || !v || !w || !s || !gsh) return fail(GHOST_ERR_ARG, "null argument");
  if (itype < 0 || itype > 10) return fail(GHOST_ERR_ARG, "itype %d not in 0..10", itype);
  return havg(c, u, v, w, s, fo, bv, itype, gsh);
}

// tbouss (pseudospec3D_bouss.f90:611-711): the z-average, maximum and
// minimum over z of each of the 11 havgcomp profiles
int ghost_tbouss(ghost_ctx *c, const void *u, const void *v, const void *w, const void *s, double fo, double bv,
                 double avg[11], double mx[11], double mn[11]) {
  CTX_CHECK(c);
  if (!u || !v || !w || !s || !avg || !mx || !mn) return fail(GHOST_ERR_ARG, "null argument");
  std::vector<double> gsh(c->nz);
  for (int q = 0; q < 11; ++q) {
    GB_CHECK(havg(c, u, v, w, s, fo, bv, q, gsh.data()));
    double sum = 0.0, hi = gsh[0], lo = gsh[0];
    for (int k = 0; k < c->nz; ++k) {
      sum += gsh[k];
      hi = std::max(hi, gsh[k]);
      lo = std::min(lo, gsh[k]);
    }
    avg[q] = sum / (double)c->nz;
    mx[q] = hi;
    mn[q] = lo;
  }
  return GHOST_OK;
}

// specpara / specperp (pseudospec3D_rot.f90:25-686): E[3 nb] and H[3 nb]
// (total, horizontal, vertical) for kin 0/1 and hel 1
static int aniso_spec(ghost_ctx *c, int mode, const void *a, const void *b, const void *cc, int kin, int hel,
                      double *Ek, double *Hk) {
  CTX_CHECK(c);
  if (!a || !b || !cc) return fail(GHOST_ERR_ARG, "null field");
  if (kin < 0 || kin > 2) return fail(GHOST_ERR_ARG, "kin %d not in 0..2", kin);
  if (kin <= 1 && !Ek) return fail(GHOST_ERR_ARG, "null Ek");
  if (hel == 1 && !Hk) return fail(GHOST_ERR_ARG, "null Hk");
  if (c->nruns != 1) return fail(GHOST_ERR_STATE, "batched contexts: one spectrum per run");
  const int nb = mode == 0 ? c->nz / 2 + 1 : c->nmaxperp / 2 + 1;
  Staging st(c);
  const void *da, *db, *dc;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  const bool sp = c->precision == GHOST_SINGLE;
  auto run = [&](int kind, double *o) {
    return sp ? aniso_dev<float>(c, kind, mode, nb, da, db, dc, nullptr, nullptr, nullptr, o)
              : aniso_dev<double>(c, kind, mode, nb, da, db, dc, nullptr, nullptr, nullptr, o);
  };
  if (kin <= 1) GB_CHECK(run(kin == 1 ? AN_KIN : AN_CURL, Ek));
  if (hel == 1) GB_CHECK(run(AN_HEL, Hk));
  return st.finish();
}

// entpara/entperp/heltpara/heltperp (pseudospec3D_rot.f90:689-1328): the
// transfer sums binned by |kz| (mode 0) or k_perp (mode 1); out[nb]
static int aniso_transfer(ghost_ctx *c, int mode, int kind, const void *a, const void *b, const void *cc,
                          const void *d, const void *e, const void *f, double *out) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !d || !e || !f || !out) return fail(GHOST_ERR_ARG, "null argument");
  if (c->nruns != 1) return fail(GHOST_ERR_STATE, "batched contexts: one spectrum per run");
  const int nb = mode == 0 ? c->nz / 2 + 1 : c->nmaxperp / 2 + 1;
  Staging st(c);
  const void *da, *db, *dc, *dd, *de, *df;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  GB_CHECK(st.map(d, c->cbytes, 1, &dd));
  GB_CHECK(st.map(e, c->cbytes, 1, &de));
  GB_CHECK(st.map(f, c->cbytes, 1, &df));
  std::vector<double> three((size_t)3 * nb);
  GB_CHECK(c->precision == GHOST_SINGLE ? aniso_dev<float>(c, kind, mode, nb, da, db, dc, dd, de, df, three.data())
                                        : aniso_dev<double>(c, kind, mode, nb, da, db, dc, dd, de, df, three.data()));
  for (int q = 0; q < nb; ++q) out[q] = three[q];
  return st.finish();
}

int ghost_specpara(ghost_ctx *c, const void *a, const void *b, const void *cc, int kin, int hel, double *Ek,
                   double *Hk) {
  return aniso_spec(c, 0, a, b, cc, kin, hel, Ek, Hk);
}
int ghost_specperp(ghost_ctx *c, const void *a, const void *b, const void *cc, int kin, int hel, double *Ek,
                   double *Hk) {
  return aniso_spec(c, 1, a, b, cc, kin, hel, Ek, Hk);
}
int ghost_entpara(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                  const void *f, int kin, double *Ek) {
  if (kin < 0 || kin > 4) return fail(GHOST_ERR_ARG, "kin %d not in 0..4", kin);
  return aniso_transfer(c, 0, kin == 0 ? RED_CROSS_K2 : RED_CROSS, a, b, cc, d, e, f, Ek);
}
int ghost_entperp(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                  const void *f, int kin, double *Ek) {
  if (kin < 0 || kin > 4) return fail(GHOST_ERR_ARG, "kin %d not in 0..4", kin);
  return aniso_transfer(c, 1, kin == 0 ? RED_CROSS_K2 : RED_CROSS, a, b, cc, d, e, f, Ek);
}
int ghost_heltpara(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                   const void *f, int kin, double *Hk) {
  if (kin < 0 || kin > 1) return fail(GHOST_ERR_ARG, "kin %d not in 0..1", kin);
  return aniso_transfer(c, 0, RED_CURL_CROSS, a, b, cc, d, e, f, Hk);
}
int ghost_heltperp(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, const void *e,
                   const void *f, int kin, double *Hk) {
  if (kin < 0 || kin > 1) return fail(GHOST_ERR_ARG, "kin %d not in 0..1", kin);
  return aniso_transfer(c, 1, RED_CURL_CROSS, a, b, cc, d, e, f, Hk);
}

int ghost_hdcheck(ghost_ctx *c, const void *vx, const void *vy, const void *vz, const void *fx, const void *fy,
                  const void *fz, int hel, int chk, double out[5]) {
  CTX_CHECK(c);
  if (!vx || !vy || !vz || !fx || !fy || !fz || !out) return fail(GHOST_ERR_ARG, "null argument");
  Staging st(c);
  const void *a, *b, *cc, *d, *e, *f;
  GB_CHECK(st.map(vx, c->cbytes, 1, &a));
  GB_CHECK(st.map(vy, c->cbytes, 1, &b));
  GB_CHECK(st.map(vz, c->cbytes, 1, &cc));
  GB_CHECK(st.map(fx, c->cbytes, 1, &d));
  GB_CHECK(st.map(fy, c->cbytes, 1, &e));
  GB_CHECK(st.map(fz, c->cbytes, 1, &f));
  const bool sp = c->precision == GHOST_SINGLE;
  auto red = [&](int kind, const void *p, const void *q, const void *r, double *o) {
    return sp ? reduce_dev<float>(c, kind, a, b, cc, p, q, r, o) : reduce_dev<double>(c, kind, a, b, cc, p, q, r, o);
  };
  for (int q = 0; q < 5; ++q) out[q] = 0.0;
  GB_CHECK(red(RED_ENERGY, nullptr, nullptr, nullptr, &out[0]));
  GB_CHECK(red(RED_ENSTROPHY, nullptr, nullptr, nullptr, &out[1]));
  if (hel == 1) GB_CHECK(red(RED_HELICITY, nullptr, nullptr, nullptr, &out[2]));
  GB_CHECK(red(RED_CROSS, d, e, f, &out[3]));
  if (chk == 1) GB_CHECK(red(RED_DIVERGENCE, nullptr, nullptr, nullptr, &out[4]));
  return st.finish();
}

int ghost_normalize(ghost_ctx *c, void *fx, void *fy, void *fz, double f0, int kin) {
  CTX_CHECK(c);
  if (!fx || !fy || !fz) return fail(GHOST_ERR_ARG, "null field");
  if (kin < 0 || kin > 2) return fail(GHOST_ERR_ARG, "kin %d not in 0..2", kin);
  Staging st(c);
  void *a, *b, *cc;
  GB_CHECK(st.map(fx, c->cbytes, 3, &a));
  GB_CHECK(st.map(fy, c->cbytes, 3, &b));
  GB_CHECK(st.map(fz, c->cbytes, 3, &cc));
  const int kind = kin == 1 ? RED_ENERGY : (kin == 0 ? RED_ENSTROPHY : RED_LAPLACIAN);
  double tmp;
  const bool sp = c->precision == GHOST_SINGLE;
  GB_CHECK(sp ? reduce_dev<float>(c, kind, a, b, cc, nullptr, nullptr, nullptr, &tmp)
              : reduce_dev<double>(c, kind, a, b, cc, nullptr, nullptr, nullptr, &tmp));
  GB_CHECK(GB_DISPATCH(c, scale3)(c, a, b, cc, f0, sqrt(tmp)));
  return st.finish();
}

int ghost_sharp(ghost_ctx *c, const void *a, void *b, double delta) {
  CTX_CHECK(c);
  if (!a || !b) return fail(GHOST_ERR_ARG, "null field");
  if (!(delta > 0)) return fail(GHOST_ERR_ARG, "delta must be positive");
  Staging st(c);
  const void *da;
  void *db;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 2, &db));
  GB_CHECK(GB_DISPATCH(c, sharp)(c, da, db, delta));
  return st.finish();
}

// ------------------------------------------------------------------- RK
int ghost_hd_rkstep1(ghost_ctx *c, const void *vx, const void *vy, const void *vz, void *C1, void *C2, void *C3) {
  CTX_CHECK(c);
  if (!vx || !vy || !vz || !C1 || !C2 || !C3) return fail(GHOST_ERR_ARG, "null field");
  Staging st(c);
  const void *in[3];
  void *out[3];
  const void *src[3] = {vx, vy, vz};
  void *dst[3] = {C1, C2, C3};
  for (int q = 0; q < 3; ++q) {
    GB_CHECK(st.map(src[q], c->cbytes, 1, &in[q]));
    GB_CHECK(st.map(dst[q], c->cbytes, 2, &out[q]));
    GB_CUDA(cudaMemcpyAsync(out[q], in[q], c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  return st.finish();
}

int ghost_hd_rkstep2(ghost_ctx *c, int o, double dt, double nu, void *vx, void *vy, void *vz, const void *C1,
                     const void *C2, const void *C3, const void *fx, const void *fy, const void *fz) {
  CTX_CHECK(c);
  if (!vx || !vy || !vz || !C1 || !C2 || !C3) return fail(GHOST_ERR_ARG, "null field");
  if (o < 1) return fail(GHOST_ERR_ARG, "substep o=%d must be >= 1", o);
  if ((fx == nullptr) != (fy == nullptr) || (fx == nullptr) != (fz == nullptr))
    return fail(GHOST_ERR_ARG, "forcing components must be all given or all null");
  Staging st(c);
  void *v[3];
  void *Cd[3];
  const void *f[3] = {nullptr, nullptr, nullptr};
  void *vu[3] = {vx, vy, vz};
  const void *Cu[3] = {C1, C2, C3};
  const void *fu[3] = {fx, fy, fz};
  for (int q = 0; q < 3; ++q) {
    GB_CHECK(st.map(vu[q], c->cbytes, 3, &v[q]));
    const void *t;
    GB_CHECK(st.map(Cu[q], c->cbytes, 1, &t));
    Cd[q] = (void *)t;
    if (fx) GB_CHECK(st.map(fu[q], c->cbytes, 1, &f[q]));
  }
  GB_CHECK(c->precision == GHOST_SINGLE ? hd_substep_dev<float>(c, o, dt, nu, v, Cd, fx ? f : nullptr, 0)
                                        : hd_substep_dev<double>(c, o, dt, nu, v, Cd, fx ? f : nullptr, 0));
  return st.finish();
}

// the live box of the truncation for host-array staging (none known:
// whole fields move)
static int staging_live_rows(ghost_ctx *c, Staging &st) {
  if (!c->prune_valid) GB_CHECK(c->precision == GHOST_SINGLE ? build_prune<float>(c) : build_prune<double>(c));
  if (c->prune_ok)
    st.set_live(c->prune_imax + 1, c->nxh, c->ny, c->prune_jtop, c->prune_jbot, c->nz, c->prune_ktop, c->prune_kbot,
                c->precision == GHOST_SINGLE ? 8 : 16);
  return GHOST_OK;
}

int ghost_hd_run(ghost_ctx *c, int nsteps, int ord, double dt, double nu, void *vx, void *vy, void *vz, void *C1,
                 void *C2, void *C3, const void *fx, const void *fy, const void *fz) {
  CTX_CHECK(c);
  if (!vx || !vy || !vz) return fail(GHOST_ERR_ARG, "null field");
  if (nsteps < 0 || ord < 1) return fail(GHOST_ERR_ARG, "nsteps=%d ord=%d", nsteps, ord);
  if ((fx == nullptr) != (fy == nullptr) || (fx == nullptr) != (fz == nullptr))
    return fail(GHOST_ERR_ARG, "forcing components must be all given or all null");
  if ((C1 == nullptr) != (C2 == nullptr) || (C1 == nullptr) != (C3 == nullptr))
    return fail(GHOST_ERR_ARG, "RK storage must be all given or all null");
  Staging st(c);
  // host arrays: the forcing is read only at kept modes and the run leaves v
  // zero outside them, so only their live kx rows need to cross the bus
  GB_CHECK(staging_live_rows(c, st));
  void *v[3], *Cd[3];
  const void *f[3] = {nullptr, nullptr, nullptr};
  void *vu[3] = {vx, vy, vz};
  void *Cu[3] = {C1, C2, C3};
  const void *fu[3] = {fx, fy, fz};
  for (int q = 0; q < 3; ++q) {
    GB_CHECK(st.map(vu[q], c->cbytes, Staging::IN | Staging::OUT | Staging::OUT_LIVE, &v[q]));
    if (fx) GB_CHECK(st.map(fu[q], c->cbytes, Staging::IN | Staging::IN_LIVE, &f[q]));
    if (C1) {
      GB_CHECK(st.map(Cu[q], c->cbytes, 3, &Cd[q]));
    } else {
      if (!c->rk[q]) GB_CHECK(dalloc(&c->rk[q], c->cbytes));
      Cd[q] = c->rk[q];
    }
  }
  GB_CHECK(st.resolve());  // every box is queued: the host scans v while they copy
  // The first substep of a call reads v on the whole grid (it may hold
  // modes outside the truncation); its update leaves v zero there, so the
  // later substeps skip the known zeros.
  for (int t = 0; t < nsteps; ++t)
    for (int o = ord; o >= 1; --o) {
      const bool prune = !(t == 0 && o == ord);
      GB_CHECK(c->precision == GHOST_SINGLE
                   ? hd_substep_dev<float>(c, o, dt, nu, v, Cd, fx ? f : nullptr, o == ord, prune)
                   : hd_substep_dev<double>(c, o, dt, nu, v, Cd, fx ? f : nullptr, o == ord, prune));
    }
  return st.finish();
}

// Tile variants tried by the autotuners (bit 0: y tiles 16 z-lines wide;
// bit 1: z CTAs of 128 threads; bits 1 and 2: two-stage z ring, three CTAs
// per SM; bit 3: two-stage y ring with a second exchange buffer; bit 4: y
// passes with 16 values per thread; bits 1, 2 and 5: one-stage z ring, four
// CTAs per SM, for lines of 256 points or more; bits 3, 4 and 6: the FP32 y
// inverse in tiles of 4 z-lines, four CTAs per SM).
static const int kTileCfgs[] = {0, 1, 2, 3, 6, 7, 8, 14, 16, 22, 24, 30, 38, 46, 62, 126};

// a variant with bit 5 runs the same kernels as without it on z lines
// shorter than 256 points, and one with bit 6 the same as without it on FP64
// or y lines shorter than 256 points: the autotuners skip those
static bool tile_cfg_distinct(const ghost_ctx *c, int cfg) {
  return (!(cfg & 32) || c->nz >= 256) && (!(cfg & 64) || (c->precision == GHOST_SINGLE && c->ny >= 256));
}

int ghost_ctx_set_tile_cfg(ghost_ctx *c, int cfg) {
  CTX_CHECK(c);
  if (cfg < 0 || cfg > 511) return fail(GHOST_ERR_ARG, "tile variant %d not in 0..511", cfg);
  c->tile_cfg = cfg;
  return GHOST_OK;
}

int ghost_ctx_get_tile_cfg(const ghost_ctx *c, int *cfg) {
  CTX_CHECK(c);
  if (!cfg) return fail(GHOST_ERR_ARG, "null output");
  *cfg = c->tile_cfg;
  return GHOST_OK;
}

int ghost_hd_autotune(ghost_ctx *c, int ord, double dt, double nu, const void *vx, const void *vy, const void *vz,
                      const void *fx, const void *fy, const void *fz, int *cfg_out) {
  CTX_CHECK(c);
  if (!vx || !vy || !vz || ord < 1) return fail(GHOST_ERR_ARG, "bad argument");
  if ((fx == nullptr) != (fy == nullptr) || (fx == nullptr) != (fz == nullptr))
    return fail(GHOST_ERR_ARG, "forcing components must be all given or all null");
  const void *vu[3] = {vx, vy, vz}, *fu[3] = {fx, fy, fz};
  for (int q = 0; q < 3; ++q)
    if (!is_device_ptr(vu[q]) || (fx && !is_device_ptr(fu[q])))
      return fail(GHOST_ERR_ARG, "ghost_hd_autotune takes device arrays");
  // time on a copy: the caller's v does not advance
  void *w[3] = {nullptr, nullptr, nullptr}, *Cd[3];
  int st = GHOST_OK;
  for (int q = 0; q < 3 && !st; ++q) st = dalloc(&w[q], c->cbytes);
  for (int q = 0; q < 3 && !st; ++q) {
    if (!c->rk[q]) st = dalloc(&c->rk[q], c->cbytes);
    Cd[q] = c->rk[q];
  }
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best = 1e30f;
  int best_cfg = c->tile_cfg;
  for (int cfg : kTileCfgs) {
    if (st) break;
    if (!tile_cfg_distinct(c, cfg)) continue;
    c->tile_cfg = cfg;
    float tot = 0.f;
    for (int rep = 0; rep < 3 && !st; ++rep) {
      for (int q = 0; q < 3; ++q) cudaMemcpyAsync(w[q], vu[q], c->cbytes, cudaMemcpyDeviceToDevice, c->stream);
      cudaEventRecord(a, c->stream);
      for (int o = ord; o >= 1 && !st; --o)
        st = c->precision == GHOST_SINGLE
                 ? hd_substep_dev<float>(c, o, dt, nu, w, Cd, fx ? fu : nullptr, o == ord, o != ord)
                 : hd_substep_dev<double>(c, o, dt, nu, w, Cd, fx ? fu : nullptr, o == ord, o != ord);
      cudaEventRecord(b, c->stream);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0) tot += ms;  // the first repetition warms up
    }
    if (!st && tot < best) {
      best = tot;
      best_cfg = cfg;
    }
  }
  c->tile_cfg = best_cfg;
  cudaStreamSynchronize(c->stream);
  for (void *p : w) cudaFree(p);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  GB_CHECK(st);
  if (cfg_out) *cfg_out = best_cfg;
  return check_status(c);
}

int ghost_init_random_solenoidal(ghost_ctx *c, int32_t *seed, double kdn, double kup, int shape, double amp, void *ox,
                                 void *oy, void *oz) {
  CTX_CHECK(c);
  if (!seed || !ox || !oy || !oz) return fail(GHOST_ERR_ARG, "null argument");
  if (shape != 0 && shape != 1) return fail(GHOST_ERR_ARG, "shape %d not in 0..1", shape);
  Staging st(c);
  void *a, *b, *cc;
  GB_CHECK(st.map(ox, c->cbytes, 2, &a));
  GB_CHECK(st.map(oy, c->cbytes, 2, &b));
  GB_CHECK(st.map(oz, c->cbytes, 2, &cc));
  GB_CHECK(c->precision == GHOST_SINGLE ? init_random_impl<float>(c, seed, kdn, kup, shape, amp, a, b, cc)
                                        : init_random_impl<double>(c, seed, kdn, kup, shape, amp, a, b, cc));
  return st.finish();
}

// ----------------------------------------------------------- Boussinesq
int ghost_advect3(ghost_ctx *c, const void *a, const void *b, const void *cc, const void *d, void *e) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !d || !e) return fail(GHOST_ERR_ARG, "null field");
  Staging st(c);
  const void *da, *db, *dc, *dd;
  void *de;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  GB_CHECK(st.map(d, c->cbytes, 1, &dd));
  GB_CHECK(st.map(e, c->cbytes, 2, &de));
  GB_CHECK(c->precision == GHOST_SINGLE ? advect3_dev<float>(c, da, db, dc, dd, de)
                                        : advect3_dev<double>(c, da, db, dc, dd, de));
  return st.finish();
}

static int bouss_args(ghost_ctx *c, Staging &st, void *vx, void *vy, void *vz, void *th, const void *fx,
                      const void *fy, const void *fz, const void *fs, void *v[4], const void *f[4], bool *have_f) {
  if (!vx || !vy || !vz || !th) return fail(GHOST_ERR_ARG, "null field");
  if ((fx == nullptr) != (fy == nullptr) || (fx == nullptr) != (fz == nullptr))
    return fail(GHOST_ERR_ARG, "forcing components must be all given or all null");
  void *vu[4] = {vx, vy, vz, th};
  const void *fu[4] = {fx, fy, fz, fs};
  *have_f = fx != nullptr || fs != nullptr;
  for (int q = 0; q < 4; ++q) {
    GB_CHECK(st.map(vu[q], c->cbytes, 3, &v[q]));
    GB_CHECK(st.map(fu[q], c->cbytes, 1, &f[q]));
  }
  return GHOST_OK;
}

int ghost_bouss_rkstep2(ghost_ctx *c, int o, double dt, double nu, double kappa, double omegaz, double xmom,
                        double xtemp, void *vx, void *vy, void *vz, void *th, const void *C1, const void *C2,
                        const void *C3, const void *C20, const void *fx, const void *fy, const void *fz,
                        const void *fs) {
  CTX_CHECK(c);
  if (o < 1) return fail(GHOST_ERR_ARG, "substep o=%d must be >= 1", o);
  if (!C1 || !C2 || !C3 || !C20) return fail(GHOST_ERR_ARG, "null RK storage");
  Staging st(c);
  void *v[4], *Cd[4];
  const void *f[4];
  bool have_f;
  GB_CHECK(bouss_args(c, st, vx, vy, vz, th, fx, fy, fz, fs, v, f, &have_f));
  const void *Cu[4] = {C1, C2, C3, C20};
  for (int q = 0; q < 4; ++q) {
    const void *t;
    GB_CHECK(st.map(Cu[q], c->cbytes, 1, &t));
    Cd[q] = (void *)t;
  }
  GB_CHECK(c->precision == GHOST_SINGLE
               ? bouss_substep_dev<float>(c, o, dt, nu, kappa, omegaz, xmom, xtemp, v, Cd, have_f ? f : nullptr, 0)
               : bouss_substep_dev<double>(c, o, dt, nu, kappa, omegaz, xmom, xtemp, v, Cd, have_f ? f : nullptr, 0));
  return st.finish();
}

// The passive-scalar solver (PHD_SOL, include/phd_rkstep1/2.f90): the
// rotating Boussinesq step without rotation, buoyancy or heat current is
// GHOST's PHD step term for term.
int ghost_phd_run(ghost_ctx *c, int nsteps, int ord, double dt, double nu, double kappa, void *vx, void *vy, void *vz,
                  void *th, const void *fx, const void *fy, const void *fz, const void *fs) {
  return ghost_bouss_run(c, nsteps, ord, dt, nu, kappa, 0.0, 0.0, 0.0, vx, vy, vz, th, fx, fy, fz, fs);
}

int ghost_bouss_run(ghost_ctx *c, int nsteps, int ord, double dt, double nu, double kappa, double omegaz,
                    double xmom, double xtemp, void *vx, void *vy, void *vz, void *th, const void *fx,
                    const void *fy, const void *fz, const void *fs) {
  CTX_CHECK(c);
  if (nsteps < 0 || ord < 1) return fail(GHOST_ERR_ARG, "nsteps=%d ord=%d", nsteps, ord);
  Staging st(c);
  void *v[4], *Cd[4];
  const void *f[4];
  bool have_f;
  GB_CHECK(bouss_args(c, st, vx, vy, vz, th, fx, fy, fz, fs, v, f, &have_f));
  for (int q = 0; q < 4; ++q) {
    if (!c->rk[q]) GB_CHECK(dalloc(&c->rk[q], c->cbytes));
    Cd[q] = c->rk[q];
  }
  for (int t = 0; t < nsteps; ++t)
    for (int o = ord; o >= 1; --o) {
      const bool prune = !(t == 0 && o == ord);
      GB_CHECK(c->precision == GHOST_SINGLE
                   ? bouss_substep_dev<float>(c, o, dt, nu, kappa, omegaz, xmom, xtemp, v, Cd, have_f ? f : nullptr,
                                              o == ord, prune)
                   : bouss_substep_dev<double>(c, o, dt, nu, kappa, omegaz, xmom, xtemp, v, Cd, have_f ? f : nullptr,
                                               o == ord, prune));
    }
  return st.finish();
}

}  // extern "C"

// ------------------------------------------------- no-allocation spectrum
// Partial sums of ghost_spectrumc_noalloc: nblk blocks write one
// histogram row of nbins each, then the final row follows them; nblk is
// chosen per call so that the (nblk + 1) rows fit the static array.  Every
// slot a call reads was written earlier by that same call, so nothing needs
// clearing between calls.
static_assert(2 * GHOST_SPECTRUM_NOALLOC_MAX_BINS <= GHOST_SPECTRUM_NOALLOC_DOUBLES,
              "static spectrum scratch too small for the advertised shell count");
static int noalloc_blocks(size_t n, int nbins) {
  const int fit = GHOST_SPECTRUM_NOALLOC_DOUBLES / nbins - 1;  // rows left after the final one
  return std::max(1, std::min(std::min(grid1d(n), 148 * 4), fit));
}
static __device__ __align__(256) double g_spectrum_scratch[GHOST_SPECTRUM_NOALLOC_DOUBLES];

static std::mutex g_spectrum_scratch_mu;
static void *g_spectrum_scratch_addr[128];

// Device address of the static array on the current device, looked up
// once per device (in host code the symbol is only a host-side stand-in).
// The cached address belongs to the device's primary context: after
// cudaDeviceReset the module reloads elsewhere, so a process that resets a
// device must not call ghost_spectrumc_noalloc on it again.
static int spectrum_scratch_address(int dev, double **out) {
  if (dev < 0 || dev >= 128) return fail(GHOST_ERR_STATE, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_spectrum_scratch_mu);
  if (!g_spectrum_scratch_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_spectrum_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return fail(GHOST_ERR_CUDA, "cudaGetSymbolAddress(spectrum scratch): %s", cudaGetErrorString(e));
    }
    g_spectrum_scratch_addr[dev] = p;
  }
  *out = (double *)g_spectrum_scratch_addr[dev];
  return GHOST_OK;
}

template <typename R>
static int spectrum_noalloc_dev(ghost_ctx *c, double *scratch, int kind, const void *a, const void *b, const void *cc,
                                double *out_host) {
  const int nbins = c->nmax / 2 + 1;
  // every run of a batched context, as ghost_spectrumc sums them
  const size_t n = c->ntot;
  const int nblk = noalloc_blocks(n, nbins);
  RedArgs<R> ra{(const cx<R> *)a, (const cx<R> *)b, (const cx<R> *)cc, nullptr, nullptr, nullptr};
  const size_t smem = (size_t)(256 / 32) * nbins * sizeof(double);
  GB_CUDA(cudaFuncSetAttribute(spectrum_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  spectrum_kernel<R><<<nblk, 256, smem, c->stream>>>(kparams<R>(c), ra, kind, n, nbins, (R)c->Dkk, (R)0.501f,
                                                     scratch);
  GB_CHECK(post_launch(c));
  double *fin = scratch + (size_t)nblk * nbins;
  finalize_kernel<<<1, 256, 0, c->stream>>>(scratch, nblk, nbins, fin);
  GB_CHECK(post_launch(c));
  GB_CUDA(cudaMemcpyAsync(out_host, fin, sizeof(double) * nbins, cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return GHOST_OK;
}

extern "C" {

int ghost_spectrumc_noalloc(ghost_ctx *c, const void *a, const void *b, const void *cc, int kin, int hel, double *Ek,
                            double *Hk) {
  CTX_CHECK(c);
  if (!a || !b || !cc) return fail(GHOST_ERR_ARG, "null field");
  if (kin < 0 || kin > 2) return fail(GHOST_ERR_ARG, "kin %d not in 0..2", kin);
  if (kin <= 1 && !Ek) return fail(GHOST_ERR_ARG, "null Ek");
  if (hel == 1 && !Hk) return fail(GHOST_ERR_ARG, "null Hk");
  if (!is_device_ptr(a) || !is_device_ptr(b) || !is_device_ptr(cc))
    return fail(GHOST_ERR_ARG, "ghost_spectrumc_noalloc needs device arrays (host arrays would need staging buffers)");
  const int nbins = c->nmax / 2 + 1;
  if (nbins > GHOST_SPECTRUM_NOALLOC_MAX_BINS)
    return fail(GHOST_ERR_SIZE, "%d spectral shells (nmax/2+1) exceed the static scratch limit of %d (nmax <= %d)",
                nbins, GHOST_SPECTRUM_NOALLOC_MAX_BINS, 2 * GHOST_SPECTRUM_NOALLOC_MAX_BINS - 1);
  int dev = -1;
  GB_CUDA(cudaGetDevice(&dev));
  if (dev != c->device) return fail(GHOST_ERR_STATE, "current device %d is not the context's device %d", dev, c->device);
  double *scratch = nullptr;
  GB_CHECK(spectrum_scratch_address(dev, &scratch));
  const bool sp = c->precision == GHOST_SINGLE;
  if (kin <= 1) {
    const int kind = kin == 1 ? RED_ENERGY : RED_ENSTROPHY;
    GB_CHECK(sp ? spectrum_noalloc_dev<float>(c, scratch, kind, a, b, cc, Ek)
                : spectrum_noalloc_dev<double>(c, scratch, kind, a, b, cc, Ek));
  }
  if (hel == 1)
    GB_CHECK(sp ? spectrum_noalloc_dev<float>(c, scratch, RED_HELICITY, a, b, cc, Hk)
                : spectrum_noalloc_dev<double>(c, scratch, RED_HELICITY, a, b, cc, Hk));
  return GHOST_OK;
}


// ------------------------------------------------------------- batches
int ghost_ctx_create_batch(int nx, int ny, int nz, int nruns, int precision, ghost_ctx **out) {
  if (nruns < 1) return fail(GHOST_ERR_ARG, "nruns=%d", nruns);
  GB_CHECK(ghost_ctx_create(nx, ny, nz, 1, 1, 1, 0, precision, out));
  ghost_ctx *c = *out;
  c->nruns = nruns;
  c->ntot = c->nspec * (size_t)nruns;
  c->cbytes = c->ntot * 2 * (c->precision == GHOST_SINGLE ? 4 : 8);
  refresh_kparams(c);
  return GHOST_OK;
}

int ghost_batch_set_nu(ghost_ctx *c, const double *nu) {
  CTX_CHECK(c);
  if (!nu) return fail(GHOST_ERR_ARG, "null nu");
  const size_t rs = c->precision == GHOST_SINGLE ? 4 : 8;
  if (!c->nu_run) GB_CHECK(dalloc(&c->nu_run, rs * c->nruns));
  std::vector<unsigned char> h(rs * c->nruns);
  for (int r = 0; r < c->nruns; ++r) {
    if (rs == 4) ((float *)h.data())[r] = (float)nu[r];
    else ((double *)h.data())[r] = nu[r];
  }
  GB_CUDA(cudaMemcpyAsync(c->nu_run, h.data(), h.size(), cudaMemcpyHostToDevice, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  refresh_kparams(c);
  return GHOST_OK;
}

int ghost_batch_energy(ghost_ctx *c, const void *a, const void *b, const void *cc, int kin, double *out) {
  CTX_CHECK(c);
  if (!a || !b || !cc || !out) return fail(GHOST_ERR_ARG, "null argument");
  if (kin < 0 || kin > 2) return fail(GHOST_ERR_ARG, "kin %d not in 0..2", kin);
  Staging st(c);
  const void *da, *db, *dc;
  GB_CHECK(st.map(a, c->cbytes, 1, &da));
  GB_CHECK(st.map(b, c->cbytes, 1, &db));
  GB_CHECK(st.map(cc, c->cbytes, 1, &dc));
  const int kind = kin == 1 ? RED_ENERGY : (kin == 0 ? RED_ENSTROPHY : RED_LAPLACIAN);
  GB_CHECK(c->precision == GHOST_SINGLE ? batch_reduce_dev<float>(c, kind, da, db, dc, out)
                                        : batch_reduce_dev<double>(c, kind, da, db, dc, out));
  return st.finish();
}

int ghost_batch_init_random_solenoidal(ghost_ctx *c, int32_t *seeds, double kdn, double kup, int shape, double amp,
                                       void *ox, void *oy, void *oz) {
  CTX_CHECK(c);
  if (!seeds || !ox || !oy || !oz) return fail(GHOST_ERR_ARG, "null argument");
  if (shape != 0 && shape != 1) return fail(GHOST_ERR_ARG, "shape %d not in 0..1", shape);
  Staging st(c);
  void *a, *b, *cc;
  GB_CHECK(st.map(ox, c->cbytes, 2, &a));
  GB_CHECK(st.map(oy, c->cbytes, 2, &b));
  GB_CHECK(st.map(oz, c->cbytes, 2, &cc));
  std::vector<int32_t> in(seeds, seeds + c->nruns);
  GB_CHECK(c->precision == GHOST_SINGLE
               ? batch_init_random_dev<float>(c, in.data(), seeds, kdn, kup, shape, amp, a, b, cc)
               : batch_init_random_dev<double>(c, in.data(), seeds, kdn, kup, shape, amp, a, b, cc));
  return st.finish();
}

}  // extern "C"

// ------------------------------------------------------------ ensembles
struct ghost_ensemble {
  int ncls = 0, precision = 0;
  // 1: each pass is one launch over every class (ensemble.cuh); 0: each
  // class runs its own launches on its own stream
  int multi = 0;
  int n[8] = {0}, nruns[8] = {0};
  ghost_ctx *cls[8] = {nullptr};
  void *v[8][3] = {{nullptr}};
  cudaStream_t main = nullptr, streams[8] = {nullptr};
  cudaEvent_t fork = nullptr, join[8] = {nullptr};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_ord = 0;
  double graph_dt = 0.0;
  bool stepped = false;  // one uncaptured step done: fields dealiased, tables and scratch built
};

namespace gb {
// one RK step (ord substeps, RK1 copy folded in) of one class on its stream
static int ensemble_class_step(ghost_ensemble *e, int q, int ord, double dt, bool prune_all) {
  ghost_ctx *c = e->cls[q];
  void *v[3] = {e->v[q][0], e->v[q][1], e->v[q][2]};
  for (int k = 0; k < 3; ++k)
    if (!c->rk[k]) GB_CHECK(dalloc(&c->rk[k], c->cbytes));
  void *C[3] = {c->rk[0], c->rk[1], c->rk[2]};
  for (int o = ord; o >= 1; --o) {
    const bool prune = prune_all || o != ord;
    GB_CHECK(c->precision == GHOST_SINGLE ? hd_substep_dev<float>(c, o, dt, 0.0, v, C, nullptr, o == ord, prune)
                                          : hd_substep_dev<double>(c, o, dt, 0.0, v, C, nullptr, o == ord, prune));
  }
  return GHOST_OK;
}

// ---- one launch per pass over all classes (ensemble.cuh)
// Persistent CTAs of a multi-class launch: per_sm CTAs on each SM; the SM
// slots are shared among the classes in proportion to their tiles (each
// class gets at least one).  Returns the grid, per_sm times the SM count.
template <class P> static int ens_split(ghost_ctx *c0, int per_sm, const long *tiles, P &p) {
  const int nsm = sm_count(c0), nc = p.ncls;
  long tot = 0;
  for (int q = 0; q < nc; ++q) tot += tiles[q];
  int sum = 0;
  for (int q = 0; q < nc; ++q) {
    p.nb[q] = std::max(1, (int)((double)nsm * (double)tiles[q] / (double)std::max<long>(1, tot)));
    sum += p.nb[q];
  }
  while (sum > nsm) {  // take slots from the class with the most
    int m = 0;
    for (int q = 1; q < nc; ++q)
      if (p.nb[q] > p.nb[m]) m = q;
    --p.nb[m];
    --sum;
  }
  while (sum < nsm) {  // give slots to the class with the most tiles per slot
    int m = 0;
    for (int q = 1; q < nc; ++q)
      if ((double)tiles[q] / p.nb[q] > (double)tiles[m] / p.nb[m]) m = q;
    ++p.nb[m];
    ++sum;
  }
  int start = 0;
  for (int q = 0; q < nc; ++q) {
    p.b0[q] = start;
    start += p.nb[q];
  }
  p.nsm = nsm;
  p.per = std::max(1, per_sm);
  return p.per * nsm;
}

template <typename R> static int ens_T(int N, int E) { return N / (E < N ? E : N); }

template <typename R, class Op>
static int ens_launch_z(ghost_ensemble *e, ZMulti<R, Op> &P, const long *tiles) {
  size_t smem = 0;
  for (int q = 0; q < P.ncls; ++q) {
    switch (P.n[q]) {
      case 16: smem = std::max(smem, ens_z_smem<R, 16, Op>(2)); break;
      case 32: smem = std::max(smem, ens_z_smem<R, 32, Op>(2)); break;
      case 64: smem = std::max(smem, ens_z_smem<R, 64, Op>(2)); break;
      case 128: smem = std::max(smem, ens_z_smem<R, 128, Op>(2)); break;
      default: return fail(GHOST_ERR_STATE, "no multi-class z pass for %d-point lines", P.n[q]);
    }
  }
  auto kern = zmulti_kernel<R, Op>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per = 0;
  GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kEnsThreads, smem));
  const int grid = ens_split(e->cls[0], per, tiles, P);
  kern<<<grid, kEnsThreads, smem, e->main>>>(P);
  return post_launch(e->cls[0]);
}

template <typename R, int S> static int ens_launch_y(ghost_ensemble *e, YMulti<R> &P, const long *tiles) {
  size_t smem = 0;
  for (int q = 0; q < P.ncls; ++q) {
    switch (P.n[q]) {
      case 16: smem = std::max(smem, ens_y_smem<R, 16>()); break;
      case 32: smem = std::max(smem, ens_y_smem<R, 32>()); break;
      case 64: smem = std::max(smem, ens_y_smem<R, 64>()); break;
      case 128: smem = std::max(smem, ens_y_smem<R, 128>()); break;
      default: return fail(GHOST_ERR_STATE, "no multi-class y pass for %d-point lines", P.n[q]);
    }
  }
  auto kern = ymulti_kernel<R, S>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per = 0;
  GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kEnsThreads, smem));
  const int grid = ens_split(e->cls[0], per, tiles, P);
  kern<<<grid, kEnsThreads, smem, e->main>>>(P);
  return post_launch(e->cls[0]);
}

template <typename R> static int ens_launch_x(ghost_ensemble *e, XMulti<R> &P, const long *tiles) {
  size_t smem = 0;
  for (int q = 0; q < P.ncls; ++q) {
    switch (P.n[q]) {
      case 16: smem = std::max(smem, ens_x_smem<R, 16>()); break;
      case 32: smem = std::max(smem, ens_x_smem<R, 32>()); break;
      case 64: smem = std::max(smem, ens_x_smem<R, 64>()); break;
      case 128: smem = std::max(smem, ens_x_smem<R, 128>()); break;
      default: return fail(GHOST_ERR_STATE, "no multi-class x pass for %d-point lines", P.n[q]);
    }
  }
  auto kern = xmulti_kernel<R>;
  GB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per = 0;
  GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kEnsThreads, smem));
  const int grid = ens_split(e->cls[0], per, tiles, P);
  kern<<<grid, kEnsThreads, smem, e->main>>>(P);
  return post_launch(e->cls[0]);
}

// x-pass tile parameters of a class (its own launch_x_fused would use the same)
template <typename R> static int ens_x_yb_of(int NX) {
  switch (NX) {
    case 16: return ens_x_yb<R, 16>();
    case 32: return ens_x_yb<R, 32>();
    case 64: return ens_x_yb<R, 64>();
    case 128: return ens_x_yb<R, 128>();
  }
  return 1;
}
static int ens_y_kb_of(int N) {
  switch (N) {
    case 16: return ens_y_kb<16>();
    case 32: return ens_y_kb<32>();
    case 64: return ens_y_kb<64>();
    case 128: return ens_y_kb<128>();
  }
  return 1;
}

// One substep (include/hd_rkstep2.f90, hd_rkstep1 folded in when copy) of
// every class: the five passes of hd_substep_dev, each one launch over all
// classes on the ensemble's main stream.
template <typename R> static int ens_substep_multi(ghost_ensemble *e, int o, double dt, int copy, bool prune) {
  const int nc = e->ncls;
  void *w[kEnsMaxCls][6];
  Prune pr[kEnsMaxCls];
  void *C[kEnsMaxCls][3];
  const unsigned U = sizeof(R) == 4 ? 1 : 2;
  for (int q = 0; q < nc; ++q) {
    ghost_ctx *c = e->cls[q];
    GB_CHECK(scratch(c, 6, w[q]));
    GB_CHECK(prune_plan<R>(c, prune, &pr[q]));
    for (int k = 0; k < 3; ++k) {
      if (!c->rk[k]) GB_CHECK(dalloc(&c->rk[k], c->cbytes));
      C[q][k] = c->rk[k];
    }
  }
  long tiles[kEnsMaxCls];
  // Z inverse
  {
    ZMulti<R, ZInv<R, 0>> P{};
    P.ncls = nc;
    for (int q = 0; q < nc; ++q) {
      ghost_ctx *c = e->cls[q];
      ZInv<R, 0> &zi = P.cl[q].op;
      for (int k = 0; k < 3; ++k) {
        zi.v.p[k] = (const cx<R> *)e->v[q][k];
        zi.cpy.p[k] = (cx<R> *)C[q][k];
      }
      for (int k = 0; k < 6; ++k) zi.w.p[k] = (cx<R> *)w[q][k];
      zi.kp = kparams<R>(c);
      zi.copy = copy;
      P.n[q] = c->nz;
      P.cl[q].tw = (const cx<R> *)c->tw_z;
      P.cl[q].lines = pr[q].lines;
      P.cl[q].nlines = pr[q].lines ? pr[q].nlines : c->ny * c->nxh * c->nruns;
      P.cl[q].ctl = pipe_ctl(c);
      const int lpb = kEnsThreads / ens_T<R>(c->nz, zE<R>());
      tiles[q] = (P.cl[q].nlines + lpb - 1) / lpb;
    }
    GB_CHECK((ens_launch_z<R, ZInv<R, 0>>(e, P, tiles)));
  }
  // Y inverse (6 fields) and, below, Y forward (3 fields)
  auto ypass = [&](auto sgn, int nf) -> int {
    constexpr int S = decltype(sgn)::value;
    YMulti<R> P{};
    P.ncls = nc;
    for (int q = 0; q < nc; ++q) {
      ghost_ctx *c = e->cls[q];
      YClass<R> &k = P.cl[q];
      const int N = c->ny, kb = ens_y_kb_of(N);
      k.rb = (pr[q].jpos && S > 0) ? std::min(32, N / 2) : std::min(N, 256);
      for (int f = 0; f < nf; ++f) {
        k.fld.p[f] = (cx<R> *)w[q][f];
        GB_CHECK(field_map(c, w[q][f], kEnsYBZ * U, k.rb, 1, &k.maps.m[f]));
      }
      k.tw = (const cx<R> *)c->tw_y;
      k.nz = c->nz;
      k.ni = pr[q].jpos ? pr[q].ni : c->nxh;
      k.nf = nf;
      k.nruns = c->nruns;
      k.nxh = c->nxh;
      k.jpos = pr[q].jpos;
      k.jneg = pr[q].jneg;
      k.ctl = pipe_ctl(c);
      P.n[q] = N;
      tiles[q] = (long)(c->nz / kEnsYBZ) * ((k.ni + kb - 1) / kb) * c->nruns * nf;
    }
    return ens_launch_y<R, S>(e, P, tiles);
  };
  GB_CHECK(ypass(std::integral_constant<int, +1>(), 6));
  // X: omega x v
  {
    XMulti<R> P{};
    P.ncls = nc;
    for (int q = 0; q < nc; ++q) {
      ghost_ctx *c = e->cls[q];
      XClass<R> &k = P.cl[q];
      const int M = c->nx / 2, yb = ens_x_yb_of<R>(c->nx), bz = ens_xBZ<R>();
      if (c->ny % yb != 0) return fail(GHOST_ERR_SIZE, "ny=%d not a multiple of the x tile's %d rows", c->ny, yb);
      const int nrows = pr[q].rows > 0 ? pr[q].rows : M + 1;
      const int nbox = (nrows + 255) / 256;
      const int align = std::max(1, 128 / (yb * bz * (int)sizeof(cx<R>)));
      const int rb = ((nrows + nbox - 1) / nbox + align - 1) / align * align;
      if (nbox * rb > M + 8 || rb > 256) return fail(GHOST_ERR_STATE, "x-pass box plan %d x %d exceeds the tile", nbox, rb);
      for (int f = 0; f < 6; ++f) GB_CHECK(field_map(c, w[q][f], bz * U, yb, rb, &k.maps.m[f]));
      for (int f = 0; f < 3; ++f) k.out.p[f] = (cx<R> *)w[q][f];
      const R nn = (R)c->nx * (R)c->ny * (R)c->nz_glob;
      k.scale = (R)1 / (nn * nn);
      k.tw = (const cx<R> *)c->tw_x;
      k.ny = c->ny;
      k.nz = c->nz;
      k.rows = nrows;
      k.nbox = nbox;
      k.rb = rb;
      k.nruns = c->nruns;
      k.nxh = c->nxh;
      k.ctl = pipe_ctl(c);
      P.n[q] = c->nx;
      tiles[q] = (long)(c->nz / bz) * (c->ny / yb) * c->nruns;
    }
    GB_CHECK(ens_launch_x<R>(e, P, tiles));
  }
  GB_CHECK(ypass(std::integral_constant<int, -1>(), 3));
  // Z forward: nonlhd3, laplak3 and the truncated update
  {
    ZMulti<R, ZFwdHD<R>> P{};
    P.ncls = nc;
    for (int q = 0; q < nc; ++q) {
      ghost_ctx *c = e->cls[q];
      ZFwdHD<R> &zf = P.cl[q].op;
      for (int k = 0; k < 3; ++k) {
        zf.nl.p[k] = (const cx<R> *)w[q][k];
        zf.v.p[k] = (cx<R> *)e->v[q][k];
        zf.c0.p[k] = (const cx<R> *)C[q][k];
        zf.f.p[k] = nullptr;
      }
      zf.kp = kparams<R>(c);
      zf.dt = (R)dt;
      zf.nu = (R)0;
      zf.rmp = (R)1 / (R)o;
      P.n[q] = c->nz;
      P.cl[q].tw = (const cx<R> *)c->tw_z;
      P.cl[q].lines = pr[q].lines;
      P.cl[q].nlines = pr[q].lines ? pr[q].nlines : c->ny * c->nxh * c->nruns;
      P.cl[q].ctl = pipe_ctl(c);
      const int lpb = kEnsThreads / ens_T<R>(c->nz, zE<R>());
      tiles[q] = (P.cl[q].nlines + lpb - 1) / lpb;
    }
    GB_CHECK((ens_launch_z<R, ZFwdHD<R>>(e, P, tiles)));
  }
  e->cls[0]->launches += 5;
  return GHOST_OK;
}

// The ensemble can run its passes as multi-class launches: at most
// kEnsMaxCls classes, cubic grids of 16..128 points per side.
static bool ens_multi_ok(const ghost_ensemble *e) {
  if (e->ncls > kEnsMaxCls) return false;
  for (int q = 0; q < e->ncls; ++q)
    if (e->n[q] < 16 || e->n[q] > 128) return false;
  return true;
}

// one RK step of every class in multi-class mode
static int ensemble_multi_step(ghost_ensemble *e, int ord, double dt, bool prune_all) {
  for (int o = ord; o >= 1; --o) {
    const bool prune = prune_all || o != ord;
    GB_CHECK(e->precision == GHOST_SINGLE ? ens_substep_multi<float>(e, o, dt, o == ord ? 1 : 0, prune)
                                          : ens_substep_multi<double>(e, o, dt, o == ord ? 1 : 0, prune));
  }
  return GHOST_OK;
}

static int ensemble_capture(ghost_ensemble *e, int ord, double dt) {
  if (e->exec) {
    cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
  }
  if (e->graph) {
    cudaGraphDestroy(e->graph);
    e->graph = nullptr;
  }
  GB_CUDA(cudaStreamBeginCapture(e->main, cudaStreamCaptureModeThreadLocal));
  int st = GHOST_OK;
  if (e->multi) {
    st = ensemble_multi_step(e, ord, dt, true);
  } else if (cudaEventRecord(e->fork, e->main) != cudaSuccess) {
    st = fail(GHOST_ERR_CUDA, "event record in capture");
  }
  for (int q = 0; q < e->ncls && st == GHOST_OK && !e->multi; ++q) {
    if (cudaStreamWaitEvent(e->streams[q], e->fork, 0) != cudaSuccess) {
      st = fail(GHOST_ERR_CUDA, "stream wait in capture");
      break;
    }
    st = ensemble_class_step(e, q, ord, dt, true);
    if (st == GHOST_OK && cudaEventRecord(e->join[q], e->streams[q]) != cudaSuccess)
      st = fail(GHOST_ERR_CUDA, "event record in capture");
    if (st == GHOST_OK && cudaStreamWaitEvent(e->main, e->join[q], 0) != cudaSuccess)
      st = fail(GHOST_ERR_CUDA, "join in capture");
  }
  cudaGraph_t g = nullptr;
  cudaError_t ce = cudaStreamEndCapture(e->main, &g);
  if (st != GHOST_OK) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return st;
  }
  if (ce != cudaSuccess || !g) {
    cudaGetLastError();
    return fail(GHOST_ERR_CUDA, "stream capture of the ensemble step failed: %s", cudaGetErrorString(ce));
  }
  e->graph = g;
  GB_CUDA(cudaGraphInstantiate(&e->exec, g, 0));
  e->graph_ord = ord;
  e->graph_dt = dt;
  return GHOST_OK;
}
}  // namespace gb

extern "C" {

int ghost_ensemble_create(int nclasses, const int *n, const int *nruns, int precision, ghost_ensemble **out) {
  if (!out || !n || !nruns) return fail(GHOST_ERR_ARG, "null argument");
  if (nclasses < 1 || nclasses > 8) return fail(GHOST_ERR_ARG, "nclasses=%d not in 1..8", nclasses);
  *out = nullptr;
  ghost_ensemble *e = new ghost_ensemble();
  e->ncls = nclasses;
  e->precision = precision;
  int st = GHOST_OK;
  if (cudaStreamCreateWithFlags(&e->main, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess)
    st = fail(GHOST_ERR_CUDA, "stream/event creation failed");
  for (int q = 0; q < nclasses && st == GHOST_OK; ++q) {
    e->n[q] = n[q];
    e->nruns[q] = nruns[q];
    st = ghost_ctx_create_batch(n[q], n[q], n[q], nruns[q], precision, &e->cls[q]);
    if (st != GHOST_OK) break;
    if (cudaStreamCreateWithFlags(&e->streams[q], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->join[q], cudaEventDisableTiming) != cudaSuccess) {
      st = fail(GHOST_ERR_CUDA, "stream/event creation failed");
      break;
    }
    e->cls[q]->stream = e->streams[q];
    for (int k = 0; k < 3 && st == GHOST_OK; ++k) {
      st = dalloc(&e->v[q][k], e->cls[q]->cbytes);
      if (st == GHOST_OK && cudaMemset(e->v[q][k], 0, e->cls[q]->cbytes) != cudaSuccess)
        st = fail(GHOST_ERR_CUDA, "memset failed");
    }
  }
  if (st != GHOST_OK) {
    ghost_ensemble_destroy(e);
    return st;
  }
  e->multi = 0;  // ghost_ensemble_autotune keeps the faster mode
  *out = e;
  return GHOST_OK;
}

int ghost_ensemble_set_mode(ghost_ensemble *e, int multi) {
  if (!e) return fail(GHOST_ERR_ARG, "null ensemble");
  if (multi != 0 && multi != 1) return fail(GHOST_ERR_ARG, "mode %d not 0 or 1", multi);
  if (multi && !ens_multi_ok(e))
    return fail(GHOST_ERR_ARG, "one launch per pass needs at most %d classes of 16..128 points per side", kEnsMaxCls);
  if (multi != e->multi && e->exec) {  // the captured step belongs to the other mode
    cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
  }
  e->multi = multi;
  return GHOST_OK;
}

int ghost_ensemble_get_mode(const ghost_ensemble *e, int *multi) {
  if (!e || !multi) return fail(GHOST_ERR_ARG, "null argument");
  *multi = e->multi;
  return GHOST_OK;
}

int ghost_ensemble_destroy(ghost_ensemble *e) {
  if (!e) return GHOST_OK;
  if (e->main) cudaStreamSynchronize(e->main);
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  for (int q = 0; q < e->ncls; ++q) {
    if (e->streams[q]) cudaStreamSynchronize(e->streams[q]);
    for (int k = 0; k < 3; ++k) cudaFree(e->v[q][k]);
    if (e->cls[q]) ghost_ctx_destroy(e->cls[q]);
    if (e->streams[q]) cudaStreamDestroy(e->streams[q]);
    if (e->join[q]) cudaEventDestroy(e->join[q]);
  }
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->main) cudaStreamDestroy(e->main);
  delete e;
  return GHOST_OK;
}

int ghost_ensemble_fields(ghost_ensemble *e, int q, void **vx, void **vy, void **vz) {
  if (!e || q < 0 || q >= e->ncls || !vx || !vy || !vz) return fail(GHOST_ERR_ARG, "bad argument");
  *vx = e->v[q][0];
  *vy = e->v[q][1];
  *vz = e->v[q][2];
  return GHOST_OK;
}

int ghost_ensemble_class(ghost_ensemble *e, int q, ghost_ctx **ctx) {
  if (!e || q < 0 || q >= e->ncls || !ctx) return fail(GHOST_ERR_ARG, "bad argument");
  *ctx = e->cls[q];
  return GHOST_OK;
}

int ghost_ensemble_init(ghost_ensemble *e, const int32_t *seeds, double kdn, double kup_frac, int shape, double amp,
                        const double *nu) {
  if (!e || !seeds || !nu) return fail(GHOST_ERR_ARG, "null argument");
  int off = 0;
  for (int q = 0; q < e->ncls; ++q) {
    std::vector<int32_t> s(seeds + off, seeds + off + e->nruns[q]);
    GB_CHECK(ghost_batch_init_random_solenoidal(e->cls[q], s.data(), kdn, kup_frac * e->n[q], shape, amp, e->v[q][0],
                                                e->v[q][1], e->v[q][2]));
    GB_CHECK(ghost_batch_set_nu(e->cls[q], nu + off));
    off += e->nruns[q];
  }
  e->stepped = false;
  return GHOST_OK;
}

// Times one step of every class in each mode (the classes' own launches on
// their streams, and one launch per pass over all classes) on a copy of the
// state and keeps the faster mode.
static int ensemble_pick_mode(ghost_ensemble *e, int ord, double dt) {
  void *save[kEnsMaxCls][3] = {};
  int st = GHOST_OK;
  for (int q = 0; q < e->ncls && st == GHOST_OK; ++q)
    for (int k = 0; k < 3 && st == GHOST_OK; ++k) {
      st = dalloc(&save[q][k], e->cls[q]->cbytes);
      if (st == GHOST_OK && cudaMemcpyAsync(save[q][k], e->v[q][k], e->cls[q]->cbytes, cudaMemcpyDeviceToDevice,
                                            e->main) != cudaSuccess)
        st = fail(GHOST_ERR_CUDA, "state copy failed");
    }
  auto restore = [&] {
    for (int q = 0; q < e->ncls; ++q)
      for (int k = 0; k < 3; ++k)
        if (save[q][k]) cudaMemcpyAsync(e->v[q][k], save[q][k], e->cls[q]->cbytes, cudaMemcpyDeviceToDevice, e->main);
  };
  cudaEvent_t a = nullptr, b = nullptr;
  if (st == GHOST_OK && (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess))
    st = fail(GHOST_ERR_CUDA, "event creation failed");
  float t[2] = {0.f, 0.f};
  for (int multi = 0; multi < 2 && st == GHOST_OK; ++multi) {
    for (int rep = 0; rep < 3 && st == GHOST_OK; ++rep) {
      restore();
      cudaEventRecord(a, e->main);
      if (multi) {
        st = ensemble_multi_step(e, ord, dt, true);
      } else {
        cudaEventRecord(e->fork, e->main);
        for (int q = 0; q < e->ncls && st == GHOST_OK; ++q) {
          cudaStreamWaitEvent(e->streams[q], e->fork, 0);
          st = ensemble_class_step(e, q, ord, dt, true);
          cudaEventRecord(e->join[q], e->streams[q]);
          cudaStreamWaitEvent(e->main, e->join[q], 0);
        }
      }
      cudaEventRecord(b, e->main);
      if (cudaEventSynchronize(b) != cudaSuccess) st = fail(GHOST_ERR_CUDA, "mode timing failed");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0) t[multi] += ms;  // the first repetition warms up
    }
  }
  restore();
  cudaStreamSynchronize(e->main);
  for (int q = 0; q < e->ncls; ++q)
    for (int k = 0; k < 3; ++k) cudaFree(save[q][k]);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  GB_CHECK(st);
  e->multi = t[1] < t[0] ? 1 : 0;
  for (int q = 0; q < e->ncls; ++q) GB_CHECK(check_status(e->cls[q]));
  return GHOST_OK;
}

int ghost_ensemble_autotune(ghost_ensemble *e, int ord, double dt, int *cfg_out) {
  if (!e || ord < 1) return fail(GHOST_ERR_ARG, "bad argument");
  for (int q = 0; q < e->ncls; ++q) {
    ghost_ctx *c = e->cls[q];
    // tune on a copy of the state: the ensemble itself does not advance
    void *save[3] = {nullptr, nullptr, nullptr};
    for (int k = 0; k < 3; ++k) {
      GB_CHECK(dalloc(&save[k], c->cbytes));
      GB_CUDA(cudaMemcpyAsync(save[k], e->v[q][k], c->cbytes, cudaMemcpyDeviceToDevice, c->stream));
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    int best_cfg = 0;
    int st = GHOST_OK;
    for (int cfg : kTileCfgs) {
      if (st != GHOST_OK) break;
      if (!tile_cfg_distinct(c, cfg)) continue;
      c->tile_cfg = cfg;
      float tot = 0.f;
      for (int rep = 0; rep < 3 && st == GHOST_OK; ++rep) {
        for (int k = 0; k < 3; ++k) cudaMemcpyAsync(e->v[q][k], save[k], c->cbytes, cudaMemcpyDeviceToDevice, c->stream);
        cudaEventRecord(a, c->stream);
        st = ensemble_class_step(e, q, ord, dt, false);
        cudaEventRecord(b, c->stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0) tot += ms;  // first repetition warms up
      }
      if (tot < best) {
        best = tot;
        best_cfg = cfg;
      }
    }
    c->tile_cfg = best_cfg;
    if (cfg_out) cfg_out[q] = best_cfg;
    for (int k = 0; k < 3; ++k) cudaMemcpyAsync(e->v[q][k], save[k], c->cbytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    for (int k = 0; k < 3; ++k) cudaFree(save[k]);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    GB_CHECK(st);
    GB_CHECK(check_status(c));
  }
  if (ens_multi_ok(e)) GB_CHECK(ensemble_pick_mode(e, ord, dt));
  if (e->exec) {  // a new tile choice needs a new graph
    cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
  }
  return GHOST_OK;
}

int ghost_ensemble_run(ghost_ensemble *e, int nsteps, int ord, double dt) {
  if (!e || nsteps < 0 || ord < 1) return fail(GHOST_ERR_ARG, "bad argument");
  int done = 0;
  if (!e->stepped && nsteps > 0) {
    // one uncaptured step: reads every mode once, builds tables and scratch
    if (e->multi) {
      GB_CHECK(ensemble_multi_step(e, ord, dt, false));
      GB_CUDA(cudaStreamSynchronize(e->main));
    } else {
      for (int q = 0; q < e->ncls; ++q) GB_CHECK(ensemble_class_step(e, q, ord, dt, false));
    }
    for (int q = 0; q < e->ncls; ++q) GB_CUDA(cudaStreamSynchronize(e->streams[q]));
    e->stepped = true;
    done = 1;
  }
  if (done < nsteps) {
    if (!e->exec || e->graph_ord != ord || e->graph_dt != dt) GB_CHECK(ensemble_capture(e, ord, dt));
    for (int q = 0; q < e->ncls; ++q) GB_CUDA(cudaStreamSynchronize(e->streams[q]));
    for (; done < nsteps; ++done) {
      GB_CUDA(cudaGraphLaunch(e->exec, e->main));
      if (e->multi)
        e->cls[0]->launches += 5LL * ord;
      else
        for (int q = 0; q < e->ncls; ++q) e->cls[q]->launches += 5LL * ord;
    }
    GB_CUDA(cudaStreamSynchronize(e->main));
  }
  for (int q = 0; q < e->ncls; ++q) GB_CHECK(check_status(e->cls[q]));
  return GHOST_OK;
}

int ghost_ensemble_energy(ghost_ensemble *e, int kin, double *out) {
  if (!e || !out) return fail(GHOST_ERR_ARG, "null argument");
  int off = 0;
  for (int q = 0; q < e->ncls; ++q) {
    GB_CHECK(ghost_batch_energy(e->cls[q], e->v[q][0], e->v[q][1], e->v[q][2], kin, out + off));
    off += e->nruns[q];
  }
  return GHOST_OK;
}

}  // extern "C"

// =====================================================================
// Slab decomposition of one run over ranks (GHOST's MPI layout).
//
// GHOST splits the spectral arrays into kx-slabs (rows ista..iend of
// 1..nx/2+1) and the real arrays into z-slabs (planes ksta..kend of 1..nz),
// both by range() (fftp-3/fftp.f90, main3D.fpp:634-635), and every 3D
// transform moves data between the two with one all-to-all
// (fftp-3/fftp3D.fpp:158-201, 255-278, 434-488).  Here a rank holds:
//   spec: a context over its kx-slab (nz, ny, nxh_loc), kx row i of a local
//         field being global row i + ista: the Z passes and the Y passes
//         of the HD substep run on it;
//   real: a context over its z-slab (nz_loc, ny, nxh): the fused X pass
//         runs on it, normalised by the global grid.
// One substep is front (Z inverse, Y inverse on 6 fields) -> pack ->
// all-to-all -> unpack -> X pass -> pack -> all-to-all -> unpack -> back
// (Y forward, Z forward and the truncated update).  The exchange itself
// belongs to the caller (NCCL all-to-all, or copies between ranks held by
// one process); the library packs and unpacks the blocks.
// Buffers are peer-major: the chunk for (or from) peer p holds the nf
// fields' blocks one after the other.
//   dir 0 (kx-slab -> z-slab): send to p: my rows x all ky x p's planes
//         (nxh_loc x ny x nz_p); receive from p: p's rows x ny x my planes,
//         which land as rows ista_p.. of the z-slab field.
//   dir 1 (z-slab -> kx-slab): the reverse.
// A pruned substep (every one after the first of a run, as in
// ghost_hd_run) runs the passes with the pruning tables of the rank's slab
// and moves only the kx rows below rows_glob, which hold every live mode.
// Slab contexts run the slab entry points only.
// =====================================================================
struct ghost_slab {
  ghost_ctx *spec = nullptr;
  ghost_ctx *real = nullptr;
  int rank = 0, nranks = 1;
  std::vector<int> ista, nxhl, ksta, nzl;  // per rank, 0-based starts
  int rows_glob = 0;  // kx rows 0..rows_glob-1 hold every mode that survives the truncation
  bool self_direct = false;  // pack/unpack skip the rank's own block (ghost_slab_exchange_self moves it)
  // kx rows of rank r that a pruned exchange moves: the live prefix of its slab
  int live_rows(int r, bool prune) const {
    return prune ? std::max(0, std::min(rows_glob - ista[r], nxhl[r])) : nxhl[r];
  }
};

namespace gb {

// range() of GHOST (fftp-3/fftp.f90), 1-based inclusive bounds
static void slab_range(int n1, int n2, int nprocs, int irank, int *ista, int *iend) {
  const int w1 = (n2 - n1 + 1) / nprocs, w2 = (n2 - n1 + 1) % nprocs;
  *ista = irank * w1 + n1 + std::min(irank, w2);
  *iend = *ista + w1 - 1;
  if (w2 > irank) *iend += 1;
}

static int slab_dev_ptrs(const void *const *p, int n) {
  if (!p) return fail(GHOST_ERR_ARG, "null field array");
  for (int q = 0; q < n; ++q) {
    if (!p[q]) return fail(GHOST_ERR_ARG, "null field %d", q);
    if (!is_device_ptr(p[q])) return fail(GHOST_ERR_ARG, "slab fields must be device arrays (field %d)", q);
    if (((uintptr_t)p[q] & 15u) != 0) return fail(GHOST_ERR_ARG, "field %d is not 16-byte aligned", q);
  }
  return GHOST_OK;
}

// kx rows holding a mode with kn2 <= kmax: row i's smallest kn2 is at ky = 0
// (the same rounding as the pruning tables and the kernels)
template <typename R> static int slab_rows_glob(const ghost_ctx *c) {
  const KParams<R> &kp = kparams<R>(c);
  int rows = 0;
  for (int i = 0; i < kp.nx / 2 + 1; ++i) {
    const R a = (R)(i < kp.nx / 2 ? i : i - kp.nx);
    volatile R aa = a * a, bb = (R)0;
    R k2;
    if (kp.anis) {
      volatile R x = kp.rmp * aa, y = kp.rmq * bb;
      volatile R t = x + y;
      k2 = t + (R)0;
    } else {
      volatile R t = aa + bb;
      k2 = t + (R)0;
    }
    if (!(k2 <= kp.kmax)) break;
    rows = i + 1;
  }
  return rows;
}

template <typename R>
static int slab_front_dev(ghost_ctx *c, const void *const v[3], void *const C[3], int copy, bool prune,
                          void *const w[6], bool with_y = true) {
  Prune pr;
  GB_CHECK(prune_plan<R>(c, prune, &pr));
  ZInv<R, 0> zi{};
  for (int q = 0; q < 3; ++q) {
    zi.v.p[q] = (const cx<R> *)v[q];
    zi.cpy.p[q] = copy ? (cx<R> *)C[q] : nullptr;
  }
  for (int q = 0; q < 6; ++q) zi.w.p[q] = (cx<R> *)w[q];
  zi.kp = kparams<R>(c);
  zi.copy = copy;
  GB_CHECK(launch_z<R>(c, zi, pr));
  if (!with_y) return GHOST_OK;
  Fields<R> fy{};
  for (int q = 0; q < 6; ++q) fy.p[q] = (cx<R> *)w[q];
  return launch_y<R, +1>(c, fy, 6, pr);
}

// the Y pass of nf fields of the kx-slab (sign +1 inverse, -1 forward)
template <typename R>
static int slab_y_dev(ghost_ctx *c, int sign, int nf, bool prune, void *const *w) {
  Prune pr;
  GB_CHECK(prune_plan<R>(c, prune, &pr));
  Fields<R> fy{};
  for (int q = 0; q < nf; ++q) fy.p[q] = (cx<R> *)w[q];
  return sign > 0 ? launch_y<R, +1>(c, fy, nf, pr) : launch_y<R, -1>(c, fy, nf, pr);
}

// Z forward and the truncated update (the back phase without its Y pass)
template <typename R>
static int slab_back_z_dev(ghost_ctx *c, int o, double dt, double nu, bool prune, void *const w[3], void *const v[3],
                           const void *const C[3], const void *const f[3]) {
  Prune pr;
  GB_CHECK(prune_plan<R>(c, prune, &pr));
  ZFwdHD<R> zf{};
  for (int q = 0; q < 3; ++q) {
    zf.nl.p[q] = (const cx<R> *)w[q];
    zf.v.p[q] = (cx<R> *)v[q];
    zf.c0.p[q] = (const cx<R> *)C[q];
    zf.f.p[q] = f ? (const cx<R> *)f[q] : nullptr;
  }
  zf.kp = kparams<R>(c);
  zf.dt = (R)dt;
  zf.nu = (R)nu;
  zf.rmp = (R)1 / (R)o;
  return launch_z<R>(c, zf, pr);
}

template <typename R>
static int slab_back_dev(ghost_ctx *c, int o, double dt, double nu, bool prune, void *const w[3], void *const v[3],
                         const void *const C[3], const void *const f[3]) {
  GB_CHECK(slab_y_dev<R>(c, -1, 3, prune, w));
  return slab_back_z_dev<R>(c, o, dt, nu, prune, w, v, C, f);
}

}  // namespace gb

#define SLAB_CHECK(s) \
  do {                \
    if (!(s)) return fail(GHOST_ERR_ARG, "null slab"); \
  } while (0)

extern "C" {

int ghost_slab_range(int n1, int n2, int nprocs, int irank, int *ista, int *iend) {
  if (!ista || !iend) return fail(GHOST_ERR_ARG, "null output");
  if (nprocs < 1 || irank < 0 || irank >= nprocs || n2 < n1)
    return fail(GHOST_ERR_ARG, "range(%d,%d,%d,%d)", n1, n2, nprocs, irank);
  slab_range(n1, n2, nprocs, irank, ista, iend);
  return GHOST_OK;
}

int ghost_slab_create(int nx, int ny, int nz, double Lx, double Ly, double Lz, int arbsize, int precision, int rank,
                      int nranks, ghost_slab **out) {
  if (!out) return fail(GHOST_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (nranks < 1 || rank < 0 || rank >= nranks) return fail(GHOST_ERR_ARG, "rank %d of %d", rank, nranks);
  if (!pow2_ok(nx) || !pow2_ok(ny) || !pow2_ok(nz))
    return fail(GHOST_ERR_SIZE, "grid %dx%dx%d: each n must be a power of two in [16,1024]", nx, ny, nz);
  const int nxh = nx / 2 + 1;
  if (nranks > nxh) return fail(GHOST_ERR_SIZE, "%d ranks for %d kx rows", nranks, nxh);
  ghost_slab *s = new ghost_slab();
  s->rank = rank;
  s->nranks = nranks;
  for (int r = 0; r < nranks; ++r) {
    int a, b, ka, kb;
    slab_range(1, nxh, nranks, r, &a, &b);
    slab_range(1, nz, nranks, r, &ka, &kb);
    s->ista.push_back(a - 1);
    s->nxhl.push_back(b - a + 1);
    s->ksta.push_back(ka - 1);
    s->nzl.push_back(kb - ka + 1);
    if ((kb - ka + 1) % 8 != 0) {
      delete s;
      return fail(GHOST_ERR_SIZE, "z-slab of %d planes on rank %d: every slab must hold a multiple of 8", kb - ka + 1, r);
    }
  }
  int st = ghost_ctx_create(nx, ny, nz, Lx, Ly, Lz, arbsize, precision, &s->spec);
  if (st == GHOST_OK) st = ghost_ctx_create(nx, ny, nz, Lx, Ly, Lz, arbsize, precision, &s->real);
  if (st != GHOST_OK) {
    ghost_ctx_destroy(s->spec);
    delete s;
    return st;
  }
  const size_t rs = precision == GHOST_SINGLE ? 4 : 8;
  ghost_ctx *c = s->spec;  // kx-slab: local rows, global kx through i0
  c->nxh = s->nxhl[rank];
  c->i0 = s->ista[rank];
  c->nspec = c->ntot = (size_t)nz * ny * c->nxh;
  c->cbytes = c->nspec * 2 * rs;
  refresh_kparams(c);
  s->rows_glob = precision == GHOST_SINGLE ? slab_rows_glob<float>(c) : slab_rows_glob<double>(c);
  c = s->real;  // z-slab: local planes, the x pass normalised by the global nz
  c->nz = s->nzl[rank];
  c->nspec = c->ntot = (size_t)c->nz * ny * nxh;
  c->cbytes = c->nspec * 2 * rs;
  c->nreal = (size_t)nx * ny * c->nz;
  c->rbytes = c->nreal * rs;
  refresh_kparams(c);
  *out = s;
  return GHOST_OK;
}

int ghost_slab_destroy(ghost_slab *s) {
  if (!s) return GHOST_OK;
  int a = ghost_ctx_destroy(s->spec), b = ghost_ctx_destroy(s->real);
  delete s;
  return a != GHOST_OK ? a : b;
}

int ghost_slab_layout(const ghost_slab *s, int *ista, int *nxh_loc, int *ksta, int *nz_loc) {
  SLAB_CHECK(s);
  for (int r = 0; r < s->nranks; ++r) {
    if (ista) ista[r] = s->ista[r];
    if (nxh_loc) nxh_loc[r] = s->nxhl[r];
    if (ksta) ksta[r] = s->ksta[r];
    if (nz_loc) nz_loc[r] = s->nzl[r];
  }
  return GHOST_OK;
}

int ghost_slab_rows(const ghost_slab *s, int *rows) {
  SLAB_CHECK(s);
  if (!rows) return fail(GHOST_ERR_ARG, "null output");
  *rows = s->rows_glob;
  return GHOST_OK;
}

int ghost_slab_launch_count(const ghost_slab *s, long long *count) {
  SLAB_CHECK(s);
  if (!count) return fail(GHOST_ERR_ARG, "null output");
  *count = s->spec->launches + (s->real != s->spec ? s->real->launches : 0);
  return GHOST_OK;
}

int ghost_slab_set_stream(ghost_slab *s, void *stream) {
  SLAB_CHECK(s);
  s->spec->stream = s->real->stream = (cudaStream_t)stream;
  return GHOST_OK;
}

int ghost_slab_synchronize(ghost_slab *s) {
  SLAB_CHECK(s);
  GB_CHECK(ghost_ctx_synchronize(s->spec));
  return ghost_ctx_synchronize(s->real);
}

int ghost_slab_hd_front(ghost_slab *s, const void *const v[3], void *const C[3], int copy, int prune,
                        void *const w[6]) {
  SLAB_CHECK(s);
  GB_CHECK(slab_dev_ptrs(v, 3));
  GB_CHECK(slab_dev_ptrs((const void *const *)w, 6));
  if (copy) GB_CHECK(slab_dev_ptrs((const void *const *)C, 3));
  ghost_ctx *c = s->spec;
  return c->precision == GHOST_SINGLE ? slab_front_dev<float>(c, v, C, copy, prune != 0, w)
                                      : slab_front_dev<double>(c, v, C, copy, prune != 0, w);
}

int ghost_slab_hd_xpass(ghost_slab *s, int prune, const void *const in[6], void *const out[3]) {
  SLAB_CHECK(s);
  GB_CHECK(slab_dev_ptrs(in, 6));
  GB_CHECK(slab_dev_ptrs((const void *const *)out, 3));
  ghost_ctx *c = s->real;
  const int rows = prune ? s->rows_glob : 0;  // a pruned substep reads and writes the live kx rows only
  if (prune && rows == 0) return GHOST_OK;
  return c->precision == GHOST_SINGLE ? launch_x<float, X_HD>(c, nullptr, nullptr, in, out, rows)
                                      : launch_x<double, X_HD>(c, nullptr, nullptr, in, out, rows);
}

int ghost_slab_hd_back(ghost_slab *s, int o, double dt, double nu, int prune, void *const w[3], void *const v[3],
                       const void *const C[3], const void *const f[3]) {
  SLAB_CHECK(s);
  if (o < 1) return fail(GHOST_ERR_ARG, "substep o=%d", o);
  GB_CHECK(slab_dev_ptrs((const void *const *)w, 3));
  GB_CHECK(slab_dev_ptrs((const void *const *)v, 3));
  GB_CHECK(slab_dev_ptrs(C, 3));
  if (f && !f[0]) f = nullptr;  // no forcing (a Fortran caller passes three null pointers)
  if (f) GB_CHECK(slab_dev_ptrs(f, 3));
  ghost_ctx *c = s->spec;
  return c->precision == GHOST_SINGLE ? slab_back_dev<float>(c, o, dt, nu, prune != 0, w, v, C, f)
                                      : slab_back_dev<double>(c, o, dt, nu, prune != 0, w, v, C, f);
}

int ghost_slab_pack(ghost_slab *s, int dir, int nf, int prune, const void *const *fields, void *send) {
  SLAB_CHECK(s);
  if ((dir != 0 && dir != 1) || nf < 1 || nf > 16 || !send) return fail(GHOST_ERR_ARG, "pack dir=%d nf=%d", dir, nf);
  GB_CHECK(slab_dev_ptrs(fields, nf));
  if (!is_device_ptr(send)) return fail(GHOST_ERR_ARG, "send buffer must be a device array");
  ghost_ctx *c = s->spec;
  const size_t es = c->precision == GHOST_SINGLE ? 8 : 16;
  const int me = s->rank, ny = c->ny, nz = c->nz_glob;
  const bool pr = prune != 0;
  unsigned char *dst = (unsigned char *)send;
  for (int p = 0; p < s->nranks; ++p)
    for (int f = 0; f < nf && !(s->self_direct && p == me); ++f) {
      const unsigned char *src = (const unsigned char *)fields[f];
      if (dir == 0) {  // my (live) kx rows, p's z planes, from a (nxh_loc, ny, nz) field
        const size_t w = (size_t)s->nzl[p] * es, h = (size_t)s->live_rows(me, pr) * ny;
        if (h > 0)
          GB_CUDA(cudaMemcpy2DAsync(dst, w, src + (size_t)s->ksta[p] * es, (size_t)nz * es, w, h,
                                    cudaMemcpyDeviceToDevice, c->stream));
        dst += w * h;
      } else {  // p's (live) kx rows of a (nxh, ny, nz_loc) field: contiguous
        const size_t n = (size_t)s->live_rows(p, pr) * ny * s->nzl[me] * es;
        if (n > 0)
          GB_CUDA(cudaMemcpyAsync(dst, src + (size_t)s->ista[p] * ny * s->nzl[me] * es, n, cudaMemcpyDeviceToDevice,
                                  c->stream));
        dst += n;
      }
    }
  return GHOST_OK;
}

int ghost_slab_unpack(ghost_slab *s, int dir, int nf, int prune, const void *recv, void *const *fields) {
  SLAB_CHECK(s);
  if ((dir != 0 && dir != 1) || nf < 1 || nf > 16 || !recv) return fail(GHOST_ERR_ARG, "unpack dir=%d nf=%d", dir, nf);
  GB_CHECK(slab_dev_ptrs((const void *const *)fields, nf));
  if (!is_device_ptr(recv)) return fail(GHOST_ERR_ARG, "receive buffer must be a device array");
  ghost_ctx *c = s->spec;
  const size_t es = c->precision == GHOST_SINGLE ? 8 : 16;
  const int me = s->rank, ny = c->ny, nz = c->nz_glob;
  const bool pr = prune != 0;
  const unsigned char *src = (const unsigned char *)recv;
  for (int p = 0; p < s->nranks; ++p)
    for (int f = 0; f < nf && !(s->self_direct && p == me); ++f) {
      unsigned char *dst = (unsigned char *)fields[f];
      if (dir == 0) {  // p's (live) kx rows of my z planes: rows ista_p.. of a (nxh, ny, nz_loc) field
        const size_t n = (size_t)s->live_rows(p, pr) * ny * s->nzl[me] * es;
        if (n > 0)
          GB_CUDA(cudaMemcpyAsync(dst + (size_t)s->ista[p] * ny * s->nzl[me] * es, src, n, cudaMemcpyDeviceToDevice,
                                  c->stream));
        src += n;
      } else {  // my (live) kx rows of p's z planes into a (nxh_loc, ny, nz) field
        const size_t w = (size_t)s->nzl[p] * es, h = (size_t)s->live_rows(me, pr) * ny;
        if (h > 0)
          GB_CUDA(cudaMemcpy2DAsync(dst + (size_t)s->ksta[p] * es, (size_t)nz * es, src, w, w, h,
                                    cudaMemcpyDeviceToDevice, c->stream));
        src += w * h;
      }
    }
  return GHOST_OK;
}

int ghost_slab_set_self_direct(ghost_slab *s, int on) {
  SLAB_CHECK(s);
  s->self_direct = on != 0;
  return GHOST_OK;
}

int ghost_slab_exchange_self(ghost_slab *s, int dir, int nf, int prune, const void *const *in, void *const *out) {
  SLAB_CHECK(s);
  if ((dir != 0 && dir != 1) || nf < 1 || nf > 16) return fail(GHOST_ERR_ARG, "exchange_self dir=%d nf=%d", dir, nf);
  GB_CHECK(slab_dev_ptrs(in, nf));
  GB_CHECK(slab_dev_ptrs((const void *const *)out, nf));
  ghost_ctx *c = s->spec;
  const size_t es = c->precision == GHOST_SINGLE ? 8 : 16;
  const int me = s->rank, ny = c->ny, nz = c->nz_glob;
  // my live kx rows of my z planes: (rows, ny, nz) at z offset ksta in the
  // kx-slab, (rows, ny, nz_loc) at row ista in the z-slab
  const size_t w = (size_t)s->nzl[me] * es, h = (size_t)s->live_rows(me, prune != 0) * ny;
  if (h == 0) return GHOST_OK;
  const size_t zoff = (size_t)s->ksta[me] * es, roff = (size_t)s->ista[me] * ny * w;
  for (int f = 0; f < nf; ++f) {
    const unsigned char *src = (const unsigned char *)in[f];
    unsigned char *dst = (unsigned char *)out[f];
    if (dir == 0)
      GB_CUDA(cudaMemcpy2DAsync(dst + roff, w, src + zoff, (size_t)nz * es, w, h, cudaMemcpyDeviceToDevice, c->stream));
    else
      GB_CUDA(cudaMemcpy2DAsync(dst + zoff, (size_t)nz * es, src + roff, w, w, h, cudaMemcpyDeviceToDevice, c->stream));
  }
  return GHOST_OK;
}

int ghost_slab_hd_front_z(ghost_slab *s, const void *const v[3], void *const C[3], int copy, int prune,
                          void *const w[6]) {
  SLAB_CHECK(s);
  GB_CHECK(slab_dev_ptrs(v, 3));
  GB_CHECK(slab_dev_ptrs((const void *const *)w, 6));
  if (copy) GB_CHECK(slab_dev_ptrs((const void *const *)C, 3));
  ghost_ctx *c = s->spec;
  return c->precision == GHOST_SINGLE ? slab_front_dev<float>(c, v, C, copy, prune != 0, w, false)
                                      : slab_front_dev<double>(c, v, C, copy, prune != 0, w, false);
}

int ghost_slab_ypass(ghost_slab *s, int sign, int nf, int prune, void *const *fields) {
  SLAB_CHECK(s);
  if ((sign != 1 && sign != -1) || nf < 1 || nf > 9) return fail(GHOST_ERR_ARG, "ypass sign=%d nf=%d", sign, nf);
  GB_CHECK(slab_dev_ptrs((const void *const *)fields, nf));
  ghost_ctx *c = s->spec;
  return c->precision == GHOST_SINGLE ? slab_y_dev<float>(c, sign, nf, prune != 0, fields)
                                      : slab_y_dev<double>(c, sign, nf, prune != 0, fields);
}

int ghost_slab_hd_back_z(ghost_slab *s, int o, double dt, double nu, int prune, void *const w[3], void *const v[3],
                         const void *const C[3], const void *const f[3]) {
  SLAB_CHECK(s);
  if (o < 1) return fail(GHOST_ERR_ARG, "substep o=%d", o);
  GB_CHECK(slab_dev_ptrs((const void *const *)w, 3));
  GB_CHECK(slab_dev_ptrs((const void *const *)v, 3));
  GB_CHECK(slab_dev_ptrs(C, 3));
  if (f && !f[0]) f = nullptr;
  if (f) GB_CHECK(slab_dev_ptrs(f, 3));
  ghost_ctx *c = s->spec;
  return c->precision == GHOST_SINGLE ? slab_back_z_dev<float>(c, o, dt, nu, prune != 0, w, v, C, f)
                                      : slab_back_z_dev<double>(c, o, dt, nu, prune != 0, w, v, C, f);
}

}  // extern "C"
