// io.cu -- GHOST's binary field files (restart and output IO).
//
// GHOST stores every field as one raw binary file <dir>/<name>.NNNN.out
// (mpiio/binary_io.f90:13-186, names from main3D.fpp:2678 with
// fmtext = '(i4.4)', pseudo/pseudospec3D_mod.fpp:40): the real array
// r(nx,ny,nz) in Fortran order (x fastest), GP precision, native byte
// order, no header (disp = 0).  Each MPI rank writes its z-slab through a
// subarray view, so the file is the whole array in that order whatever the
// rank count.  Restart reads may byte-swap (iswap, gutils_mod.fpp:114-151).
//
//   ghost_io_write / ghost_io_read       io_write / io_read of a real field
//   ghost_io_output                      one field of the output step
//                                        (main3D.fpp:2678-2709): the real
//                                        field of v/(nx ny nz), then io_write
//   ghost_io_restart                     one field of the restart
//                                        (main3D.fpp:2155-2161): io_read,
//                                        then fftp3d_real_to_complex
// Field pointers may be device or host memory.  The transforms run on the
// device; the files go through host memory.
#include <stdio.h>
#include <string.h>

#include <vector>

#include "../../include/ghost_b200.h"
#include "common.cuh"
#include "internal.cuh"

namespace gb {

template <typename R> __global__ void io_scale_kernel(cx<R> *x, size_t n, R s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = mk(x[i].x * s, x[i].y * s);
}

static void byte_swap(unsigned char *p, size_t nvals, size_t es) {
  for (size_t q = 0; q < nvals; ++q, p += es)
    for (size_t a = 0, b = es - 1; a < b; ++a, --b) {
      const unsigned char t = p[a];
      p[a] = p[b];
      p[b] = t;
    }
}

static size_t real_bytes(const ghost_ctx *c) { return c->rbytes; }
static size_t elem_bytes(const ghost_ctx *c) { return c->precision == GHOST_SINGLE ? 4 : 8; }

// write nbytes of host memory (byte-swapped when swap) to path
static int write_file(const char *path, const void *host, size_t nbytes, size_t es, int swap) {
  std::vector<unsigned char> tmp;
  const unsigned char *src = (const unsigned char *)host;
  if (swap) {
    tmp.assign(src, src + nbytes);
    byte_swap(tmp.data(), nbytes / es, es);
    src = tmp.data();
  }
  FILE *fh = fopen(path, "wb");
  if (!fh) return fail(GHOST_ERR_IO, "io_write: cannot open %s for writing", path);
  const size_t w = fwrite(src, 1, nbytes, fh);
  const int cl = fclose(fh);
  if (w != nbytes || cl != 0) return fail(GHOST_ERR_IO, "io_write: short write to %s", path);
  return GHOST_OK;
}

// read exactly nbytes from path into host memory (byte-swapped when swap)
static int read_file(const char *path, void *host, size_t nbytes, size_t es, int swap) {
  FILE *fh = fopen(path, "rb");
  if (!fh) return fail(GHOST_ERR_IO, "io_read: cannot open %s for reading", path);
  if (fseek(fh, 0, SEEK_END) != 0) {
    fclose(fh);
    return fail(GHOST_ERR_IO, "io_read: cannot seek in %s", path);
  }
  const long sz = ftell(fh);
  rewind(fh);
  if (sz < 0 || (size_t)sz != nbytes) {
    fclose(fh);
    return fail(GHOST_ERR_SIZE, "io_read: %s holds %ld bytes, the grid needs %zu", path, sz, nbytes);
  }
  const size_t r = fread(host, 1, nbytes, fh);
  fclose(fh);
  if (r != nbytes) return fail(GHOST_ERR_IO, "io_read: short read from %s", path);
  if (swap) byte_swap((unsigned char *)host, nbytes / es, es);
  return GHOST_OK;
}

static int aligned_dev(const void *p) {
  if (((uintptr_t)p & 15u) != 0) return fail(GHOST_ERR_ARG, "device array %p is not 16-byte aligned", p);
  return GHOST_OK;
}

template <typename R> static int output_dev(ghost_ctx *c, const void *spec, const char *path, int swap) {
  // w[0] is used by the transform itself; w[1] holds v/(nx ny nz), w[2] the real field
  void *w[3];
  GB_CHECK(scratch(c, 3, w));
  const bool dev = is_device_ptr(spec);
  if (dev) GB_CHECK(aligned_dev(spec));
  GB_CUDA(cudaMemcpyAsync(w[1], spec, c->cbytes, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
  // rmp = 1/(nx ny nz) in GP (main3D.fpp:2680-2681)
  const R rmp = (R)1 / ((R)c->nx * (R)c->ny * (R)c->nz);
  io_scale_kernel<R><<<grid1d(c->nspec), 256, 0, c->stream>>>((cx<R> *)w[1], c->nspec, rmp);
  GB_CHECK(post_launch(c));
  GB_CHECK(c2r_dev<R>(c, w[1], w[2]));
  std::vector<unsigned char> host(real_bytes(c));
  GB_CUDA(cudaMemcpyAsync(host.data(), w[2], real_bytes(c), cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  GB_CHECK(check_status(c));
  return write_file(path, host.data(), real_bytes(c), elem_bytes(c), swap);
}

template <typename R> static int restart_dev(ghost_ctx *c, const char *path, int swap, void *spec) {
  void *w[3];
  GB_CHECK(scratch(c, 3, w));
  std::vector<unsigned char> host(real_bytes(c));
  GB_CHECK(read_file(path, host.data(), real_bytes(c), elem_bytes(c), swap));
  GB_CUDA(cudaMemcpyAsync(w[1], host.data(), real_bytes(c), cudaMemcpyHostToDevice, c->stream));
  const bool dev = is_device_ptr(spec);
  if (dev) GB_CHECK(aligned_dev(spec));
  void *out = dev ? spec : w[2];
  GB_CHECK(r2c_dev<R>(c, w[1], out));
  if (!dev) GB_CUDA(cudaMemcpyAsync(spec, out, c->cbytes, cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return check_status(c);
}

}  // namespace gb

using namespace gb;

#define IO_CHECK(c, p)                                                       \
  do {                                                                       \
    if (!(c)) return fail(GHOST_ERR_ARG, "null context");                    \
    if (!(p)) return fail(GHOST_ERR_ARG, "null path");                       \
    if ((c)->nruns != 1) return fail(GHOST_ERR_STATE, "batched contexts hold several runs: one file per run"); \
  } while (0)

extern "C" {

int ghost_io_filename(const char *dir, const char *name, int index, int width, char *buf, size_t len) {
  if (!dir || !name || !buf) return fail(GHOST_ERR_ARG, "null argument");
  if (index < 0 || width < 1 || width > 18) return fail(GHOST_ERR_ARG, "index %d / width %d", index, width);
  // Fortran (iW.W): zero-padded to W digits; a wider number prints as W asterisks
  char num[32];
  long long lim = 1;
  for (int q = 0; q < width; ++q) lim *= 10;
  if (index >= lim)
    memset(num, '*', (size_t)width), num[width] = 0;
  else
    snprintf(num, sizeof num, "%0*d", width, index);
  const int n = snprintf(buf, len, "%s/%s.%s.out", dir, name, num);
  if (n < 0 || (size_t)n >= len) return fail(GHOST_ERR_ARG, "file name needs %d bytes", n + 1);
  return GHOST_OK;
}

int ghost_io_write(ghost_ctx *c, const void *real, const char *path, int swap) {
  IO_CHECK(c, path);
  if (!real) return fail(GHOST_ERR_ARG, "null field");
  const size_t nb = real_bytes(c);
  if (!is_device_ptr(real)) return write_file(path, real, nb, elem_bytes(c), swap);
  std::vector<unsigned char> host(nb);
  GB_CUDA(cudaMemcpyAsync(host.data(), real, nb, cudaMemcpyDeviceToHost, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return write_file(path, host.data(), nb, elem_bytes(c), swap);
}

int ghost_io_read(ghost_ctx *c, const char *path, int swap, void *real) {
  IO_CHECK(c, path);
  if (!real) return fail(GHOST_ERR_ARG, "null field");
  const size_t nb = real_bytes(c);
  if (!is_device_ptr(real)) return read_file(path, real, nb, elem_bytes(c), swap);
  std::vector<unsigned char> host(nb);
  GB_CHECK(read_file(path, host.data(), nb, elem_bytes(c), swap));
  GB_CUDA(cudaMemcpyAsync(real, host.data(), nb, cudaMemcpyHostToDevice, c->stream));
  GB_CUDA(cudaStreamSynchronize(c->stream));
  return GHOST_OK;
}

int ghost_io_output(ghost_ctx *c, const void *spec, const char *path, int swap) {
  IO_CHECK(c, path);
  if (!spec) return fail(GHOST_ERR_ARG, "null field");
  return c->precision == GHOST_SINGLE ? output_dev<float>(c, spec, path, swap) : output_dev<double>(c, spec, path, swap);
}

int ghost_io_restart(ghost_ctx *c, const char *path, int swap, void *spec) {
  IO_CHECK(c, path);
  if (!spec) return fail(GHOST_ERR_ARG, "null field");
  return c->precision == GHOST_SINGLE ? restart_dev<float>(c, path, swap, spec) : restart_dev<double>(c, path, swap, spec);
}

}  // extern "C"
