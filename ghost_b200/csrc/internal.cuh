// internal.cuh -- device-path entry points of api.cu shared with the other
// translation units of the library (les.cu).  Explicit instantiations for
// float and double live at the end of api.cu's gb namespace.
#pragma once
#include "common.cuh"

namespace gb {

int dalloc(void **p, size_t bytes);
// scratch spectral fields 0..n-1 of the context (each cbytes); the 3D
// transforms and substeps below use them, so callers keep their own
// buffers for anything that must survive a call
int scratch(ghost_ctx *c, int n, void **out);
int post_launch(ghost_ctx *c);
int check_status(ghost_ctx *c);
bool is_device_ptr(const void *p);
int grid1d(size_t n);

template <typename R> const KParams<R> &kparams(const ghost_ctx *c);
// unnormalised 3D transforms on device arrays (c2r keeps its input)
template <typename R> int r2c_dev(ghost_ctx *c, const void *in, void *out);
template <typename R> int c2r_dev(ghost_ctx *c, const void *in, void *out);
// the LES closure's input rows x[q][10] (gradients times gs, delta) of a
// spectral velocity, through spectral work fields spec[9]
template <typename R>
int grad9_features_dev(ghost_ctx *c, const void *const v[3], void *const spec[9], float *x, float gs, float delta);
// six real fields to spectra (x per field, one y and one z pass for all six)
template <typename R> int r2c6_dev(ghost_ctx *c, const void *const in[6], void *const out[6]);
// one fused HD substep (include/hd_rkstep2.f90; hd_rkstep1 folded in with copy)
template <typename R>
int hd_substep_dev(ghost_ctx *c, int o, double dt, double nu, void *const v[3], void *const C[3], const void *const f[3],
                   int copy, bool prune = false);
// reductions of ops.cuh (kind 0: <|v|^2>) into one host double
template <typename R>
int reduce_dev(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, const void *d, const void *e,
               const void *f, double *out_host);
// kinetic (kind 1) shell spectrum into out_host[nmax/2+1]
template <typename R>
int spectrum_dev(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, double *out_host);
// the same into a device array, without synchronising
template <typename R>
int spectrum_dev_async(ghost_ctx *c, int kind, const void *a, const void *b, const void *cc, double *out_dev);

}  // namespace gb

namespace gb {
template <> const KParams<float> &kparams<float>(const ghost_ctx *c);
template <> const KParams<double> &kparams<double>(const ghost_ctx *c);
}  // namespace gb
