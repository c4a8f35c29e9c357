// ensemble.cuh -- one launch per pass for every size class of an ensemble.
//
// An ensemble holds batched contexts of different grids (config 3: 128 runs
// of 32^3, 96 of 64^3, 32 of 128^3).  Each pass of the fused substep (Z
// inverse, Y inverse, X, Y forward, Z forward) runs as ONE kernel over all
// classes.  The launch has per CTAs for each of nsm SM slots; class c owns
// the slots [b0[c], b0[c] + nb[c]), and CTA b (slot b % nsm, round b / nsm)
// works for the class owning its slot, as CTA round nb[c] + slot - b0[c] of
// that class's per nb[c] persistent CTAs, with the class's own line length
// (a switch over the supported lengths picks the templated pass body).  The
// hardware fills the SMs slot by slot, round after round, so the CTAs
// resident on one SM tend to run one class's code: the instruction cache
// then holds one pass body per SM instead of several.  Every class runs the same CTA size, NTH threads:
//   Z pass: NTH / (N/E) lines of N points per tile;
//   Y pass: BZ z-lines of NTH / (BZ N/E) consecutive kx per tile;
//   X pass: BZ z-values of NTH / (BZ (N/2)/E) consecutive y per tile;
// so the arithmetic of a line is the one of the class's own launch.
#pragma once
#include "passes.cuh"

namespace gb {

constexpr int kEnsMaxCls = 4;   // classes one launch covers
constexpr int kEnsThreads = 128;  // CTA size of every class

template <typename R> constexpr int ens_zE() { return sizeof(R) == 4 ? 8 : 4; }
template <typename R> constexpr int ens_xE() { return sizeof(R) == 4 ? 8 : 4; }
template <typename R> constexpr int ens_xBZ() { return sizeof(R) == 4 ? 8 : 4; }
constexpr int kEnsYBZ = 8;
constexpr int kEnsXStages = 4;  // the X pass's ring: four fields in flight, as the classes' own launches

// the class a CTA works for, its index among that class's CTAs, and their number
struct EnsCta {
  int c, vb, nvb;
};
template <class P> __device__ __forceinline__ EnsCta ens_cta(const P &p) {
  const int slot = (int)blockIdx.x % p.nsm, round = (int)blockIdx.x / p.nsm;
  int c = 0;
  while (c + 1 < p.ncls && slot >= p.b0[c + 1]) ++c;
  return EnsCta{c, round * p.nb[c] + (slot - p.b0[c]), p.per * p.nb[c]};
}

// ------------------------------------------------------------------ Z
template <typename R, class Op> struct ZClass {
  Op op;
  const cx<R> *tw;
  const int *lines;
  int nlines;
  PipeCtl ctl;
};
template <typename R, class Op> struct ZMulti {
  int ncls, nsm, per;
  int n[kEnsMaxCls], b0[kEnsMaxCls], nb[kEnsMaxCls];
  ZClass<R, Op> cl[kEnsMaxCls];
};
template <typename R, int N, int NTH> constexpr int ens_z_lpb() { return NTH / (N / (ens_zE<R>() < N ? ens_zE<R>() : N)); }
template <typename R, int N, class Op> constexpr size_t ens_z_smem(int stages) {
  constexpr int E = ens_zE<R>() < N ? ens_zE<R>() : N;
  return ZGeom<R, N, E, ens_z_lpb<R, N, kEnsThreads>(), Op::NLOAD>::smem_bytes(stages);
}

template <typename R, int N, class Op> __device__ __forceinline__ void ens_z_run(const ZClass<R, Op> &k, int vb, int nvb) {
  constexpr int E = ens_zE<R>() < N ? ens_zE<R>() : N;
  zpipe_body<R, N, E, ens_z_lpb<R, N, kEnsThreads>(), 2>(vb, nvb, k.op, k.tw, k.lines, k.nlines, k.ctl);
}

template <typename R, class Op>
__global__ void __launch_bounds__(kEnsThreads) zmulti_kernel(const __grid_constant__ ZMulti<R, Op> P) {
  const EnsCta k = ens_cta(P);
  switch (P.n[k.c]) {
    case 16: ens_z_run<R, 16>(P.cl[k.c], k.vb, k.nvb); break;
    case 32: ens_z_run<R, 32>(P.cl[k.c], k.vb, k.nvb); break;
    case 64: ens_z_run<R, 64>(P.cl[k.c], k.vb, k.nvb); break;
    case 128: ens_z_run<R, 128>(P.cl[k.c], k.vb, k.nvb); break;
  }
}

// ------------------------------------------------------------------ Y
template <typename R> struct YClass {
  FieldMaps maps;
  Fields<R> fld;
  const cx<R> *tw;
  int nz, ni, nf, nruns, nxh, rb;
  const int *jpos, *jneg;
  PipeCtl ctl;
};
template <typename R> struct YMulti {
  int ncls, nsm, per;
  int n[kEnsMaxCls], b0[kEnsMaxCls], nb[kEnsMaxCls];
  YClass<R> cl[kEnsMaxCls];
};
template <int N> constexpr int ens_y_kb() {
  constexpr int E = N < 8 ? N : 8;
  return kEnsThreads / (kEnsYBZ * (N / E));
}
template <typename R, int N> constexpr size_t ens_y_smem() {
  constexpr int E = N < 8 ? N : 8;
  return YGeom<R, N, E, kEnsYBZ, false, ens_y_kb<N>()>::smem_bytes(3);
}

template <typename R, int N, int S> __device__ __forceinline__ void ens_y_run(const YClass<R> &k, int vb, int nvb) {
  constexpr int E = N < 8 ? N : 8;
  ypipe_body<R, N, E, kEnsYBZ, 3, S, false, ens_y_kb<N>()>(vb, nvb, k.maps, k.maps, k.fld, k.tw, k.nz, k.ni, k.nf,
                                                           k.nruns, k.nxh, k.jpos, k.jneg, k.rb, 0, k.ctl);
}

template <typename R, int S>
__global__ void __launch_bounds__(kEnsThreads) ymulti_kernel(const __grid_constant__ YMulti<R> P) {
  const EnsCta k = ens_cta(P);
  switch (P.n[k.c]) {
    case 16: ens_y_run<R, 16, S>(P.cl[k.c], k.vb, k.nvb); break;
    case 32: ens_y_run<R, 32, S>(P.cl[k.c], k.vb, k.nvb); break;
    case 64: ens_y_run<R, 64, S>(P.cl[k.c], k.vb, k.nvb); break;
    case 128: ens_y_run<R, 128, S>(P.cl[k.c], k.vb, k.nvb); break;
  }
}

// ------------------------------------------------------------------ X
template <typename R> struct XClass {
  FieldMaps maps;
  Fields<R> out;
  const cx<R> *tw;
  int ny, nz, rows, nbox, rb, nruns, nxh;
  R scale;
  PipeCtl ctl;
};
template <typename R> struct XMulti {
  int ncls, nsm, per;
  int n[kEnsMaxCls], b0[kEnsMaxCls], nb[kEnsMaxCls];
  XClass<R> cl[kEnsMaxCls];
};
template <typename R, int NX> constexpr int ens_x_E() { return ens_xE<R>() < NX / 2 ? ens_xE<R>() : NX / 2; }
template <typename R, int NX> constexpr int ens_x_yb() {
  return kEnsThreads / (ens_xBZ<R>() * (NX / 2 / ens_x_E<R, NX>()));
}
template <typename R, int NX> constexpr size_t ens_x_smem() {
  return XGeom<R, NX, ens_xBZ<R>(), ens_x_yb<R, NX>()>::smem_bytes(kEnsXStages);
}

template <typename R, int NX> __device__ __forceinline__ void ens_x_run(const XClass<R> &k, int vb, int nvb) {
  xpipe_nl_body<R, NX, ens_x_E<R, NX>(), ens_xBZ<R>(), 0, kEnsXStages, ens_x_yb<R, NX>()>(
      vb, nvb, k.maps, k.out, k.tw, k.ny, k.nz, k.scale, k.rows, k.nbox, k.rb, k.nruns, k.nxh, k.ctl);
}

template <typename R>
__global__ void __launch_bounds__(kEnsThreads) xmulti_kernel(const __grid_constant__ XMulti<R> P) {
  const EnsCta k = ens_cta(P);
  switch (P.n[k.c]) {
    case 16: ens_x_run<R, 16>(P.cl[k.c], k.vb, k.nvb); break;
    case 32: ens_x_run<R, 32>(P.cl[k.c], k.vb, k.nvb); break;
    case 64: ens_x_run<R, 64>(P.cl[k.c], k.vb, k.nvb); break;
    case 128: ens_x_run<R, 128>(P.cl[k.c], k.vb, k.nvb); break;
  }
}

}  // namespace gb
