// fft_core.cuh -- register-resident Stockham FFT stages for one line.
//
// A line of N complex values is held by T = N/E threads, E values each:
// thread t owns elements t + T*e (e = 0..E-1).  Every stage of radix R
// (R = E, or the remainder 2/4 for the last stage) reads that pattern,
// applies twiddles, does R-point DFTs in registers and writes either to
// the shared-memory exchange buffer (intermediate stages) or straight back
// into the same register pattern (last stage).  So the first stage can be
// fed directly from coalesced global loads and the last stage stores
// directly with the same pattern: a transform costs (#stages - 1) shared
// memory exchanges and nothing else.
//
// Stage with span L (product of the previous radices), butterfly b in
// [0, N/R): inputs b + m*N/R, twiddle W^(k*m*N/(L*R)) with k = b mod L,
// outputs (b/L)*L*R + k + r*L  (Stockham autosort; no bit reversal).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {

template <typename R> struct cx_of;
template <> struct cx_of<float> { using type = float2; };
template <> struct cx_of<double> { using type = double2; };
template <typename R> using cx = typename cx_of<R>::type;

__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
// a * (S*i), S = +-1
template <int S, typename C> __device__ __forceinline__ C mul_si(C a) {
  return S > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
// tw holds forward twiddles exp(-2 pi i e/N); sign +1 uses their conjugate
template <int S, typename C> __device__ __forceinline__ C twmul(C a, C w) {
  return S < 0 ? cmul(a, w) : cmulc(a, w);
}

template <typename C> struct rsqrt2_of;
template <> struct rsqrt2_of<float2> { static __device__ __forceinline__ float v() { return 0.70710678118654752440f; } };
template <> struct rsqrt2_of<double2> { static __device__ __forceinline__ double v() { return 0.70710678118654752440; } };

// In-register DFTs, y_r = sum_m x_m exp(S 2 pi i m r / R), in place.
template <int S, typename C> __device__ __forceinline__ void dft2(C &a, C &b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}
template <int S, typename C> __device__ __forceinline__ void dft4(C &x0, C &x1, C &x2, C &x3) {
  C a0 = cadd(x0, x2), a1 = csub(x0, x2);
  C b0 = cadd(x1, x3), b1 = mul_si<S>(csub(x1, x3));
  x0 = cadd(a0, b0);
  x2 = csub(a0, b0);
  x1 = cadd(a1, b1);
  x3 = csub(a1, b1);
}
template <int S, typename C> __device__ __forceinline__ void dft8(C (&v)[8]) {
  // split into pairs (m, m+4), then 4-point DFTs of the sums and of the
  // differences twiddled by W8^m
  C u0 = cadd(v[0], v[4]), d0 = csub(v[0], v[4]);
  C u1 = cadd(v[1], v[5]), d1 = csub(v[1], v[5]);
  C u2 = cadd(v[2], v[6]), d2 = csub(v[2], v[6]);
  C u3 = cadd(v[3], v[7]), d3 = csub(v[3], v[7]);
  const auto h = rsqrt2_of<C>::v();
  // W8^1 = h (1 + S i), W8^2 = S i, W8^3 = h (-1 + S i)
  C e1 = S > 0 ? mk(h * (d1.x - d1.y), h * (d1.x + d1.y)) : mk(h * (d1.x + d1.y), h * (d1.y - d1.x));
  C e2 = mul_si<S>(d2);
  C e3 = S > 0 ? mk(-h * (d3.x + d3.y), h * (d3.x - d3.y)) : mk(h * (d3.y - d3.x), -h * (d3.x + d3.y));
  dft4<S>(u0, u1, u2, u3);
  dft4<S>(d0, e1, e2, e3);
  v[0] = u0; v[2] = u1; v[4] = u2; v[6] = u3;
  v[1] = d0; v[3] = e1; v[5] = e2; v[7] = e3;
}

template <int R, int S, typename C> __device__ __forceinline__ void dftR(C (&v)[R]) {
  if constexpr (R == 2) {
    dft2<S>(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4<S>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft8<S>(v);
  } else {
    static_assert(R == 2 || R == 4 || R == 8, "radix");
  }
}

// radix of the stage with span L for an N-point transform, E per thread:
// E (at most 8, the largest in-register DFT; with E = 16 a thread runs two
// radix-8 butterflies per stage), or the remainder 2/4 for the last stage
template <int N, int E, int L> struct stage_radix {
  static constexpr int rem = N / L;
  static constexpr int RM = E < 8 ? E : 8;
  static constexpr int value = (rem % RM == 0) ? RM : rem;
};

// Butterflies of one stage.  Writes outputs to `dst(idx, val)` unless this
// is the last stage, in which case they go back into x.
template <typename C, int N, int E, int L, int S, int TWS, class Dst>
__device__ __forceinline__ void fft_stage(C (&x)[E], int t, const C *__restrict__ tw, Dst dst) {
  constexpr int T = N / E;
  constexpr int R = stage_radix<N, E, L>::value;
  constexpr int NB = E / R;
  constexpr bool LAST = (L * R == N);
  C y[E];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int b = t + q * T;
    const int k = b & (L - 1);
    C v[R];
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = x[q + m * NB];
    if constexpr (L > 1) {
      if constexpr (sizeof(C) == 8 && R >= 4) {
        // FP32: one table load, the other powers by products of depth <= 3
        // (shared-memory loads, not FMAs, limit these kernels)
        C w[R];
        w[1] = tw[(k * (N / (L * R))) * TWS];
        w[2] = cmul(w[1], w[1]);
        w[3] = cmul(w[2], w[1]);
        if constexpr (R == 8) {
          w[4] = cmul(w[2], w[2]);
          w[5] = cmul(w[4], w[1]);
          w[6] = cmul(w[4], w[2]);
          w[7] = cmul(w[4], w[3]);
        }
#pragma unroll
        for (int m = 1; m < R; ++m) v[m] = twmul<S>(v[m], w[m]);
      } else {
#pragma unroll
        for (int m = 1; m < R; ++m) v[m] = twmul<S>(v[m], tw[(k * m * (N / (L * R))) * TWS]);
      }
    }
    dftR<R, S>(v);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; ++r) y[q + r * NB] = v[r];
    } else {
      const int base = (b / L) * L * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) dst(base + r * L, v[r]);
    }
  }
  if constexpr (LAST) {
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = y[e];
  }
}

// number of shared-memory exchanges of an N-point transform, E per thread
template <int N, int E, int L = 1> constexpr int fft_exchanges() {
  constexpr int R = stage_radix<N, E, L>::value;
  if constexpr (L * R == N)
    return 0;
  else
    return 1 + fft_exchanges<N, E, L * R>();
}

// An exchange buffer in two halves used alternately: a half is written again
// only after the barrier that follows the other half's write, by which time
// every thread has read it, so an exchange needs one barrier instead of two.
// slot(idx, half) gives the thread's slot; the phase lives with the caller
// and persists across transforms (all threads of the CTA share the schedule).
template <typename C, class Slot> struct DualBuf {
  Slot slot;
  int *ph;
  __device__ __forceinline__ C &operator()(int idx) const { return slot(idx, *ph); }
  __device__ __forceinline__ void flip() const { *ph ^= 1; }
};
template <class B> struct is_dual_buf { static constexpr bool value = false; };
template <typename C, class Slot> struct is_dual_buf<DualBuf<C, Slot>> { static constexpr bool value = true; };
template <typename C, class Slot> __device__ __forceinline__ DualBuf<C, Slot> dual_buf(Slot s, int *ph) {
  return DualBuf<C, Slot>{s, ph};
}

// Full N-point transform of the line held in x (pattern t + T*e).
//   buf(idx) -> C& : this thread's line slot in shared memory
//   sync()         : barrier over every thread taking part (all lines of
//                    the CTA run the same schedule)
//   tw             : forward twiddles of a table of size N*TWS
template <typename C, int N, int E, int S, int TWS = 1, int L = 1, class Buf, class Sync>
__device__ __forceinline__ void line_fft(C (&x)[E], int t, const C *__restrict__ tw, Buf buf, Sync sync) {
  constexpr int T = N / E;
  constexpr int R = stage_radix<N, E, L>::value;
  constexpr bool LAST = (L * R == N);
  if constexpr (LAST) {
    fft_stage<C, N, E, L, S, TWS>(x, t, tw, [](int, C) {});
  } else {
    fft_stage<C, N, E, L, S, TWS>(x, t, tw, [&](int idx, C v) { buf(idx) = v; });
    sync();
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] = buf(t + T * e);
    if constexpr (is_dual_buf<Buf>::value)
      buf.flip();
    else
      sync();
    line_fft<C, N, E, S, TWS, L * R>(x, t, tw, buf, sync);
  }
}

// line_fft whose first exchange barrier is first() instead of sync(): a
// pipelined pass folds its wait agreement (__syncthreads_or) and its stage
// refill into that barrier.  Needs at least one exchange.
template <typename C, int N, int E, int S, int TWS = 1, class Buf, class Sync0, class Sync>
__device__ __forceinline__ void line_fft_first(C (&x)[E], int t, const C *__restrict__ tw, Buf buf, Sync0 first,
                                               Sync sync) {
  static_assert(fft_exchanges<N, E>() > 0, "no exchange barrier to fold into");
  constexpr int T = N / E;
  constexpr int R = stage_radix<N, E, 1>::value;
  fft_stage<C, N, E, 1, S, TWS>(x, t, tw, [&](int idx, C v) { buf(idx) = v; });
  first();
#pragma unroll
  for (int e = 0; e < E; ++e) x[e] = buf(t + T * e);
  if constexpr (is_dual_buf<Buf>::value)
    buf.flip();
  else
    sync();
  line_fft<C, N, E, S, TWS, R>(x, t, tw, buf, sync);
}

}  // namespace gb
