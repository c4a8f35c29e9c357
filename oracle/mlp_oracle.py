"""CPU restatement of the subgrid-stress MLP (10 -> 64 -> 64 -> 6, GELU).

TEST INFRASTRUCTURE ONLY: tests/ and __graft_entry__.smoke() use it as the
checker of the tensor-core kernels in ghost_b200/csrc/mlp.cu.  The product
never imports it.

The network has no counterpart in GHOST; its definition is the one the
C-ABI header states (ghost_b200.h, "Learned subgrid-stress closure"):
parameters packed as W1[64][10], b1[64], W2[64][64], b2[64], W3[6][64],
b3[6]; y = W x + b; GELU(z) = z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
(the tanh form of Hendrycks and Gimpel); loss = mean of the
squared error over B*6 values; Adam with beta1 0.9, beta2 0.999, eps 1e-8
and bias correction.

Two modes:
  emulate=False  exact float64 arithmetic (pins the gradient by finite
                 differences, and is the precision-free reference);
  emulate=True   rounds to bfloat16 exactly where the kernel stores BF16
                 operands (inputs, weights, activations, dY, dZ2, dZ1) and
                 keeps everything else in float32 / float64 accumulation.
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT = 10, 64, 6
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NOUT, NH)), ("b3", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n]).reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name]).ravel() for name, _ in SHAPES])


GELU_C, GELU_A = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_d(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def _q(a, emulate):
    return bf16(a) if emulate else a


def _mm(a, b, emulate):
    # products accumulate in float64 either way; the kernel accumulates in
    # float32 (the difference is far below one bf16 ulp of the results)
    r = a.astype(np.float64) @ b.astype(np.float64)
    return r.astype(np.float32) if emulate else r


def forward(p: np.ndarray, x: np.ndarray, emulate: bool = False, cache: bool = False):
    w = unpack(p)
    dt = np.float32 if emulate else np.float64
    W1, W2, W3 = (_q(w[k].astype(dt), emulate) for k in ("W1", "W2", "W3"))
    b1, b2, b3 = (w[k].astype(dt) for k in ("b1", "b2", "b3"))
    X = _q(np.asarray(x, dtype=dt), emulate)
    Z1 = (_mm(X, W1.T, emulate) + b1).astype(dt)
    H1 = _q(gelu(Z1).astype(dt), emulate)
    Z2 = (_mm(H1, W2.T, emulate) + b2).astype(dt)
    H2 = _q(gelu(Z2).astype(dt), emulate)
    Y = (_mm(H2, W3.T, emulate) + b3).astype(dt)
    if cache:
        return Y, dict(X=X, Z1=Z1, H1=H1, Z2=Z2, H2=H2, W2=W2, W3=W3)
    return Y


def gradients(p: np.ndarray, x: np.ndarray, t: np.ndarray, emulate: bool = False):
    """(gradient vector, loss) of mean((mlp(x) - t)^2)."""
    Y, c = forward(p, x, emulate, cache=True)
    dt = np.float32 if emulate else np.float64
    B = x.shape[0]
    e = (Y - np.asarray(t, dtype=dt)).astype(dt)
    loss = float(np.mean(e.astype(np.float64) ** 2))
    dY = _q((e * dt(2.0 / (B * NOUT))).astype(dt), emulate)
    dH2 = _mm(dY, c["W3"], emulate)
    dZ2 = _q((dH2 * gelu_d(c["Z2"]).astype(dt)).astype(dt), emulate)
    dH1 = _mm(dZ2, c["W2"], emulate)
    dZ1 = _q((dH1 * gelu_d(c["Z1"]).astype(dt)).astype(dt), emulate)
    g = dict(W1=_mm(dZ1.T, c["X"], emulate), b1=dZ1.astype(np.float64).sum(0),
             W2=_mm(dZ2.T, c["H1"], emulate), b2=dZ2.astype(np.float64).sum(0),
             W3=_mm(dY.T, c["H2"], emulate), b3=dY.astype(np.float64).sum(0))
    return pack(g).astype(np.float64), loss


def adam(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (float32, as the kernel); returns new (p, m, v)."""
    p, m, v, g = (np.asarray(a, dtype=np.float32) for a in (p, m, v, g))
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    mh = m / np.float32(1 - b1 ** step)
    vh = v / np.float32(1 - b2 ** step)
    return p - np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps)), m, v


def glorot(seed: int) -> np.ndarray:
    """A seeded parameter vector with the kernel library's initial scales
    (Glorot-uniform weights, zero biases); the values differ from the
    library's own host RNG."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SHAPES:
        if name.startswith("W"):
            a = np.sqrt(6.0 / (shape[0] + shape[1]))
            d[name] = rng.uniform(-a, a, shape)
        else:
            d[name] = np.zeros(shape)
    return pack(d).astype(np.float32)
