"""The MLP oracle against its pins: float64 gradients against central finite
differences, the bfloat16 rounding against torch's conversion, the emulated
(BF16-operand) gradients against the exact ones, and Adam's first step."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def _batch(seed, B):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((B, M.NIN)), 0.5 * rng.standard_normal((B, M.NOUT))


def test_parameter_count():
    assert M.NPARAM == 5254


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 10000),
                        np.array([1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 0.0], np.float32)])
    ref = torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16).float().numpy()
    assert np.array_equal(M.bf16(x), ref)


def test_gradient_matches_finite_differences():
    p = M.glorot(1).astype(np.float64)
    p[M.NH * M.NIN:M.NH * M.NIN + M.NH] = 0.1  # nonzero b1 exercises the bias path
    x, t = _batch(2, 37)
    g, _ = M.gradients(p, x, t)
    rng = np.random.default_rng(5)
    idx = rng.choice(M.NPARAM, 60, replace=False)
    h = 1e-6
    for q in idx:
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        lp = np.mean((M.forward(pp, x) - t) ** 2)
        lm = np.mean((M.forward(pm, x) - t) ** 2)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[q]) <= 1e-7 + 1e-5 * abs(fd), (q, fd, g[q])


def test_emulated_gradient_close_to_exact():
    p = M.glorot(4)
    x, t = _batch(6, 4096)
    ge, le = M.gradients(p, x.astype(np.float32), t.astype(np.float32), emulate=True)
    gx, lx = M.gradients(p.astype(np.float64), x, t)
    assert abs(le - lx) / lx < 1e-2
    assert np.linalg.norm(ge - gx) / np.linalg.norm(gx) < 3e-2


def test_adam_first_step_is_signed_lr():
    p = M.glorot(7)
    g = np.random.default_rng(8).standard_normal(M.NPARAM).astype(np.float32)
    z = np.zeros_like(p)
    p1, m, v = M.adam(p, z, z, g, 1, 1e-3)
    # bias-corrected first step: m_hat = g, v_hat = g^2 -> step = lr * g / (|g| + eps)
    np.testing.assert_allclose(p - p1, 1e-3 * np.sign(g), rtol=1e-4, atol=1e-9)
