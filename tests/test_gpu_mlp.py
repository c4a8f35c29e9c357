"""The tensor-core MLP kernels (ghost_mlp_*) against the CPU oracle: forward
outputs, loss and gradients (BF16 operands, FP32 accumulation) on ragged and
full batches, Adam updates, and that training reduces the loss.

Tolerances: against the oracle that rounds the same operands to BF16, 2e-3
(relative L2; only accumulation order differs, which flips an occasional
BF16 rounding); against exact FP64 arithmetic, 3e-2 (the BF16 error)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _data(seed, B):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((B, M.NIN)).astype(np.float32)
    t = (0.5 * rng.standard_normal((B, M.NOUT))).astype(np.float32)
    return x, t


def _mlp(p):
    from ghost_b200.les import MLP
    m = MLP(seed=0)
    m.params = p
    return m


@pytest.mark.parametrize("B", [1, 100, 1000, 65536])
def test_forward_matches_oracle(B):
    import torch
    p = M.glorot(11)
    p[M.NH * M.NIN:M.NH * M.NIN + M.NH] = np.linspace(-0.2, 0.2, M.NH)
    x, _ = _data(12, B)
    m = _mlp(p)
    y = m.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(y, M.forward(p, x, emulate=True)) < 2e-3
    assert rel_l2(y, M.forward(p.astype(np.float64), x.astype(np.float64))) < 3e-2


@pytest.mark.parametrize("B", [100, 4097, 65536])
def test_gradients_match_oracle(B):
    import torch
    p = M.glorot(21)
    x, t = _data(22, B)
    m = _mlp(p)
    g, loss = m.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    ge, le = M.gradients(p, x, t, emulate=True)
    gx, lx = M.gradients(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - le) / le < 1e-5
    assert rel_l2(g, ge) < 2e-3
    assert rel_l2(g, gx) < 3e-2
    # per-tensor, so that a small block (b3, W1) cannot hide in the total
    o = 0
    for name, shape in M.SHAPES:
        n = int(np.prod(shape))
        assert rel_l2(g[o:o + n], ge[o:o + n]) < 5e-3, name
        o += n


def test_adam_steps_match_oracle():
    import torch
    p = M.glorot(31)
    x, t = _data(32, 8192)
    m = _mlp(p)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    pm, mm, vm = p.copy(), np.zeros_like(p), np.zeros_like(p)
    for step in range(1, 4):
        ge, _ = M.gradients(pm, x, t, emulate=True)
        pm, mm, vm = M.adam(pm, mm, vm, ge, step, 1e-3)
        m.train_step(xd, td, 1e-3)
    # Adam's first steps move every weight by about lr; compare the moves
    assert rel_l2(m.params - p, pm - p) < 2e-2


def test_training_reduces_loss():
    import torch
    teacher = M.glorot(41)
    x, _ = _data(42, 65536)
    t = M.forward(teacher.astype(np.float64), x.astype(np.float64)).astype(np.float32)
    m = _mlp(M.glorot(43))
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    first = m.train_step(xd, td, 3e-3)
    for _ in range(300):
        m.train_step(xd, td, 3e-3, want_loss=False)
    last = m.train_step(xd, td, 3e-3)
    assert last < 0.2 * first, (first, last)


def test_bad_arguments():
    import ctypes

    import torch
    from ghost_b200 import GhostError
    from ghost_b200._lib import check
    m = _mlp(M.glorot(1))
    with pytest.raises(ValueError):
        m.forward(torch.zeros((4, 9), device="cuda"))
    with pytest.raises(GhostError):
        check(m.lib.ghost_mlp_forward(m.h, None, None, 4), "ghost_mlp_forward")
    host = np.zeros((4, 10), np.float32)
    y = torch.zeros((4, 6), device="cuda")
    with pytest.raises(GhostError):  # host arrays are refused, not staged
        check(m.lib.ghost_mlp_forward(m.h, host.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(y.data_ptr()), 4),
              "ghost_mlp_forward")
