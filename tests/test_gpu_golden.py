"""The CUDA library against the committed golden fixtures (tests/golden):
the same seeded inputs through the C ABI, compared with the stored oracle
outputs.  FP64 tolerances follow the parity bar (1e-12 after one step, 1e-9
after 100); FP32 runs are held to 1e-5 per the fast-path bound."""
import os

import numpy as np
import pytest

from tests.conftest import rel_l2
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def low_modes(a, m=8):
    idx = np.r_[0:m, -m:0]
    return a[:m][:, idx][:, :, idx]


def test_hd64_cfg0_trajectory():
    from ghost_b200 import Ghost
    gold = load("hd64_cfg0")
    g = Ghost(64, precision="fp64")
    V = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000, 1.0, 64 / 3.0, 1, 1.0, *V)
    done = 0
    tol = {0: 1e-13, 1: 1e-12, 10: 1e-11, 100: 1e-9}
    for n in (0, 1, 10, 100):
        if n > done:
            g.hd_run(n - done, 2, 1e-3, 2e-3, *V)
            done = n
        h = [to_host(x) for x in V]
        assert rel_l2(np.stack([low_modes(x) for x in h]), gold[f"modes_{n}"]) <= tol[n], n
        planes = np.stack([np.sqrt(np.sum(np.abs(x) ** 2, axis=(1, 2))) for x in h])
        assert rel_l2(planes, gold[f"planes_{n}"]) <= tol[n], n
        assert abs(g.energy(*V, 1) - gold[f"E_{n}"]) <= tol[n] * gold[f"E_{n}"]
        assert abs(g.energy(*V, 0) - gold[f"W_{n}"]) <= tol[n] * gold[f"W_{n}"]
        Ek, _ = g.spectrumc(*V, 1, 1)
        assert rel_l2(Ek, gold[f"Ek_{n}"]) <= tol[n], n


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_hd16_forced_rk4(prec):
    from ghost_b200 import Ghost
    gold = load("hd16_forced")
    g = Ghost(16, precision=prec)
    V = [to_dev(x.astype(g.cdtype_np)) for x in gold["v0"]]
    F = [to_dev(x.astype(g.cdtype_np)) for x in gold["f"]]
    g.hd_run(5, 4, 5e-4, 1e-3, *V, *F)
    err = rel_l2([to_host(x) for x in V], list(gold["v5"]))
    assert err <= (1e-12 if prec == "fp64" else 1e-5), err


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_bouss16_rk4(prec):
    from ghost_b200 import Ghost
    gold = load("bouss16")
    g = Ghost(16, 16, 16, 1.0, 1.0, 0.25, arbsize=True, precision=prec)
    V = [to_dev(x.astype(g.cdtype_np)) for x in gold["v0"]]
    TH = g.czeros()
    g.bouss_run(3, 4, 2.5e-4, 5e-4, 5e-4, 0.5, 8.0, 8.0, *V, TH)
    err = rel_l2([to_host(x) for x in V], list(gold["v3"]))
    assert err <= (1e-12 if prec == "fp64" else 1e-5), err
    assert rel_l2(to_host(TH), gold["th3"]) <= (1e-12 if prec == "fp64" else 1e-5)


@pytest.mark.parametrize("tag,shape", [("a", (16, 16, 16)), ("b", (32, 16, 16))])
def test_fft_fixture(tag, shape):
    from ghost_b200 import GHOST_COMPLEX_TO_REAL, GHOST_REAL_TO_COMPLEX, Ghost
    gold = load("fft")
    g = Ghost(*shape, precision="fp64")
    out = g.czeros()
    g.fftp3d_real_to_complex(g.fftp3d_create_plan(shape, GHOST_REAL_TO_COMPLEX), to_dev(gold[f"r_{tag}"]), out)
    assert rel_l2(to_host(out), gold[f"c_{tag}"]) <= 1e-14
    r = g.rzeros()
    g.fftp3d_complex_to_real(g.fftp3d_create_plan(shape, GHOST_COMPLEX_TO_REAL), to_dev(gold[f"c_{tag}"]), r)
    assert rel_l2(to_host(r), gold[f"rr_{tag}"]) <= 1e-14


def test_mlp_fixture():
    import torch
    from ghost_b200.les import MLP
    gold = load("mlp")
    m = MLP(0)
    m.params = gold["params"]
    x, t = torch.from_numpy(gold["x"]).cuda(), torch.from_numpy(gold["t"]).cuda()
    y = m.forward(x).cpu().numpy()
    assert rel_l2(y, gold["y_bf16"]) < 2e-3
    assert rel_l2(y, gold["y_exact"]) < 3e-2
    grad, loss = m.gradients(x, t)
    assert rel_l2(grad, gold["grad_bf16"]) < 2e-3
    assert rel_l2(grad, gold["grad_exact"]) < 3e-2
    assert abs(loss - float(gold["loss_bf16"])) < 1e-5 * float(gold["loss_bf16"])
