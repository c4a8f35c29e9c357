"""The oracle against the committed golden fixtures (tests/golden/*.npz,
made by tests/golden/make_golden.py): the oracle must reproduce them, and the
fixtures must satisfy the physical pins they are supposed to carry."""
import os

import numpy as np
import pytest

from tests.conftest import rel_l2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


@pytest.fixture(scope="module")
def regenerated():
    import sys
    sys.path.insert(0, GOLD)
    import make_golden
    from oracle.oracle import Oracle, build
    build()
    return make_golden, Oracle


def test_fixture_files_present():
    for name in ("hd64_cfg0", "hd16_forced", "bouss16", "fft", "mlp"):
        assert os.path.exists(os.path.join(GOLD, name + ".npz")), name


def test_oracle_reproduces_hd64(regenerated):
    mg, Oracle = regenerated
    new, old = mg.hd64_cfg0(Oracle), load("hd64_cfg0")
    for k in old:
        tol = 1e-13 if k.endswith("_0") else 1e-11
        assert rel_l2(new[k], old[k]) <= tol, k


def test_oracle_reproduces_small_runs(regenerated):
    mg, Oracle = regenerated
    for name, fn in (("hd16_forced", mg.hd16_forced), ("bouss16", mg.bouss16), ("fft", mg.fft)):
        new, old = fn(Oracle), load(name)
        for k in old:
            assert rel_l2(new[k], old[k]) <= 1e-12, (name, k)


def test_oracle_reproduces_mlp(regenerated):
    mg, _ = regenerated
    new, old = mg.mlp(), load("mlp")
    for k in old:
        assert rel_l2(np.asarray(new[k], np.float64), np.asarray(old[k], np.float64)) <= 1e-6, k


def test_hd64_fixture_physics():
    g = load("hd64_cfg0")
    # unit <|v|^2>, decay without forcing, spectrum sums to the energy
    assert abs(g["E_0"] - 1.0) < 1e-12
    assert g["E_0"] > g["E_1"] > g["E_10"] > g["E_100"] > 0.9 * g["E_0"]
    for n in (0, 1, 10, 100):
        assert abs(np.sum(g[f"Ek_{n}"]) - g[f"E_{n}"]) < 1e-12 * g[f"E_{n}"]
    # energy() returns <|v|^2> and <|w|^2>: d<|v|^2>/dt = -2 nu <|w|^2>, over the first 10 steps
    dEdt = (g["E_10"] - g["E_0"]) / 0.01
    rate = -2 * 2e-3 * 0.5 * (g["W_0"] + g["W_10"])
    assert abs(dEdt - rate) < 1e-4 * abs(rate)


def test_fft_fixture_parseval():
    g = load("fft")
    for tag in ("a", "b"):
        r, rr = g[f"r_{tag}"], g[f"rr_{tag}"]
        assert rel_l2(rr / r.size, r) < 1e-14
