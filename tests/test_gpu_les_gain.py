"""What the trained network gains: the whole learned-closure workflow at a
reduced size (128^3 forced DNS -> 32^3 LES with kc = 10, 12 snapshots),
trained on the GPU by the library's own kernels, and judged a posteriori
against the filtered DNS spectra.  The LES with the network must track the
filtered DNS spectrum better than the same LES without a closure, and the
network must explain most of the subgrid-stress variance it was not
trained on."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.timeout(900)
def test_mlp_closure_beats_no_closure():
    from ghost_b200.les_experiment import run
    res = run(dns_n=128, les_n=32, kc=10, nu_dns=5e-3, dt=1e-3, les_dt_ratio=4, spinup=1500, nsnap=12,
              snap_every=40, val_snaps=2, train_steps=1500, batch=16384, lr=2e-3, models=("none", "mlp", "edqnm"),
              log=lambda *a: None)
    tr = res["training"]
    # held-out stresses: the network explains most of their variance
    assert tr["val_loss"] < 0.5 * tr["val_loss_zero_model"], tr
    les = res["les"]
    assert les["mlp"]["finite"] and les["none"]["finite"]
    e_mlp = les["mlp"]["error_time_avg"]["mean"]
    e_none = les["none"]["error_time_avg"]["mean"]
    assert e_mlp < e_none, (e_mlp, e_none)
    # the LES is cheaper per unit of simulated time than the DNS it replaces
    assert res["cost"]["mlp_speedup_vs_dns"] > 1.0
