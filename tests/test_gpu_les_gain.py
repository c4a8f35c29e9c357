"""What the trained network gains: the whole learned-closure workflow at a
reduced size (128^3 forced DNS -> 32^3 LES with kc = 10, 12 snapshots),
trained on the GPU by the library's own kernels, and judged a posteriori
against the filtered DNS spectra.

The network must predict held-out (deviatoric) subgrid stresses better than
the best constant, and the LES that uses it must track the filtered DNS
spectrum shell by shell better than the same LES without a closure.  The
spectral network (a learned eddy viscosity per shell, trained on the
a-priori transfer of the same snapshots) must track it better still."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.timeout(900)
def test_mlp_closure_beats_no_closure():
    from ghost_b200.les_experiment import run
    res = run(dns_n=128, les_n=32, kc=10, nu_dns=5e-3, dt=1e-3, les_dt_ratio=4, spinup=1500, nsnap=12,
              snap_every=40, val_snaps=2, train_steps=1500, batch=16384, lr=2e-3,
              models=("none", "mlp", "mlp_spectral"), log=print)
    tr = res["training"]
    assert tr["val_loss"] < 0.9 * tr["val_loss_mean_model"], tr
    assert min(tr["val_correlation"]) > 0.3, tr["val_correlation"]
    les = res["les"]
    assert les["mlp"]["finite"] and les["none"]["finite"]
    e_mlp = les["mlp"]["error_time_avg"]["mean"]
    e_none = les["none"]["error_time_avg"]["mean"]
    print("per-shell spectrum error: mlp", e_mlp, "none", e_none)
    assert e_mlp < 0.8 * e_none, (e_mlp, e_none)
    ts = res["training_spectral"]
    assert ts["val_loss"] < 0.1 * ts["val_loss_zero_model"], ts
    assert les["mlp_spectral"]["finite"]
    e_spec = les["mlp_spectral"]["error_time_avg"]
    print("spectral closure:", e_spec["mean"], e_spec["energy_weighted"])
    assert e_spec["mean"] < 0.8 * e_mlp, (e_spec["mean"], e_mlp)
    assert e_spec["energy_weighted"] < les["none"]["error_time_avg"]["energy_weighted"]
