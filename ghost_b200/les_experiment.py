"""The learned-closure LES workflow, end to end on one GPU.

    python -m ghost_b200.les_experiment [--dns-n 512 --les-n 128 --kc 42 ...] [--out result.json]

1. DNS: forced HD turbulence on the fine grid (FP32 fast path): seeded
   random solenoidal velocity with E(k) ~ k^4 exp(-2(k/2)^2), <|v|^2> = 1;
   constant random solenoidal forcing on 2 <= |k| <= 3 with <|f|^2> = 1;
   RK4.  After a spin-up, `nsnap` snapshots `snap_every` steps apart.
2. Data: every snapshot gives one sample per coarse grid point
   (ghost_les_samples): the nine resolved velocity gradients and the filter
   width in, the six subgrid stresses tau = filt(u u) - ubar ubar out, for
   the sharp filter at kc.  The filtered spectra of the snapshots are the
   reference the LES is judged against.
3. Training: the tensor-core MLP (ghost_mlp_*) with Adam on random batches
   of the samples (inputs scaled by their rms, stresses by theirs), the last
   snapshots held out for validation.  A second network of the same shape
   learns a spectral eddy viscosity: from the shell inputs of each
   snapshot's filtered spectrum (ghost_les_spectral_features) to the
   a-priori nu_t(k) = -S(k)/D(k) of that snapshot, S the subgrid energy
   transfer of shell k and D its sum of k^2 |ubar|^2, in units of
   sqrt(E(kc)/kc); for an LES at a lower viscosity than the DNS the
   difference nu_dns - nu_les joins the target.
4. LES: from the filtered first snapshot, the coarse grid is advanced over
   the same time window with no closure, GHOST's EDQNM eddy viscosity, and
   the trained networks; spectra at the snapshot times.
5. Report: spectrum errors of each LES against the filtered DNS
   (|E_les(k)/E_dns(k) - 1| over 1 <= k <= kc, time-averaged spectra), and
   the device time per unit of simulated time of the DNS and of each LES.

Synthetic seeded inputs throughout; no external data.
"""
from __future__ import annotations

import argparse
import json
import time


def spectrum_errors(E_les, E_dns, kc):
    import numpy as np
    a = np.asarray(E_les)[:kc]
    b = np.asarray(E_dns)[:kc]
    r = np.abs(a / b - 1.0)
    return {"mean": float(r.mean()), "max": float(r.max()), "rms": float(np.sqrt(np.mean(r ** 2))),
            # the same over the inertial shells k <= kc/2, and weighted by energy
            "mean_k_le_kc_half": float(r[:kc // 2].mean()),
            "energy_weighted": float(np.abs(a - b).sum() / b.sum()),
            "per_k": r.tolist()}


def run(dns_n=512, les_n=128, kc=42, nu_dns=1e-3, nu_les=None, dt=5e-4, les_dt_ratio=4, ord=4, spinup=4000,
        nsnap=40, snap_every=100, val_snaps=4, train_steps=4000, batch=65536, lr=2e-3, seed=7, kolmo=1.4,
        models=("none", "edqnm", "mlp", "mlp_cal", "mlp_spectral"), deviatoric=True, spec_train_steps=3000,
        spec_lr=3e-3, fallback=False, spectral_from=None, log=print):
    import numpy as np
    import torch

    from ghost_b200 import Ghost
    from ghost_b200.les import LES, MLP

    to_np = lambda t: t.detach().cpu().numpy()  # noqa: E731

    nu_les = nu_dns if nu_les is None else nu_les
    if snap_every % les_dt_ratio:
        raise ValueError("snap_every must be a multiple of les_dt_ratio")
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    out = {"config": dict(dns_n=dns_n, les_n=les_n, kc=kc, nu_dns=nu_dns, nu_les=nu_les, dt=dt,
                          les_dt=dt * les_dt_ratio, ord=ord, spinup=spinup, nsnap=nsnap, snap_every=snap_every,
                          val_snaps=val_snaps, train_steps=train_steps, batch=batch, lr=lr, seed=seed,
                          kolmo=kolmo, deviatoric=deviatoric, spec_train_steps=spec_train_steps, spec_lr=spec_lr,
                          fallback=fallback, precision="fp32")}

    # ---- 1. DNS
    g = Ghost(dns_n, precision="fp32")
    v = [g.czeros() for _ in range(3)]
    f = [g.czeros() for _ in range(3)]
    g.init_random_solenoidal(1000, 1.0, dns_n / 3.0, 1, 1.0, *v)
    g.init_random_solenoidal(2000, 2.0, 3.0, 0, 1.0, *f)
    e0, e1 = ev(), ev()
    e0.record(stream)
    g.hd_run(spinup, ord, dt, nu_dns, *v, *f)
    e1.record(stream)
    e1.synchronize()
    dns_ms = e0.elapsed_time(e1)
    out["dns"] = {"spinup_ms": dns_ms, "ms_per_step": dns_ms / max(1, spinup),
                  "energy_after_spinup": g.energy(*v, 1)}
    log(f"DNS spin-up {spinup} steps: {dns_ms / max(1, spinup):.3f} ms/step, <|v|^2> = {out['dns']['energy_after_spinup']:.4f}")

    # ---- 2. snapshots -> samples and filtered spectra
    c = Ghost(les_n, precision="fp32")
    les = LES(c, kc)
    rows = les_n ** 3
    X = torch.empty((nsnap, rows, 10), dtype=torch.float32, device=dev)
    T = torch.empty((nsnap, rows, 6), dtype=torch.float32, device=dev)
    E_dns = []
    S_sgs, D_sgs = [], []
    v0 = None
    fl = [les.truncate(g, x) for x in f]
    for s in range(nsnap):
        if s:
            g.hd_run(snap_every, ord, dt, nu_dns, *v, *f)
        les.samples(g, *v, 1.0, X[s], T[s])
        ub = [les.truncate(g, x) for x in v]
        E_dns.append(c.spectrumc(*ub, 1, 0)[0])
        # the subgrid energy transfer of each shell, S(k) = sum Re(ubar . conj F)
        # with F = P(-div tau), and D(k) = sum k^2 |ubar|^2 (entrans's kin = 1
        # and kin = 0 sums): an eddy force -nu_t(k) k^2 ubar transfers
        # -nu_t(k) D(k), so nu_t(k) = -S(k)/D(k) reproduces it shell by shell
        Fs = les.tau_force(T[s], 1.0)
        S_sgs.append(c.entrans(*ub, *Fs, 1))
        D_sgs.append(c.entrans(*ub, *ub, 0))
        del Fs
        if s == 0:
            v0 = [x.clone() for x in ub]
    torch.cuda.synchronize()
    E_dns = np.array(E_dns)
    S_sgs, D_sgs = np.array(S_sgs), np.array(D_sgs)
    t0 = spinup * dt
    # release the DNS grid before training and the LES runs
    del v, f
    g.close()
    torch.cuda.empty_cache()

    # ---- 3. training
    ntr = nsnap - val_snaps
    if deviatoric:
        # the isotropic part of tau is a pressure: -P div (q I) = 0, so the
        # network is trained on the trace-free stress only
        tr3 = T[:, :, :3].sum(-1, keepdim=True) / 3.0
        T[:, :, :3] -= tr3
        del tr3
    gs = float(1.0 / X[:ntr, :, :9].pow(2).mean().sqrt())
    ts = float(1.0 / T[:ntr].pow(2).mean().sqrt())
    X[:, :, :9] *= gs
    T *= ts
    Xtr, Ttr = X[:ntr].reshape(-1, 10), T[:ntr].reshape(-1, 6)
    Xva, Tva = X[ntr:].reshape(-1, 10), T[ntr:].reshape(-1, 6)
    mlp = MLP(seed)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    xb = torch.empty((batch, 10), dtype=torch.float32, device=dev)
    tb = torch.empty((batch, 6), dtype=torch.float32, device=dev)
    vb = min(Xva.shape[0], 1 << 20)
    val_idx = torch.randperm(Xva.shape[0], generator=gen, device=dev)[:vb]
    xv, tv = Xva[val_idx].contiguous(), Tva[val_idx].contiguous()

    def val_loss():
        _, l = mlp.gradients(xv, tv)
        return l

    loss_hist = []
    e0.record(stream)
    for step in range(train_steps):
        idx = torch.randint(0, Xtr.shape[0], (batch,), generator=gen, device=dev)
        torch.index_select(Xtr, 0, idx, out=xb)
        torch.index_select(Ttr, 0, idx, out=tb)
        # cosine decay of the step size
        lr_s = lr * 0.5 * (1.0 + np.cos(np.pi * step / train_steps))
        want = step % 500 == 0 or step == train_steps - 1
        l = mlp.train_step(xb, tb, lr_s, want_loss=want)
        if want:
            loss_hist.append((step, l, val_loss()))
    e1.record(stream)
    e1.synchronize()
    train_ms = e0.elapsed_time(e1)
    # the mean-stress baseline: loss of predicting tau = 0 (the scaled stresses have unit rms)
    out["training"] = {"samples": int(Xtr.shape[0]), "val_samples": int(vb), "steps": train_steps,
                       "ms": train_ms, "ms_per_step": train_ms / max(1, train_steps),
                       "grad_scale": gs, "tau_scale": ts, "history": loss_hist,
                       "val_loss": loss_hist[-1][2] if loss_hist else None,
                       "val_loss_zero_model": float(tv.pow(2).mean()),
                       "val_loss_mean_model": float((tv - Ttr.mean(0)).pow(2).mean())}
    # correlation of predicted and true stresses on the validation set
    yv = mlp.forward(xv)
    corr = [float(torch.corrcoef(torch.stack([yv[:, m], tv[:, m]]))[0, 1]) for m in range(6)]
    out["training"]["val_correlation"] = corr
    # subgrid dissipation Pi = -tau_ab S_ab (S the resolved strain): the part
    # of the stress that drains resolved energy; correlation and mean ratio
    g = xv[:, :9].reshape(-1, 3, 3)
    S = 0.5 * (g + g.transpose(1, 2))
    w = torch.tensor([1.0, 1.0, 1.0, 2.0, 2.0, 2.0], device=dev)
    Sv = torch.stack([S[:, 0, 0], S[:, 1, 1], S[:, 2, 2], S[:, 0, 1], S[:, 0, 2], S[:, 1, 2]], 1)
    pi_true = -(tv * Sv * w).sum(1)
    pi_pred = -(yv * Sv * w).sum(1)
    out["training"]["dissipation_corr"] = float(torch.corrcoef(torch.stack([pi_pred, pi_true]))[0, 1])
    out["training"]["dissipation_mean_ratio"] = float(pi_pred.mean() / pi_true.mean())
    # a priori dissipation calibration, on training samples: the factor that
    # makes the network's mean subgrid dissipation equal the data's
    cal_idx = torch.randint(0, Xtr.shape[0], (min(Xtr.shape[0], 1 << 20),), generator=gen, device=dev)
    xc, tc = Xtr[cal_idx].contiguous(), Ttr[cal_idx].contiguous()
    yc = mlp.forward(xc)
    gc = xc[:, :9].reshape(-1, 3, 3)
    Sc = 0.5 * (gc + gc.transpose(1, 2))
    Scv = torch.stack([Sc[:, 0, 0], Sc[:, 1, 1], Sc[:, 2, 2], Sc[:, 0, 1], Sc[:, 0, 2], Sc[:, 1, 2]], 1)
    cal = float((tc * Scv * w).sum(1).mean() / (yc * Scv * w).sum(1).mean())
    out["training"]["dissipation_calibration"] = cal
    del xc, tc, yc
    log(f"trained {train_steps} steps in {train_ms:.0f} ms: val loss {out['training']['val_loss']:.4f} "
        f"(zero model {out['training']['val_loss_zero_model']:.4f}), corr {np.round(corr, 3).tolist()}")
    del X, T, Xtr, Ttr, Xva, Tva
    torch.cuda.empty_cache()

    # ---- 3b. the spectral network: shell inputs of each snapshot's filtered
    # spectrum -> nu_t(k) / sqrt(E(kc)/kc), trained on the a-priori eddy
    # viscosity of the training snapshots.  An LES at a lower viscosity than
    # the DNS must also dissipate what the DNS's extra viscosity did on the
    # resolved shells: nu_t(k) = -S(k)/D(k) + (nu_dns - nu_les)
    nu_ap = -S_sgs[:, :kc] / D_sgs[:, :kc] + (nu_dns - nu_les)
    vel = np.sqrt(np.maximum(E_dns[:, kc - 1], 0.0) / kc)
    xs = torch.cat([les.spectral_features(torch.tensor(E_dns[q], device=dev)) for q in range(nsnap)])
    ys0 = nu_ap / vel[:, None]
    so = float(1.0 / np.sqrt(np.mean(ys0[:ntr] ** 2)))
    ys = torch.zeros((nsnap * kc, 6), dtype=torch.float32, device=dev)
    ys[:, 0] = torch.tensor((ys0 * so).ravel(), dtype=torch.float32, device=dev)
    xs_tr, ys_tr = xs[:ntr * kc].contiguous(), ys[:ntr * kc].contiguous()
    xs_va, ys_va = xs[ntr * kc:].contiguous(), ys[ntr * kc:].contiguous()
    mlp_s = MLP(seed + 1)
    e0.record(stream)
    if spectral_from is not None:
        # a spectral network trained elsewhere (another cutoff or grid): its
        # inputs and output are in units of kc and sqrt(E(kc)/kc), so it is
        # used as it is, with its own output scale
        mlp_s.params = np.asarray(spectral_from["params"], dtype=np.float32)
        so = 1.0 / float(spectral_from["out_scale"])
        ys[:, 0] = torch.tensor((ys0 * so).ravel(), dtype=torch.float32, device=dev)
        xs_va, ys_va = xs[ntr * kc:].contiguous(), ys[ntr * kc:].contiguous()
        spec_train_steps = 0
    for step in range(spec_train_steps):
        lr_s = spec_lr * 0.5 * (1.0 + np.cos(np.pi * step / spec_train_steps))
        mlp_s.train_step(xs_tr, ys_tr, lr_s, want_loss=False)
    e1.record(stream)
    e1.synchronize()
    pred = to_np(mlp_s.forward(xs))[:, 0].reshape(nsnap, kc) / so
    _, lva = mlp_s.gradients(xs_va, ys_va)
    out["training_spectral"] = {
        "samples": int(ntr * kc), "steps": spec_train_steps, "ms": e0.elapsed_time(e1), "out_scale": 1.0 / so,
        # the losses count the five unused (zero-target) outputs too
        "val_loss": lva, "val_loss_zero_model": float(ys_va.pow(2).mean()),
        "nu_t_apriori_mean": (nu_ap[:ntr].mean(0)).tolist(),
        "nu_t_apriori_std": (nu_ap[:ntr].std(0)).tolist(),
        "nu_t_pred_val_mean": (pred[ntr:] * vel[ntr:, None]).mean(0).tolist(),
    }
    log(f"spectral network: val loss {lva:.4g} (zero model {out['training_spectral']['val_loss_zero_model']:.4g}); "
        f"a-priori nu_t(kc) {nu_ap[:ntr, -1].mean():.4g}")

    # ---- 4. LES runs over the snapshot window
    les_dt = dt * les_dt_ratio
    sub = snap_every // les_dt_ratio
    out["les"] = {}
    for model in models:
        vl = [x.clone() for x in v0]
        if model == "mlp":
            les.set_model("mlp", mlp, grad_scale=gs, tau_scale=1.0 / ts, delta=1.0, kolmo=kolmo)
        elif model == "mlp_cal":
            les.set_model("mlp", mlp, grad_scale=gs, tau_scale=cal / ts, delta=1.0, kolmo=kolmo)
        elif model == "mlp_spectral":
            les.set_model("mlp_spectral", mlp_s, tau_scale=1.0 / so, kolmo=kolmo)
        if model.startswith("mlp"):
            les.set_fallback(fallback)  # a learned closure that blows up hands over to EDQNM
        elif model == "edqnm":
            les.set_model("edqnm", kolmo=kolmo)
        else:
            les.set_model("none")
        les.set_time(t0)
        spectra = [c.spectrumc(*vl, 1, 0)[0]]
        ms = 0.0
        ok = True
        for s in range(1, nsnap):
            e0.record(stream)
            les.run(sub, ord, les_dt, nu_les, *vl, *fl)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            spectra.append(c.spectrumc(*vl, 1, 0)[0])
            if not np.all(np.isfinite(spectra[-1])):
                ok = False
                break
        spectra = np.array(spectra)
        steps = (len(spectra) - 1) * sub
        res = {"finite": ok, "steps": steps, "ms": ms, "ms_per_step": ms / max(1, steps),
               "energy_final": float(np.sum(spectra[-1]))}
        if model.startswith("mlp") and fallback:
            res["closure_at_end"], res["fell_back_at_step"] = les.status()
        if ok:
            res["error_time_avg"] = spectrum_errors(spectra[1:].mean(0), E_dns[1:].mean(0), kc)
            res["error_final"] = spectrum_errors(spectra[-1], E_dns[-1], kc)
            res["spectrum_time_avg"] = spectra[1:].mean(0)[:kc + 1].tolist()
        out["les"][model] = res
        log(f"LES {model}: {res['ms_per_step']:.3f} ms/step, "
            + (f"time-avg spectrum error mean {res['error_time_avg']['mean']:.3f} max {res['error_time_avg']['max']:.3f}"
               if ok else "diverged"))
    out["dns_spectrum_time_avg"] = E_dns[1:].mean(0)[:kc + 1].tolist()
    # where the learned closure's time goes: inputs, network, stress divergence
    if "mlp" in models:
        vl = [x.clone() for x in v0]
        xf = les.features(*vl, gs, 1.0)
        yf = mlp.forward(xf)
        parts = {"features": lambda: les.features(*vl, gs, 1.0, x=xf), "network": lambda: mlp.forward(xf, yf),
                 "stress_force": lambda: les.tau_force(yf, 1.0 / ts)}
        timing = {}
        for name, fn in parts.items():
            fn()
            e0.record(stream)
            for _ in range(10):
                fn()
            e1.record(stream)
            e1.synchronize()
            timing[name] = e0.elapsed_time(e1) / 10
        out["closure_ms_per_substep"] = timing
        log(f"MLP closure per substep: {timing}")
    # cost per unit of simulated time
    dns_per_t = out["dns"]["ms_per_step"] / dt
    out["cost"] = {"dns_ms_per_time_unit": dns_per_t}
    for model, res in out["les"].items():
        les_per_t = res["ms_per_step"] / les_dt
        out["cost"][f"{model}_ms_per_time_unit"] = les_per_t
        out["cost"][f"{model}_speedup_vs_dns"] = dns_per_t / les_per_t if les_per_t > 0 else None
    out["mlp_params"] = mlp.params.tolist()
    out["mlp_spectral_params"] = mlp_s.params.tolist()
    if spectral_from is not None:
        out["training_spectral"]["trained_on"] = spectral_from.get("from")
    les.close()
    c.close()
    mlp.close()
    mlp_s.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--dns-n", type=int, default=512)
    ap.add_argument("--les-n", type=int, default=128)
    ap.add_argument("--kc", type=int, default=42)
    ap.add_argument("--nu-dns", type=float, default=1e-3)
    ap.add_argument("--nu-les", type=float, default=None)
    ap.add_argument("--dt", type=float, default=5e-4)
    ap.add_argument("--les-dt-ratio", type=int, default=4)
    ap.add_argument("--spinup", type=int, default=4000)
    ap.add_argument("--nsnap", type=int, default=40)
    ap.add_argument("--snap-every", type=int, default=100)
    ap.add_argument("--train-steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--val-snaps", type=int, default=4)
    ap.add_argument("--full-stress", action="store_true", help="train on tau with its trace")
    ap.add_argument("--fallback", action="store_true", help="learned closures hand over to EDQNM on a blow-up")
    ap.add_argument("--spectral-from", default=None,
                    help="a result file (--out) whose spectral network is used instead of training one")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    spec = None
    if a.spectral_from:
        r0 = json.load(open(a.spectral_from))
        spec = {"params": r0["mlp_spectral_params"], "out_scale": r0["training_spectral"]["out_scale"],
                "from": r0["config"]}
    t = time.time()
    res = run(dns_n=a.dns_n, les_n=a.les_n, kc=a.kc, nu_dns=a.nu_dns, nu_les=a.nu_les, dt=a.dt,
              les_dt_ratio=a.les_dt_ratio, spinup=a.spinup, nsnap=a.nsnap, snap_every=a.snap_every,
              train_steps=a.train_steps, batch=a.batch, lr=a.lr, val_snaps=a.val_snaps,
              deviatoric=not a.full_stress, fallback=a.fallback, spectral_from=spec)
    res["wall_s"] = time.time() - t
    summary = {k: res[k] for k in ("config", "dns", "cost")}
    summary["training"] = {k: v for k, v in res["training"].items() if k != "history"}
    summary["training_spectral"] = {k: v for k, v in res["training_spectral"].items() if not isinstance(v, list)}
    summary["les"] = {m: {k: v for k, v in r.items() if k not in ("spectrum_time_avg",)} for m, r in res["les"].items()}
    for m in summary["les"].values():
        for k in ("error_time_avg", "error_final"):
            if k in m:
                m[k] = {kk: vv for kk, vv in m[k].items() if kk != "per_k"}
    print(json.dumps(summary))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
