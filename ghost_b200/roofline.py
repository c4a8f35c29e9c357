"""Algorithmic bytes of the fused HD substep, the numerator of the HBM
rooflines that bench.py and the ensemble bench report.

For a cubic n^3 grid with the 2/3 truncation (kn2 <= n^2/9, the library's
float32 rounding of kmax), the pruned passes touch these fractions of a
spectral field C = (n/2+1) n^2 complex values: f_line of the (kx, ky)
z-lines, f_row of the kx rows and f_keep of the modes.  Per substep of an
RK step of order `ord` the five passes move (in units of C):
    Z inverse  (9 + 3/ord) f_line    v in, v and curl v out (+ the RK copy)
    Y inverse  6 (f_line + f_row)
    X fused    9 f_row               six fields in, three products out
    Y forward  3 (f_row + f_line)
    Z forward  6 f_line + 9 f_keep   (6 f_keep without forcing)
"""
from __future__ import annotations

import json
import os


def prune_fractions(n: int):
    """(f_line, f_row, f_keep) of a cubic n^3 grid: the fractions of the
    spectral grid the pruned passes touch (kz = 0 decides a z-line; a kx
    row is live if any of its lines is)."""
    import numpy as np
    nxh = n // 2 + 1
    kmax = np.float32(1.0 / 9.0) * np.float32(n * n)
    kx = np.arange(nxh, dtype=np.float64)
    kx[-1] = -(n // 2)
    ky = np.fft.fftfreq(n, 1.0 / n)
    k2 = kx[:, None] ** 2 + ky[None, :] ** 2
    live = k2 <= kmax
    f_line = live.mean()
    f_row = live.any(axis=1).mean()
    kz = np.fft.fftfreq(n, 1.0 / n)
    kept = 0
    for i in range(nxh):
        kk = k2[i][:, None] + kz[None, :] ** 2
        kept += int(((kk <= kmax) & (kk >= 3.8e-7)).sum())
    f_keep = kept / (nxh * n * n)
    return float(f_line), float(f_row), float(f_keep)


def pass_bytes(n: int, ord: int, forced: bool = True, elem_bytes: int = 8, runs: int = 1):
    """Algorithmic bytes of each pass of one pruned substep (dict)."""
    f_line, f_row, f_keep = prune_fractions(n)
    cb = (n // 2 + 1) * n * n * elem_bytes * runs
    return {"z_inv": (9 + 3 / ord) * f_line * cb,
            "y_inv": 6 * (f_line + f_row) * cb,
            "x_nl": 9 * f_row * cb,
            "y_fwd": 3 * (f_row + f_line) * cb,
            "z_fwd": (6 * f_line + (9 if forced else 6) * f_keep) * cb}


def measured_hbm_peak():
    """(GB/s, "measured" | "fallback"): MEASURED_PEAKS.json's hbm_gbs at the
    repository root, or the fallback figure of this GPU pool."""
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def live_box(n: int):
    """(live kx rows, y-lines from the top, y-lines from the bottom, kz values
    from the top, kz values from the bottom) of a cubic n^3 grid's
    truncation: the box of the spectral field that holds every kept mode
    (the host-array staging of ghost_hd_run moves only this box, its z
    blocks rounded out to 16-byte words)."""
    import numpy as np
    kmax = np.float32(1.0 / 9.0) * np.float32(n * n)
    nxh = n // 2 + 1
    kx = np.arange(nxh, dtype=np.float64)
    kx[-1] = -(n // 2)
    ky = np.fft.fftfreq(n, 1.0 / n)
    live = (kx[:, None] ** 2 + ky[None, :] ** 2) <= kmax
    rows = int(np.nonzero(live.any(axis=1))[0].max()) + 1
    jt = int(live[:, : n // 2].sum(axis=1).max())
    jb = int(live[:, n // 2:].sum(axis=1).max())
    kz = np.fft.fftfreq(n, 1.0 / n)
    zl = kz ** 2 <= kmax
    kt = int(zl[: n // 2].sum())
    kb = int(zl[n // 2:].sum())
    return rows, jt, jb, kt, kb


def slab_exchange_bytes(n: int, nranks: int, elem_bytes: int = 8):
    """Bytes that must cross the links in one pruned substep of the slab run
    (ghost_b200.slab) of a cubic n^3 grid over nranks ranks: the six front
    fields (v, curl v) kx-slab -> z-slab and the three products back, the
    live kx rows only, each rank's own block excluded.  Returns the largest
    over the ranks of max(bytes sent, bytes received), the per-direction
    load of the busiest GPU."""
    from .slab import exchange_counts, live_rows, slab_layout
    ista, nxhl, _, nzl = slab_layout(n, n, nranks)
    lr = live_rows(ista, nxhl, live_box(n)[0])
    worst = 0
    for r in range(nranks):
        s0, r0 = exchange_counts(lr, nzl, n, r, 0, 6, self_direct=True)
        s1, r1 = exchange_counts(lr, nzl, n, r, 1, 3, self_direct=True)
        worst = max(worst, sum(s0) + sum(s1), sum(r0) + sum(r1))
    return worst * elem_bytes


def slab_roofline(n: int, nranks: int, ms_per_step: float, xch_ms_per_substep: float, ord: int = 4,
                  elem_bytes: int = 8, link_gbs: float = 770.0):
    """Roofline of the slab-decomposed run (no per-pass timers there): each
    rank's share of the pruned step's algorithmic bytes (pass_bytes x ord /
    nranks) over the measured step time, against the HBM peak, and the
    exchange's link bytes per substep (slab_exchange_bytes) over the
    measured exchange time, against the peer copy bandwidth link_gbs (GB/s
    per direction, measured on this kind of machine)."""
    peak, kind = measured_hbm_peak()
    step_bytes = ord * sum(pass_bytes(n, ord, True, elem_bytes).values()) / nranks
    ach = step_bytes / (ms_per_step * 1e-3) / 1e9
    xb = slab_exchange_bytes(n, nranks, elem_bytes)
    xach = xb / (xch_ms_per_substep * 1e-3) / 1e9 if xch_ms_per_substep > 0 else None
    return {"bound": "hbm", "kernel": f"whole RK{ord} step, one rank's share of the pruned passes",
            "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": kind,
            "bytes_per_rank_per_step": step_bytes, "traffic": None,
            "exchange": {"bytes_per_substep": xb, "achieved": xach, "peak": link_gbs, "unit": "GB/s",
                         "frac": None if xach is None else xach / link_gbs,
                         "peak_kind": "measured peer copy per direction"}}
