"""CPU restatement of the reference's gamma index (TEST INFRASTRUCTURE ONLY).

Oracle for ``pbd_gamma_index``.  Only ``tests/`` and ``bench.py``'s CPU legs may import it;
the product path never does.  Follows gamma.py:41-60 (``dta_offsets``: integer offsets
within the DTA ball, at most ``max_vox`` voxels per axis) and gamma.py:81-164
(``gamma_index``) in float64 NumPy: for each offset the evaluated dose is shifted with zero
fill, the squared distance term (|o|/DTA)^2 is added to the squared dose term
((E - R) / dose_crit)^2 and the running minimum kept with ``np.minimum`` (NaN-propagating);
the statistics run over the low-dose mask (R >= thr * ref_max, else R > 0) with
``np.percentile``'s 'linear' method.  Pinned against fixtures made by the reference itself
(tests/golden/gamma.npz).
"""
from __future__ import annotations

import numpy as np


def dta_offsets(spacing, dta_cm, max_vox=6):
    """Offsets (K, 3) and distances (K,) in the reference's loop order (gamma.py:41-60)."""
    dz, dy, dx = spacing
    h = [min(int(np.floor(dta_cm / s + 1e-9)), max_vox) for s in (dz, dy, dx)]
    offs, dists = [], []
    for a in range(-h[0], h[0] + 1):
        for b in range(-h[1], h[1] + 1):
            for c in range(-h[2], h[2] + 1):
                d = np.sqrt((a * dz) ** 2 + (b * dy) ** 2 + (c * dx) ** 2)
                if d <= dta_cm + 1e-12:
                    offs.append((a, b, c))
                    dists.append(d)
    return np.array(offs, dtype=np.int64), np.array(dists, dtype=np.float64)


def shifted(a, off):
    """out[r] = a[r + off], zero where r + off leaves the grid (gamma.py:63-75)."""
    out = np.zeros_like(a)
    src, dst = [], []
    for o, n in zip(off, a.shape):
        o = int(o)
        src.append(slice(max(0, o), n + min(0, o)))
        dst.append(slice(max(0, -o), n + min(0, -o)))
    out[tuple(dst)] = a[tuple(src)]
    return out


def gamma_index(reference, evaluation, spacing=(0.2, 0.2, 0.2), dose_crit_pct=3.0,
                dta_mm=3.0, threshold_pct=10.0, normalization="global", ref_dose=None,
                max_vox=6):
    """Same keys as the reference's result, maps included."""
    ref = np.asarray(reference, dtype=np.float64)
    ev = np.asarray(evaluation, dtype=np.float64)
    if ref.shape != ev.shape:
        raise ValueError("shape mismatch")
    dta_cm = dta_mm / 10.0
    ref_max = float(ref.max()) if ref_dose is None else float(ref_dose)
    if ref_max <= 0:
        raise ValueError("reference dose max <= 0")
    if normalization == "global":
        crit = dose_crit_pct / 100.0 * ref_max * np.ones_like(ref)
    else:
        crit = dose_crit_pct / 100.0 * np.maximum(ref, 1e-12)
    mask = ref >= (threshold_pct / 100.0) * ref_max
    if mask.sum() == 0:
        mask = ref > 0
    offs, dists = dta_offsets(spacing, dta_cm, max_vox)
    g2 = np.full(ref.shape, np.inf)
    for off, dist in zip(offs, dists):
        dd = (shifted(ev, off) - ref) / crit
        dr = dist / dta_cm
        np.minimum(g2, dr * dr + dd * dd, out=g2)
    gamma = np.sqrt(g2)
    gm = gamma[mask]
    passed = gm <= 1.0
    return {
        "pass_rate": float(passed.mean() * 100.0) if gm.size else float("nan"),
        "gamma_mean": float(gm.mean()),
        "gamma_max": float(gm.max()),
        "gamma_p95": float(np.percentile(gm, 95)),
        "gamma_p99": float(np.percentile(gm, 99)),
        "n_eval": int(gm.size),
        "n_pass": int(passed.sum()),
        "ref_max": ref_max,
        "n_dta_offsets": len(offs),
        "gamma": gamma,
        "mask": mask,
    }
