"""Generate tests/golden/gamma.npz by running the REFERENCE's gamma index itself.

Run in a container where the reference checkout is available (read-only):

    python tests/golden/make_golden_gamma.py /root/reference

Inputs are seeded synthetic dose-like fields (sums of 3-D Gaussians with a depth
gradient; the evaluation is a shifted, rescaled, noisy copy), so no data leaves the
reference.  For each case the archive holds the inputs, the reference's statistics and
either its full gamma map and mask (small grids) or SHA-256 digests of their bytes
(larger grids).  The GPU box never needs the reference.
"""
from __future__ import annotations

import hashlib
import importlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STATS = ("pass_rate", "gamma_mean", "gamma_max", "gamma_p95", "gamma_p99", "n_eval", "n_pass",
         "ref_max", "n_dta_offsets")


def import_gamma(ref_dir):
    tmp = tempfile.mkdtemp(prefix="pbdose_ref_")
    os.symlink(os.path.abspath(ref_dir), os.path.join(tmp, "pbdose"))
    sys.path.insert(0, tmp)
    return importlib.import_module("pbdose.gamma")


def field(shape, spacing, seed, n_blobs=4):
    """A smooth non-negative dose-like field on a (nz, ny, nx) grid."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    dz, dy, dx = spacing
    z = np.arange(nz) * dz
    y = (np.arange(ny) - (ny - 1) / 2) * dy
    x = (np.arange(nx) - (nx - 1) / 2) * dx
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    d = np.zeros(shape)
    for _ in range(n_blobs):
        cz, cy, cx = rng.uniform(0.2, 0.8) * z[-1], rng.uniform(-0.3, 0.3) * (y[-1] - y[0]), \
            rng.uniform(-0.3, 0.3) * (x[-1] - x[0])
        s = rng.uniform(0.3, 0.9)
        d += rng.uniform(0.5, 1.5) * np.exp(-((Z - cz) ** 2 + (Y - cy) ** 2 + (X - cx) ** 2)
                                            / (2 * s * s))
    return d * (1.0 + 0.3 * Z / max(z[-1], 1e-9))


def evaluation_of(ref, seed, shift=(1, 0, -1), scale=1.02, noise=0.01):
    rng = np.random.default_rng(seed)
    ev = np.roll(ref, shift, axis=(0, 1, 2)) * 0.5 + ref * 0.5
    return ev * scale + noise * ref.max() * rng.standard_normal(ref.shape)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(ref_dir):
    G = import_gamma(ref_dir)
    small = (10, 12, 14)
    cases = []
    arrays = {}

    inputs = {}

    def key_of(a):
        # inputs are stored once; float32-exact ones as float32
        for k, v in inputs.items():
            if v.shape == a.shape and np.array_equal(v, a, equal_nan=True):
                return k
        k = f"in{len(inputs)}"
        inputs[k] = a
        f32 = a.astype(np.float32)
        exact = np.array_equal(f32.astype(np.float64), a, equal_nan=True)
        arrays[k] = f32 if exact else a
        return k

    def add(name, ref, ev, spacing, kw, full_maps):
        r = G.gamma_index(ref, ev, spacing=spacing, **kw)
        ref_key, ev_key = key_of(ref), key_of(ev)
        if full_maps:
            arrays[f"{name}__gamma"] = r["gamma"]
            arrays[f"{name}__mask"] = r["mask"]
        meta = {"name": name, "ref": ref_key, "eval": ev_key, "spacing": list(spacing),
                "kwargs": kw, "full_maps": full_maps,
                "stats": {k: r[k] for k in STATS},
                "gamma_sha256": digest(r["gamma"]), "mask_sha256": digest(r["mask"])}
        cases.append(meta)

    sp = (0.2, 0.2, 0.2)
    ref = field(small, sp, 1)
    ev = evaluation_of(ref, 2)
    add("g3_3", ref, ev, sp, {"dose_crit_pct": 3.0, "dta_mm": 3.0}, True)
    add("g2_2", ref, ev, sp, {"dose_crit_pct": 2.0, "dta_mm": 2.0}, True)
    add("local3_3", ref, ev, sp, {"dose_crit_pct": 3.0, "dta_mm": 3.0,
                                  "normalization": "local"}, True)
    add("thr0", ref, ev, sp, {"threshold_pct": 0.0}, True)
    add("refdose", ref, ev, sp, {"ref_dose": 0.8 * float(ref.max())}, True)
    add("fallback", ref, ev, sp, {"ref_dose": 3.0 * float(ref.max()), "threshold_pct": 50.0},
        True)
    ev_nan = ev.copy()
    ev_nan[3, 4, 5] = np.nan
    ev_nan[7, 1, 2] = np.nan
    add("nan", ref, ev_nan, sp, {}, True)
    sp_a = (0.25, 0.2, 0.15)
    ref_a = field(small, sp_a, 3)
    add("aniso", ref_a, evaluation_of(ref_a, 4, shift=(0, 1, 1)), sp_a, {}, True)
    sp1 = (0.1, 0.1, 0.1)
    ref1 = field(small, sp1, 5)
    ev1 = evaluation_of(ref1, 6, shift=(2, -1, 1), noise=0.03)
    add("dta5_1mm", ref1, ev1, sp1, {"dta_mm": 5.0}, True)
    add("cap_8mm", ref1, ev1, sp1, {"dta_mm": 8.0, "dose_crit_pct": 1.0}, True)
    mid = (64, 32, 32)
    ref_m = field(mid, sp, 7, n_blobs=6).astype(np.float32).astype(np.float64)
    ev_m = evaluation_of(ref_m, 8, shift=(1, 1, 0)).astype(np.float32).astype(np.float64)
    add("mid_3_3", ref_m, ev_m, sp, {}, False)
    add("mid_2_2_local", ref_m, ev_m, sp, {"dose_crit_pct": 2.0, "dta_mm": 2.0,
                                          "normalization": "local"}, False)
    crit = G.gamma_pass_rate_vs_criteria(ref, ev, spacing=sp)
    arrays["criteria_pass_rates"] = np.array([c["pass_rate"] for c in crit])
    arrays["criteria"] = np.array([[c["dose_pct"], c["dta_mm"]] for c in crit])
    arrays["cases_json"] = np.array(json.dumps(cases))
    out = os.path.join(HERE, "gamma.npz")
    np.savez_compressed(out, **arrays)
    print(f"wrote {out}: {len(cases)} cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
