"""Gamma index, host side (no GPU): the oracle against fixtures made by the reference's own
gamma.py (bit for bit), the library's offset table against the reference's dta_offsets
(including spacings where Python's ``x ** 2`` and ``x * x`` round differently), and
argument validation of the C ABI before any device work."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import golden, load_pkg
from oracle import gamma_ref as gr

STATS = ("pass_rate", "gamma_mean", "gamma_max", "gamma_p95", "gamma_p99", "n_eval", "n_pass",
         "ref_max", "n_dta_offsets")


def cases():
    z = golden("gamma.npz")
    return z, json.loads(str(z["cases_json"]))


def same(a, b):
    return (a == b) or (a != a and b != b)


@pytest.mark.parametrize("idx", range(12))
def test_oracle_matches_reference_fixtures(idx):
    import hashlib
    z, cs = cases()
    c = cs[idx]
    ref = z[c["ref"]].astype(np.float64)
    ev = z[c["eval"]].astype(np.float64)
    r = gr.gamma_index(ref, ev, spacing=tuple(c["spacing"]), **c["kwargs"])
    for k in STATS:
        assert same(r[k], c["stats"][k]), (c["name"], k, r[k], c["stats"][k])
    assert hashlib.sha256(r["gamma"].tobytes()).hexdigest() == c["gamma_sha256"]
    assert hashlib.sha256(r["mask"].tobytes()).hexdigest() == c["mask_sha256"]
    if c["full_maps"]:
        assert np.array_equal(r["gamma"], z[c["name"] + "__gamma"], equal_nan=True)
        assert np.array_equal(r["mask"], z[c["name"] + "__mask"])


def test_oracle_criteria_sweep_matches_fixture():
    z, cs = cases()
    c = cs[0]
    ref = z[c["ref"]].astype(np.float64)
    ev = z[c["eval"]].astype(np.float64)
    got = [gr.gamma_index(ref, ev, spacing=(0.2, 0.2, 0.2), dose_crit_pct=dp, dta_mm=dt)["pass_rate"]
           for dp, dt in z["criteria"]]
    assert got == z["criteria_pass_rates"].tolist()


@pytest.fixture(scope="module")
def pb():
    pkg = load_pkg()
    if not os.path.exists(pkg._lib.LIB_PATH):
        pytest.skip("library not built")
    return pkg


# spacings where (a*d)**2 (libm pow, what the reference evaluates) and (a*d)*(a*d) differ
ODD = [(0.3176, 0.1176, 0.0794), (0.3813, 0.2, 0.1), (0.1, 0.1, 0.1), (0.25, 0.2, 0.15),
       (0.2, 0.2, 0.2), (0.0794, 0.0794, 0.0794)]


@pytest.mark.parametrize("spacing", ODD)
@pytest.mark.parametrize("dta_mm", [2.0, 3.0, 5.0, 8.0])
def test_offset_table_matches_reference_offsets(pb, spacing, dta_mm):
    spec = pb.gamma.gamma_spec(spacing, dta_mm=dta_mm)
    n, radii, w = pb.gamma.offsets_table(spec)
    offs, dists = gr.dta_offsets(spacing, dta_mm / 10.0)
    assert n == len(offs)
    dta_cm = dta_mm / 10.0
    want = np.full((7, 7, 7), -1.0)
    for (a, b, c), d in zip(offs, dists):
        dr = d / dta_cm
        want[abs(a), abs(b), abs(c)] = dr * dr
    assert np.array_equal(w, want)
    assert tuple(radii) == tuple(int(np.abs(offs[:, k]).max()) for k in range(3))
    # the product's own dta_offsets equals the reference's
    o2, d2 = pb.gamma.dta_offsets(spacing, dta_cm)
    assert np.array_equal(o2, offs) and np.array_equal(d2, dists)


def test_gamma_entry_points_validate_before_device_work(pb):
    lib = pb._lib.load()
    fake = ctypes.c_void_p(0x1000)
    ok = pb.gamma.gamma_spec()
    sz = ctypes.c_size_t(0)
    assert lib.pbd_gamma_workspace(8, 8, 8, ctypes.byref(sz)) == 0 and sz.value > 0
    assert lib.pbd_gamma_workspace(0, 8, 8, ctypes.byref(sz)) == -2

    def call(spec, nz=8, ref=fake, ev=fake, dtype=0, stats=fake, ws=fake, wsb=1 << 30):
        return lib.pbd_gamma_index(ctypes.byref(spec) if spec is not None else None, nz, 8, 8,
                                   ref, ev, dtype, None, None, stats, ws, wsb, None)

    assert call(None) == -1
    assert call(ok, nz=0) == -2
    assert call(ok, ref=None) == -1
    assert call(ok, stats=None) == -1
    assert call(ok, dtype=7) == -10
    assert call(ok, ws=None) == -7
    assert call(ok, wsb=16) == -7
    for bad in (dict(spacing=(0.0, 0.2, 0.2)), dict(spacing=(0.2, float("nan"), 0.2)),
                dict(dta_mm=0.0), dict(dose_crit_pct=float("inf")), dict(max_vox=7),
                dict(max_vox=-1)):
        assert call(pb.gamma.gamma_spec(**bad)) == -10, bad
    nan_dose = pb.gamma.gamma_spec(ref_dose=float("nan"))
    assert call(nan_dose) == -10
    with pytest.raises(ValueError):
        pb.gamma.gamma_spec(normalization="relative")
