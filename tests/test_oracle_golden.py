"""Pin the oracle (oracle/) against fixtures produced by the reference itself.

These run on the CPU.  A pass here is what makes the oracle a valid checker for
the CUDA path: every physics piece, the per-layer tables and the separable dose
agree with the reference's own outputs (tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from conftest import golden
from oracle import engine_ref as er
from oracle import physics_ref as pr


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def test_range_table_and_lookups():
    g = golden("physics.npz")
    e, r = pr.range_table()
    assert e.shape == (3797,)
    np.testing.assert_array_equal(e, g["E_tab"])
    assert rel(r, g["R_tab"]) < 1e-14
    assert rel(pr.csda_range(g["e_q"]), g["csda_q"]) < 1e-14
    assert rel(pr.energy_from_range(g["r_q"]), g["efr_q"]) < 1e-14
    assert rel(pr.stopping_power(g["e_q"]), g["stopping"]) < 1e-14
    assert rel(pr.highland_local_power(g["e_q"]), g["highland"]) < 1e-14


def test_straggling():
    g = golden("physics.npz")
    b = np.array([pr.bohr_straggling(e) for e in g["strag_e"]])
    s = np.array([pr.sigma_range(e)[0] for e in g["strag_e"]])
    assert rel(b, g["bohr"]) < 1e-13
    assert rel(s, g["sigma_R"]) < 1e-13


def test_fermi_eyges():
    g = golden("physics.npz")
    for k, e in enumerate(g["fe_e"]):
        m = pr.fermi_eyges_sigma(g["fe_z"], e, sigma_x0=0.3, return_all=True)
        assert rel(m["sigma_x"], g["fe_sigma"][k]) < 1e-13
        assert rel(m["B"], g["fe_B"][k]) < 1e-12
        assert rel(m["A2"], g["fe_A2"][k]) < 1e-12


def test_idd():
    g = golden("physics.npz")
    for k, e in enumerate(g["idd_e"]):
        o = pr.idd_fluence(g["idd_z"], e, return_all=True)
        assert rel(o["idd"], g["idd"][k]) < 1e-12
        assert abs(o["sigma_R"] - g["idd_sigma_R"][k]) < 1e-14
        assert abs(o["R0"] - g["idd_R0"][k]) < 1e-14


@pytest.mark.parametrize("cfg", [0, 1, 4])
def test_workload_luts(cfg):
    g = golden(f"luts_cfg{cfg}.npz")
    from conftest import load_pkg
    wl = load_pkg().workloads.build_workload(cfg)
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    assert rel(en, g["energies"]) < 1e-15
    if cfg == 4:
        pytest.skip("config 4 tables are checked on the GPU against the device builder")
    idd, sig = pr.layer_luts(g["z"], en)
    assert rel(idd, g["idd"]) < 1e-12
    assert rel(sig, g["sigma"]) < 1e-13


def _axes(wl):
    gr = wl["grid"]
    xv = gr["ox"] + np.arange(gr["nx"]) * gr["dx"]
    yv = gr["oy"] + np.arange(gr["ny"]) * gr["dy"]
    xs = wl["x0"] + (np.arange(wl["n_sx"]) - (wl["n_sx"] - 1) / 2.0) * wl["spot_pitch"]
    ys = wl["y0"] + (np.arange(wl["n_sy"]) - (wl["n_sy"] - 1) / 2.0) * wl["spot_pitch"]
    return xv, yv, xs, ys


def test_separable_dose_cfg0():
    from conftest import load_pkg
    wl = load_pkg().workloads.build_workload(0)
    lut = golden("luts_cfg0.npz")
    ref = golden("dose_cfg0.npz")
    d = er.separable_f64(*_axes(wl), wl["weights"], lut["idd"], lut["sigma"])
    assert rel(d, ref["dose"]) < 1e-14
    dt = er.separable_torch(*_axes(wl), wl["weights"], lut["idd"], lut["sigma"]).numpy()
    assert rel(dt, ref["dose"]) < 1e-14
    # the reference's own float32 engine sits at ~1e-7 against its float64 oracle
    assert rel(ref["dose_torch_f32"], ref["dose"]) < 1e-6


@pytest.mark.slow
def test_separable_dose_cfg1_slices():
    from conftest import load_pkg
    wl = load_pkg().workloads.build_workload(1)
    lut = golden("luts_cfg1.npz")
    ref = golden("dose_cfg1_slices.npz")
    d = er.separable_torch(*_axes(wl), wl["weights"], lut["idd"], lut["sigma"]).numpy()
    assert rel(d[ref["k"]], ref["slices"]) < 1e-13
    assert abs(d.max() - ref["dmax"]) / ref["dmax"] < 1e-13
    assert rel(d.sum(axis=(1, 2)), ref["zsum"]) < 1e-12


def test_engine_check_small_case():
    """The reference's cross-engine check (engine_check.py): naive triple loop == separable."""
    g = golden("engine_check.npz")
    xv = -3.0 + np.arange(24) * 0.25
    xs = (np.arange(3) - 1.0) * 0.5
    d = er.separable_f64(xv, xv, xs, xs, g["w"], g["idd"], g["sigma"])
    assert rel(d, g["dose_sep"]) < 1e-14
    assert rel(d, g["dose_naive"]) < 1e-12
    dn = er.naive_dose(xv, xv, 32, xs, xs, g["w"], g["idd"], g["sigma"])
    assert rel(dn, g["dose_naive"]) < 1e-13
    z = np.arange(32) * 0.25
    idd = np.stack([pr.idd_fluence(z, e) for e in g["energies"]])
    idd /= idd.max(axis=1, keepdims=True)       # engine_check uses peak-normalised IDDs
    assert rel(idd, g["idd"]) < 1e-12
