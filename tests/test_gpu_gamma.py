"""Gamma index on the device against fixtures made by the reference's own gamma.py and
against the oracle on larger grids.

Bar: the gamma map (float64), the mask, n_eval, n_pass, pass_rate, gamma_max, gamma_p95,
gamma_p99, ref_max and n_dta_offsets bit for bit (the kernel rounds every float64 operation
in the reference's order); gamma_mean within 1e-13 relative (a fixed-order device sum
against NumPy's pairwise sum).
"""
import hashlib
import json

import numpy as np
import pytest

from conftest import golden, has_gpu, load_pkg
from oracle import gamma_ref as gr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

EXACT = ("pass_rate", "gamma_max", "gamma_p95", "gamma_p99", "n_eval", "n_pass", "ref_max",
         "n_dta_offsets")
MEAN_TOL = 1e-13


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


def same(a, b):
    return (a == b) or (a != a and b != b)


def check_stats(got, want, name):
    for k in EXACT:
        assert same(got[k], want[k]), (name, k, got[k], want[k])
    a, b = got["gamma_mean"], want["gamma_mean"]
    assert (a != a and b != b) or abs(a - b) <= MEAN_TOL * abs(b), (name, a, b)


def fixture_cases():
    z = golden("gamma.npz")
    return z, json.loads(str(z["cases_json"]))


@pytest.mark.parametrize("idx", range(12))
def test_gamma_matches_reference_fixtures(pb, idx):
    z, cs = fixture_cases()
    c = cs[idx]
    ref = z[c["ref"]]
    ev = z[c["eval"]]
    r = pb.gamma.gamma_index(ref.astype(np.float64), ev.astype(np.float64),
                             spacing=tuple(c["spacing"]), **c["kwargs"])
    check_stats(r, c["stats"], c["name"])
    assert hashlib.sha256(r["gamma"].tobytes()).hexdigest() == c["gamma_sha256"], c["name"]
    assert hashlib.sha256(r["mask"].tobytes()).hexdigest() == c["mask_sha256"], c["name"]
    if c["full_maps"]:
        assert np.array_equal(r["gamma"], z[c["name"] + "__gamma"], equal_nan=True)
    if ref.dtype == np.float32 and ev.dtype == np.float32:
        # the float32 input path gives the same float64 result
        r32 = pb.gamma.gamma_index(ref, ev, spacing=tuple(c["spacing"]), **c["kwargs"])
        check_stats(r32, c["stats"], c["name"] + " f32")
        assert hashlib.sha256(r32["gamma"].tobytes()).hexdigest() == c["gamma_sha256"]


def test_criteria_sweep_and_torch_entry_point(pb):
    z, cs = fixture_cases()
    c = cs[0]
    ref = z[c["ref"]].astype(np.float64)
    ev = z[c["eval"]].astype(np.float64)
    got = pb.gamma.gamma_pass_rate_vs_criteria(ref, ev, spacing=(0.2, 0.2, 0.2))
    assert [g["pass_rate"] for g in got] == z["criteria_pass_rates"].tolist()
    assert [(g["dose_pct"], g["dta_mm"]) for g in got] == [tuple(v) for v in z["criteria"]]
    t = pb.gamma.gamma_index_torch(ref, ev, spacing=(0.2, 0.2, 0.2))
    check_stats(t, c["stats"], "torch entry point")
    assert "gamma" not in t and t["normalization"] == "global"


def smooth(shape, seed):
    rng = np.random.default_rng(seed)
    idx = np.meshgrid(*[np.linspace(-1, 1, n) for n in shape], indexing="ij")
    d = np.zeros(shape)
    for _ in range(5):
        c = rng.uniform(-0.5, 0.5, 3)
        s = rng.uniform(0.15, 0.4)
        d += rng.uniform(0.5, 1.5) * np.exp(-sum((g - ci) ** 2 for g, ci in zip(idx, c))
                                            / (2 * s * s))
    return d


@pytest.mark.parametrize("spacing,dta,crit,norm", [((0.1, 0.1, 0.1), 3.0, 3.0, "global"),
                                                   ((0.2, 0.2, 0.2), 3.0, 3.0, "global"),
                                                   ((0.2, 0.15, 0.1), 2.0, 2.0, "local")])
def test_gamma_larger_grid_vs_oracle(pb, spacing, dta, crit, norm):
    """A ragged 70 x 45 x 83 grid (no dimension a multiple of the 32 x 8 x 4 brick)."""
    shape = (70, 45, 83)
    ref = smooth(shape, 11)
    rng = np.random.default_rng(12)
    ev = (np.roll(ref, (1, -1, 2), axis=(0, 1, 2)) * 0.3 + ref * 0.7) * 1.01 \
        + 0.005 * rng.standard_normal(shape)
    want = gr.gamma_index(ref, ev, spacing=spacing, dose_crit_pct=crit, dta_mm=dta,
                          normalization=norm)
    got = pb.gamma.gamma_index(ref, ev, spacing=spacing, dose_crit_pct=crit, dta_mm=dta,
                               normalization=norm)
    check_stats(got, want, "larger grid")
    assert np.array_equal(got["gamma"], want["gamma"])
    assert np.array_equal(got["mask"], want["mask"])


def test_gamma_plan_graph_replay_and_device_inputs(pb):
    """Device-resident float32 doses through a GammaPlan, eager and replayed from a CUDA
    graph, equal the one-shot call."""
    import torch
    shape = (40, 36, 44)
    ref = smooth(shape, 21).astype(np.float32)
    ev = (ref * 1.015 + 0.01 * np.roll(ref, 1, axis=2)).astype(np.float32)
    want = pb.gamma.gamma_index(ref, ev, spacing=(0.2, 0.2, 0.2))
    rd = torch.as_tensor(ref, device="cuda")
    ed = torch.as_tensor(ev, device="cuda")
    plan = pb.gamma.GammaPlan(shape, pb.gamma.gamma_spec((0.2, 0.2, 0.2)))
    plan.run(rd, ed)
    st = plan.stats()
    assert st.status == 0 and st.pass_rate == want["pass_rate"]
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.run(rd, ed)
    torch.cuda.current_stream().wait_stream(s)
    with torch.cuda.graph(g):
        plan.run(rd, ed)
    plan.stats_dev.zero_()
    g.replay()
    st2 = plan.stats()
    for k in ("pass_rate", "gamma_mean", "gamma_max", "gamma_p95", "gamma_p99", "n_eval",
              "n_pass"):
        assert getattr(st2, k) == want[k], k
    assert np.array_equal(plan.gamma.cpu().numpy(), want["gamma"])


def test_gamma_errors(pb):
    z = np.zeros((8, 8, 8))
    with pytest.raises(ValueError):
        pb.gamma.gamma_index(z, z)                                # reference max <= 0
    with pytest.raises(ValueError):
        pb.gamma.gamma_index(-np.ones((8, 8, 8)), z)
    with pytest.raises(ValueError):
        pb.gamma.gamma_index(np.ones((8, 8, 8)), np.ones((8, 8, 9)))
    with pytest.raises(ValueError):
        # a normalisation dose with no positive reference voxel: nothing to evaluate
        pb.gamma.gamma_index(-np.ones((8, 8, 8)), z, ref_dose=1.0)
    # a plan refuses doses that are not on its device
    import torch
    plan = pb.gamma.GammaPlan((8, 8, 8), pb.gamma.gamma_spec())
    on_dev = torch.ones((8, 8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        plan.run(torch.ones((8, 8, 8), dtype=torch.float64), on_dev)
    # all-equal doses: every gamma is 0
    one = np.ones((9, 10, 11))
    r = pb.gamma.gamma_index(one, one)
    assert r["pass_rate"] == 100.0 and r["gamma_max"] == 0.0 and r["n_eval"] == one.size
