"""Host-side tests (no GPU): the C ABI library loads and exports every declared symbol,
argument validation returns the documented codes before any device work, and the
workload / model host logic matches the reference's conventions."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO, has_gpu, load_pkg

HEADER = os.path.join(REPO, "include", "pbdose_b200.h")


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


@pytest.fixture(scope="module")
def lib(pb):
    if not os.path.exists(pb._lib.LIB_PATH):
        pytest.skip("library not built")
    return pb._lib.load()


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"PBD_API\s+[\w\s\*]*?\b(pbd_\w+)\s*\(", txt)))


def test_every_declared_symbol_is_exported_and_bound(pb, lib):
    decl = declared_symbols()
    assert len(decl) >= 15
    for name in decl:
        assert hasattr(lib, name), name
    assert sorted(pb._lib.exported_symbols()) == decl


def field(pb, **kw):
    f = dict(nx=32, ny=32, nz=64, dx=0.2, dy=0.2, dz=0.2, ox=-3.1, oy=-3.1, oz=0.0, n_sx=11,
             n_sy=11, n_layers=8, dx_spot=0.5, dy_spot=0.5, x0=0.0, y0=0.0)
    f.update(kw)
    return pb._lib.Field(**f)


def test_field_validation_codes(pb, lib):
    assert lib.pbd_field_validate(ctypes.byref(field(pb))) == 0
    assert lib.pbd_field_validate(None) == -1
    assert lib.pbd_field_validate(ctypes.byref(field(pb, nx=0))) == -2
    assert lib.pbd_field_validate(ctypes.byref(field(pb, n_layers=-1))) == -2
    assert lib.pbd_field_validate(ctypes.byref(field(pb, dx=float("nan")))) == -10
    assert lib.pbd_field_validate(ctypes.byref(field(pb, dx_spot=0.0))) == -10
    assert lib.pbd_field_validate(ctypes.byref(field(pb, n_sx=5000))) == -5
    for code in range(-12, 1):
        assert lib.pbd_strerror(code)


def test_entry_points_validate_before_device_work(pb, lib):
    f = field(pb)
    sz = ctypes.c_size_t(0)
    assert lib.pbd_forward_workspace(ctypes.byref(f), 0, ctypes.byref(sz)) == 0 and sz.value > 0
    assert lib.pbd_forward_workspace(ctypes.byref(f), 99, ctypes.byref(sz)) == -10
    fake = 0x1000
    # null arrays, missing / short workspace -> errors, and nothing launched
    assert lib.pbd_forward(ctypes.byref(f), None, fake, fake, fake, 0, fake, 1 << 30, None) == -1
    assert lib.pbd_forward(ctypes.byref(f), fake, fake, fake, fake, 0, None, 0, None) == -7
    assert lib.pbd_forward(ctypes.byref(f), fake, fake, fake, fake, 0, fake, 16, None) == -7
    assert lib.pbd_adjoint(ctypes.byref(f), fake, fake, fake, fake, fake, fake, fake, fake, 0,
                           None, 0, None) == -7
    big = field(pb, n_sx=65)
    assert lib.pbd_adjoint_workspace(ctypes.byref(big), 0, ctypes.byref(sz)) == -5
    assert lib.pbd_loss_grad(ctypes.byref(f), fake, fake, fake, None, None, fake, fake, fake, fake,
                             fake, fake, fake, 0, None, 0, None) == -1
    assert lib.pbd_set_schedule(65, 0) == -10
    assert lib.pbd_set_schedule(0, 0) == 0


def test_optimizer_steps_validate_before_device_work(pb, lib):
    fake = 0x1000
    P = pb._lib.AdamParams
    ok = P(lr=0.01, beta1=0.9, beta2=0.999, eps=1e-8, lo=0.0, hi=float("inf"), grad_scale=1.0)
    st = ctypes.c_void_p(fake)
    assert lib.pbd_adam_step(None, 4, fake, fake, fake, fake, st, None, None, None, 0, None) == -1
    assert lib.pbd_adam_step(ctypes.byref(ok), 4, fake, fake, fake, fake, None, None, None, None,
                             0, None) == -1
    assert lib.pbd_adam_step(ctypes.byref(ok), 4, None, fake, fake, fake, st, None, None, None, 0,
                             None) == -1
    assert lib.pbd_adam_step(ctypes.byref(ok), -1, fake, fake, fake, fake, st, None, None, None,
                             0, None) == -2
    assert lib.pbd_adam_step(ctypes.byref(ok), 4, fake, fake, fake, fake, st, None, None, None,
                             8, None) == -1                      # history without a loss
    for bad in (dict(lr=float("nan")), dict(lr=-1.0), dict(beta1=1.0), dict(beta2=-0.1),
                dict(eps=0.0), dict(lo=1.0, hi=0.0), dict(grad_scale=float("inf"))):
        kw = dict(lr=0.01, beta1=0.9, beta2=0.999, eps=1e-8, lo=0.0, hi=1.0, grad_scale=1.0)
        kw.update(bad)
        assert lib.pbd_adam_step(ctypes.byref(P(**kw)), 4, fake, fake, fake, fake, st, None, None,
                                 None, 0, None) == -10, bad
    # n == 0 enqueues nothing and succeeds
    assert lib.pbd_adam_step(ctypes.byref(ok), 0, None, None, None, None, st, None, None, None, 0,
                             None) == 0
    assert lib.pbd_scenario_combine(2, 3, 4, fake, fake, fake, None, None) == -10
    assert lib.pbd_scenario_combine(0, 0, 4, fake, fake, fake, None, None) == -2
    assert lib.pbd_scenario_combine(1, 129, 4, fake, fake, fake, None, None) == -2
    assert lib.pbd_scenario_combine(1, 3, 4, None, fake, fake, None, None) == -1
    assert lib.pbd_scenario_combine(1, 3, 4, fake, None, fake, None, None) == -1
    assert lib.pbd_scenario_combine(1, 3, 0, None, fake, None, None, None) == 0


def test_batched_loss_grad_validation(pb, lib):
    jobs = (pb._lib.GradJob * 129)()
    for k in range(129):
        jobs[k].field = field(pb)
    sz = ctypes.c_size_t(0)
    assert lib.pbd_loss_grad_batch_workspace(jobs, 129, 1, ctypes.byref(sz)) == -9
    assert lib.pbd_loss_grad_batch_workspace(jobs, 0, 1, ctypes.byref(sz)) == -2
    assert lib.pbd_loss_grad_batch_workspace(jobs, 4, 0, ctypes.byref(sz)) == -5   # fp32
    assert lib.pbd_loss_grad_batch_workspace(jobs, 4, 1, ctypes.byref(sz)) == 0 and sz.value > 0
    jobs[2].grad_range = 0x1000                       # range gradient on some jobs only
    assert lib.pbd_loss_grad_batch_workspace(jobs, 4, 1, ctypes.byref(sz)) == -10
    jobs[2].grad_range = None
    assert lib.pbd_loss_grad_batch(jobs, 4, 1, ctypes.c_void_p(0x1000), sz.value, None) == -1


def test_batch_limits(pb, lib):
    jobs = (pb._lib.Job * 129)()
    for k in range(129):
        jobs[k].field = field(pb)
    sz = ctypes.c_size_t(0)
    assert lib.pbd_forward_batch_workspace(jobs, 129, 0, ctypes.byref(sz)) == -9
    assert lib.pbd_forward_batch_workspace(jobs, 0, 0, ctypes.byref(sz)) == -2
    assert lib.pbd_forward_batch_workspace(jobs, 4, 0, ctypes.byref(sz)) == 0
    assert lib.pbd_forward_batch(jobs, 4, 0, ctypes.c_void_p(0x1000), sz.value, None) == -1


def test_lut_spec_validation(pb, lib):
    s = pb.physics.lut_spec(64, 0.0, 0.2)
    sz = ctypes.c_size_t(0)
    assert lib.pbd_lut_workspace(ctypes.byref(s), 8, ctypes.byref(sz)) == 0 and sz.value > 0
    bad = pb.physics.lut_spec(64, 0.0, -0.2)
    assert lib.pbd_lut_workspace(ctypes.byref(bad), 8, ctypes.byref(sz)) == -10
    assert lib.pbd_lut_workspace(ctypes.byref(s), 0, ctypes.byref(sz)) == -2
    with pytest.raises(ValueError):
        pb.physics.lut_spec(64, 0.0, 0.2, idd_model=pb.physics.IDDModel(straggling_model="x"))


# ----------------------------------------------------------------------- host logic
def test_workloads(pb):
    W = pb.workloads
    w0 = W.build_workload(0)
    assert w0["weights"].shape == (8, 11, 11) and w0["weights"].dtype == np.float32
    assert 0.5 <= w0["weights"].min() and w0["weights"].max() <= 1.5
    w1 = W.build_workload(1)
    assert w1["weights"].shape == (40, 41, 41)
    lw = w1["weights"].mean(axis=(1, 2))
    assert lw[0] < 0.33 and lw[-1] > 0.95 and np.all(np.diff(lw) > 0)
    np.testing.assert_array_equal(W.build_workload(1)["weights"], w1["weights"])
    w2 = W.build_workload(2)
    m, p = w2["mask"], w2["presc"]
    assert m.shape == (128, 128, 128)
    assert set(np.unique(m).tolist()) == {0.0, float(np.float32(0.2)), 1.0}
    assert np.all(p[m == 1.0] == 2.0) and np.all(p[m != 1.0] == 0.0)
    assert (m == 1.0).sum() == 31 * 30 * 30  # z centres 8.0..14.0 cm, x/y within +-3 cm
    w4 = W.build_workload(4)
    assert w4["weights"].shape == (60, 61, 61) and w4["grid"]["nz"] == 256
    fields = W.robust_fields()
    assert [f["weights"].shape for f in fields] == [(16, 21, 21), (28, 33, 33), (40, 41, 41),
                                                   (48, 41, 51)]
    sc = W.robust_scenarios()
    assert len(sc) == 25 and len(set(sc)) == 25 and (0.0, 0.0, 0.0, 1.0) in sc
    spots, layers = W.fd_sample(w2)
    assert spots.shape == (64, 3) and len(layers) == 8


def test_model_api_host_parts(pb):
    M = pb.model
    g = M.DoseGrid.centered(128, 0.2)
    assert g.shape == (128, 128, 128) and g.n_vox == 128**3
    assert g.ox == -(127 * 0.2 / 2.0)
    np.testing.assert_array_equal(g.x, g.ox + np.arange(128) * 0.2)
    assert g.z[0] == 0.0
    lat = M.SpotLattice(41, 41, 40, 0.25, 0.25)
    np.testing.assert_array_equal(lat.spot_x, 0.0 + (np.arange(41) - 20.0) * 0.25)
    assert lat.n_spots == 67240
    x, y, l, w = lat.flat_spot_table()
    assert x.shape == (67240,)
    fw = M.flat_field_weights(41, 41, 3)
    assert fw.shape == (3, 41, 41) and fw.min() >= 0.0
    prob = M.PBProblem(g, lat, np.zeros((40, 128)), np.ones((40, 128)))
    f = prob.field_descriptor()
    assert (f.nx, f.n_layers, f.dx_spot) == (128, 40, 0.25)
    c = pb.engines.operation_counts(prob, active_pairs=2727)
    assert abs(2 * c["separable_exact"] - 4.837e9) / 4.837e9 < 1e-3


def test_no_cpu_path(pb):
    if has_gpu():
        pytest.skip("checks the CPU-only behaviour")
    M = pb.model
    g = M.DoseGrid(8, 8, 8, 0.2, 0.2, 0.2)
    lat = M.SpotLattice(3, 3, 1, 0.5, 0.5, weights=np.ones((1, 3, 3)))
    prob = M.PBProblem(g, lat, np.ones((1, 8)), np.ones((1, 8)))
    with pytest.raises(RuntimeError):
        pb.engines.torch_separable(prob, "cuda")
    with pytest.raises(RuntimeError):
        pb.physics.csda_range(100.0)


def test_tensor_argument_checks():
    """The host-side check every plan applies to a tensor it hands to the library: refused
    unless it has the expected element count, dtype, device and a contiguous layout."""
    import torch
    pkg = load_pkg()
    chk, cpu = pkg._lib.check_arg, torch.device("cpu")
    t = torch.zeros((4, 5), dtype=torch.float32)
    assert chk(t, "t", 20, torch.float32, cpu) is t
    with pytest.raises(ValueError):
        chk(t, "t", 21, torch.float32, cpu)
    with pytest.raises(ValueError):
        chk(t.double(), "t", 20, torch.float32, cpu)
    with pytest.raises(ValueError):
        chk(t.t(), "t", 20, torch.float32, cpu)
    with pytest.raises(TypeError):
        chk(np.zeros(20, dtype=np.float32), "t", 20, torch.float32, cpu)
    with pytest.raises(ValueError):
        chk(t, "t", 20, torch.float32, torch.device("cuda", 0))
    assert pkg._lib.same_device(cpu, torch.device("cpu"))
    assert not pkg._lib.same_device(cpu, torch.device("cuda"))


def test_tuning_cache_and_schedule(pb, lib, tmp_path, monkeypatch):
    """The tuner's host side: the JSON cache (round trip; a missing or corrupt file reads as
    empty), the geometry key, lookup, and the schedule context -- its layers per forward unit
    reach the library (the forward's workspace grows with the number of layer chunks) and are
    reset on exit, also after an exception."""
    import types
    tun = pb.tuning
    cache = tmp_path / "sub" / "tuning.json"
    monkeypatch.setenv("PBD_TUNING_CACHE", str(cache))
    assert tun.cache_path() == str(cache)
    assert tun._load() == {}
    f = pb._lib.Field(nx=128, ny=128, nz=128, dx=0.2, dy=0.2, dz=0.2, ox=-12.7, oy=-12.7,
                      oz=0.0, n_sx=41, n_sy=41, n_layers=40, dx_spot=0.25, dy_spot=0.25,
                      x0=0.0, y0=0.0)
    plan = types.SimpleNamespace(field=f, precision=1, active_pairs=lambda: 2727)
    key = tun.geometry_key(plan, "loss_grad")
    assert key == "loss_grad|128x128x128|41x41x40|p1|a2727"
    assert tun.lookup(plan, "loss_grad") is None
    tun._store({key: {"schedule": [24, 4], "ms": 0.35}})
    assert tun.lookup(plan, "loss_grad") == (24, 4)
    assert tun.lookup(plan, "forward") is None
    cache.write_text("{not json")
    assert tun._load() == {} and tun.lookup(plan, "loss_grad") is None

    def fwd_ws():
        n = ctypes.c_size_t(0)
        assert lib.pbd_forward_workspace(ctypes.byref(f), 1, ctypes.byref(n)) == 0
        return n.value

    base = fwd_ws()
    with tun.schedule(8, 4):
        small_units = fwd_ws()
    assert small_units > base and fwd_ws() == base
    with pytest.raises(RuntimeError):
        with tun.schedule(8, 4):
            raise RuntimeError("inside")
    assert fwd_ws() == base


def test_packed_result_layout(pb):
    """grad_w, grad_range and loss in one buffer: each at a 256-byte boundary, no overlap,
    typed views that write exactly their own bytes, and a too-small buffer refused."""
    import torch
    eng = pb.engines
    offs, sizes, span = eng.packed_result_layout(41 * 41 * 40, 40)
    assert all(o % 256 == 0 for o in offs)
    assert sizes == (4 * 67240, 160, 8)
    assert all(offs[i] + sizes[i] <= offs[i + 1] for i in range(2))
    assert span == offs[2] + 8
    buf = torch.zeros(span, dtype=torch.uint8)
    v = eng.packed_result_views(buf, (40, 41, 41), 40)
    assert v["grad_w"].shape == (40, 41, 41) and v["grad_w"].is_contiguous()
    assert v["grad_range"].shape == (40,) and v["loss"].shape == ()
    v["grad_w"].fill_(1.0)
    v["grad_range"].fill_(2.0)
    v["loss"].fill_(3.0)
    raw = buf.numpy()
    assert np.array_equal(raw[offs[0]:offs[0] + sizes[0]].view(np.float32),
                          np.ones(67240, np.float32))
    assert np.array_equal(raw[offs[1]:offs[1] + sizes[1]].view(np.float32),
                          np.full(40, 2.0, np.float32))
    assert raw[offs[2]:offs[2] + 8].view(np.float64)[0] == 3.0
    gaps = np.ones(span, bool)
    for o, n in zip(offs, sizes):
        gaps[o:o + n] = False
    assert not raw[gaps].any()
    assert v["packed"].numel() == span
    with pytest.raises(ValueError):
        eng.packed_result_views(torch.zeros(span - 1, dtype=torch.uint8), (40, 41, 41), 40)


def test_engine_host_utilities_match_oracle(pb):
    """The reference's host utilities kept in engines.py (lateral_kernel, relative_error,
    normalize_dose, operation_counts) against the oracle's restatements and the FLOP count the
    bench credits (2 x 2727 active pairs x (nsx nsy ny + nx nsx ny) at 128^3 / 41x41x40)."""
    import torch
    from oracle import engine_ref as er
    E, M = pb.engines, pb.model
    rng = np.random.default_rng(9)
    vox = np.linspace(-3.0, 3.0, 17)
    spots = np.linspace(-2.0, 2.0, 5)
    sig = rng.uniform(0.2, 0.6, (3, 4))
    sig[0, 0] = 0.0                                  # clipped at 1e-9
    assert np.array_equal(E.lateral_kernel(vox, spots, sig), er.lateral_kernel(vox, spots, sig))
    raw = E.lateral_kernel(vox, spots, 0.4, normalized=False)
    assert np.array_equal(raw, np.exp(-(vox[:, None] - spots[None, :]) ** 2 / (2 * 0.4 ** 2)))
    a = rng.standard_normal((6, 7, 8))
    b = rng.standard_normal((6, 7, 8))
    mask = rng.random((6, 7, 8)) < 0.3
    for m in (None, mask, np.zeros_like(mask)):
        assert E.relative_error(a, b, m) == er.relative_error(a, b, m)
    assert E.relative_error(torch.as_tensor(a), torch.as_tensor(b)) == er.relative_error(a, b)
    d = np.abs(b)
    nd, ref = E.normalize_dose(d)
    assert ref == d.max() and nd.max() == 1.0
    roi = np.zeros_like(mask)
    roi[2, 3, 4] = True
    nd2, ref2 = E.normalize_dose(d, "roi_max", roi)
    assert ref2 == d[2, 3, 4] and np.array_equal(nd2, d / d[2, 3, 4])
    grid = M.DoseGrid(128, 128, 128, 0.2, 0.2, 0.2, -12.7, -12.7, 0.0)
    lat = M.SpotLattice(41, 41, 40, 0.25, 0.25, weights=np.ones((40, 41, 41)))
    prob = M.PBProblem(grid, lat, np.ones((40, 128)), np.full((40, 128), 0.4))
    oc = E.operation_counts(prob, active_pairs=2727)
    assert 2 * oc["separable_exact"] == 4837218048 and oc["pairs"] == 2727
    assert E.operation_counts(prob)["pairs"] == 40 * 128
    assert oc["naive"] == 41 * 41 * 40 * 128 ** 3


def test_model_builders_match_reference_fixture(pb):
    """DoseGrid axes, SpotLattice positions, the flat spot table (default seeded weights) and
    flat_field_weights equal the reference's own model.py outputs bit for bit
    (tests/golden/builders.npz, made by tests/golden/make_golden_builders.py)."""
    from conftest import golden
    z = golden("builders.npz")
    M = pb.model
    grids = {"centered_z": M.DoseGrid.centered(64, 0.25),
             "centered_xyz": M.DoseGrid.centered(33, 0.3, axis="xyz"),
             "aniso": M.DoseGrid(20, 30, 40, 0.15, 0.2, 0.3, -1.4, -2.9, 0.5)}
    for name, g in grids.items():
        for ax in ("x", "y", "z"):
            assert np.array_equal(getattr(g, ax), z[f"{name}__{ax}"]), (name, ax)
        assert [g.nx, g.ny, g.nz, g.n_vox] == z[f"{name}__dims"].tolist()
    lat = M.SpotLattice(7, 5, 3, 0.4, 0.6, x0=0.07, y0=-0.11)
    assert np.array_equal(lat.spot_x, z["lat__spot_x"])
    assert np.array_equal(lat.spot_y, z["lat__spot_y"])
    for got, key in zip(lat.flat_spot_table(), ("x", "y", "l", "w")):
        assert np.array_equal(got, z[f"lat__table_{key}"]), key
    assert np.array_equal(M.flat_field_weights(41, 41, 4), z["flat_default"])
    assert np.array_equal(M.flat_field_weights(21, 21, 3, field_half_width=3.0, spot_spacing=0.4,
                                               edge=0.5, radial_falloff=0.1, layer_jitter=0.3,
                                               seed=7), z["flat_args"])
    assert np.array_equal(M.flat_field_weights(15, 15, 2, layer_jitter=0.0), z["flat_nojitter"])


def test_reference_arm_json_contract():
    """``bench.py --impl reference`` (the oracle's CPU port, host cores only) prints one JSON
    line with the bench contract's keys: the metric and unit of the device arm, at least three
    warm-up evaluations, a cpu_baseline describing the run and an e2e object with no copies."""
    import json
    import subprocess
    import sys
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True,
                       timeout=600, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "grad_evals/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["warmup"] >= 3 and d["steps"] == 1
    assert d["metric"].startswith("fwd+adjoint dose-gradient evals/s")
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_depth_axis_check(pb):
    """The device table builder takes a uniform depth axis (nz, z0, dz); layer_luts derives it
    from the caller's axis and refuses what it cannot represent."""
    ua = pb.physics._uniform_axis
    assert ua(np.arange(64) * 0.2) == (64, 0.0, (63 * 0.2) / 63)
    assert ua([3.5]) == (1, 3.5, 1.0)
    n, z0, dz = ua(0.1 + np.arange(10) * 0.25)
    assert n == 10 and z0 == 0.1 and abs(dz - 0.25) < 1e-15
    for bad in ([], [[0.0, 1.0]], [0.0, 0.1, 0.3]):
        with pytest.raises(ValueError):
            ua(bad)
