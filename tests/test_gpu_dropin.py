"""The drop-in boundary against the float64 oracle, on the GPU.

* A problem object that carries only what the reference's engine reads
  (engines.py:227-234, 257-259: grid nx, ny, nz, x, y; lattice n_sx, n_sy, n_layers,
  spot_x, spot_y, ensure_weights(); idd, sigma) goes through ``torch_separable`` and
  ``DosePlan`` unchanged -- the reference's own PBProblem has no method of this package.
* ``dtype=torch.float64`` (the reference's float64 mode, engines.py:223-224) returns a
  float64 dose computed in FP64 on the device: 1e-12 of max against the oracle and the
  reference's own float64 dose of the 32x32x64 workload.
* ``allow_tf32=True`` keeps the accuracy the reference's flag kept (1.51e-7,
  benchmark_full.json:68-81): <= 1e-6 of max on the clinical field.
* ``layer_chunk`` is per call: two plans with different work-item sizes, called on two
  streams, both match the oracle.
* Bounded device waits: with the schedulers held (test hook) every wait runs out, the call's
  outputs are NaN and the status query reports PBD_ERR_TIMEOUT; the next call is correct.

Tolerances: float32 doses 1e-6 of max (the accuracy bound for FP32 and split forms), float64 doses 1e-12.
"""
import ctypes
from types import SimpleNamespace

import numpy as np
import pytest

from conftest import golden, has_gpu, load_pkg
from oracle import engine_ref as er

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

F32_TOL = 1e-6
F64_TOL = 1e-12


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


def _bare_problem(grid, lattice, idd, sigma):
    """Only the attributes the reference's torch_separable reads."""
    g = SimpleNamespace(nx=grid.nx, ny=grid.ny, nz=grid.nz, x=grid.x.copy(), y=grid.y.copy())
    w = np.asarray(lattice.ensure_weights(), dtype=np.float64).copy()
    lat = SimpleNamespace(n_sx=lattice.n_sx, n_sy=lattice.n_sy, n_layers=lattice.n_layers,
                          spot_x=lattice.spot_x.copy(), spot_y=lattice.spot_y.copy(),
                          ensure_weights=lambda: w)
    return SimpleNamespace(grid=g, lattice=lat, idd=np.asarray(idd), sigma=np.asarray(sigma))


def _cfg0(pb):
    wl = pb.workloads.build_workload(0)
    lut = golden("luts_cfg0.npz")
    return wl, pb.model.problem_from_workload(wl, lut["energies"], lut["idd"], lut["sigma"])


def test_bare_problem_through_torch_separable_and_plan(pb):
    wl, prob = _cfg0(pb)
    bare = _bare_problem(prob.grid, prob.lattice, prob.idd, prob.sigma)
    ref = golden("dose_cfg0.npz")["dose"]              # the reference's own float64 dose
    d = pb.engines.torch_separable(bare, "cuda").cpu().numpy()
    assert rel(d, ref) < F32_TOL
    plan = pb.engines.DosePlan(bare, tables="problem")
    assert rel(plan.forward().cpu().numpy(), ref) < F32_TOL
    # a ragged grid with an offset lattice: the field comes from the axes alone
    M = pb.model
    rng = np.random.default_rng(11)
    grid = M.DoseGrid(37, 70, 9, 0.15, 0.2, 0.3, -2.7, -6.9, 0.0)
    w = rng.uniform(0.1, 1.0, (3, 13, 29))
    lat = M.SpotLattice(29, 13, 3, 0.25, 0.3, x0=0.07, y0=-0.11, weights=w)
    idd = rng.uniform(0.0, 5.0, (3, 9))
    sig = rng.uniform(0.2, 0.8, (3, 9))
    bare = _bare_problem(grid, lat, idd, sig)
    ref = er.separable_f64(grid.x, grid.y, lat.spot_x, lat.spot_y, w, idd, sig)
    assert rel(pb.engines.torch_separable(bare, "cuda").cpu().numpy(), ref) < F32_TOL


def test_float64_dose(pb):
    import torch
    wl, prob = _cfg0(pb)
    d = pb.engines.torch_separable(prob, "cuda", dtype=torch.float64)
    assert d.dtype == torch.float64 and d.shape == prob.grid.shape
    err = rel(d.cpu().numpy(), golden("dose_cfg0.npz")["dose"])
    print(f"float64 dose vs the reference's float64 dose: {err:.2e}")
    assert err < F64_TOL
    # clinical field (five slices of the reference's float64 dose + the oracle on the rest)
    wl1 = pb.workloads.build_workload(1)
    lut = golden("luts_cfg1.npz")
    p1 = pb.model.problem_from_workload(wl1, lut["energies"], lut["idd"], lut["sigma"])
    d1 = pb.engines.torch_separable(p1, "cuda", dtype=torch.float64).cpu().numpy()
    sl = golden("dose_cfg1_slices.npz")
    for k, z in enumerate(sl["k"]):
        assert float(np.max(np.abs(d1[int(z)] - sl["slices"][k]))) <= F64_TOL * float(sl["dmax"])
    assert abs(float(d1.max()) - float(sl["dmax"])) <= F64_TOL * float(sl["dmax"])
    ragged = pb.model.PBProblem(
        pb.model.DoseGrid(150, 70, 5, 0.15, 0.2, 0.3, -11.0, -6.9, 0.0),
        pb.model.SpotLattice(61, 13, 4, 0.25, 0.3, x0=0.05, y0=-0.1,
                             weights=np.random.default_rng(3).uniform(0.1, 1.0, (4, 13, 61))),
        np.random.default_rng(4).uniform(0.0, 5.0, (4, 5)),
        np.random.default_rng(5).uniform(0.2, 0.8, (4, 5)))
    g, L = ragged.grid, ragged.lattice
    ref = er.separable_f64(g.x, g.y, L.spot_x, L.spot_y, L.weights, ragged.idd, ragged.sigma)
    got = pb.engines.torch_separable(ragged, "cuda", dtype=torch.float64).cpu().numpy()
    assert rel(got, ref) < F64_TOL


def test_allow_tf32_keeps_fp32_accuracy(pb):
    wl = pb.workloads.build_workload(1)
    lut = golden("luts_cfg1.npz")
    prob = pb.model.problem_from_workload(wl, lut["energies"], lut["idd"], lut["sigma"])
    d = pb.engines.torch_separable(prob, "cuda", allow_tf32=True).cpu().numpy()
    sl = golden("dose_cfg1_slices.npz")
    worst = 0.0
    for k, z in enumerate(sl["k"]):
        worst = max(worst, float(np.max(np.abs(d[int(z)] - sl["slices"][k]))) / float(sl["dmax"]))
    print(f"allow_tf32=True: {worst:.2e} of max on the reference's slices")
    assert worst < F32_TOL
    # the default (no flag) is the same split form
    d0 = pb.engines.torch_separable(prob, "cuda").cpu().numpy()
    assert np.array_equal(d0, d)


def test_layer_chunk_per_call_on_two_streams(pb):
    import torch
    wl, prob = _cfg0(pb)
    ref = golden("dose_cfg0.npz")["dose"]
    a = pb.engines.DosePlan(prob, tables="problem", precision="tf32x3")
    b = pb.engines.DosePlan(prob, tables="problem", precision="tf32x3")
    a.schedule, b.schedule = (2, 0), (5, 0)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    outs = []
    for _ in range(3):
        with torch.cuda.stream(s1):
            oa = a.forward()
        with torch.cuda.stream(s2):
            ob = b.forward()
        outs.append((oa, ob))
    torch.cuda.synchronize()
    for oa, ob in outs:
        assert rel(oa.cpu().numpy(), ref) < F32_TOL
        assert rel(ob.cpu().numpy(), ref) < F32_TOL
    # torch_separable's layer_chunk leaves no setting behind for later calls
    d = pb.engines.torch_separable(prob, "cuda", layer_chunk=3).cpu().numpy()
    assert rel(d, ref) < F32_TOL
    lib = pb._lib.load()
    f = pb._lib.field_of(prob)
    n1, n2 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert lib.pbd_forward_workspace(ctypes.byref(f), 1, ctypes.byref(n1)) == 0
    pb._lib.call("pbd_set_schedule", 0, 0)
    assert lib.pbd_forward_workspace(ctypes.byref(f), 1, ctypes.byref(n2)) == 0
    assert n1.value == n2.value


@pytest.mark.parametrize("prec", ["tf32x3", "bf16", "fp16x3"])
def test_timeout_status_and_recovery(pb, prec):
    """Every bounded wait of the tensor-core forward and adjoint runs out (schedulers held by
    the test hook, 50 ms limit): outputs NaN, status PBD_ERR_TIMEOUT, PbdError raised; the
    next call with the hook cleared is correct.  With fp16x3 the forward's status header is
    cleared by its pack kernel (no install kernel), so the recovery checks that as well."""
    import torch
    wl, prob = _cfg0(pb)
    ref = golden("dose_cfg0.npz")["dose"]
    plan = pb.engines.DosePlan(prob, tables="problem", precision=prec)
    good = plan.forward().clone()
    g = torch.ones(prob.grid.shape, dtype=torch.float32, device="cuda")
    gw_good, _ = plan.adjoint(g, with_range=False)
    torch.cuda.synchronize()
    plan.check("fwd")
    plan.check("adj")
    try:
        pb._lib.test_hook(50_000_000, hold=True)
        bad = plan.forward()
        assert pb._lib.workspace_status(plan.ws._bufs["fwd"]) == pb._lib.PBD_ERR_TIMEOUT
        with pytest.raises(pb._lib.PbdError) as e:
            plan.check("fwd")
        assert e.value.code == pb._lib.PBD_ERR_TIMEOUT
        assert torch.isnan(bad).all()
        gw_bad, _ = plan.adjoint(g, with_range=False)
        assert pb._lib.workspace_status(plan.ws._bufs["adj"]) == pb._lib.PBD_ERR_TIMEOUT
        assert torch.isnan(gw_bad).all()
    finally:
        pb._lib.test_hook(0, hold=False)
    again = plan.forward()
    gw_again, _ = plan.adjoint(g, with_range=False)
    torch.cuda.synchronize()
    plan.check("fwd")
    plan.check("adj")
    assert torch.equal(again, good)
    assert torch.equal(gw_again, gw_good)
    if prec in ("tf32x3", "fp16x3"):
        assert rel(again.cpu().numpy(), ref) < F32_TOL


def test_adjoint_unit_size_leaves_the_gradient_bit_identical(pb):
    """The single-job tensor-core adjoint derives its unit size on the device from the active
    pairs (20 layers on the clinical field).  A pair's products do not depend on the unit that
    carries it, and the reduce sums in a fixed order, so dL/dW, dL/dR and the loss equal, bit for
    bit, those of explicit unit sizes (4 and 9 layers), with the forward unchanged."""
    import torch
    wl = pb.workloads.build_workload(2)
    prob = pb.model.problem_from_workload(wl)
    m = torch.as_tensor(wl["mask"], device="cuda")
    p = torch.as_tensor(wl["presc"], device="cuda")
    outs = {}
    for sched in (None, (20, 4), (20, 9)):
        plan = pb.engines.DosePlan(prob, tables="device", precision="fp16x3")
        plan.schedule = sched
        o = plan.loss_grad(m, p)
        torch.cuda.synchronize()
        outs[sched] = {k: v.clone() for k, v in o.items() if torch.is_tensor(v)}
    base = outs[None]
    for sched in ((20, 4), (20, 9)):
        for k in ("grad_w", "grad_range", "loss"):
            assert torch.equal(outs[sched][k], base[k]), (sched, k)
