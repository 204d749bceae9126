"""Heterogeneous media on the device: the WED ray trace against fixtures made with the
reference's own wed_from_density_path and against the oracle; in water the heterogeneous
dose reproduces the homogeneous engine; in a slab phantom (bone and lung slabs) it matches
the float64 oracle (depth dose evaluated at the WED, lateral widths of water).

Tolerances: WED 1e-13 of max; doses 1e-6 of max (FP32 and TF32x3, like the homogeneous
engine)."""
import numpy as np
import pytest

from conftest import golden, has_gpu, load_pkg
from oracle import hetero_ref as hr
from oracle import physics_ref as pr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("case", [0, 1, 2])
def test_wed_raytrace_matches_reference_fixture(pb, case):
    z = golden("hetero.npz")
    rho, want = z[f"rho{case}"], z[f"wed{case}"]
    oz, dz = z[f"grid{case}"]
    grid = {"nz": rho.shape[0], "ny": rho.shape[1], "nx": rho.shape[2], "oz": oz, "dz": dz}
    got = pb.hetero.wed_raytrace(rho, grid).cpu().numpy()
    assert rel(got, want) <= 1e-13


def _cfg0(pb):
    wl = pb.workloads.build_workload(0)
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    return wl, en, pb.model.problem_from_workload(wl, energies=en)


def test_water_reproduces_homogeneous_dose(pb):
    import torch
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    wed = pb.hetero.wed_raytrace(rho, g)
    zc = np.maximum(g.oz + np.arange(g.nz) * g.dz, 0.0)[:, None, None]
    assert np.max(np.abs(wed.cpu().numpy() - zc)) <= 1e-12
    for prec in ("fp32", "tf32x3"):
        plan = pb.hetero.WedPlan(prob, precision=prec)
        d_wed = plan.forward(wed)
        d_ref = pb.engines.DosePlan(prob, tables="device", precision=prec).forward()
        torch.cuda.synchronize()
        assert rel(d_wed.cpu().numpy(), d_ref.cpu().numpy()) < 1e-6, prec
        # a host WED map is uploaded: the same dose
        assert torch.equal(plan.forward(wed.cpu().numpy()), d_wed), prec


def test_slab_phantom_vs_oracle(pb):
    """Bone (1.6) from 2 to 3 cm and lung (0.25) from 4 to 5.4 cm; with a lateral edge."""
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    zc = g.oz + np.arange(g.nz) * g.dz
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    rho[(zc >= 2.0) & (zc < 3.0)] = 1.6
    lung = (zc >= 4.0) & (zc < 5.4)
    rho[lung, :, : g.nx // 2] = 0.25                    # lung only on one side
    wed_ref = hr.wed_ref(rho, g.oz, g.dz)
    sig = pr.layer_luts(zc, en)[1]
    want = hr.dose_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y, wl["weights"], en, sig,
                       wed_ref)
    wed = pb.hetero.wed_raytrace(rho, g)
    assert rel(wed.cpu().numpy(), wed_ref) <= 1e-13
    for prec in ("fp32", "tf32x3"):
        d = pb.hetero.WedPlan(prob, precision=prec).forward(wed).cpu().numpy()
        err = rel(d, want)
        print(f"{prec}: heterogeneous dose max rel err {err:.2e}")
        assert err < 1e-6, prec
    # the slabs move the dose: not the water result
    d_water = pb.engines.DosePlan(prob, tables="device", precision="fp32").forward().cpu().numpy()
    assert rel(d, d_water) > 1e-2


def test_one_shot_entry_point_equals_plan(pb):
    """pbd_forward_wed (curves rebuilt inside its workspace) gives the plan's dose (curves
    built once by pbd_build_wed_curves) bit for bit, call after call, also from a workspace
    whose base is not 256-byte aligned."""
    import ctypes
    import torch
    lib = pb._lib
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    zc = g.oz + np.arange(g.nz) * g.dz
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    rho[(zc >= 1.0) & (zc < 2.5), :, g.nx // 3:] = 0.4
    wed = pb.hetero.wed_raytrace(rho, g)
    plan = pb.hetero.WedPlan(prob, precision="tf32x3")
    a = plan.forward(wed).clone()
    b = plan.forward(wed).clone()
    out = torch.empty_like(a)
    lib.call("pbd_forward_wed", ctypes.byref(plan.field), ctypes.byref(plan.spec),
             lib.ptr(plan.energies), None, lib.ptr(plan.w), lib.ptr(plan.sigma), lib.ptr(wed),
             lib.ptr(out), plan.precision, lib.ptr(plan.ws), plan.ws.numel(),
             lib.stream_handle(plan.device))
    torch.cuda.synchronize()
    assert torch.equal(a, b) and torch.equal(a, out)
    # a workspace whose base is only 8-byte aligned: the library aligns its sub-arrays itself
    need = plan.ws.numel()
    raw = torch.empty(need + 64, dtype=torch.uint8, device=plan.device)
    out2 = torch.empty_like(a)
    lib.call("pbd_forward_wed", ctypes.byref(plan.field), ctypes.byref(plan.spec),
             lib.ptr(plan.energies), None, lib.ptr(plan.w), lib.ptr(plan.sigma), lib.ptr(wed),
             lib.ptr(out2), plan.precision, ctypes.c_void_p(raw.data_ptr() + 8), need,
             lib.stream_handle(plan.device))
    torch.cuda.synchronize()
    assert torch.equal(a, out2)


def test_ragged_grid_random_medium_vs_oracle(pb):
    """A 29 x 23 x 37 grid (24,679 voxels: the last 1024-voxel tile holds 103, not a multiple
    of 4) in a random medium (rho 0.2 to 2.0) that takes some voxels past every layer's range."""
    wl = dict(pb.workloads.build_workload(0))
    nx, ny, nz = 29, 23, 37
    wl["grid"] = {"nx": nx, "ny": ny, "nz": nz, "dx": 0.15, "dy": 0.2, "dz": 0.3,
                  "ox": -(nx - 1) * 0.075, "oy": -(ny - 1) * 0.1, "oz": 0.0}
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    prob = pb.model.problem_from_workload(wl, energies=en)
    g = prob.grid
    rng = np.random.default_rng(29)
    rho = rng.uniform(0.2, 2.0, (nz, ny, nx)).astype(np.float32)
    zc = g.oz + np.arange(g.nz) * g.dz
    wed_ref = hr.wed_ref(rho, g.oz, g.dz)
    sig = pr.layer_luts(zc, en)[1]
    want = hr.dose_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y, wl["weights"], en, sig,
                       wed_ref)
    wed = pb.hetero.wed_raytrace(rho, g)
    assert rel(wed.cpu().numpy(), wed_ref) <= 1e-13
    assert wed_ref.max() > 1.2 * wl["r_max"]               # past every layer's range
    for prec in ("fp32", "tf32x3"):
        d = pb.hetero.WedPlan(prob, precision=prec).forward(wed).cpu().numpy()
        err = rel(d, want)
        print(f"ragged {prec}: heterogeneous dose max rel err {err:.2e}")
        assert err < 1e-6, prec


def test_nan_and_out_of_range_wed(pb):
    """A NaN WED gives a NaN dose at that voxel only (np.interp propagates NaN); the other
    voxels -- the NaN's tile included, which then streams every layer -- keep their values bit
    for bit.  WED maps beyond every layer's curve, or negative, give a dose of exactly 0 (no
    (layer, slice) is active, nothing is written or read)."""
    import torch
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    wed = pb.hetero.wed_raytrace(np.ones((g.nz, g.ny, g.nx), dtype=np.float32), g)
    plan = pb.hetero.WedPlan(prob, precision="tf32x3")
    base = plan.forward(wed).clone()
    w2 = wed.clone()
    w2[5, 3, 4] = float("nan")
    d = plan.forward(w2)
    torch.cuda.synchronize()
    nan = torch.isnan(d)
    assert nan.sum().item() == 1 and bool(nan[5, 3, 4])
    keep = ~nan
    assert torch.equal(d[keep], base[keep])
    for fill in (1e3, -1.0):
        z = plan.forward(torch.full_like(wed, fill))
        torch.cuda.synchronize()
        assert torch.count_nonzero(z).item() == 0, fill


def test_gradient_vs_oracle(pb):
    """dL/dW of the heterogeneous dose (pbd_adjoint_wed) for a random dL/dD in the slab
    phantom against float64 autograd through the oracle's dose.  Tolerance 1e-4 of max
    (the adjoint's split-BF16 products); with a positive dL/dD, sum(dL/dW * W) equals
    <dL/dD, D> (D is linear in W) to 1e-5."""
    import torch
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    zc = g.oz + np.arange(g.nz) * g.dz
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    rho[(zc >= 2.0) & (zc < 3.0)] = 1.6
    rho[(zc >= 4.0) & (zc < 5.4), :, : g.nx // 2] = 0.25
    wed_np = hr.wed_ref(rho, g.oz, g.dz)
    sig = pr.layer_luts(zc, en)[1]
    rng = np.random.default_rng(3)
    grad = rng.standard_normal((g.nz, g.ny, g.nx)).astype(np.float32)
    want = hr.grad_w_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y, wl["weights"], en,
                         sig, wed_np, grad.astype(np.float64))
    wed = pb.hetero.wed_raytrace(rho, g)
    pos = np.abs(grad) + 0.1
    for prec in ("fp32", "tf32x3", "fp16x3"):
        plan = pb.hetero.WedPlan(prob, precision=prec)
        got = plan.adjoint(torch.as_tensor(grad, device="cuda"), wed).cpu().numpy()
        err = rel(got, want)
        print(f"{prec}: heterogeneous dL/dW max rel err {err:.2e}")
        assert err < 1e-4, prec
        d = plan.forward(wed).double().cpu().numpy()
        gp = plan.adjoint(torch.as_tensor(pos, device="cuda"), wed).double().cpu().numpy()
        lhs = float(np.sum(gp * wl["weights"]))
        rhs = float(np.sum(pos * d))
        assert abs(lhs - rhs) <= 1e-5 * abs(rhs), (prec, lhs, rhs)


def _slab(g):
    zc = g.oz + np.arange(g.nz) * g.dz
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    rho[(zc >= 2.0) & (zc < 3.0)] = 1.6
    rho[(zc >= 4.0) & (zc < 5.4), :, : g.nx // 2] = 0.25
    return zc, rho


def test_range_gradient_vs_oracle(pb):
    """dL/dW and dL/d(range shift) of the heterogeneous dose in one call
    (pbd_adjoint_wed_range) for a random dL/dD in the slab phantom, against the oracle: dL/dW
    by float64 autograd, dL/dR by the chain rule through the central differences at +-h of the
    depth curves (at the WED) and of the widths (float64, autograd for the widths' part).
    Tolerance 1e-4 of max for both (the adjoint's split-BF16 products; FP32 well inside)."""
    import torch
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    zc, rho = _slab(g)
    wed_np = hr.wed_ref(rho, g.oz, g.dz)
    rng = np.random.default_rng(5)
    grad = rng.standard_normal((g.nz, g.ny, g.nx)).astype(np.float32)
    h = 0.005
    want_r = hr.grad_range_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y, wl["weights"],
                               en, zc, wed_np, grad.astype(np.float64), h)
    sig = pr.layer_luts(zc, en)[1]
    want_w = hr.grad_w_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y, wl["weights"], en,
                           sig, wed_np, grad.astype(np.float64))
    wed = pb.hetero.wed_raytrace(rho, g)
    for prec in ("fp32", "tf32x3", "fp16x3"):
        plan = pb.hetero.WedPlan(prob, precision=prec, fd_step=h)
        gw, gr = plan.adjoint(torch.as_tensor(grad, device="cuda"), wed, with_range=True)
        ew, er_ = rel(gw.cpu().numpy(), want_w), rel(gr.cpu().numpy(), want_r)
        print(f"{prec}: heterogeneous dL/dW {ew:.2e}, dL/dR {er_:.2e} of max")
        assert ew < 1e-4, prec
        assert er_ < 1e-4, prec
        # the dL/dW of the range call equals the plain adjoint's
        gw1 = plan.adjoint(torch.as_tensor(grad, device="cuda"), wed)
        assert torch.equal(gw, gw1), prec


def test_range_gradient_in_water_equals_homogeneous(pb):
    """In water (rho = 1, WED = depth) the heterogeneous dL/dR equals the homogeneous
    adjoint's dL/dR through the depth tables' range derivatives (the same central differences
    at the grid depths): 1e-4 of max, and dL/dW likewise."""
    import torch
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    wed = pb.hetero.wed_raytrace(rho, g)
    grad = torch.as_tensor(np.random.default_rng(6).standard_normal((g.nz, g.ny, g.nx)),
                           dtype=torch.float32, device="cuda")
    for prec in ("fp32", "tf32x3"):
        hp = pb.hetero.WedPlan(prob, precision=prec, fd_step=0.005)
        gw, gr = hp.adjoint(grad, wed, with_range=True)
        dp = pb.engines.DosePlan(prob, tables="device", precision=prec, fd_step=0.005)
        gw0, gr0 = dp.adjoint(grad, with_range=True)
        torch.cuda.synchronize()
        assert rel(gw.cpu().numpy(), gw0.cpu().numpy()) < 1e-4, prec
        assert rel(gr.cpu().numpy(), gr0.cpu().numpy()) < 1e-4, prec
