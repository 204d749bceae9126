"""Tensor-core (tcgen05) forward against the float64 oracle, every precision mode.

Tolerances (max |dD| / max D against float64):
  tf32x3, fp16x3:    1e-6   -- the accuracy bound for the split forms
  bf16x3:            5e-5   -- reported; the split with bf16 parts keeps ~16 mantissa bits
  tf32:              5e-3   -- one TF32 product (10-bit mantissa)
  bf16:              5e-2   -- one BF16 product (7-bit mantissa)
"""
import numpy as np
import pytest

from conftest import golden, has_gpu, load_pkg
from oracle import engine_ref as er
from oracle import physics_ref as pr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

TOL = {"tf32x3": 1e-6, "fp16x3": 1e-6, "bf16x3": 5e-5, "tf32": 5e-3, "bf16": 5e-2}


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


@pytest.mark.parametrize("prec", ["tf32x3", "fp16x3", "bf16x3", "tf32", "bf16"])
def test_tc_forward_cfg0(pb, prec):
    wl = pb.workloads.build_workload(0)
    lut = golden("luts_cfg0.npz")
    prob = pb.model.problem_from_workload(wl, lut["energies"], lut["idd"], lut["sigma"])
    d = pb.engines.torch_separable(prob, "cuda", precision=prec).cpu().numpy()
    err = rel(d, golden("dose_cfg0.npz")["dose"])
    print(f"cfg0 {prec}: max_rel_err {err:.3e}")
    assert err < TOL[prec]


@pytest.mark.parametrize("prec", ["tf32x3", "fp16x3", "bf16x3", "tf32", "bf16"])
def test_tc_forward_cfg1(pb, prec):
    wl = pb.workloads.build_workload(1)
    lut = golden("luts_cfg1.npz")
    prob = pb.model.problem_from_workload(wl, lut["energies"], lut["idd"], lut["sigma"])
    d = pb.engines.torch_separable(prob, "cuda", precision=prec).cpu().numpy()
    ref = er.separable_torch(prob.grid.x, prob.grid.y, prob.lattice.spot_x, prob.lattice.spot_y,
                             wl["weights"], lut["idd"], lut["sigma"]).numpy()
    err = rel(d, ref)
    print(f"cfg1 {prec}: max_rel_err {err:.3e}")
    assert err < TOL[prec]


@pytest.mark.parametrize("prec", ["tf32x3", "fp16x3"])
@pytest.mark.parametrize("shape", [(1, 1, 1, 1, 1, 1), (150, 70, 33, 61, 13, 5),
                                   (37, 129, 9, 5, 64, 3), (200, 200, 3, 61, 61, 2),
                                   (128, 96, 12, 51, 41, 70)])
def test_tc_forward_ragged(pb, shape, prec):
    nx, ny, nz, nsx, nsy, nl = shape
    rng = np.random.default_rng(sum(shape) + 1)
    M = pb.model
    grid = M.DoseGrid(nx, ny, nz, 0.15, 0.2, 0.3, -(nx - 1) * 0.075, -(ny - 1) * 0.1, 0.0)
    w = rng.uniform(0.1, 1.0, (nl, nsy, nsx))
    lat = M.SpotLattice(nsx, nsy, nl, 0.25, 0.3, x0=0.07, y0=-0.11, weights=w)
    idd = rng.uniform(0.0, 5.0, (nl, nz))
    idd[rng.random((nl, nz)) < 0.3] = 0.0
    sig = rng.uniform(0.2, 0.8, (nl, nz))
    prob = M.PBProblem(grid, lat, idd, sig)
    d = pb.engines.torch_separable(prob, "cuda", precision=prec).cpu().numpy()
    ref = er.separable_f64(grid.x, grid.y, lat.spot_x, lat.spot_y, w, idd, sig)
    if np.max(np.abs(ref)) == 0:
        assert np.all(d == 0)
    else:
        assert rel(d, ref) < TOL[prec]


def test_tc_rejects_large_lattice(pb):
    M = pb.model
    grid = M.DoseGrid(16, 16, 4, 0.2, 0.2, 0.2)
    lat = M.SpotLattice(65, 3, 1, 0.25, 0.25, weights=np.ones((1, 3, 65)))
    prob = M.PBProblem(grid, lat, np.ones((1, 4)), np.ones((1, 4)))
    with pytest.raises(RuntimeError):
        pb.engines.torch_separable(prob, "cuda", precision="tf32x3")
    d = pb.engines.torch_separable(prob, "cuda", precision="fp32")   # the FP32 path chunks it
    assert d.shape == (4, 16, 16)


@pytest.mark.parametrize("prec", ["tf32x3", "fp16x3"])
def test_tc_loss_grad_and_batch(pb, prec):
    import torch
    wl = pb.workloads.build_workload(0)
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    prob = pb.model.problem_from_workload(wl, energies=en)
    ref_plan = pb.engines.DosePlan(prob, tables="device", precision="fp32")
    tc_plan = pb.engines.DosePlan(prob, tables="device", precision=prec)
    mask, presc = pb.workloads.target_loss_arrays(wl["grid"], half=1.0, shell=1.0, depth=5.0)
    m = torch.as_tensor(mask, device="cuda")
    p = torch.as_tensor(presc * 100.0, device="cuda")
    a = ref_plan.loss_grad(m, p)
    b = tc_plan.loss_grad(m, p)
    assert rel(b["dose"].cpu().numpy(), a["dose"].cpu().numpy()) < 1e-6
    assert rel(b["grad_w"].cpu().numpy(), a["grad_w"].cpu().numpy()) < 1e-5
    scen = [(0, 0, 0, 1.0), (0.3, -0.3, 0.3, 1.035)]
    b32 = pb.robust.ScenarioBatch([prob], scen, precision="fp32")
    btc = pb.robust.ScenarioBatch([prob], scen, precision=prec)
    b32.run()
    btc.run()
    torch.cuda.synchronize()
    for d0, d1 in zip(b32.doses, btc.doses):
        assert rel(d1.cpu().numpy(), d0.cpu().numpy()) < 1e-6


# ----------------------------------------------------------------------- adjoint
def _oracle_grads(prob, w, idd, sig, didd, dsig, mask, presc):
    import torch
    from oracle import engine_ref as er
    wt = torch.tensor(np.asarray(w, np.float64), requires_grad=True)
    it = torch.tensor(np.asarray(idd, np.float64), requires_grad=True)
    st = torch.tensor(np.asarray(sig, np.float64), requires_grad=True)
    d = er.separable_torch(prob.grid.x, prob.grid.y, prob.lattice.spot_x, prob.lattice.spot_y,
                           wt, it, st)
    er.masked_quadratic_loss(d, torch.as_tensor(mask, dtype=torch.float64),
                             torch.as_tensor(presc, dtype=torch.float64)).backward()
    gr = (it.grad.numpy() * didd).sum(1) + (st.grad.numpy() * dsig).sum(1)
    return wt.grad.numpy(), gr


@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3"])
def test_tc_adjoint_cfg0(pb, prec):
    import torch
    wl = pb.workloads.build_workload(0)
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    prob = pb.model.problem_from_workload(wl, energies=en)
    plan = pb.engines.DosePlan(prob, tables="device", precision=prec)
    mask, presc = pb.workloads.target_loss_arrays(wl["grid"], half=1.0, shell=1.0, depth=5.0)
    presc = presc * 100.0
    out = plan.loss_grad(torch.as_tensor(mask, device="cuda"), torch.as_tensor(presc, device="cuda"))
    gw_ref, gr_ref = _oracle_grads(prob, wl["weights"], plan.idd.cpu().numpy(),
                                   plan.sigma.cpu().numpy(), plan.didd.cpu().numpy(),
                                   plan.dsig.cpu().numpy(), mask, presc)
    ew = rel(out["grad_w"].cpu().numpy(), gw_ref)
    er_ = rel(out["grad_range"].cpu().numpy(), gr_ref)
    print(f"cfg0 adjoint {prec}: grad_w {ew:.3e} grad_range {er_:.3e}")
    assert ew < 1e-4 and er_ < 1e-4
    gw2, gr2 = plan.adjoint(out["grad_dose"])
    assert rel(gw2.cpu().numpy(), out["grad_w"].cpu().numpy()) < 1e-6


@pytest.mark.slow
@pytest.mark.parametrize("prec", ["tf32x3", "bf16x3"])
def test_tc_adjoint_clinical(pb, prec):
    import torch
    wl = pb.workloads.build_workload(2)
    lut = golden("luts_cfg1.npz")
    prob = pb.model.problem_from_workload(wl, energies=lut["energies"])
    plan = pb.engines.DosePlan(prob, tables="device", precision=prec)
    out = plan.loss_grad(torch.as_tensor(wl["mask"], device="cuda"),
                         torch.as_tensor(wl["presc"], device="cuda"))
    gw_ref, gr_ref = _oracle_grads(prob, wl["weights"], plan.idd.cpu().numpy(),
                                   plan.sigma.cpu().numpy(), plan.didd.cpu().numpy(),
                                   plan.dsig.cpu().numpy(), wl["mask"], wl["presc"])
    ew = rel(out["grad_w"].cpu().numpy(), gw_ref)
    er_ = rel(out["grad_range"].cpu().numpy(), gr_ref)
    print(f"clinical adjoint {prec}: grad_w {ew:.3e} grad_range {er_:.3e}")
    assert ew < 1e-4 and er_ < 1e-4


def test_tc_adjoint_wide_lattice(pb):
    """51 spots in x (padded to 64): the tensor-core adjoint covers lattices up to 64 x 64
    spots; its dL/dW agrees with the FP32 adjoint within the gradient tolerance."""
    import torch
    M = pb.model
    rng = np.random.default_rng(9)
    grid = M.DoseGrid(64, 64, 24, 0.2, 0.2, 0.25, -6.3, -6.3, 0.0)
    en = pr.layer_energies(3, 3.0, 5.0)
    w = rng.uniform(0.5, 1.5, (3, 11, 51))
    lat = M.SpotLattice(51, 11, 3, 0.25, 0.25, energies=en, weights=w)
    idd, sig = pr.layer_luts(grid.z, en)
    prob = M.PBProblem(grid, lat, idd, sig)
    plan = pb.engines.DosePlan(prob, tables="device", precision="tf32x3")
    g = torch.randn(grid.shape, device="cuda", dtype=torch.float32,
                    generator=torch.Generator(device="cuda").manual_seed(3))
    gw, _ = plan.adjoint(g)
    ref = pb.engines.DosePlan(prob, tables="device", precision="fp32").adjoint(g)[0]
    assert rel(gw.cpu().numpy(), ref.cpu().numpy()) < 1e-4


def test_loss_grad_graph_replay_matches_eager(pb):
    """LossGradGraph: the captured loss gradient, with the weight upload and the result
    download inside the graph, equals an eager call, also after the host weights change; with
    the packed host results (one download for grad_w, grad_range and loss) as well."""
    import torch
    wl = pb.workloads.build_workload(0)
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    prob = pb.model.problem_from_workload(wl, energies=en)
    plan = pb.engines.DosePlan(prob, tables="device", precision="tf32x3")
    mask, presc = pb.workloads.target_loss_arrays(wl["grid"], half=1.0, shell=1.0, depth=5.0)
    m = torch.as_tensor(mask, device="cuda")
    p = torch.as_tensor(presc * 100.0, device="cuda")
    w_host = torch.tensor(wl["weights"], dtype=torch.float32).pin_memory()
    gw_host = torch.empty_like(w_host).pin_memory()
    loss_host = torch.empty((), dtype=torch.float64).pin_memory()
    g = pb.engines.LossGradGraph(plan, m, p, host_w=w_host,
                                 host_out={"grad_w": gw_host, "loss": loss_host})
    # the packed host results: grad_w, grad_range and loss downloaded by one copy
    plan16 = pb.engines.DosePlan(prob, tables="device", precision="fp16x3")
    w16_host = torch.tensor(wl["weights"], dtype=torch.float32).pin_memory()
    hres = plan16.alloc_host_results()
    g16 = pb.engines.LossGradGraph(plan16, m, p, host_w=w16_host, host_out=hres)
    assert len(g16._copies) == 1
    for scale in (1.0, 1.1):
        w_host.mul_(scale)
        w16_host.mul_(scale)
        g.replay()
        g16.replay()
        torch.cuda.synchronize()
        ref = plan.loss_grad(m, p, w=w_host.cuda())
        ref16 = plan16.loss_grad(m, p, w=w16_host.cuda())
        torch.cuda.synchronize()
        assert rel(gw_host.numpy(), ref["grad_w"].cpu().numpy()) == 0.0
        assert float(loss_host) == float(ref["loss"].item())
        assert torch.equal(hres["grad_w"], ref16["grad_w"].cpu())
        assert torch.equal(hres["grad_range"], ref16["grad_range"].cpu())
        assert float(hres["loss"]) == float(ref16["loss"].item())


# ----------------------------------------------------------------------- precision study
# The 200x200x256 / 61x61x60 field (1 mm voxels, 223,260 beams) in every precision mode
# against the float64 oracle fed the reference's own tables (luts_cfg4.npz).  Bounds: FP32
# and TF32x3 at the 1e-6-of-max accuracy bound; the reduced modes pinned at ~5x their measured
# error (BF16x3 2.0e-6, TF32 2.7e-4, BF16 2.1e-3); the FP64 kernel at 1e-12.
CFG4_TOL = {"fp32": 1e-6, "tf32x3": 1e-6, "fp16x3": 1e-6, "bf16x3": 1e-5, "tf32": 1e-3,
            "bf16": 1e-2}


@pytest.fixture(scope="module")
def cfg4(pb):
    wl = pb.workloads.build_workload(4)
    lut = golden("luts_cfg4.npz")
    prob = pb.model.problem_from_workload(wl, lut["energies"], lut["idd"], lut["sigma"])
    g, L = prob.grid, prob.lattice
    ref = er.separable_torch(g.x, g.y, L.spot_x, L.spot_y, wl["weights"], lut["idd"],
                             lut["sigma"], layer_chunk=4).numpy()
    return prob, ref


@pytest.mark.parametrize("prec", ["fp32", "tf32x3", "fp16x3", "bf16x3", "tf32", "bf16"])
def test_precision_study_cfg4(pb, cfg4, prec):
    prob, ref = cfg4
    d = pb.engines.torch_separable(prob, "cuda", precision=prec).cpu().numpy()
    err = rel(d, ref)
    print(f"cfg4 {prec}: max_rel_err {err:.3e}")
    assert err < CFG4_TOL[prec]


def test_float64_kernel_cfg4(pb, cfg4):
    import torch
    prob, ref = cfg4
    d = pb.engines.torch_separable(prob, "cuda", dtype=torch.float64).cpu().numpy()
    err = rel(d, ref)
    print(f"cfg4 float64 kernel: max_rel_err {err:.3e}")
    assert err < 1e-12
