"""On-device plan optimisation: the projected Adam step and the scenario combination
against the oracle (bit for bit: both are FP32 with every operation rounded separately),
graph replay against eager iterations (bit for bit: the library is deterministic), the
nominal weight trajectory against the oracle's float64-gradient Adam loop, range-shift
optimisation with the tables rebuilt inside the graph, and the robust min-max / mean loop.

Tolerances: Adam step and combination exact; trajectory of 12 steps (FP32 adjoint gradient
vs float64 autograd, relative error ~1e-6) within 1e-5 relative on the loss history and
5e-5 absolute on the weights (lr 0.02, weights ~1).
"""
import math

import numpy as np
import pytest

from conftest import has_gpu, load_pkg
from oracle import optim_ref as orf
from oracle import physics_ref as pr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


def _adam_call(pb, cfg, x, m, v, g, state, x64=None, loss=None, hist=None):
    import ctypes
    _lib = pb._lib
    p = cfg.params()
    _lib.call("pbd_adam_step", ctypes.byref(p), int(x.numel()), _lib.ptr(x), _lib.ptr(m),
              _lib.ptr(v), _lib.ptr(g), _lib.ptr(state), _lib.ptr(x64), _lib.ptr(loss),
              _lib.ptr(hist), 0 if hist is None else int(hist.numel()), _lib.stream_handle())


@pytest.mark.parametrize("n", [1, 1023, 10007])
def test_adam_step_bit_exact_vs_oracle(pb, n):
    import torch
    rng = np.random.default_rng(n)
    cfg = pb.optimize.Adam(lr=0.03, beta1=0.85, beta2=0.995, eps=1e-7, lo=0.1, hi=1.8,
                           grad_scale=0.5)
    x0 = rng.uniform(0.0, 2.0, n).astype(np.float32)
    x = torch.tensor(x0, device="cuda")
    m = torch.zeros_like(x)
    v = torch.zeros_like(x)
    x64 = torch.zeros(n, dtype=torch.float64, device="cuda")
    state = torch.zeros(2, dtype=torch.int32, device="cuda")
    hist = torch.zeros(8, dtype=torch.float64, device="cuda")
    xr, mr, vr = x0.copy(), np.zeros(n, np.float32), np.zeros(n, np.float32)
    kw = dict(lr=cfg.lr, beta1=cfg.beta1, beta2=cfg.beta2, eps=cfg.eps, lo=cfg.lo, hi=cfg.hi,
              grad_scale=cfg.grad_scale)
    losses = []
    for t in range(1, 6):
        g = (rng.standard_normal(n) * 10.0 ** rng.integers(-20, 4, n)).astype(np.float32)
        g[rng.random(n) < 0.05] = 0.0
        loss = torch.tensor(float(rng.uniform(1, 2)), dtype=torch.float64, device="cuda")
        losses.append(float(loss))
        _adam_call(pb, cfg, x, m, v, torch.tensor(g, device="cuda"), state, x64, loss, hist)
        xr, mr, vr = orf.adam_step(xr, mr, vr, g, t, **kw)
    torch.cuda.synchronize()
    assert np.array_equal(x.cpu().numpy(), xr)
    assert np.array_equal(m.cpu().numpy(), mr)
    assert np.array_equal(v.cpu().numpy(), vr)
    assert np.array_equal(x64.cpu().numpy(), xr.astype(np.float64))
    assert state.cpu().tolist() == [5, 0]
    assert hist.cpu().numpy()[:5].tolist() == losses
    assert np.all(hist.cpu().numpy()[5:] == 0.0)


def test_adam_step_unbounded_box_and_zero_length(pb):
    import torch
    cfg = pb.optimize.Adam(lr=0.1, lo=-math.inf, hi=math.inf)
    x = torch.tensor([-5.0, 0.0, 5.0], device="cuda")
    m, v = torch.zeros_like(x), torch.zeros_like(x)
    state = torch.zeros(2, dtype=torch.int32, device="cuda")
    g = torch.tensor([1.0, -1.0, 0.0], device="cuda")
    _adam_call(pb, cfg, x, m, v, g, state)
    e = torch.empty(0, device="cuda")
    _adam_call(pb, cfg, e, e, e, e, state)          # n = 0: nothing launched
    torch.cuda.synchronize()
    xr, _, _ = orf.adam_step([-5.0, 0.0, 5.0], [0, 0, 0], [0, 0, 0], [1.0, -1.0, 0.0], 1,
                             lr=0.1, lo=-np.inf, hi=np.inf)
    assert np.array_equal(x.cpu().numpy(), xr)
    assert state.cpu().tolist() == [1, 0]


@pytest.mark.parametrize("mode", ["mean", "max"])
def test_scenario_combine_vs_oracle(pb, mode):
    import torch
    _lib = pb._lib
    rng = np.random.default_rng(3)
    s_n, n = 5, 3001
    grads = rng.standard_normal((s_n, n)).astype(np.float32)
    losses = np.array([1.0, 3.5, 2.0, 3.5, 0.5])      # tie: scenario 1 is the first maximum
    gd = torch.tensor(grads, device="cuda")
    ld = torch.tensor(losses, device="cuda")
    out = torch.empty(n, device="cuda")
    out_loss = torch.zeros((), dtype=torch.float64, device="cuda")
    _lib.call("pbd_scenario_combine", _lib.OBJ[mode], s_n, n, _lib.ptr(gd), _lib.ptr(ld),
              _lib.ptr(out), _lib.ptr(out_loss), _lib.stream_handle())
    torch.cuda.synchronize()
    gr, lr_ = orf.scenario_combine(mode, grads, losses)
    assert np.array_equal(out.cpu().numpy(), gr)
    assert float(out_loss) == lr_
    if mode == "max":
        assert np.array_equal(out.cpu().numpy(), grads[1])


def _cfg0(pb, precision="fp32"):
    import torch
    wl = pb.workloads.build_workload(0)
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    prob = pb.model.problem_from_workload(wl, energies=en)
    mask, presc = pb.workloads.target_loss_arrays(wl["grid"], half=1.0, shell=1.0, depth=5.0)
    m = torch.as_tensor(mask, device="cuda")
    p = torch.as_tensor(presc * 100.0, device="cuda")
    return wl, prob, m, p, mask, presc * 100.0


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_plan_optimizer_graph_equals_eager(pb, precision):
    import torch
    wl, prob, m, p, _, _ = _cfg0(pb)
    runs = []
    for graph in (False, True):
        plan = pb.engines.DosePlan(prob, tables="device", precision=precision)
        opt = pb.optimize.PlanOptimizer(plan, m, p, adam=pb.optimize.Adam(lr=0.02),
                                        max_iter=16, graph=graph)
        h = opt.run(10)
        runs.append((h, plan.w.cpu().numpy()))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    h = runs[0][0]
    assert h.shape == (10,) and h[-1] < 0.8 * h[0]


def test_plan_optimizer_trajectory_vs_oracle(pb):
    import torch
    wl, prob, m, p, mask, presc = _cfg0(pb)
    plan = pb.engines.DosePlan(prob, tables="device", precision="fp32")
    idd = plan.idd.cpu().numpy()
    sig = plan.sigma.cpu().numpy()
    w0 = plan.w.cpu().numpy().copy()
    opt = pb.optimize.PlanOptimizer(plan, m, p, adam=pb.optimize.Adam(lr=0.02), max_iter=12)
    h = opt.run(12)
    g = prob.grid
    w_ref, h_ref = orf.optimize_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y, w0, idd,
                                    sig, mask, presc, 12, lr=0.02, lo=0.0)
    rel_h = np.max(np.abs(h - h_ref) / np.abs(h_ref))
    dw = np.max(np.abs(plan.w.cpu().numpy() - w_ref))
    print(f"loss history max rel {rel_h:.2e}; weights max abs diff {dw:.2e}")
    assert rel_h < 1e-5
    assert dw < 5e-5


def test_plan_optimizer_range_shifts(pb):
    """Weights and per-layer range shifts together: the tables are rebuilt inside the graph;
    graph and eager runs agree exactly, the loss falls, the shifts stay in their box, and
    the final tables equal a fresh device build at the final shifts."""
    import torch
    wl, prob, m, p, _, _ = _cfg0(pb)
    runs = []
    for graph in (False, True):
        plan = pb.engines.DosePlan(prob, tables="device", precision="fp32")
        opt = pb.optimize.PlanOptimizer(
            plan, m, p, adam=pb.optimize.Adam(lr=0.02),
            range_adam=pb.optimize.Adam(lr=0.02, lo=-0.3, hi=0.3), max_iter=8, graph=graph)
        h = opt.run(8)
        runs.append((h, plan.w.cpu().numpy(), opt.range_shift.cpu().numpy(),
                     opt.range_shift64.cpu().numpy(), plan, opt))
    for a, b in zip(runs[0][:4], runs[1][:4]):
        assert np.array_equal(a, b)
    h, _, rs, rs64, plan, opt = runs[1]
    assert h[-1] < h[0]
    assert np.all(np.abs(rs) <= 0.3) and np.any(rs != 0.0)
    assert np.array_equal(rs64, rs.astype(np.float64))
    # the graph leaves the tables at the shifts of the last gradient evaluation; rebuild
    # once more at the final shifts and compare with a fresh build
    opt.builder.build(opt.range_shift64)
    g = prob.grid
    t = pb.physics.build_tables(g.nz, g.oz, g.dz, plan.energies, range_shift=opt.range_shift64,
                                fd_step=plan.fd_step)
    torch.cuda.synchronize()
    assert torch.equal(t.idd, plan.idd) and torch.equal(t.sigma, plan.sigma)
    assert torch.equal(t.didd_dr, plan.didd) and torch.equal(t.dsigma_dr, plan.dsig)


@pytest.mark.parametrize("objective", ["max", "mean"])
def test_robust_optimizer(pb, objective):
    import torch
    wl, prob, m, p, _, _ = _cfg0(pb)
    scen = [(0.0, 0.0, 0.0, 1.0), (0.3, -0.3, 0.3, 1.035), (-0.3, 0.0, -0.3, 0.965)]
    runs = []
    for graph in (False, True):
        b = pb.robust.ScenarioBatch([prob], scen, precision="fp32", with_grad=True)
        first = [float(o["loss"]) for o in b.loss_grad_all(m, p)]
        opt = pb.optimize.RobustOptimizer(b, m, p, objective=objective,
                                          adam=pb.optimize.Adam(lr=0.02), max_iter=8, graph=graph)
        h = opt.run(8)
        runs.append((h, b.weights[0].cpu().numpy(), first))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    h, _, first = runs[0]
    want = max(first) if objective == "max" else sum(first) / len(first)
    assert h.shape == (1, 8)
    assert h[0, 0] == pytest.approx(want, rel=1e-12)
    assert h[0, -1] < h[0, 0]
