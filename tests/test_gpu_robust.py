"""Fields x scenarios: batched forward (direct and partial-slice modes), the per-job
loop, and per-job loss gradients with CUDA-graph replay, against the float64 oracle.

Tolerances (max |d| / max |ref| against float64): doses 1e-5 for fp32 and 1e-6 for
tf32x3 batches; grad_w and grad_range 1e-5 (fp32 adjoint, float32 accumulation).
"""
import numpy as np
import pytest

from conftest import has_gpu, load_pkg
from oracle import engine_ref as er
from oracle import physics_ref as pr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

DOSE_TOL = {"fp32": 1e-5, "tf32x3": 1e-6}
GRAD_TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


def _fields(pb):
    """An 11x11x8 field and a ragged 9x13 field of 70 layers (more than one 64-layer chunk
    per slice, so the batch takes its partial-slice path) on one 32x32x64 grid."""
    a = pb.workloads.build_workload(0)
    rng = np.random.default_rng(7)
    b = pb.workloads._base(a["grid"], 9, 13, 70, 0.45, 3.0, 10.0,
                           rng.uniform(0.5, 1.5, (70, 13, 9)), "32x32x64 / 9x13x70")
    out = []
    for wl in (a, b):
        en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
        out.append((wl, en, pb.model.problem_from_workload(wl, energies=en)))
    return out


SCEN = [(0.0, 0.0, 0.0, 1.0), (0.3, -0.3, 0.3, 1.035), (-0.3, 0.0, -0.3, 0.965)]


def _oracle_dose(prob, wl, en, s):
    g = prob.grid
    sx, sy, sz, sc = s
    idd, sig = pr.scenario_luts(g.oz - sz, g.dz, g.nz, en, depth_scale=sc)
    return er.separable_f64(g.x, g.y, prob.lattice.spot_x + sx, prob.lattice.spot_y + sy,
                            wl["weights"], idd, sig)


@pytest.mark.parametrize("prec", ["fp32", "tf32x3"])
def test_batch_two_fields_vs_oracle_and_loop(pb, prec):
    import torch
    fields = _fields(pb)
    b = pb.robust.ScenarioBatch([p for _, _, p in fields], SCEN, precision=prec)
    b.run()
    loop = b.loop_forward(prec)
    torch.cuda.synchronize()
    for k in range(b.n_jobs):
        wl, en, prob = fields[k // len(SCEN)]
        ref = _oracle_dose(prob, wl, en, SCEN[k % len(SCEN)])
        err = rel(b.doses[k].cpu().numpy(), ref)
        print(f"{prec} job {k}: batch max_rel_err {err:.3e}")
        assert err < DOSE_TOL[prec]
        assert rel(loop[k].cpu().numpy(), ref) < DOSE_TOL[prec]


def test_batch_gradients_vs_oracle_and_graph_replay(pb):
    import torch
    wl, en, prob = _fields(pb)[0]
    b = pb.robust.ScenarioBatch([prob], SCEN, precision="fp32", with_grad=True)
    mask, presc = pb.workloads.target_loss_arrays(wl["grid"], half=1.0, shell=1.0, depth=5.0)
    m = torch.as_tensor(mask, device="cuda")
    p = torch.as_tensor(presc * 100.0, device="cuda")
    outs = b.loss_grad_all(m, p)
    torch.cuda.synchronize()
    eager = [{k: v.clone() for k, v in o.items()} for o in outs]
    g = prob.grid
    for k, s in enumerate(SCEN):
        sx, sy, sz, sc = s
        t = b.tables[k]
        wt = torch.tensor(wl["weights"].astype(np.float64), requires_grad=True)
        it = torch.tensor(t.idd.cpu().numpy(), requires_grad=True)
        st = torch.tensor(t.sigma.cpu().numpy(), requires_grad=True)
        d = er.separable_torch(g.x, g.y, prob.lattice.spot_x + sx, prob.lattice.spot_y + sy,
                               wt, it, st)
        loss = er.masked_quadratic_loss(d, torch.as_tensor(mask, dtype=torch.float64),
                                        torch.as_tensor(presc * 100.0, dtype=torch.float64))
        loss.backward()
        gr = ((it.grad * t.didd_dr.cpu().double()).sum(1)
              + (st.grad * t.dsigma_dr.cpu().double()).sum(1)).numpy()
        o = eager[k]
        assert abs(float(o["loss"]) - float(loss)) / abs(float(loss)) < GRAD_TOL
        assert rel(o["grad_w"].cpu().numpy(), wt.grad.numpy()) < GRAD_TOL
        assert rel(o["grad_range"].cpu().numpy(), gr) < GRAD_TOL
    b.capture_loss_grad(m, p)
    b.replay_loss_grad()
    torch.cuda.synchronize()
    for o0, o1 in zip(eager, b.grad_outputs):
        for key in ("loss", "grad_w", "grad_range", "grad_dose"):
            assert torch.equal(o0[key], o1[key]), key


def test_batched_loss_grad_vs_per_job_and_oracle(pb):
    """pbd_loss_grad_batch (all forwards in one launch, all adjoints in another) on two
    fields x three scenarios -- the 70-layer field takes the chunked forward -- against the
    per-job tensor-core calls and the float64 oracle; graph replay equals the eager call.
    Tolerances: loss 1e-6 relative, grad_w / grad_range 1e-4 of max (split-BF16 adjoint)."""
    import torch
    fields = _fields(pb)
    probs = [p for _, _, p in fields]
    mask, presc = pb.workloads.target_loss_arrays(fields[0][0]["grid"], half=1.0, shell=1.0,
                                                  depth=5.0)
    m = torch.as_tensor(mask, device="cuda")
    p = torch.as_tensor(presc * 100.0, device="cuda")
    b = pb.robust.ScenarioBatch(probs, SCEN, precision="tf32x3", with_grad=True)
    per = [{k: v.clone() for k, v in o.items()} for o in b.loss_grad_all(m, p, batched=False)]
    outs = b.loss_grad_all(m, p, batched=True)
    torch.cuda.synchronize()
    bat = [{k: v.clone() for k, v in o.items()} for o in outs]
    g = probs[0].grid
    for k in range(b.n_jobs):
        wl, en, prob = fields[k // len(SCEN)]
        sx, sy, sz, sc = SCEN[k % len(SCEN)]
        o, q = bat[k], per[k]
        assert abs(float(o["loss"]) - float(q["loss"])) <= 1e-6 * abs(float(q["loss"])), k
        assert rel(o["grad_w"].cpu().numpy(), q["grad_w"].cpu().numpy()) < 1e-4, k
        assert rel(o["grad_range"].cpu().numpy(), q["grad_range"].cpu().numpy()) < 1e-4, k
        t = b.tables[k]
        wt = torch.tensor(wl["weights"].astype(np.float64), requires_grad=True)
        it = torch.tensor(t.idd.cpu().numpy(), requires_grad=True)
        st = torch.tensor(t.sigma.cpu().numpy(), requires_grad=True)
        d = er.separable_torch(g.x, g.y, prob.lattice.spot_x + sx, prob.lattice.spot_y + sy,
                               wt, it, st)
        loss = er.masked_quadratic_loss(d, torch.as_tensor(mask, dtype=torch.float64),
                                        torch.as_tensor(presc * 100.0, dtype=torch.float64))
        loss.backward()
        gr = ((it.grad * t.didd_dr.cpu().double()).sum(1)
              + (st.grad * t.dsigma_dr.cpu().double()).sum(1)).numpy()
        print(f"job {k}: loss rel {abs(float(o['loss']) - float(loss)) / float(loss):.2e}, "
              f"grad_w {rel(o['grad_w'].cpu().numpy(), wt.grad.numpy()):.2e}")
        assert abs(float(o["loss"]) - float(loss)) <= 1e-6 * abs(float(loss)), k
        assert rel(o["grad_w"].cpu().numpy(), wt.grad.numpy()) < 1e-4, k
        assert rel(o["grad_range"].cpu().numpy(), gr) < 1e-4, k
    b.capture_loss_grad(m, p)
    b.replay_loss_grad()
    torch.cuda.synchronize()
    for o0, o1 in zip(bat, b.grad_outputs):
        for key in ("loss", "grad_w", "grad_range", "grad_dose"):
            assert torch.equal(o0[key], o1[key]), key


def test_batch_without_grad_tables_refuses_gradients(pb):
    import torch
    _, _, prob = _fields(pb)[0]
    b = pb.robust.ScenarioBatch([prob], SCEN[:1])
    z = torch.zeros((prob.grid.nz, prob.grid.ny, prob.grid.nx), device="cuda")
    with pytest.raises(RuntimeError):
        b.loss_grad_all(z, z)


@pytest.mark.parametrize("world", [2, 3])
def test_slab_plans_sum_to_full_field(pb, world):
    """Every depth slab of one field, run one after another on this device (no process
    group: ``reduce=False``), sums to the single-plan loss and gradients."""
    import torch
    wl, en, prob = _fields(pb)[0]
    mask, presc = pb.workloads.target_loss_arrays(wl["grid"], half=1.0, shell=1.0, depth=5.0)
    m = torch.as_tensor(mask, device="cuda")
    p = torch.as_tensor(presc * 100.0, device="cuda")
    full = pb.engines.DosePlan(prob, tables="device", precision="fp32").loss_grad(m, p)
    parts = [pb.distributed.SlabPlan(prob, rank=r, world=world, precision="fp32")
             for r in range(world)]
    assert [s.bounds[r] for r, s in enumerate(parts)] == parts[0].bounds
    outs = [s.loss_grad(m, p, reduce=False) for s in parts]
    dose = torch.cat([s.forward() for s in parts])
    torch.cuda.synchronize()
    loss = sum(float(o[0]) for o in outs)
    gw = sum(o[1].double() for o in outs)
    gr = sum(o[2].double() for o in outs)
    assert abs(loss - float(full["loss"])) / abs(float(full["loss"])) < 1e-6
    assert rel(gw.cpu().numpy(), full["grad_w"].cpu().numpy()) < 1e-5
    assert rel(gr.cpu().numpy(), full["grad_range"].cpu().numpy()) < 1e-5
    assert rel(dose.cpu().numpy(), full["dose"].cpu().numpy()) < 1e-6
    with pytest.raises(RuntimeError):
        parts[0].loss_grad(m, p)       # world > 1 without a process group


# ------------------------------------------------------------- the full robust workload
# 4 uneven fields (21x21x16, 33x33x28, 41x41x40, 51x41x48 spots x layers) x 25 scenarios on
# 128^3 voxels: the batched forward (one persistent launch) and the batched loss gradient
# (one forward + one adjoint launch for all 100 jobs), every job against the float64 oracle.
# * Tables: every distinct (depth shift, range scaling) pair of every field, built on the
#   device, against the oracle's scenario tables: 1e-9 of max.
# * Dose: each job's dose on 8 depth slices (including the slice of its maximum) against the
#   oracle's separable sum fed the job's own tables: 1e-6 of max (TF32x3).
# * Gradients: each job's loss, dL/dW and dL/dR against float64 autograd through the
#   oracle's torch engine: loss 1e-6 relative, dL/dW and dL/dR 1e-4 of max (split-BF16
#   adjoint).
CFG3_SLICES = (0, 17, 40, 63, 85, 100, 127)


@pytest.fixture(scope="module")
def cfg3(pb):
    import torch
    fields = pb.workloads.robust_fields()
    scen = pb.workloads.robust_scenarios()
    probs = pb.robust.robust_problems(fields)
    b = pb.robust.ScenarioBatch(probs, scen, precision="tf32x3", with_grad=True)
    b.run()
    g = fields[0]["grid"]
    m_np, p_np = pb.workloads.target_loss_arrays(g)
    m = torch.as_tensor(m_np, device="cuda")
    p = torch.as_tensor(p_np, device="cuda")
    outs = b.loss_grad_all(m, p)
    torch.cuda.synchronize()
    doses = [d.cpu().numpy() for d in b.doses]
    grads = [{k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in o.items()}
             for o in outs]
    return fields, scen, probs, b, doses, grads, m_np, p_np


def test_cfg3_tables_vs_oracle(pb, cfg3):
    fields, scen, probs, b, *_ = cfg3
    seen = set()
    for k in range(b.n_jobs):
        fi, si = divmod(k, len(scen))
        sx, sy, sz, sc = scen[si]
        if (fi, sz, sc) in seen:
            continue
        seen.add((fi, sz, sc))
        g = probs[fi].grid
        en = probs[fi].lattice.energies
        idd, sig = pr.scenario_luts(g.oz - sz, g.dz, g.nz, en, depth_scale=sc)
        t = b.tables[k]
        assert rel(t.idd.cpu().numpy(), idd) < 1e-9, (fi, sz, sc)
        assert rel(t.sigma.cpu().numpy(), sig) < 1e-9, (fi, sz, sc)
    assert len(seen) == 4 * 9


def test_cfg3_doses_vs_oracle(pb, cfg3):
    fields, scen, probs, b, doses, *_ = cfg3
    worst = 0.0
    for k in range(b.n_jobs):
        fi, si = divmod(k, len(scen))
        sx, sy, sz, sc = scen[si]
        prob, t, d = probs[fi], b.tables[k], doses[k]
        g, L = prob.grid, prob.lattice
        zs = sorted(set(CFG3_SLICES) | {int(np.argmax(d.reshape(g.nz, -1).max(axis=1)))})
        idd = t.idd.cpu().numpy()[:, zs]
        sig = t.sigma.cpu().numpy()[:, zs]
        ref = er.separable_f64(g.x, g.y, L.spot_x + sx, L.spot_y + sy, fields[fi]["weights"],
                               idd, sig)
        err = float(np.max(np.abs(d[zs] - ref)) / np.max(np.abs(ref)))
        worst = max(worst, err)
        assert err < DOSE_TOL["tf32x3"], (k, err)
    print(f"cfg3: worst dose error over 100 jobs {worst:.2e}")


def test_cfg3_gradients_vs_oracle(pb, cfg3):
    import torch
    fields, scen, probs, b, doses, grads, m_np, p_np = cfg3
    mask = torch.as_tensor(m_np, dtype=torch.float64)
    presc = torch.as_tensor(p_np, dtype=torch.float64)
    worst = [0.0, 0.0, 0.0]
    for k in range(b.n_jobs):
        fi, si = divmod(k, len(scen))
        sx, sy, sz, sc = scen[si]
        prob, t, o = probs[fi], b.tables[k], grads[k]
        g, L = prob.grid, prob.lattice
        wt = torch.tensor(fields[fi]["weights"].astype(np.float64), requires_grad=True)
        it = torch.tensor(t.idd.cpu().numpy(), requires_grad=True)
        st = torch.tensor(t.sigma.cpu().numpy(), requires_grad=True)
        d = er.separable_torch(g.x, g.y, L.spot_x + sx, L.spot_y + sy, wt, it, st)
        loss = er.masked_quadratic_loss(d, mask, presc)
        loss.backward()
        gr = ((it.grad * t.didd_dr.cpu().double()).sum(1)
              + (st.grad * t.dsigma_dr.cpu().double()).sum(1)).numpy()
        e = (abs(float(o["loss"]) - float(loss)) / abs(float(loss)),
             rel(o["grad_w"], wt.grad.numpy()), rel(o["grad_range"], gr))
        worst = [max(a, c) for a, c in zip(worst, e)]
        assert e[0] <= 1e-6, (k, e)
        assert e[1] < 1e-4, (k, e)
        assert e[2] < 1e-4, (k, e)
    print(f"cfg3: worst loss / dL/dW / dL/dR errors over 100 jobs {worst}")
