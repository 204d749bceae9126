"""Multi-rank host logic on CPU (gloo, world size 2): depth-slab partition, the one
gradient all-reduce, slab gather, loss gather and the weighted robust reduction.

Each rank stands in for its GPU with the oracle's float64 gradient of its own depth
slab (the quantity the slab's kernels produce); the reduced result must equal the
oracle's gradient of the whole field.  The CUDA side of ``SlabPlan`` is covered by the
GPU tests (``test_gpu_robust.py``), which run all slabs of a field on one device.
"""
import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest

from conftest import load_pkg
from oracle import engine_ref as er
from oracle import physics_ref as pr

H = 0.005


def _case():
    pb = load_pkg()
    wl = pb.workloads.build_workload(0)
    g = wl["grid"]
    z = g["oz"] + np.arange(g["nz"]) * g["dz"]
    x = g["ox"] + np.arange(g["nx"]) * g["dx"]
    y = g["oy"] + np.arange(g["ny"]) * g["dy"]
    xs = (np.arange(wl["n_sx"]) - (wl["n_sx"] - 1) / 2.0) * wl["spot_pitch"]
    ys = (np.arange(wl["n_sy"]) - (wl["n_sy"] - 1) / 2.0) * wl["spot_pitch"]
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    idd, sig = pr.layer_luts(z, en)
    ip, sp = pr.layer_luts(z, en, range_shift=np.full(len(en), H))
    im, sm = pr.layer_luts(z, en, range_shift=np.full(len(en), -H))
    mask, presc = pb.workloads.target_loss_arrays(g, half=1.0, shell=1.0, depth=5.0)
    return dict(pb=pb, wl=wl, x=x, y=y, xs=xs, ys=ys, idd=idd, sig=sig,
                didd=(ip - im) / (2 * H), dsig=(sp - sm) / (2 * H),
                mask=mask.astype(np.float64), presc=presc.astype(np.float64) * 100.0)


def _oracle_grad(c, z0, z1):
    import torch
    w = torch.tensor(c["wl"]["weights"].astype(np.float64), requires_grad=True)
    it = torch.tensor(c["idd"][:, z0:z1], requires_grad=True)
    st = torch.tensor(c["sig"][:, z0:z1], requires_grad=True)
    d = er.separable_torch(c["x"], c["y"], c["xs"], c["ys"], w, it, st)
    loss = er.masked_quadratic_loss(d, torch.tensor(c["mask"][z0:z1]),
                                    torch.tensor(c["presc"][z0:z1]))
    loss.backward()
    gr = ((it.grad * torch.tensor(c["didd"][:, z0:z1])).sum(1)
          + (st.grad * torch.tensor(c["dsig"][:, z0:z1])).sum(1))
    return loss.detach(), w.grad, gr, d.detach()


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        c = _case()
        D = c["pb"].distributed
        bounds = D.slab_bounds((c["idd"] != 0).sum(0), world)
        z0, z1 = bounds[rank]
        loss, gw, gr, dose = _oracle_grad(c, z0, z1)
        L, GW, GR = D.allreduce_gradients(loss, gw.float(), gr.float())
        full = D.gather_slabs(dose, bounds)
        jobs = D.shard_jobs(5, world)
        mine = torch.tensor([10.0 * k for k in jobs[rank]])
        losses = D.gather_losses(mine, [len(j) for j in jobs])
        grads = [torch.full((3,), float(k)) for k in jobs[rank]]
        weights = [1.0 / (1 + k) for k in jobs[rank]]
        rw = D.reduce_weighted(grads, weights)
        torch.save({"bounds": bounds, "loss": L, "grad_w": GW, "grad_range": GR, "dose": full,
                    "losses": losses, "rw": rw}, os.path.join(out_dir, f"rank{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_bounds_partition():
    pb = load_pkg()
    D = pb.distributed
    rng = np.random.default_rng(0)
    for nz, world in [(128, 2), (128, 8), (64, 3), (5, 8), (1, 1), (7, 7)]:
        cost = rng.integers(0, 41, nz)
        b = D.slab_bounds(cost, world)
        assert len(b) == world and b[0][0] == 0 and b[-1][1] == nz
        assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
        assert all(z0 <= z1 for z0, z1 in b)
        if nz >= world:
            assert all(z1 > z0 for z0, z1 in b)
    cost = np.r_[np.full(40, 40.0), np.linspace(40, 0, 88)]
    b = D.slab_bounds(cost, 4)
    per = [cost[z0:z1].sum() for z0, z1 in b]
    assert max(per) - min(per) <= 2 * cost.max()
    with pytest.raises(ValueError):
        D.slab_bounds([1.0, -1.0], 2)
    assert [len(r) for r in D.shard_jobs(100, 8)] == [13] * 4 + [12] * 4
    assert [list(r) for r in D.shard_jobs(2, 3)] == [[0], [1], []]


def test_single_rank_reductions_are_identity():
    import torch
    D = load_pkg().distributed
    gw = torch.arange(6, dtype=torch.float32).reshape(2, 3)
    L, GW, GR = D.allreduce_gradients(torch.tensor(2.5, dtype=torch.float64), gw,
                                      torch.ones(2))
    assert float(L) == 2.5 and torch.equal(GW, gw) and torch.equal(GR, torch.ones(2))
    assert torch.equal(D.gather_slabs(gw, [(0, 2)]), gw)


def test_two_rank_gloo_slab_gradient_matches_full_field():
    import torch
    import torch.multiprocessing as mp
    world = 2
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = [torch.load(os.path.join(out, f"rank{r}.pt")) for r in range(world)]
    c = _case()
    nz = c["idd"].shape[1]
    loss, gw, gr, dose = _oracle_grad(c, 0, nz)
    for r in res:
        assert r["bounds"][0][0] == 0 and r["bounds"][-1][1] == nz
        assert r["bounds"][0][1] > 0 and r["bounds"][0][1] < nz
        assert abs(float(r["loss"]) - float(loss)) <= 1e-12 * abs(float(loss))
        # float32 on the way in and out of the float64 all-reduce
        assert float((r["grad_w"].double() - gw).abs().max() / gw.abs().max()) < 1e-6
        assert float((r["grad_range"].double() - gr).abs().max() / gr.abs().max()) < 1e-6
        assert torch.allclose(r["dose"], dose, rtol=0, atol=1e-12 * float(dose.abs().max()))
        assert torch.equal(r["losses"], torch.tensor([0.0, 10.0, 20.0, 30.0, 40.0],
                                                     dtype=torch.float64))
        expect = sum(k / (1.0 + k) for k in range(5))
        assert torch.allclose(r["rw"], torch.full((3,), expect), rtol=1e-6)
