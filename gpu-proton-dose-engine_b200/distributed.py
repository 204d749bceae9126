"""Multi-GPU sharding of the separable dose: one process per GPU over ``torch.distributed``.

The reference computes on one device; its per-layer engine (engines.py:208-283) is
separable in depth, and fields or scenarios are independent, so both partitions below
leave the dose itself without any exchange:

* depth slabs of one field (``SlabPlan``): slice k of the dose depends only on slice k
  of the depth tables, so rank r computes slices [z0_r, z1_r) on its own.  The gradient
  dL/dW = sum over slices is the one exchange: a single all-reduce of
  L*nsy*nsx + L + 1 float64 values (dL/dW, dL/dR, the loss), 538 KB for 41x41x40.
* jobs (fields x scenarios, ``shard_jobs``): fully independent.  A robust objective
  needs the per-job losses (``gather_losses``, an all-gather of n_jobs values) and, for
  its gradient, one weighted all-reduce (``reduce_weighted``).

Slabs are cut by cost, not by slice count: a slice costs its number of active layers
(IDD != 0), which falls with depth beyond the shallowest Bragg peaks.  The reductions
are plain tensor functions (NCCL on CUDA tensors, gloo on host tensors), so the host
logic runs on CPU process groups too.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from . import physics as ph
from .model import DoseGrid, PBProblem


# ----------------------------------------------------------------------------- partitions
def slab_bounds(cost, world: int) -> list:
    """Contiguous depth slabs [(z0, z1), ...], one per rank, of near-equal total cost.

    ``cost[k]`` >= 0 is the work of slice k.  Cut points are the first slices whose
    prefix cost reaches r/world of the total; every slab keeps at least one slice while
    there are at least ``world`` slices (otherwise the last ranks get empty slabs)."""
    c = np.asarray(cost, dtype=np.float64).reshape(-1)
    nz = c.size
    if world < 1:
        raise ValueError("world must be >= 1")
    if np.any(c < 0):
        raise ValueError("slice costs must be non-negative")
    c = c + 1e-9 * max(float(c.max(initial=0.0)), 1.0)    # empty slices still cost something
    pref = np.concatenate([[0.0], np.cumsum(c)])
    total = pref[-1]
    cuts = [0]
    for r in range(1, world):
        k = int(np.searchsorted(pref, total * r / world, side="left"))
        lo = cuts[-1] + (1 if nz >= world else 0)
        hi = nz - (world - r) if nz >= world else nz
        cuts.append(int(min(max(k, lo), max(hi, lo))))
    cuts.append(nz)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def shard_jobs(n_jobs: int, world: int) -> list:
    """Contiguous job ranges, one per rank, sizes differing by at most one."""
    base, extra = divmod(int(n_jobs), int(world))
    out, s = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append(range(s, s + n))
        s += n
    return out


# ----------------------------------------------------------------------------- reductions
def _dist():
    import torch.distributed as dist
    return dist


def _world(group):
    dist = _dist()
    return dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1


def allreduce_gradients(loss, grad_w, grad_range=None, group=None):
    """Sum the loss and gradients of every rank in one all-reduce (float64 on the wire).

    Returns (loss float64 scalar, grad_w, grad_range) as new tensors of the inputs'
    dtypes on the inputs' device; with one rank (or no process group) the sums are the
    inputs themselves."""
    import torch
    gw = grad_w.reshape(-1)
    parts = [loss.reshape(1).to(torch.float64), gw.to(torch.float64)]
    if grad_range is not None:
        parts.append(grad_range.reshape(-1).to(torch.float64))
    buf = torch.cat(parts)
    if _world(group) > 1:
        _dist().all_reduce(buf, op=_dist().ReduceOp.SUM, group=group)
    n = gw.numel()
    out_loss = buf[0].clone()
    out_w = buf[1:1 + n].to(grad_w.dtype).reshape(grad_w.shape)
    out_r = None if grad_range is None else buf[1 + n:].to(grad_range.dtype)
    return out_loss, out_w, out_r


def gather_losses(local_losses, counts, group=None):
    """All ranks' per-job losses in job order.  ``counts[r]`` = jobs of rank r."""
    import torch
    local = torch.as_tensor(local_losses).reshape(-1).to(torch.float64)
    world = _world(group)
    if world == 1:
        return local.clone()
    m = max(counts)
    pad = torch.zeros(m, dtype=torch.float64, device=local.device)
    pad[:local.numel()] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    _dist().all_gather(bufs, pad, group=group)
    return torch.cat([b[:c] for b, c in zip(bufs, counts)])


def reduce_weighted(grads, weights, group=None):
    """sum_k weights[k] * grads[k] over this rank's jobs, then summed over ranks
    (one all-reduce).  ``grads``: tensors of one shape; ``weights``: this rank's
    entries of the global job weights."""
    import torch
    if len(grads) == 0:
        raise ValueError("reduce_weighted needs the gradient shape: pass at least one tensor")
    acc = torch.zeros(grads[0].shape, dtype=torch.float64, device=grads[0].device)
    for g, a in zip(grads, weights):
        acc += float(a) * g.to(torch.float64)
    if _world(group) > 1:
        _dist().all_reduce(acc, op=_dist().ReduceOp.SUM, group=group)
    return acc.to(grads[0].dtype)


def gather_slabs(local, bounds, group=None):
    """Full (nz, ...) array from every rank's slab ``local`` (shape (z1-z0, ...))."""
    import torch
    world = _world(group)
    if world == 1:
        return local.clone()
    m = max(z1 - z0 for z0, z1 in bounds)
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    _dist().all_gather(bufs, pad, group=group)
    return torch.cat([b[:z1 - z0] for b, (z0, z1) in zip(bufs, bounds)])


# ----------------------------------------------------------------------------- depth slabs
class SlabPlan:
    """This rank's depth slab of one field, resident on its GPU.

    The full-depth tables (and their range derivatives) are built once on the device,
    the slab's columns are kept, and a ``DosePlan`` runs the slab as a field of its own
    (grid origin moved to the slab's first slice).  ``loss_grad`` reduces the loss and
    gradients over all ranks unless ``reduce=False``."""

    def __init__(self, problem: PBProblem, *, rank: int = 0, world: int = 1, group=None,
                 precision: str | None = None, device=None, fd_step: float = 0.005):
        from . import engines
        torch = _lib.require_cuda()
        self.torch = torch
        self.device = torch.device(device or "cuda")
        self.rank, self.world, self.group = int(rank), int(world), group
        g, L = problem.grid, problem.lattice
        if L.energies is None:
            raise ValueError("slab plans build their tables from lattice.energies")
        t = ph.build_tables(g.nz, g.oz, g.dz, L.energies, fd_step=fd_step, device=self.device)
        cost = (t.idd != 0).sum(0).cpu().numpy()
        self.bounds = slab_bounds(cost, self.world)
        self.z0, self.z1 = self.bounds[self.rank]
        self.shape = (g.nz, g.ny, g.nx)
        self.n_layers = L.n_layers
        self.w_shape = (L.n_sy, L.n_sx)
        self.plan = None
        if self.z1 > self.z0:
            sg = DoseGrid(g.nx, g.ny, self.z1 - self.z0, g.dx, g.dy, g.dz, g.ox, g.oy,
                          g.oz + self.z0 * g.dz)
            sl = slice(self.z0, self.z1)
            sub = PBProblem(sg, L, t.idd[:, sl].cpu().numpy(), t.sigma[:, sl].cpu().numpy(),
                            meta=dict(problem.meta or {}, slab=(self.z0, self.z1)))
            kw = {} if precision is None else {"precision": precision}
            self.plan = engines.DosePlan(sub, tables="problem", device=self.device, **kw)
            self.plan.idd = t.idd[:, sl].contiguous()
            self.plan.sigma = t.sigma[:, sl].contiguous()
            self.plan.didd = t.didd_dr[:, sl].contiguous()
            self.plan.dsig = t.dsigma_dr[:, sl].contiguous()

    def _slab(self, a):
        torch = self.torch
        a = a if torch.is_tensor(a) else torch.as_tensor(np.asarray(a, dtype=np.float32))
        return a[self.z0:self.z1].to(self.device, torch.float32).contiguous()

    def forward(self, w=None):
        """This rank's slab of the dose, shape (z1 - z0, ny, nx)."""
        torch = self.torch
        if self.plan is None:
            return torch.zeros((0,) + self.shape[1:], dtype=torch.float32, device=self.device)
        return self.plan.forward(w=w)

    def gather_dose(self, w=None):
        """The full dose on every rank (all-gather of the slabs)."""
        return gather_slabs(self.forward(w), self.bounds, self.group)

    def loss_grad(self, mask, presc, w=None, reduce: bool = True):
        """L = sum m (D - P)^2 over the whole field and dL/dW, dL/dR on every rank.
        ``mask`` / ``presc``: full-grid (nz, ny, nx) arrays; each rank reads its slab."""
        torch = self.torch
        if self.plan is not None:
            o = self.plan.loss_grad(self._slab(mask), self._slab(presc), w=w)
            loss, gw, gr = o["loss"], o["grad_w"], o["grad_range"]
        else:
            nsy, nsx = self.w_shape
            loss = torch.zeros((), dtype=torch.float64, device=self.device)
            gw = torch.zeros((self.n_layers, nsy, nsx), dtype=torch.float32, device=self.device)
            gr = torch.zeros(self.n_layers, dtype=torch.float32, device=self.device)
        if not reduce:
            return loss, gw, gr
        if self.world > 1 and _world(self.group) != self.world:
            raise RuntimeError("world > 1 needs an initialised process group of that size")
        return allreduce_gradients(loss, gw, gr, self.group)
