"""Plan optimisation on the device: projected Adam over a field's spot weights (and,
optionally, its per-layer range shifts) for the nominal plan loss, or over the fields of a
scenario batch for a robust objective (mean or worst case over scenarios).

No counterpart in the reference, which computes dose only: this is the caller that makes
the adjoint useful.  Every iteration is

    [rebuild the depth tables at the current range shifts]   (pbd_build_luts)
    loss L = sum m (D - P)^2 and dL/dW, dL/dR                 (pbd_loss_grad, per job)
    [combine the scenario gradients]                          (pbd_scenario_combine)
    projected Adam on W [and on the range shifts]             (pbd_adam_step)

and keeps all of its state on the device (moments, step count, loss history), so the
iteration is captured once into a CUDA graph and ``step()`` replays it with no host work.
``history()`` returns the loss of the gradient applied at each step (the loss at the
start of that step).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import physics as ph


@dataclass
class Adam:
    """Projected Adam settings (Kingma & Ba 2015, Algorithm 1; the box [lo, hi] after each
    step).  Spot weights default to the non-negative orthant."""
    lr: float = 0.01
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    lo: float = 0.0
    hi: float = math.inf
    grad_scale: float = 1.0

    def params(self) -> _lib.AdamParams:
        return _lib.AdamParams(lr=self.lr, beta1=self.beta1, beta2=self.beta2, eps=self.eps,
                               lo=self.lo, hi=self.hi, grad_scale=self.grad_scale)


class _AdamState:
    """Moments and step counter of one parameter vector, on the device."""

    def __init__(self, torch, x, cfg: Adam, max_iter: int, x64=None):
        self.x, self.x64, self.cfg = x, x64, cfg
        self.p = cfg.params()
        self.m = torch.zeros_like(x)
        self.v = torch.zeros_like(x)
        self.state = torch.zeros(2, dtype=torch.int32, device=x.device)
        self.hist = torch.zeros(max(max_iter, 1), dtype=torch.float64, device=x.device)
        self.max_iter = max_iter

    def step(self, grad, loss, stream):
        _lib.call("pbd_adam_step", ctypes.byref(self.p), int(self.x.numel()), _lib.ptr(self.x),
                  _lib.ptr(self.m), _lib.ptr(self.v), _lib.ptr(grad), _lib.ptr(self.state),
                  _lib.ptr(self.x64), _lib.ptr(loss), _lib.ptr(self.hist), self.max_iter, stream)

    def steps_done(self) -> int:
        return int(self.state[0].item())


class _Loop:
    """Shared driver: one iteration enqueued by ``_iteration``, optionally captured."""

    torch = None
    device = None

    def _setup_graph(self, graph: bool):
        self.graph = None
        if graph:
            torch = self.torch
            self._prepare()               # allocations and lookups outside the capture
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._iteration()
            self.graph = g

    def _prepare(self):
        pass

    def step(self, n: int = 1):
        """Enqueue ``n`` iterations on the current stream."""
        if self._done + n > self.max_iter:
            raise ValueError(f"the loss history holds {self.max_iter} iterations")
        for _ in range(n):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._iteration()
        self._done += n

    def run(self, n_iter: int):
        """Run ``n_iter`` iterations and return the loss history so far (host array)."""
        self.step(n_iter)
        self.torch.cuda.synchronize(self.device)
        return self.history()


class PlanOptimizer(_Loop):
    """Nominal plan optimisation of one field (``engines.DosePlan``).

    ``mask`` / ``presc``: (nz, ny, nx) float32 device tensors of the loss
    L = sum m (D - P)^2.  ``range_adam``: also optimise the per-layer range shifts (needs a
    plan with device tables); their tables are rebuilt on the device every iteration.
    The plan's weights ``plan.w`` are the optimised parameters (updated in place)."""

    def __init__(self, plan, mask, presc, *, adam: Adam | None = None,
                 range_adam: Adam | None = None, max_iter: int = 1000, graph: bool = True):
        torch = _lib.require_cuda()
        self.torch, self.plan, self.device = torch, plan, plan.device
        self.mask, self.presc = mask, presc
        self.max_iter = int(max_iter)
        self._done = 0
        self.out = plan.alloc_outputs()
        self.w = plan.w
        self.w_opt = _AdamState(torch, self.w, adam or Adam(), self.max_iter)
        self.r_opt = None
        self.builder = None
        if range_adam is not None:
            if plan.tables_mode != "device" or plan.fd_step <= 0:
                raise ValueError("range optimisation needs device tables with range derivatives")
            g = plan.problem.grid
            nl = int(self.w.shape[0])
            rs = plan.range_shift
            self.range_shift64 = (torch.zeros(nl, dtype=torch.float64, device=self.device)
                                  if rs is None else rs.clone().contiguous())
            self.range_shift = self.range_shift64.to(torch.float32)
            self.builder = ph.TableBuilder(g.nz, g.oz, g.dz, plan.energies, fd_step=plan.fd_step,
                                           device=self.device)
            t = self.builder.build(self.range_shift64)
            plan.idd, plan.sigma, plan.didd, plan.dsig = t.idd, t.sigma, t.didd_dr, t.dsigma_dr
            plan.range_shift = None       # the plan's tables now follow range_shift64
            plan._tuned = False
            self.r_opt = _AdamState(torch, self.range_shift, range_adam, self.max_iter,
                                    x64=self.range_shift64)
        self._setup_graph(graph)

    def _prepare(self):
        self.plan.loss_grad(self.mask, self.presc, w=self.w, outputs=self.out)

    def _iteration(self):
        st = _lib.stream_handle(self.device)
        if self.builder is not None:
            self.builder.build(self.range_shift64)
        o = self.plan.loss_grad(self.mask, self.presc, w=self.w, outputs=self.out)
        self.w_opt.step(o["grad_w"], o["loss"], st)
        if self.r_opt is not None:
            self.r_opt.step(o["grad_range"], o["loss"], st)

    def history(self):
        """Loss at the start of each completed iteration (float64, host)."""
        n = self.w_opt.steps_done()
        return self.w_opt.hist[:min(n, self.max_iter)].cpu().numpy()


class RobustOptimizer(_Loop):
    """Robust optimisation over a ``robust.ScenarioBatch`` built with ``with_grad=True``:
    every field's weights (shared by its scenarios) follow projected Adam on the mean
    (``objective="mean"``) or the worst-case (``"max"``, min-max) loss over its scenarios.
    ``mask`` / ``presc`` are shared by all jobs (same grid)."""

    def __init__(self, batch, mask, presc, *, objective: str = "max", adam: Adam | None = None,
                 max_iter: int = 1000, graph: bool = True):
        torch = _lib.require_cuda()
        if objective not in _lib.OBJ:
            raise ValueError(f"objective must be one of {sorted(_lib.OBJ)}")
        self.torch, self.batch, self.device = torch, batch, batch.device
        self.mask, self.presc = mask, presc
        self.mode = _lib.OBJ[objective]
        self.max_iter = int(max_iter)
        self._done = 0
        self.outs = batch.alloc_grad_outputs()
        self.n_scen = len(batch.scenarios)
        cfg = adam or Adam()
        self.fields = []
        for f, w in enumerate(batch.weights):
            self.fields.append({
                "w": w,
                "grad": torch.empty_like(w),
                "loss": torch.zeros((), dtype=torch.float64, device=self.device),
                "opt": _AdamState(torch, w, cfg, self.max_iter),
            })
        self._setup_graph(graph)

    def _prepare(self):
        self.batch.loss_grad_all(self.mask, self.presc)

    def _iteration(self):
        st = _lib.stream_handle(self.device)
        self.batch.loss_grad_all(self.mask, self.presc)
        for f, fd in enumerate(self.fields):
            grads = self.batch.field_grads[f]
            losses = self.batch.field_losses[f]
            _lib.call("pbd_scenario_combine", self.mode, self.n_scen, int(fd["w"].numel()),
                      _lib.ptr(grads), _lib.ptr(losses), _lib.ptr(fd["grad"]),
                      _lib.ptr(fd["loss"]), st)
            fd["opt"].step(fd["grad"], fd["loss"], st)

    def history(self):
        """(n_fields, iterations) objective value at the start of each iteration."""
        n = min(self.fields[0]["opt"].steps_done(), self.max_iter)
        return np.stack([fd["opt"].hist[:n].cpu().numpy() for fd in self.fields])
