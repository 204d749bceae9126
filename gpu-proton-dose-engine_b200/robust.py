"""Robust scenarios and several fields in one persistent launch.

No counterpart in the reference (it computes one nominal field at a time).  A
scenario perturbs a field by a lateral setup shift (sub-voxel lattice offset), a shift
of the water surface along the beam, and a range (stopping-power) scaling; its depth
tables are rebuilt on the device for the shifted / scaled water-equivalent depths
(``pbd_lut_spec.z0`` and ``depth_scale``).  All (field, scenario) jobs then run as one
persistent ``pbd_forward_batch`` launch, whose device-side scheduler balances the
uneven fields, and the whole batch can be captured into a CUDA graph and replayed.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import physics as ph


@dataclass
class Scenario:
    dx: float = 0.0      # lateral setup shift of the beam, cm
    dy: float = 0.0
    dz: float = 0.0      # water surface moved deeper by dz, cm
    scale: float = 1.0   # water-equivalent depth scaling (range scaling)


class ScenarioBatch:
    """Fields x scenarios on one device, forward dose of every job per ``run()``."""

    def __init__(self, problems, scenarios, *, precision="fp32", device=None,
                 with_grad: bool = False, fd_step: float = 0.005):
        torch = _lib.require_cuda()
        self.torch = torch
        self.device = torch.device(device or "cuda")
        self.precision = _lib.precision_code(precision)
        self.problems = list(problems)
        self.scenarios = [s if isinstance(s, Scenario) else Scenario(*s) for s in scenarios]
        n_jobs = len(self.problems) * len(self.scenarios)
        if n_jobs > _lib.MAX_JOBS:
            raise ValueError(f"{n_jobs} jobs exceed the per-launch limit {_lib.MAX_JOBS}")
        self.jobs = (_lib.Job * n_jobs)()
        self.keep = []
        self.doses = []
        self.tables = []
        self.weights = []
        k = 0
        for p in self.problems:
            g, L = p.grid, p.lattice
            w = torch.as_tensor(np.ascontiguousarray(L.ensure_weights(), dtype=np.float32),
                                device=self.device)
            self.weights.append(w)
            for s in self.scenarios:
                t = ph.build_tables(g.nz, g.oz - s.dz, g.dz, L.energies, depth_scale=s.scale,
                                    anchor_surface=True, device=self.device,
                                    fd_step=fd_step if with_grad else 0.0)
                d = torch.empty((g.nz, g.ny, g.nx), dtype=torch.float32, device=self.device)
                f = _lib.field_of(p)
                f.x0 = L.x0 + s.dx
                f.y0 = L.y0 + s.dy
                self.jobs[k] = _lib.Job(field=f, w=_lib.ptr(w), idd=_lib.ptr(t.idd),
                                        sigma=_lib.ptr(t.sigma), dose=_lib.ptr(d))
                self.keep += [w, t.idd, t.sigma]
                self.tables.append(t)
                self.doses.append(d)
                k += 1
        self.n_jobs = n_jobs
        self.graph = None

    def run(self):
        """Enqueue the batched forward on the current stream (the workspace follows the
        schedule in force, see ``tuning.schedule``)."""
        need = _lib.query("pbd_forward_batch_workspace", self.jobs, self.n_jobs, self.precision)
        ws = self._ws("fwd_batch", need)
        _lib.call("pbd_forward_batch", self.jobs, self.n_jobs, self.precision, _lib.ptr(ws),
                  ws.numel(), _lib.stream_handle(self.device))
        return self.doses

    def capture(self):
        """Capture one batched forward into a CUDA graph (replay with ``replay()``)."""
        torch = self.torch
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.run()          # warm-up outside capture (kernel attributes, lazy loading)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.doses

    def job_problem(self, k) -> tuple:
        """(problem, scenario) of job ``k``."""
        return self.problems[k // len(self.scenarios)], self.scenarios[k % len(self.scenarios)]

    # -- plain per-job loop (the comparison the batch is measured against) -------------
    def loop_forward(self, precision="fp32"):
        """One ``pbd_forward`` call per job on the current stream (shared workspace, calls
        ordered on the stream), e.g. the plain FP32 kernel looped over the scenarios."""
        prec = _lib.precision_code(precision)
        need = max(_lib.query("pbd_forward_workspace", ctypes.byref(self.jobs[k].field), prec)
                   for k in range(self.n_jobs))
        ws = self._ws("loop", need)
        out = []
        for k in range(self.n_jobs):
            j = self.jobs[k]
            d = self._loop_out(k)
            _lib.call("pbd_forward", ctypes.byref(j.field), j.w, j.idd, j.sigma, _lib.ptr(d),
                      prec, _lib.ptr(ws), ws.numel(), _lib.stream_handle(self.device))
            out.append(d)
        return out

    def _loop_out(self, k):
        if not hasattr(self, "_loop_doses"):
            self._loop_doses = [torch_empty_like(d) for d in self.doses]
        return self._loop_doses[k]

    def _ws(self, name, nbytes):
        bufs = self.__dict__.setdefault("_wsbufs", {})
        b = bufs.get(name)
        if b is None or b.numel() < nbytes:
            b = self.torch.empty(max(nbytes, 256), dtype=self.torch.uint8, device=self.device)
            bufs[name] = b
        return b

    # -- gradients of every job ----------------------------------------------------------
    def alloc_grad_outputs(self):
        """Per-job gradient outputs.  The dL/dW and loss of one field's scenarios are views
        of one contiguous block, ``field_grads[f]`` (S, L, nsy, nsx) and
        ``field_losses[f]`` (S,), which a robust objective combines in one call."""
        if getattr(self, "grad_outputs", None):
            return self.grad_outputs
        torch = self.torch
        n_s = len(self.scenarios)
        self.field_grads, self.field_losses = [], []
        outs = []
        for fi in range(len(self.problems)):
            f = self.jobs[fi * n_s].field
            gw = torch.empty((n_s, f.n_layers, f.n_sy, f.n_sx), dtype=torch.float32,
                             device=self.device)
            ls = torch.zeros(n_s, dtype=torch.float64, device=self.device)
            self.field_grads.append(gw)
            self.field_losses.append(ls)
            for si in range(n_s):
                outs.append({"grad_dose": torch.empty((f.nz, f.ny, f.nx), dtype=torch.float32,
                                                      device=self.device),
                             "loss": ls[si],
                             "grad_w": gw[si],
                             "grad_range": torch.zeros(f.n_layers, dtype=torch.float32,
                                                       device=self.device)})
        self.grad_outputs = outs
        return outs

    def loss_grad_all(self, mask, presc, batched=None):
        """Forward, masked quadratic loss and adjoint of every (field, scenario) job on the
        current stream.  ``mask`` / ``presc``: one (nz, ny, nx) pair for all jobs (same grid).

        ``batched`` (default: for the tensor-core precisions): every job's forward in one
        persistent launch and every adjoint in another (``pbd_loss_grad_batch``); otherwise
        one ``pbd_loss_grad`` call per job with a shared workspace."""
        nvox = {p.grid.nz * p.grid.ny * p.grid.nx for p in self.problems}
        if len(nvox) != 1:
            raise ValueError("one mask and prescription need every field on the same grid")
        n = nvox.pop()
        _lib.check_arg(mask, "mask", n, self.torch.float32, self.device)
        _lib.check_arg(presc, "presc", n, self.torch.float32, self.device)
        if not getattr(self, "grad_outputs", None):
            self.alloc_grad_outputs()
        if batched is None:
            batched = self.precision != _lib.PREC["fp32"]
        if batched:
            return self._loss_grad_batched(mask, presc)
        need = max(_lib.query("pbd_loss_grad_workspace", ctypes.byref(self.jobs[k].field),
                              self.precision) for k in range(self.n_jobs))
        ws = self._ws("grad", need)
        st = _lib.stream_handle(self.device)
        for k in range(self.n_jobs):
            j, t, o = self.jobs[k], self.tables[k], self.grad_outputs[k]
            if t.didd_dr is None:
                raise RuntimeError("build the batch with with_grad=True for gradients")
            _lib.call("pbd_loss_grad", ctypes.byref(j.field), j.w, j.idd, j.sigma,
                      _lib.ptr(t.didd_dr), _lib.ptr(t.dsigma_dr), _lib.ptr(mask), _lib.ptr(presc),
                      j.dose, _lib.ptr(o["grad_dose"]), _lib.ptr(o["loss"]), _lib.ptr(o["grad_w"]),
                      _lib.ptr(o["grad_range"]), self.precision, _lib.ptr(ws), ws.numel(), st)
        return self.grad_outputs

    def _loss_grad_batched(self, mask, presc):
        key = (_lib.ptr(mask), _lib.ptr(presc))
        if getattr(self, "_gjobs_key", None) != key:
            gj = (_lib.GradJob * self.n_jobs)()
            for k in range(self.n_jobs):
                j, t, o = self.jobs[k], self.tables[k], self.grad_outputs[k]
                if t.didd_dr is None:
                    raise RuntimeError("build the batch with with_grad=True for gradients")
                gj[k] = _lib.GradJob(field=j.field, w=j.w, idd=j.idd, sigma=j.sigma,
                                     didd_dr=_lib.ptr(t.didd_dr), dsigma_dr=_lib.ptr(t.dsigma_dr),
                                     mask=_lib.ptr(mask), presc=_lib.ptr(presc), dose=j.dose,
                                     grad_dose=_lib.ptr(o["grad_dose"]), loss=_lib.ptr(o["loss"]),
                                     grad_w=_lib.ptr(o["grad_w"]),
                                     grad_range=_lib.ptr(o["grad_range"]))
            self._gjobs, self._gjobs_key = gj, key
            self._gjobs_refs = (mask, presc)
        need = _lib.query("pbd_loss_grad_batch_workspace", self._gjobs, self.n_jobs,
                          self.precision)
        ws = self._ws("grad_batch", need)
        _lib.call("pbd_loss_grad_batch", self._gjobs, self.n_jobs, self.precision, _lib.ptr(ws),
                  ws.numel(), _lib.stream_handle(self.device))
        return self.grad_outputs

    def capture_loss_grad(self, mask, presc):
        """Capture ``loss_grad_all`` into a CUDA graph (replay with ``replay_loss_grad``)."""
        torch = self.torch
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.loss_grad_all(mask, presc)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.loss_grad_all(mask, presc)
        self.grad_graph = g
        return g

    def replay_loss_grad(self):
        self.grad_graph.replay()
        return self.grad_outputs


def torch_empty_like(t):
    return t.new_empty(t.shape)


def robust_problems(fields):
    """PBProblem of each workload field (``workloads.robust_fields``), tables on the device."""
    from .model import problem_from_workload
    return [problem_from_workload(f) for f in fields]
