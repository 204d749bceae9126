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
from .model import PBProblem


@dataclass
class Scenario:
    dx: float = 0.0      # lateral setup shift of the beam, cm
    dy: float = 0.0
    dz: float = 0.0      # water surface moved deeper by dz, cm
    scale: float = 1.0   # water-equivalent depth scaling (range scaling)


class ScenarioBatch:
    """Fields x scenarios on one device, forward dose of every job per ``run()``."""

    def __init__(self, problems, scenarios, *, precision="fp32", device=None):
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
        k = 0
        for p in self.problems:
            g, L = p.grid, p.lattice
            w = torch.as_tensor(np.ascontiguousarray(L.ensure_weights(), dtype=np.float32),
                                device=self.device)
            for s in self.scenarios:
                t = ph.build_tables(g.nz, g.oz - s.dz, g.dz, L.energies, depth_scale=s.scale,
                                    anchor_surface=True, device=self.device)
                d = torch.empty((g.nz, g.ny, g.nx), dtype=torch.float32, device=self.device)
                f = p.field_descriptor()
                f.x0 = L.x0 + s.dx
                f.y0 = L.y0 + s.dy
                self.jobs[k] = _lib.Job(field=f, w=_lib.ptr(w), idd=_lib.ptr(t.idd),
                                        sigma=_lib.ptr(t.sigma), dose=_lib.ptr(d))
                self.keep += [w, t.idd, t.sigma]
                self.doses.append(d)
                k += 1
        self.n_jobs = n_jobs
        nbytes = _lib.query("pbd_forward_batch_workspace", self.jobs, n_jobs, self.precision)
        self.ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        self.graph = None

    def run(self):
        """Enqueue the batched forward on the current stream."""
        _lib.call("pbd_forward_batch", self.jobs, self.n_jobs, self.precision, _lib.ptr(self.ws),
                  self.ws.numel(), _lib.stream_handle(self.device))
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
