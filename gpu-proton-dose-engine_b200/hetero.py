"""Heterogeneous media: water-equivalent depth (WED) and the dose that uses it.

The reference treats water only: ``physics.wed_from_density_path`` (physics.py:421-423) is a
stub, WED = sum of rho * L along one path, and its README lists heterogeneous media as not
implemented.  Here, on the device:

* ``wed_raytrace(rho, grid)`` -- WED at every voxel centre along the beam axis (+z) through a
  relative stopping-power map: the reference's sum of rho * L over the path from depth 0 to
  the voxel centre, voxel k filling [z_k - dz/2, z_k + dz/2], water above the first voxel
  (``pbd_wed_raytrace``).  rho = 1 gives WED = depth.
* ``WedPlan(problem).forward(wed)`` -- the dose with each layer's depth dose evaluated at the
  voxel's WED instead of its geometric depth: the same smoothed depth curve and interpolation
  as the depth tables (physics.py:328-387), the lateral widths of water at the geometric
  depth (a broad-beam ray-casting approximation; the lateral scattering in the material is
  not modelled) (``pbd_build_wed_curves`` once, then ``pbd_forward_wed_curves``).  In water it
  reproduces the homogeneous dose.  ``WedPlan(problem).adjoint(grad_dose, wed)`` gives dL/dW
  (``pbd_adjoint_wed``), and with ``with_range=True`` also dL/d(range shift) per layer
  (``pbd_adjoint_wed_range``: the depth curves' and the widths' central differences at +-h),
  for plan optimisation in the medium.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from . import physics as ph


def wed_from_density_path(densities, lengths) -> float:
    """WED = sum rho_i L_i (the reference's helper, physics.py:421-423), host NumPy."""
    return float(np.sum(np.asarray(densities) * np.asarray(lengths)))


def wed_raytrace(rho, grid, device=None):
    """WED (cm, float64 device tensor (nz, ny, nx)) of a relative stopping-power map
    ``rho`` (nz, ny, nx) on ``grid`` (a DoseGrid or a dict with nz, ny, nx, oz, dz)."""
    torch = _lib.require_cuda()
    dev = torch.device(device or "cuda")
    g = grid if isinstance(grid, dict) else {k: getattr(grid, k) for k in ("nz", "ny", "nx", "oz", "dz")}
    r = rho.to(dev, torch.float32).contiguous() if torch.is_tensor(rho) else \
        torch.as_tensor(np.ascontiguousarray(rho, dtype=np.float32), device=dev)
    shape = (int(g["nz"]), int(g["ny"]), int(g["nx"]))
    if tuple(r.shape) != shape:
        raise ValueError(f"rho has shape {tuple(r.shape)}, the grid {shape}")
    wed = torch.empty(shape, dtype=torch.float64, device=dev)
    _lib.call("pbd_wed_raytrace", shape[0], shape[1], shape[2], float(g["oz"]), float(g["dz"]),
              _lib.ptr(r), _lib.ptr(wed), _lib.stream_handle(dev))
    return wed


class WedPlan:
    """One field in a heterogeneous medium: the lateral widths of water at the geometric
    depths and the layers' depth curves (``pbd_build_wed_curves``), built once on the device,
    and the workspaces of ``pbd_forward_wed_curves`` and (on first use) ``pbd_adjoint_wed``."""

    def __init__(self, problem, *, precision: str = "tf32x3", device=None,
                 idd_model: ph.IDDModel = ph.DEFAULT_IDD, sigma_x0: float = 0.30,
                 fd_step: float = 0.005):
        torch = _lib.require_cuda()
        self.torch = torch
        self.device = torch.device(device or "cuda")
        self.problem = problem
        g, L = problem.grid, problem.lattice
        if L.energies is None:
            raise ValueError("the heterogeneous dose needs lattice.energies")
        self.field = _lib.field_of(problem)
        self.precision = _lib.precision_code(precision)
        self.spec = ph.lut_spec(g.nz, g.oz, g.dz, idd_model=idd_model, sigma_x0=sigma_x0)
        self.energies = torch.as_tensor(np.asarray(L.energies, dtype=np.float64), device=self.device)
        self.sigma = ph.build_tables(g.nz, g.oz, g.dz, L.energies, idd_model=idd_model,
                                     sigma_x0=sigma_x0, device=self.device).sigma
        self.w = torch.as_tensor(np.ascontiguousarray(L.ensure_weights(), dtype=np.float32),
                                 device=self.device)
        nbytes = _lib.query("pbd_forward_wed_workspace", ctypes.byref(self.field),
                            ctypes.byref(self.spec), self.precision)
        self.ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        self.adj_ws = None
        self.range_ws = None
        self.idd_model, self.sigma_x0, self.fd_step = idd_model, sigma_x0, float(fd_step)
        self.curves_pm = None   # the curves at range shifts +h and -h, built on first use
        self.dsigma_dr = None
        # the depth curves depend on the energies only: built once, reused by every call
        cbytes = _lib.query("pbd_wed_curves_workspace", ctypes.byref(self.spec), len(L.energies))
        self.curves = torch.empty(cbytes, dtype=torch.uint8, device=self.device)
        self._build_curves(self.curves, None)
        self.shape = (g.nz, g.ny, g.nx)
        self.nvox = g.nz * g.ny * g.nx

    def _build_curves(self, out, shift):
        _lib.call("pbd_build_wed_curves", ctypes.byref(self.spec), int(self.energies.numel()),
                  _lib.ptr(self.energies), _lib.ptr(shift), _lib.ptr(out), out.numel(),
                  _lib.stream_handle(self.device))

    def _range_tables(self):
        """The curves at range shifts +-h and the widths' range derivative (once per plan)."""
        if self.curves_pm is None:
            torch = self.torch
            g = self.problem.grid
            h = self.fd_step
            n = int(self.energies.numel())
            pm = []
            for sign in (1.0, -1.0):
                c = torch.empty_like(self.curves)
                self._build_curves(c, torch.full((n,), sign * h, dtype=torch.float64,
                                                 device=self.device))
                pm.append(c)
            self.curves_pm = tuple(pm)
            self.dsigma_dr = ph.build_tables(g.nz, g.oz, g.dz, self.problem.lattice.energies,
                                             idd_model=self.idd_model, sigma_x0=self.sigma_x0,
                                             fd_step=h, device=self.device).dsigma_dr
        return self.curves_pm, self.dsigma_dr

    def _wed(self, wed):
        """The WED map as a contiguous float64 device tensor (host data is uploaded)."""
        torch = self.torch
        if not torch.is_tensor(wed):
            wed = torch.as_tensor(np.ascontiguousarray(wed, dtype=np.float64))
        if tuple(wed.shape) != self.shape or wed.dtype != torch.float64:
            raise ValueError("wed must be a float64 tensor of the grid's shape")
        return wed.to(self.device).contiguous()

    def _weights(self, w):
        torch = self.torch
        if w is None:
            return self.w
        wt = torch.as_tensor(w, dtype=torch.float32, device=self.device).contiguous()
        return _lib.check_arg(wt, "w", self.w.numel(), torch.float32, self.device)

    def forward(self, wed, w=None, out=None):
        """Dose (float32 device tensor (nz, ny, nx)) for the WED map ``wed`` (float64 tensor or
        array of the grid's shape, e.g. from ``wed_raytrace``), on the current stream."""
        torch = self.torch
        wd = self._wed(wed)
        wt = self._weights(w)
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        _lib.check_arg(out, "out", self.nvox, torch.float32, self.device)
        _lib.call("pbd_forward_wed_curves", ctypes.byref(self.field), ctypes.byref(self.spec),
                  _lib.ptr(self.curves), self.curves.numel(), _lib.ptr(wt), _lib.ptr(self.sigma),
                  _lib.ptr(wd), _lib.ptr(out), self.precision, _lib.ptr(self.ws),
                  self.ws.numel(), _lib.stream_handle(self.device))
        return out

    def adjoint(self, grad_dose, wed, w=None, with_range: bool = False):
        """dL/dW (float32 device tensor (L, nsy, nsx)) of the heterogeneous dose for the
        dL/dD ``grad_dose`` ((nz, ny, nx)) and the WED map ``wed`` (``pbd_adjoint_wed``).
        ``with_range=True`` returns (dL/dW, dL/dR), dL/dR (L,) float32 the gradient in each
        layer's range shift (``pbd_adjoint_wed_range``)."""
        torch = self.torch
        wd = self._wed(wed)
        wt = self._weights(w)
        g = torch.as_tensor(grad_dose).to(self.device, torch.float32).contiguous()
        _lib.check_arg(g, "grad_dose", self.nvox, torch.float32, self.device)
        if with_range:
            (cp, cm), dsig = self._range_tables()
            if self.range_ws is None:
                nbytes = _lib.query("pbd_adjoint_wed_range_workspace", ctypes.byref(self.field),
                                    ctypes.byref(self.spec), self.precision)
                self.range_ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
            gw = torch.empty_like(self.w)
            gr = torch.empty(self.w.shape[0], dtype=torch.float32, device=self.device)
            _lib.call("pbd_adjoint_wed_range", ctypes.byref(self.field), ctypes.byref(self.spec),
                      _lib.ptr(self.curves), self.curves.numel(), _lib.ptr(cp), _lib.ptr(cm),
                      self.fd_step, _lib.ptr(wt), _lib.ptr(self.sigma), _lib.ptr(dsig),
                      _lib.ptr(wd), _lib.ptr(g), _lib.ptr(gw), _lib.ptr(gr), self.precision,
                      _lib.ptr(self.range_ws), self.range_ws.numel(),
                      _lib.stream_handle(self.device))
            return gw, gr
        if self.adj_ws is None:
            nbytes = _lib.query("pbd_adjoint_wed_workspace", ctypes.byref(self.field),
                                ctypes.byref(self.spec), self.precision)
            self.adj_ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        gw = torch.empty_like(self.w)
        _lib.call("pbd_adjoint_wed", ctypes.byref(self.field), ctypes.byref(self.spec),
                  _lib.ptr(self.curves), self.curves.numel(), _lib.ptr(wt), _lib.ptr(self.sigma),
                  _lib.ptr(wd), _lib.ptr(g), _lib.ptr(gw), self.precision, _lib.ptr(self.adj_ws),
                  self.adj_ws.numel(), _lib.stream_handle(self.device))
        return gw


def dose_heterogeneous(problem, rho, *, precision: str = "tf32x3", device=None):
    """(dose, wed) of ``problem`` in the relative stopping-power map ``rho``."""
    wed = wed_raytrace(rho, problem.grid, device=device)
    plan = WedPlan(problem, precision=precision, device=device)
    return plan.forward(wed), wed
