"""Depth-LUT builder on the device (FP64) and CSDA range lookups.

Replaces the reference's per-layer host loop that fills ``PBProblem.idd`` and
``PBProblem.sigma`` (model.py:225-233: ``physics.idd_pristine(normalize=False)`` and
``physics.fermi_eyges_moments(...)["sigma_x"]``, physics.py:221-387).  The tables are
built by ``pbd_build_luts`` in the CUDA library; this module only marshals arguments.
There is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib

_STRAG = {"bohr": 0, "icru49": 1, "none": 2}


@dataclass
class IDDModel:
    """Parameters of the analytic IDD (same fields and defaults as physics.py:292-308)."""
    straggling_model: str = "bohr"
    straggling_coef: float = 0.012
    straggling_exp: float = 0.935
    energy_spread: float = 0.0033
    attenuation_length: float = 150.0
    n_fine: int = 6000
    e_cut: float = 0.05


DEFAULT_IDD = IDDModel()


def lut_spec(nz: int, z0: float, dz: float, *, sigma_x0: float = 0.30, sigma_theta0: float = 0.0,
             rho0: float = 0.0, idd_model: IDDModel = DEFAULT_IDD, depth_scale: float = 1.0,
             anchor_surface: bool = False, fd_step: float = 0.0, n_sub: int = 4,
             max_step: float = 0.02) -> _lib.LutSpec:
    if idd_model.straggling_model not in _STRAG:
        raise ValueError(f"unknown straggling model: {idd_model.straggling_model}")
    return _lib.LutSpec(nz=int(nz), z0=float(z0), dz=float(dz), depth_scale=float(depth_scale),
                        anchor_surface=int(bool(anchor_surface)), sigma_x0=float(sigma_x0),
                        sigma_theta0=float(sigma_theta0), rho0=float(rho0), fe_n_sub=int(n_sub),
                        fe_max_step=float(max_step),
                        straggling_model=_STRAG[idd_model.straggling_model],
                        strag_coef=float(idd_model.straggling_coef),
                        strag_exp=float(idd_model.straggling_exp),
                        energy_spread=float(idd_model.energy_spread),
                        atten_len=float(idd_model.attenuation_length),
                        idd_n_fine=int(idd_model.n_fine), fd_step=float(fd_step))


@dataclass
class DepthTables:
    """Per-layer depth tables on the device, float64, shape (L, nz)."""
    idd: "object"
    sigma: "object"
    didd_dr: Optional["object"] = None
    dsigma_dr: Optional["object"] = None
    fd_step: float = 0.0


def build_tables(nz: int, z0: float, dz: float, energies, *, range_shift=None,
                 fd_step: float = 0.0, device=None, **spec_kw) -> DepthTables:
    """Build IDD_l(z) and sigma_l(z) (and their range derivatives when ``fd_step`` > 0).

    ``energies`` (MeV) and ``range_shift`` (cm, per layer) may be NumPy arrays or CUDA
    tensors; the result stays on the device."""
    torch = _lib.require_cuda()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    e = torch.as_tensor(np.asarray(energies, dtype=np.float64) if not torch.is_tensor(energies)
                        else energies, dtype=torch.float64, device=dev).contiguous()
    n_layers = int(e.numel())
    sh = None
    if range_shift is not None:
        sh = torch.as_tensor(range_shift if torch.is_tensor(range_shift)
                             else np.asarray(range_shift, dtype=np.float64),
                             dtype=torch.float64, device=dev).contiguous()
        if sh.numel() != n_layers:
            raise ValueError("range_shift must have one entry per layer")
    spec = lut_spec(nz, z0, dz, fd_step=fd_step, **spec_kw)
    ws_bytes = _lib.query("pbd_lut_workspace", ctypes.byref(spec), n_layers)
    with torch.cuda.device(dev):
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        idd = torch.empty((n_layers, nz), dtype=torch.float64, device=dev)
        sig = torch.empty((n_layers, nz), dtype=torch.float64, device=dev)
        didd = dsig = None
        if fd_step > 0:
            didd = torch.empty_like(idd)
            dsig = torch.empty_like(idd)
        _lib.call("pbd_build_luts", ctypes.byref(spec), n_layers, _lib.ptr(e), _lib.ptr(sh),
                  _lib.ptr(idd), _lib.ptr(sig), _lib.ptr(didd), _lib.ptr(dsig), _lib.ptr(ws),
                  ws_bytes, _lib.stream_handle(dev))
    return DepthTables(idd=idd, sigma=sig, didd_dr=didd, dsigma_dr=dsig, fd_step=fd_step)


class TableBuilder:
    """Rebuilds one field's depth tables in place: the outputs and the workspace are
    allocated once, so ``build`` only enqueues the builder's kernels and can run inside a
    captured CUDA graph, reading the range shifts from a device float64 vector."""

    def __init__(self, nz: int, z0: float, dz: float, energies, *, fd_step: float = 0.0,
                 device=None, **spec_kw):
        torch = _lib.require_cuda()
        self.torch = torch
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.energies = torch.as_tensor(np.asarray(energies, dtype=np.float64),
                                        device=self.device).contiguous()
        self.n_layers = int(self.energies.numel())
        self.spec = lut_spec(nz, z0, dz, fd_step=fd_step, **spec_kw)
        nbytes = _lib.query("pbd_lut_workspace", ctypes.byref(self.spec), self.n_layers)
        self.ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        shape = (self.n_layers, nz)
        f64 = torch.float64
        self.tables = DepthTables(
            idd=torch.empty(shape, dtype=f64, device=self.device),
            sigma=torch.empty(shape, dtype=f64, device=self.device),
            didd_dr=torch.empty(shape, dtype=f64, device=self.device) if fd_step > 0 else None,
            dsigma_dr=torch.empty(shape, dtype=f64, device=self.device) if fd_step > 0 else None,
            fd_step=fd_step)

    def build(self, range_shift=None) -> DepthTables:
        """Enqueue the rebuild at CSDA ranges R0_l + range_shift_l (``range_shift``: a device
        float64 tensor of L entries, or None) on the current stream."""
        if range_shift is not None:
            _lib.check_arg(range_shift, "range_shift", self.n_layers, self.torch.float64,
                           self.device)
        t = self.tables
        _lib.call("pbd_build_luts", ctypes.byref(self.spec), self.n_layers, _lib.ptr(self.energies),
                  _lib.ptr(range_shift), _lib.ptr(t.idd), _lib.ptr(t.sigma), _lib.ptr(t.didd_dr),
                  _lib.ptr(t.dsigma_dr), _lib.ptr(self.ws), self.ws.numel(),
                  _lib.stream_handle(self.device))
        return t


def _uniform_axis(z):
    z = np.asarray(z, dtype=np.float64)
    if z.ndim != 1 or z.size == 0:
        raise ValueError("depth axis must be a non-empty 1-D array")
    if z.size == 1:
        return 1, float(z[0]), 1.0
    dz = (z[-1] - z[0]) / (z.size - 1)
    if not np.allclose(np.diff(z), dz, rtol=1e-9, atol=1e-12):
        raise ValueError("the device LUT builder needs a uniformly spaced depth axis")
    return z.size, float(z[0]), float(dz)


def layer_luts(z, energies, *, idd_model: IDDModel = DEFAULT_IDD, sigma_x0: float = 0.30,
               sigma_theta0: float = 0.0, range_shift=None):
    """(idd, sigma) as float64 NumPy arrays of shape (L, nz): the tables model.py:225-233
    fills, built on the device.  ``z`` is a uniformly spaced depth axis (cm)."""
    nz, z0, dz = _uniform_axis(z)
    t = build_tables(nz, z0, dz, energies, range_shift=range_shift, idd_model=idd_model,
                     sigma_x0=sigma_x0, sigma_theta0=sigma_theta0)
    return t.idd.cpu().numpy(), t.sigma.cpu().numpy()


def _lookup(values, inverse: bool):
    torch = _lib.require_cuda()
    arr = np.asarray(values, dtype=np.float64)
    src = torch.as_tensor(arr.reshape(-1), device="cuda")
    out = torch.empty_like(src)
    _lib.call("pbd_energy_from_range" if inverse else "pbd_csda_range", _lib.ptr(src),
              _lib.ptr(out), int(src.numel()), _lib.stream_handle())
    res = out.cpu().numpy().reshape(arr.shape)
    return float(res) if res.ndim == 0 else res


def csda_range(e_kin):
    """CSDA range R(E) in cm (physics.py:130-133), evaluated on the device."""
    return _lookup(e_kin, inverse=False)


def energy_from_range(r_cm):
    """Energy E(R) in MeV, the inverse table lookup (physics.py:136-139), on the device."""
    return _lookup(r_cm, inverse=True)
