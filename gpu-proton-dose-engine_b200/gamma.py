"""Gamma index on the device (Low et al. 1998 / AAPM TG-218), with the reference's API.

Replaces the reference's ``gamma.py``: ``dta_offsets`` (gamma.py:41-60), ``gamma_index``
(gamma.py:81-164), ``gamma_pass_rate_vs_criteria`` (gamma.py:197-207) and
``gamma_index_torch`` (gamma.py:213-261).  One library call (``pbd_gamma_index``) computes
the gamma map, the low-dose mask and every statistic on the device; the result equals the
reference's float64 NumPy path (gamma map, mask, counts, maximum and percentiles bit for
bit; the mean within rounding).  ``gamma_index_torch`` returns the same float64 result
(the reference's torch version rounds to float32).

``GammaPlan`` keeps the workspace and outputs of one grid resident, for repeated
comparisons of device doses (and CUDA-graph capture); its statistics stay on the device
until ``stats()`` reads them.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib

_NORM = {"global": 0, "local": 1}


def dta_offsets(spacing, dta_cm: float, max_vox: int = 6):
    """Integer voxel offsets within the DTA ball and their distances (cm), in the
    reference's order (gamma.py:41-60).  Host NumPy; the device computes the same set."""
    dz, dy, dx = spacing
    nz = min(int(np.floor(dta_cm / dz + 1e-9)), max_vox)
    ny = min(int(np.floor(dta_cm / dy + 1e-9)), max_vox)
    nx = min(int(np.floor(dta_cm / dx + 1e-9)), max_vox)
    offs, dists = [], []
    for a in range(-nz, nz + 1):
        for b in range(-ny, ny + 1):
            for c in range(-nx, nx + 1):
                d = np.sqrt((a * dz) ** 2 + (b * dy) ** 2 + (c * dx) ** 2)
                if d <= dta_cm + 1e-12:
                    offs.append((a, b, c))
                    dists.append(d)
    return np.array(offs, dtype=np.int64), np.array(dists, dtype=np.float64)


def gamma_spec(spacing=(0.2, 0.2, 0.2), dose_crit_pct: float = 3.0, dta_mm: float = 3.0,
               threshold_pct: float = 10.0, normalization: str = "global",
               ref_dose: Optional[float] = None, max_vox: int = 6) -> _lib.GammaSpec:
    if normalization not in _NORM:
        raise ValueError(f"normalization must be 'global' or 'local', not {normalization!r}")
    dz, dy, dx = (float(v) for v in spacing)
    return _lib.GammaSpec(dz=dz, dy=dy, dx=dx, dose_crit_pct=float(dose_crit_pct),
                          dta_mm=float(dta_mm), threshold_pct=float(threshold_pct),
                          normalization=_NORM[normalization],
                          use_ref_dose=int(ref_dose is not None),
                          ref_dose=0.0 if ref_dose is None else float(ref_dose),
                          max_vox=int(max_vox))


def offsets_table(spec: _lib.GammaSpec):
    """(count, radii (z, y, x), weights (|o|/DTA)^2 over (|a|,|b|,|c|), -1 outside) -- the
    table the device uses, built by the library's host code."""
    n = ctypes.c_int(0)
    radii = (ctypes.c_int * 3)()
    w = np.empty((7, 7, 7), dtype=np.float64)
    _lib.call("pbd_gamma_offsets", ctypes.byref(spec), ctypes.byref(n), radii,
              w.ctypes.data_as(ctypes.c_void_p))
    return int(n.value), tuple(radii), w


class GammaPlan:
    """Workspace and outputs for one (nz, ny, nx) grid on one device."""

    def __init__(self, shape, spec: _lib.GammaSpec, *, device=None, maps: bool = True):
        torch = _lib.require_cuda()
        self.torch = torch
        self.device = torch.device(device or "cuda")
        self.shape = tuple(int(v) for v in shape)
        if len(self.shape) != 3:
            raise ValueError("doses must be 3-D (nz, ny, nx)")
        self.spec = spec
        nz, ny, nx = self.shape
        nbytes = _lib.query("pbd_gamma_workspace", nz, ny, nx)
        self.ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        self.stats_dev = torch.zeros(ctypes.sizeof(_lib.GammaStats), dtype=torch.uint8,
                                     device=self.device)
        self.gamma = self.mask = None
        if maps:
            self.gamma = torch.empty(self.shape, dtype=torch.float64, device=self.device)
            self.mask = torch.empty(self.shape, dtype=torch.uint8, device=self.device)

    def run(self, reference, evaluation):
        """Enqueue the gamma index of two device doses of this plan's shape (float32 or
        float64, same dtype) on the current stream."""
        torch = self.torch
        if tuple(reference.shape) != self.shape or tuple(evaluation.shape) != self.shape:
            raise ValueError(f"shape mismatch: {tuple(reference.shape)} vs "
                             f"{tuple(evaluation.shape)} (plan {self.shape})")
        if reference.dtype != evaluation.dtype or reference.dtype not in (torch.float32,
                                                                          torch.float64):
            raise ValueError("reference and evaluation must both be float32 or both float64")
        dt = _lib.DTYPE["float32" if reference.dtype == torch.float32 else "float64"]
        ref = reference.contiguous()
        ev = evaluation.contiguous()
        nz, ny, nx = self.shape
        _lib.check_arg(ref, "reference", nz * ny * nx, ref.dtype, self.device)
        _lib.check_arg(ev, "evaluation", nz * ny * nx, ev.dtype, self.device)
        _lib.call("pbd_gamma_index", ctypes.byref(self.spec), nz, ny, nx, _lib.ptr(ref),
                  _lib.ptr(ev), dt, _lib.ptr(self.gamma), _lib.ptr(self.mask),
                  _lib.ptr(self.stats_dev), _lib.ptr(self.ws), self.ws.numel(),
                  _lib.stream_handle(self.device))
        self._keep = (ref, ev)
        return self.stats_dev

    def stats(self) -> _lib.GammaStats:
        """Read the statistics of the last ``run`` (synchronises with the device)."""
        raw = self.stats_dev.cpu().numpy().tobytes()
        return _lib.GammaStats.from_buffer_copy(raw)


def _to_device(a, torch, device):
    if torch.is_tensor(a):
        t = a.to(device)
        if t.dtype not in (torch.float32, torch.float64):
            t = t.to(torch.float64)
        return t
    arr = np.asarray(a)
    if arr.dtype not in (np.float32, np.float64):
        arr = arr.astype(np.float64)
    return torch.as_tensor(np.ascontiguousarray(arr), device=device)


def _result(st: _lib.GammaStats, spec, normalization):
    if st.status != 0:
        if st.n_eval == 0 and st.ref_max > 0:
            raise ValueError("no voxel passes the low-dose mask")
        raise ValueError("reference dose max <= 0")
    return {
        "pass_rate": float(st.pass_rate),
        "gamma_mean": float(st.gamma_mean),
        "gamma_max": float(st.gamma_max),
        "gamma_p95": float(st.gamma_p95),
        "gamma_p99": float(st.gamma_p99),
        "n_eval": int(st.n_eval),
        "n_pass": int(st.n_pass),
        "dose_crit_pct": spec.dose_crit_pct,
        "dta_mm": spec.dta_mm,
        "threshold_pct": spec.threshold_pct,
        "normalization": normalization,
        "ref_max": float(st.ref_max),
        "n_dta_offsets": int(st.n_dta_offsets),
    }


def _run(reference, evaluation, spec, normalization, return_maps, device):
    torch = _lib.require_cuda()
    dev = torch.device(device or "cuda")
    ref = _to_device(reference, torch, dev)
    ev = _to_device(evaluation, torch, dev)
    if tuple(ref.shape) != tuple(ev.shape):
        raise ValueError(f"shape mismatch: {tuple(ref.shape)} vs {tuple(ev.shape)}")
    if ref.dtype != ev.dtype:
        ref, ev = ref.to(torch.float64), ev.to(torch.float64)
    plan = GammaPlan(ref.shape, spec, device=dev, maps=return_maps)
    plan.run(ref, ev)
    res = _result(plan.stats(), spec, normalization)
    if return_maps:
        res["gamma"] = plan.gamma.cpu().numpy()
        res["mask"] = plan.mask.cpu().numpy().astype(bool)
        res["ref"] = ref.to(torch.float64).cpu().numpy()
        res["eval"] = ev.to(torch.float64).cpu().numpy()
    return res


def gamma_index(reference, evaluation, spacing=(0.2, 0.2, 0.2), dose_crit_pct: float = 3.0,
                dta_mm: float = 3.0, threshold_pct: float = 10.0, normalization: str = "global",
                ref_dose: Optional[float] = None, return_maps: bool = True, *,
                max_vox: int = 6, device=None) -> dict:
    """Gamma index of ``evaluation`` against ``reference`` (same (nz, ny, nx) grid; NumPy
    arrays or torch tensors), ``spacing`` = (dz, dy, dx) cm.  Same arguments, keys and
    errors as the reference's ``gamma_index`` (gamma.py:81-164)."""
    spec = gamma_spec(spacing, dose_crit_pct, dta_mm, threshold_pct, normalization, ref_dose,
                      max_vox)
    return _run(reference, evaluation, spec, normalization, return_maps, device)


def gamma_index_torch(reference, evaluation, spacing=(0.2, 0.2, 0.2),
                      dose_crit_pct: float = 3.0, dta_mm: float = 3.0,
                      threshold_pct: float = 10.0, ref_dose=None, device: str = "cuda",
                      threshold: float = 1e-6) -> dict:
    """The reference's GPU entry point (gamma.py:213-261): global normalisation, statistics
    only.  ``threshold`` is accepted and unused, as in the reference."""
    spec = gamma_spec(spacing, dose_crit_pct, dta_mm, threshold_pct, "global", ref_dose)
    return _run(reference, evaluation, spec, "global", False, device)


def gamma_pass_rate_vs_criteria(reference, evaluation, spacing=(0.2, 0.2, 0.2),
                                criteria=((3.0, 3.0), (2.0, 2.0), (1.0, 1.0),
                                          (3.0, 2.0), (2.0, 3.0)),
                                threshold_pct: float = 10.0) -> list:
    """Pass rates over several (dose %, DTA mm) criteria (gamma.py:197-207); the doses are
    uploaded once."""
    torch = _lib.require_cuda()
    dev = torch.device("cuda")
    ref = _to_device(reference, torch, dev)
    ev = _to_device(evaluation, torch, dev)
    if tuple(ref.shape) != tuple(ev.shape):
        raise ValueError(f"shape mismatch: {tuple(ref.shape)} vs {tuple(ev.shape)}")
    if ref.dtype != ev.dtype:
        ref, ev = ref.to(torch.float64), ev.to(torch.float64)
    out = []
    for dp, dt in criteria:
        spec = gamma_spec(spacing, dp, dt, threshold_pct)
        plan = GammaPlan(ref.shape, spec, device=dev, maps=False)
        plan.run(ref, ev)
        r = _result(plan.stats(), spec, "global")
        out.append({"dose_pct": dp, "dta_mm": dt, **r})
    return out
