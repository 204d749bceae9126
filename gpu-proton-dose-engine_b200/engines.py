"""Dose engines: the drop-in ``torch_separable`` and its differentiable, plan-based form.

``torch_separable`` keeps the reference's signature and return convention
(engines.py:208-283) and computes the per-layer exact separable dose with the CUDA
library.  ``DosePlan`` holds one field's geometry, weights and depth tables on the
device for repeated forward / adjoint / loss-gradient calls; ``SeparableDose`` is the
``torch.autograd.Function`` over it, differentiable in the spot weights and the
per-layer range shifts.  There is no CPU path: every function here that computes a
dose needs the built library and a CUDA device.
"""
from __future__ import annotations

import contextlib
import ctypes
import time
from typing import Optional

import numpy as np

from . import _lib
from . import physics as ph
from .model import PBProblem

INV_SQRT_2PI = 1.0 / np.sqrt(2.0 * np.pi)
# "auto": the tensor cores' hi/lo split in FP16 (FP16x3: within 1e-6 of FP64 -- 4e-7 on the
# clinical field -- and the fastest mode that meets it) for lattices they take (<= 64 x 64
# spots), else the FP32 kernel on the CUDA cores
DEFAULT_PRECISION = "auto"


def resolve_precision(precision, lattice) -> int:
    """Library precision code of ``precision`` for a lattice ("auto": see DEFAULT_PRECISION)."""
    if precision is None or str(precision).lower() == "auto":
        wide = int(lattice.n_sx) > 64 or int(lattice.n_sy) > 64
        return _lib.PREC["fp32" if wide else "fp16x3"]
    return _lib.precision_code(precision)
DEFAULT_FD_STEP = 0.005   # cm: central-difference step of the range-derivative tables

# The loss gradient's small results, in the order they sit in one packed buffer.
PACKED_RESULTS = ("grad_w", "grad_range", "loss")


def packed_result_layout(n_weights: int, n_layers: int):
    """Byte offsets and sizes of grad_w (float32), grad_range (float32) and loss (float64)
    in one packed buffer, each at a 256-byte boundary, and the bytes that span them: a single
    copy of that span moves all three results between device and host."""
    sizes = (4 * int(n_weights), 4 * int(n_layers), 8)
    offs, o = [], 0
    for n in sizes:
        offs.append(o)
        o += (n + 255) // 256 * 256
    return tuple(offs), sizes, offs[-1] + sizes[-1]


def packed_result_views(buf, w_shape, n_layers: int) -> dict:
    """Typed views of grad_w, grad_range and loss in a uint8 buffer with the packed layout
    (``buf`` is kept under the key "packed")."""
    import torch
    offs, sizes, span = packed_result_layout(int(np.prod(w_shape)), n_layers)
    if buf.dtype != torch.uint8 or buf.dim() != 1 or buf.numel() < span:
        raise ValueError(f"packed buffer must be a 1-D uint8 tensor of at least {span} bytes")
    (o0, o1, o2), (n0, n1, n2) = offs, sizes
    return {"grad_w": buf[o0:o0 + n0].view(torch.float32).view(tuple(w_shape)),
            "grad_range": buf[o1:o1 + n1].view(torch.float32),
            "loss": buf[o2:o2 + n2].view(torch.float64).view(()),
            "packed": buf[:span]}


def lateral_kernel(vox_axis, spot_axis, sigma, normalized: bool = True) -> np.ndarray:
    """Host utility with the reference's semantics (engines.py:49-61); not used by the engine,
    whose kernels generate these factors on the fly."""
    d = (np.asarray(vox_axis)[:, None] - np.asarray(spot_axis)[None, :]) ** 2
    s = np.clip(np.asarray(sigma, dtype=np.float64), 1e-9, None)
    out = np.exp(-d / (2.0 * s[..., None, None] ** 2))
    if normalized:
        out = out * (INV_SQRT_2PI / s)[..., None, None]
    return out


def relative_error(a, b, mask=None) -> dict:
    """Error of ``a`` against reference ``b`` (engines.py:364-378): max |a-b| / max |b| etc."""
    a = np.asarray(a.detach().cpu() if hasattr(a, "detach") else a, dtype=np.float64)
    b = np.asarray(b.detach().cpu() if hasattr(b, "detach") else b, dtype=np.float64)
    if mask is None:
        mask = np.ones_like(b, dtype=bool)
    d = (a - b)[mask]
    ref_max = float(np.max(np.abs(b))) or 1.0
    return {
        "max_abs_err": float(np.abs(d).max()) if d.size else 0.0,
        "max_rel_err_global": float(np.abs(d).max() / ref_max) if d.size else 0.0,
        "rms_err": float(np.sqrt((d**2).mean())) if d.size else 0.0,
        "rms_rel_global": float(np.sqrt((d**2).mean()) / ref_max) if d.size else 0.0,
        "n_vox": int(mask.sum()),
    }


def normalize_dose(d, mode: str = "max", roi=None):
    """Dose normalisation (engines.py:381-388)."""
    d = np.asarray(d, dtype=np.float64)
    ref = float(d[roi].max()) if (mode == "roi_max" and roi is not None) else float(d.max())
    return d / (ref if ref > 0 else 1.0), ref


def operation_counts(problem: PBProblem, active_pairs: Optional[int] = None) -> dict:
    """Multiply-add counts of the separable contraction, with the layer factor included
    (the reference's engines.py:83-96 counts one layer).  ``active_pairs`` = number of
    (layer, slice) pairs with non-zero IDD; default: all."""
    g, L = problem.grid, problem.lattice
    per_pair = L.n_sx * L.n_sy * g.ny + g.nx * L.n_sx * g.ny
    pairs = L.n_layers * g.nz if active_pairs is None else int(active_pairs)
    return {"naive": L.n_spots * g.n_vox, "separable_exact": per_pair * pairs, "pairs": pairs,
            "M": L.n_spots, "N_vox": g.n_vox, "L": L.n_layers}


class _Workspace:
    """Device scratch buffers cached by (name, size)."""

    def __init__(self, device):
        self.device = device
        self._bufs = {}

    def get(self, name, nbytes):
        torch = _lib.require_cuda()
        buf = self._bufs.get(name)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)
            self._bufs[name] = buf
        return buf


class DosePlan:
    """One field resident on the device: geometry, weights, depth tables, scratch.

    ``tables`` may be ("problem") the problem's own host tables (the drop-in's
    semantics), or ("device") tables rebuilt by the device LUT builder from the lattice
    energies, which also provides the range-derivative tables needed for
    dL/d(range shift)."""

    def __init__(self, problem: PBProblem, *, precision: str = DEFAULT_PRECISION,
                 tables: str = "device", fd_step: float = DEFAULT_FD_STEP, device=None,
                 range_shift=None):
        torch = _lib.require_cuda()
        self.torch = torch
        self.device = torch.device(device or "cuda")
        self.problem = problem
        self.field = _lib.field_of(problem)
        _lib.call("pbd_field_validate", ctypes.byref(self.field))
        self.precision = resolve_precision(precision, problem.lattice)
        self.fd_step = float(fd_step)
        g, L = problem.grid, problem.lattice
        self.shape = (g.nz, g.ny, g.nx)
        self.w = torch.as_tensor(np.ascontiguousarray(L.ensure_weights(), dtype=np.float32),
                                 device=self.device)
        en = getattr(L, "energies", None)
        self.energies = None if en is None else np.asarray(en, dtype=np.float64)
        self.ws = _Workspace(self.device)
        self.schedule = None          # (layers per forward item, adjoint item size) or None
        self._tuned = False           # cached tuning lookup (False = not looked up yet)
        self._tuning_off = False
        self.tables_mode = tables
        self.range_shift = None
        if tables == "problem":
            self.idd = torch.as_tensor(np.ascontiguousarray(problem.idd, dtype=np.float64),
                                       device=self.device)
            self.sigma = torch.as_tensor(np.ascontiguousarray(problem.sigma, dtype=np.float64),
                                         device=self.device)
            self.didd = self.dsig = None
        elif tables == "device":
            if self.energies is None:
                raise ValueError("device tables need lattice.energies")
            self.set_range_shift(range_shift)
        else:
            raise ValueError("tables must be 'problem' or 'device'")

    # -- tables ------------------------------------------------------------------
    def set_range_shift(self, range_shift=None):
        """(Re)build the depth tables on the device at CSDA ranges R0_l + range_shift_l."""
        torch = self.torch
        g = self.problem.grid
        if range_shift is not None:
            rs = torch.as_tensor(range_shift, dtype=torch.float64, device=self.device).reshape(-1)
            if self.range_shift is not None and torch.equal(rs, self.range_shift):
                return
        elif self.range_shift is None and getattr(self, "idd", None) is not None:
            return
        t = ph.build_tables(g.nz, g.oz, g.dz, self.energies, range_shift=range_shift,
                            fd_step=self.fd_step, device=self.device)
        self.idd, self.sigma, self.didd, self.dsig = t.idd, t.sigma, t.didd_dr, t.dsigma_dr
        self.range_shift = None if range_shift is None else rs.clone()
        self._tuned = False

    def active_pairs(self) -> int:
        return int((self.idd != 0).sum().item())

    def _sched(self):
        """Work-item sizes for this plan's calls: an explicit ``schedule``, else the tuned one
        for this geometry (looked up once per set of tables), else the library default."""
        from . import tuning
        if self._tuning_off:
            return contextlib.nullcontext()
        s = self.schedule
        if s is None:
            if self._tuned is False:
                self._tuned = tuning.lookup(self, "loss_grad")
            s = self._tuned
        return tuning.schedule(*s) if s else contextlib.nullcontext()

    # -- weights -----------------------------------------------------------------
    def _weights(self, w):
        torch = self.torch
        if w is None:
            return self.w
        if not torch.is_tensor(w):
            w = torch.as_tensor(np.asarray(w, dtype=np.float32))
        if not _lib.same_device(w.device, self.device):
            w = w.to(self.device, non_blocking=True)
        w = w.to(torch.float32).contiguous()
        return _lib.check_arg(w, "w", self.w.numel(), torch.float32, self.device)

    def _check_tables(self, idd, sigma):
        n = self.w.shape[0] * self.shape[0]
        _lib.check_arg(idd, "idd", n, self.torch.float64, self.device)
        _lib.check_arg(sigma, "sigma", n, self.torch.float64, self.device)

    # -- forward -------------------------------------------------------------------
    def forward(self, w=None, out=None, idd=None, sigma=None):
        torch = self.torch
        w = self._weights(w)
        idd = self.idd if idd is None else idd
        sigma = self.sigma if sigma is None else sigma
        self._check_tables(idd, sigma)
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        nvox = self.shape[0] * self.shape[1] * self.shape[2]
        _lib.check_arg(out, "out", nvox, torch.float32, self.device)
        with self._sched():
            nbytes = _lib.query("pbd_forward_workspace", ctypes.byref(self.field), self.precision)
            ws = self.ws.get("fwd", nbytes)
            _lib.call("pbd_forward", ctypes.byref(self.field), _lib.ptr(w), _lib.ptr(idd),
                      _lib.ptr(sigma), _lib.ptr(out), self.precision, _lib.ptr(ws), ws.numel(),
                      _lib.stream_handle(self.device))
        return out

    def forward_f64(self, w=None, out=None):
        """The dose in FP64 on the CUDA cores (pbd_forward_f64): weights, Gaussians, products
        and sums in float64.  ``w`` defaults to the plan's weights (float32 values, exact in
        float64); returns a float64 (nz, ny, nx) tensor."""
        torch = self.torch
        if w is None:
            w = self.w
        elif not torch.is_tensor(w):
            w = torch.as_tensor(np.asarray(w, dtype=np.float64))
        w = w.to(self.device, torch.float64).contiguous()
        _lib.check_arg(w, "w", self.w.numel(), torch.float64, self.device)
        self._check_tables(self.idd, self.sigma)
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float64, device=self.device)
        nvox = self.shape[0] * self.shape[1] * self.shape[2]
        _lib.check_arg(out, "out", nvox, torch.float64, self.device)
        _lib.call("pbd_forward_f64", ctypes.byref(self.field), _lib.ptr(w), _lib.ptr(self.idd),
                  _lib.ptr(self.sigma), _lib.ptr(out), _lib.stream_handle(self.device))
        return out

    def check(self, op: str = "fwd") -> None:
        """Raise PbdError(PBD_ERR_TIMEOUT) if a device wait of the plan's last ``op`` call
        ("fwd", "adj" or "lossgrad") ran out (its outputs are NaN then); synchronises."""
        ws = self.ws._bufs.get(op)
        if ws is not None:
            _lib.check_workspace(ws, f"DosePlan.{op}", _lib.stream_handle(self.device))

    # -- adjoint -------------------------------------------------------------------
    def adjoint(self, grad_dose, w=None, idd=None, sigma=None, didd=None, dsig=None,
                with_range: bool = True):
        torch = self.torch
        w = self._weights(w)
        idd = self.idd if idd is None else idd
        sigma = self.sigma if sigma is None else sigma
        didd = self.didd if didd is None else didd
        dsig = self.dsig if dsig is None else dsig
        with_range = with_range and didd is not None and dsig is not None
        self._check_tables(idd, sigma)
        if with_range:
            self._check_tables(didd, dsig)
        g = grad_dose.to(self.device, torch.float32).contiguous()
        _lib.check_arg(g, "grad_dose", self.shape[0] * self.shape[1] * self.shape[2],
                       torch.float32, self.device)
        gw = torch.empty_like(w)
        gr = torch.zeros(w.shape[0], dtype=torch.float32, device=self.device) if with_range else None
        with self._sched():
            nbytes = _lib.query("pbd_adjoint_workspace", ctypes.byref(self.field), self.precision)
            ws = self.ws.get("adj", nbytes)
            _lib.call("pbd_adjoint", ctypes.byref(self.field), _lib.ptr(w), _lib.ptr(idd),
                      _lib.ptr(sigma), _lib.ptr(didd if with_range else None),
                      _lib.ptr(dsig if with_range else None), _lib.ptr(g), _lib.ptr(gw),
                      _lib.ptr(gr), self.precision, _lib.ptr(ws), ws.numel(),
                      _lib.stream_handle(self.device))
        return gw, gr

    # -- fused loss gradient -------------------------------------------------------
    def loss_grad(self, mask, presc, w=None, outputs=None):
        """L = sum m (D - P)^2 and its gradients in one library call.

        Returns a dict of device tensors: loss (float64 scalar), dose, grad_dose,
        grad_w, grad_range (None when the plan has no range-derivative tables)."""
        torch = self.torch
        w = self._weights(w)
        o = outputs or self.alloc_outputs()
        with_range = self.didd is not None
        nvox = self.shape[0] * self.shape[1] * self.shape[2]
        f32, dev = torch.float32, self.device
        _lib.check_arg(mask, "mask", nvox, f32, dev)
        _lib.check_arg(presc, "presc", nvox, f32, dev)
        _lib.check_arg(o["dose"], "outputs['dose']", nvox, f32, dev)
        _lib.check_arg(o["grad_dose"], "outputs['grad_dose']", nvox, f32, dev)
        _lib.check_arg(o["loss"], "outputs['loss']", 1, torch.float64, dev)
        _lib.check_arg(o["grad_w"], "outputs['grad_w']", self.w.numel(), f32, dev)
        if with_range:
            _lib.check_arg(o["grad_range"], "outputs['grad_range']", self.w.shape[0], f32, dev)
        with self._sched():
            nbytes = _lib.query("pbd_loss_grad_workspace", ctypes.byref(self.field),
                                self.precision)
            ws = self.ws.get("lossgrad", nbytes)
            _lib.call("pbd_loss_grad", ctypes.byref(self.field), _lib.ptr(w), _lib.ptr(self.idd),
                      _lib.ptr(self.sigma), _lib.ptr(self.didd if with_range else None),
                      _lib.ptr(self.dsig if with_range else None), _lib.ptr(mask),
                      _lib.ptr(presc), _lib.ptr(o["dose"]), _lib.ptr(o["grad_dose"]),
                      _lib.ptr(o["loss"]), _lib.ptr(o["grad_w"]),
                      _lib.ptr(o["grad_range"] if with_range else None), self.precision,
                      _lib.ptr(ws), ws.numel(), _lib.stream_handle(self.device))
        if not with_range:
            o = dict(o, grad_range=None)
        return o

    def alloc_outputs(self, packed: bool = False):
        """Device tensors for ``loss_grad``.  With ``packed``, grad_w, grad_range and loss are
        views of one buffer (``packed_result_layout``; the buffer is under "packed"), so that
        one copy downloads all three (see ``alloc_host_results``)."""
        torch = self.torch
        nl = self.w.shape[0]
        out = {"dose": torch.empty(self.shape, dtype=torch.float32, device=self.device),
               "grad_dose": torch.empty(self.shape, dtype=torch.float32, device=self.device)}
        if packed:
            span = packed_result_layout(self.w.numel(), nl)[2]
            buf = torch.zeros(span, dtype=torch.uint8, device=self.device)
            out.update(packed_result_views(buf, tuple(self.w.shape), nl))
        else:
            out.update({"loss": torch.zeros((), dtype=torch.float64, device=self.device),
                        "grad_w": torch.empty_like(self.w),
                        "grad_range": torch.zeros(nl, dtype=torch.float32, device=self.device)})
        return out

    def alloc_host_results(self) -> dict:
        """Pinned host tensors grad_w, grad_range and loss in the packed layout of
        ``alloc_outputs(packed=True)`` (the whole buffer under "packed")."""
        torch = self.torch
        nl = self.w.shape[0]
        span = packed_result_layout(self.w.numel(), nl)[2]
        buf = torch.zeros(span, dtype=torch.uint8).pin_memory()
        return packed_result_views(buf, tuple(self.w.shape), nl)


class LossGradGraph:
    """One ``DosePlan.loss_grad`` captured into a CUDA graph, for loops that evaluate the same
    field repeatedly (plan optimisation, line searches): a replay launches the library's
    kernels without the per-call host work.

    The graph reads the weights from ``self.w`` (a device tensor owned by this object); with
    ``host_w`` (a pinned host tensor of the weights' shape) every replay first uploads it,
    and with ``host_out`` (a dict of pinned host tensors keyed like the outputs: any of
    "loss", "grad_w", "grad_range", "dose") every replay ends by downloading those results.
    The device results sit in one packed buffer; when ``host_out`` comes from
    ``DosePlan.alloc_host_results`` (its "packed" key), grad_w, grad_range and loss come back
    in one copy.  ``mask`` and ``presc`` stay referenced; change their contents in place, not
    the tensors."""

    def __init__(self, plan: "DosePlan", mask, presc, host_w=None, host_out=None):
        torch = plan.torch
        self.plan = plan
        self.mask, self.presc = mask, presc
        self.w = plan.w.clone()
        self.out = plan.alloc_outputs(packed=True)
        self.host_w, self.host_out = host_w, dict(host_out or {})
        copies = []
        packed = "packed" in self.host_out
        if packed:
            hp = self.host_out["packed"]
            if hp.numel() != self.out["packed"].numel() or hp.dtype != self.out["packed"].dtype:
                raise ValueError("host_out['packed'] does not have the packed result layout")
            copies.append((hp, self.out["packed"]))
        for k, t in self.host_out.items():
            if k == "packed" or (packed and k in PACKED_RESULTS):
                continue   # inside the packed copy
            copies.append((t, self.out[k]))
        self._copies = copies
        # first call outside the capture: workspace allocation and schedule lookup
        plan.loss_grad(mask, presc, w=self.w, outputs=self.out)
        torch.cuda.synchronize(plan.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            if host_w is not None:
                self.w.copy_(host_w, non_blocking=True)
            plan.loss_grad(mask, presc, w=self.w, outputs=self.out)
            for dst, src in self._copies:
                dst.copy_(src, non_blocking=True)

    def replay(self):
        """Enqueue one evaluation on the current stream; returns the device outputs."""
        self.graph.replay()
        return self.out


def _autograd_function():
    torch = _lib.require_cuda()

    class SeparableDose(torch.autograd.Function):
        """D(w, range_shift) with a hand-written backward (the adjoint kernel)."""

        @staticmethod
        def forward(ctx, w, range_shift, plan):
            if range_shift is not None:
                plan.set_range_shift(range_shift.detach())
            dose = plan.forward(w)
            ctx.plan = plan
            ctx.tables = (plan.idd, plan.sigma, plan.didd, plan.dsig)
            ctx.has_shift = range_shift is not None
            ctx.shift_dtype = None if range_shift is None else range_shift.dtype
            ctx.save_for_backward(w)
            return dose

        @staticmethod
        def backward(ctx, grad_dose):
            (w,) = ctx.saved_tensors
            idd, sig, didd, dsig = ctx.tables
            need_r = ctx.has_shift and ctx.needs_input_grad[1]
            gw, gr = ctx.plan.adjoint(grad_dose, w, idd, sig, didd, dsig, with_range=need_r)
            gr = gr.to(ctx.shift_dtype) if (need_r and gr is not None) else None
            return gw, gr, None

    return SeparableDose


_SEPARABLE_DOSE = None


def separable_dose(w, range_shift, plan: DosePlan):
    """Differentiable dose D(w, range_shift); gradients through the CUDA adjoint."""
    global _SEPARABLE_DOSE
    if _SEPARABLE_DOSE is None:
        _SEPARABLE_DOSE = _autograd_function()
    return _SEPARABLE_DOSE.apply(w, range_shift, plan)


def torch_separable(problem, device: str = "cuda", dtype=None, allow_tf32: bool = False,
                    per_layer: bool = True, layer_chunk: Optional[int] = None,
                    return_timing: bool = False, return_intermediates: bool = False,
                    precision: Optional[str] = None):
    """Drop-in for the reference's per-layer batched-matmul engine (engines.py:208-283).

    Same arguments and return value: a CUDA tensor D of shape (nz, ny, nx), or
    (D, seconds) with ``return_timing``.  ``problem`` may be the reference's own
    PBProblem: only ``grid``, ``lattice`` (axes, spot pitch and offsets,
    ``ensure_weights()``) and ``idd`` / ``sigma`` are read, as the reference does
    (engines.py:227-234, 257-259).  Like the reference it uploads the problem's arrays on
    every call and synchronises before returning.

    * ``dtype``: None or torch.float32 give a float32 dose from the tensor cores (split
      FP16, three products with power-of-two scaling: within 1e-6 of FP64; lattices wider
      than 64 spots use the FP32 kernel on the CUDA cores); torch.float64 gives a float64
      dose computed in FP64 on the CUDA cores (the reference's float64 mode, ~1e-15).
    * ``allow_tf32``: the reference's flag for TF32 tensor cores; its run with the flag
      kept FP32 accuracy (1.51e-7, benchmark_full.json:68-81), so it keeps the default
      split form, within 1e-6.  One-product TF32 (~1e-4) is available only as
      ``precision="tf32"``.
    * ``precision``: any mode explicitly ("fp32", "fp16x3", "tf32x3", "bf16x3", "tf32",
      "bf16").
    * ``layer_chunk``: active layers per forward work item, for this call only (the
      reference used it to bound memory; here it only sets the work granularity).

    Differences, all loud: ``device`` must be CUDA (no CPU path) and ``per_layer=False``
    (the single-sigma approximation) is not provided.  A device wait that ran out raises
    PbdError (PBD_ERR_TIMEOUT)."""
    torch = _lib.require_cuda()
    if not str(device).startswith("cuda"):
        raise RuntimeError("torch_separable: this engine runs on CUDA only (no CPU path)")
    if dtype not in (None, torch.float32, torch.float64):
        raise NotImplementedError(f"torch_separable: dtype {dtype} (float32 or float64 only)")
    if not per_layer:
        raise NotImplementedError("torch_separable: the single-sigma approximation "
                                  "(per_layer=False) is not provided; use per_layer=True")
    prec = precision or DEFAULT_PRECISION
    t0 = time.perf_counter()
    plan = DosePlan(problem, precision=prec, tables="problem", device=device)
    if layer_chunk:
        plan.schedule = (int(layer_chunk), 0)
    if dtype == torch.float64:
        dose = plan.forward_f64(np.ascontiguousarray(problem.lattice.ensure_weights(),
                                                     dtype=np.float64))
        torch.cuda.synchronize(plan.device)
    else:
        dose = plan.forward()
        plan.check("fwd")        # synchronises; raises if a device wait ran out
    t1 = time.perf_counter()
    return (dose, t1 - t0) if return_timing else dose
