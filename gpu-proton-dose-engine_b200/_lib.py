"""ctypes binding of libpbdose_b200.so (the C ABI declared in include/pbdose_b200.h).

The library is loaded lazily on first use so that the host-only parts of the package
(model types, workloads) import on machines without a GPU.  Every call that reaches
the device goes through ``call`` which raises ``PbdError`` with the library's own
message for a non-zero return code.  There is no fallback: a missing library or a
missing CUDA device is an error.
"""
from __future__ import annotations

import ctypes
import os
import threading
from ctypes import POINTER, c_char_p, c_double, c_int, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbdose_b200.so")

PBD_OK = 0
PBD_ERR_TIMEOUT = -8
PREC = {"fp32": 0, "tf32x3": 1, "tf32": 2, "bf16x3": 3, "bf16": 4, "fp16x3": 5}
MAX_JOBS = 128


class PbdError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed: {msg} (code {code})")
        self.code = code


class Field(ctypes.Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("nz", c_int),
                ("dx", c_double), ("dy", c_double), ("dz", c_double),
                ("ox", c_double), ("oy", c_double), ("oz", c_double),
                ("n_sx", c_int), ("n_sy", c_int), ("n_layers", c_int),
                ("dx_spot", c_double), ("dy_spot", c_double),
                ("x0", c_double), ("y0", c_double)]


def _uniform(axis, name):
    """(first value, spacing) of a uniform axis; its centre and spacing for a lattice."""
    import numpy as np
    a = np.asarray(axis, dtype=np.float64).reshape(-1)
    if a.size == 0:
        raise ValueError(f"{name} is empty")
    if a.size == 1:
        return float(a[0]), 1.0
    d = np.diff(a)
    step = float((a[-1] - a[0]) / (a.size - 1))
    if step <= 0 or np.max(np.abs(d - step)) > 1e-9 * max(abs(step), 1.0):
        raise ValueError(f"{name} is not a uniform increasing axis")
    return float(a[0]), step


def field_from(grid, lattice) -> Field:
    """The C ABI's pbd_field from a dose grid and a spot lattice.

    Takes the reference's DoseGrid / SpotLattice as they are (model.py:27-113): the grid's
    nx, ny, nz and origin / spacing fields (or, when an object lacks those, its voxel-centre
    axes x, y -- the attributes the reference's engine reads, engines.py:227-234) and the
    lattice's n_sx, n_sy, n_layers and pitch / offset fields (or its spot_x, spot_y
    positions).  The depth origin and spacing default to 0 and 1 when absent: the dose
    kernels do not use them (the depth tables are per slice)."""
    g, L = grid, lattice
    nx, ny, nz = int(g.nx), int(g.ny), int(g.nz)
    if all(hasattr(g, a) for a in ("ox", "dx", "oy", "dy")):
        ox, dx, oy, dy = float(g.ox), float(g.dx), float(g.oy), float(g.dy)
    else:
        ox, dx = _uniform(g.x, "grid.x")
        oy, dy = _uniform(g.y, "grid.y")
    oz = float(getattr(g, "oz", 0.0))
    dz = float(getattr(g, "dz", 1.0))
    if all(hasattr(L, a) for a in ("x0", "dx_spot", "y0", "dy_spot")):
        x0, dxs, y0, dys = float(L.x0), float(L.dx_spot), float(L.y0), float(L.dy_spot)
    else:
        import numpy as np
        sx = np.asarray(L.spot_x, dtype=np.float64)
        sy = np.asarray(L.spot_y, dtype=np.float64)
        _, dxs = _uniform(sx, "lattice.spot_x")
        _, dys = _uniform(sy, "lattice.spot_y")
        x0 = float(0.5 * (sx[0] + sx[-1]))       # spot_x = x0 + (i - (n-1)/2) dx_spot
        y0 = float(0.5 * (sy[0] + sy[-1]))
    return Field(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, dz=dz, ox=ox, oy=oy, oz=oz,
                 n_sx=int(L.n_sx), n_sy=int(L.n_sy), n_layers=int(L.n_layers),
                 dx_spot=dxs, dy_spot=dys, x0=x0, y0=y0)


def field_of(problem) -> Field:
    """pbd_field of a problem: anything with ``grid`` and ``lattice`` (the reference's
    PBProblem or this package's)."""
    return field_from(problem.grid, problem.lattice)


class LutSpec(ctypes.Structure):
    _fields_ = [("nz", c_int), ("z0", c_double), ("dz", c_double), ("depth_scale", c_double),
                ("anchor_surface", c_int),
                ("sigma_x0", c_double), ("sigma_theta0", c_double), ("rho0", c_double),
                ("fe_n_sub", c_int), ("fe_max_step", c_double),
                ("straggling_model", c_int), ("strag_coef", c_double), ("strag_exp", c_double),
                ("energy_spread", c_double), ("atten_len", c_double), ("idd_n_fine", c_int),
                ("fd_step", c_double)]


class Job(ctypes.Structure):
    _fields_ = [("field", Field), ("w", c_void_p), ("idd", c_void_p), ("sigma", c_void_p),
                ("dose", c_void_p)]


class AdamParams(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("eps", ctypes.c_float), ("lo", ctypes.c_float), ("hi", ctypes.c_float),
                ("grad_scale", ctypes.c_float)]


class GradJob(ctypes.Structure):
    _fields_ = [("field", Field), ("w", c_void_p), ("idd", c_void_p), ("sigma", c_void_p),
                ("didd_dr", c_void_p), ("dsigma_dr", c_void_p), ("mask", c_void_p),
                ("presc", c_void_p), ("dose", c_void_p), ("grad_dose", c_void_p),
                ("loss", c_void_p), ("grad_w", c_void_p), ("grad_range", c_void_p)]


OBJ = {"mean": 0, "max": 1}


class GammaSpec(ctypes.Structure):
    _fields_ = [("dz", c_double), ("dy", c_double), ("dx", c_double),
                ("dose_crit_pct", c_double), ("dta_mm", c_double), ("threshold_pct", c_double),
                ("normalization", c_int), ("use_ref_dose", c_int), ("ref_dose", c_double),
                ("max_vox", c_int)]


class GammaStats(ctypes.Structure):
    _fields_ = [("pass_rate", c_double), ("gamma_mean", c_double), ("gamma_max", c_double),
                ("gamma_p95", c_double), ("gamma_p99", c_double), ("ref_max", c_double),
                ("n_eval", ctypes.c_longlong), ("n_pass", ctypes.c_longlong),
                ("n_dta_offsets", c_int), ("mask_fallback", c_int), ("status", c_int),
                ("reserved", c_int)]


DTYPE = {"float32": 0, "float64": 1}

_SIGS = {
    "pbd_strerror": (c_char_p, [c_int]),
    "pbd_version": (c_int, []),
    "pbd_field_validate": (c_int, [POINTER(Field)]),
    "pbd_set_schedule": (c_int, [c_int, c_int]),
    "pbd_profile_begin": (c_int, []),
    "pbd_profile_end": (c_int, [POINTER(c_double), POINTER(c_int), POINTER(c_double),
                                POINTER(c_int)]),
    "pbd_launch_count": (c_int, [POINTER(ctypes.c_longlong)]),
    "pbd_workspace_status": (c_int, [c_void_p, c_size_t, POINTER(c_int), c_void_p]),
    "pbd_test_hook": (c_int, [ctypes.c_ulonglong, c_int]),
    "pbd_forward_f64": (c_int, [POINTER(Field), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "pbd_lut_workspace": (c_int, [POINTER(LutSpec), c_int, POINTER(c_size_t)]),
    "pbd_build_luts": (c_int, [POINTER(LutSpec), c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "pbd_csda_range": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "pbd_energy_from_range": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "pbd_forward_workspace": (c_int, [POINTER(Field), c_int, POINTER(c_size_t)]),
    "pbd_forward": (c_int, [POINTER(Field), c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                            c_void_p, c_size_t, c_void_p]),
    "pbd_adjoint_workspace": (c_int, [POINTER(Field), c_int, POINTER(c_size_t)]),
    "pbd_adjoint": (c_int, [POINTER(Field), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                            c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_size_t, c_void_p]),
    "pbd_loss_grad_workspace": (c_int, [POINTER(Field), c_int, POINTER(c_size_t)]),
    "pbd_loss_grad": (c_int, [POINTER(Field), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p, c_int, c_void_p, c_size_t, c_void_p]),
    "pbd_forward_noalloc": (c_int, [POINTER(Field), c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                                    c_void_p]),
    "pbd_forward_batch_workspace": (c_int, [POINTER(Job), c_int, c_int, POINTER(c_size_t)]),
    "pbd_forward_batch": (c_int, [POINTER(Job), c_int, c_int, c_void_p, c_size_t, c_void_p]),
    "pbd_loss_grad_batch_workspace": (c_int, [POINTER(GradJob), c_int, c_int, POINTER(c_size_t)]),
    "pbd_loss_grad_batch": (c_int, [POINTER(GradJob), c_int, c_int, c_void_p, c_size_t, c_void_p]),
    "pbd_wed_raytrace": (c_int, [c_int, c_int, c_int, c_double, c_double, c_void_p, c_void_p,
                                 c_void_p]),
    "pbd_forward_wed_workspace": (c_int, [POINTER(Field), POINTER(LutSpec), c_int,
                                          POINTER(c_size_t)]),
    "pbd_forward_wed": (c_int, [POINTER(Field), POINTER(LutSpec), c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_size_t, c_void_p]),
    "pbd_wed_curves_workspace": (c_int, [POINTER(LutSpec), c_int, POINTER(c_size_t)]),
    "pbd_build_wed_curves": (c_int, [POINTER(LutSpec), c_int, c_void_p, c_void_p, c_void_p,
                                     c_size_t, c_void_p]),
    "pbd_forward_wed_curves": (c_int, [POINTER(Field), POINTER(LutSpec), c_void_p, c_size_t,
                                       c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                       c_size_t, c_void_p]),
    "pbd_adjoint_wed_workspace": (c_int, [POINTER(Field), POINTER(LutSpec), c_int,
                                          POINTER(c_size_t)]),
    "pbd_adjoint_wed": (c_int, [POINTER(Field), POINTER(LutSpec), c_void_p, c_size_t, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                c_size_t, c_void_p]),
    "pbd_adjoint_wed_range_workspace": (c_int, [POINTER(Field), POINTER(LutSpec), c_int,
                                                POINTER(c_size_t)]),
    "pbd_adjoint_wed_range": (c_int, [POINTER(Field), POINTER(LutSpec), c_void_p, c_size_t,
                                      c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p,
                                      c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                      c_size_t, c_void_p]),
    "pbd_adam_step": (c_int, [POINTER(AdamParams), c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "pbd_scenario_combine": (c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p]),
    "pbd_gamma_offsets": (c_int, [POINTER(GammaSpec), POINTER(c_int), c_void_p, c_void_p]),
    "pbd_gamma_workspace": (c_int, [c_int, c_int, c_int, POINTER(c_size_t)]),
    "pbd_gamma_index": (c_int, [POINTER(GammaSpec), c_int, c_int, c_int, c_void_p, c_void_p, c_int,
                                c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
}

_lib = None
_lock = threading.Lock()


def exported_symbols():
    """Names the C ABI header declares (used by the symbol test)."""
    return sorted(_SIGS)


def load():
    """Load the shared library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                    "(there is no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def strerror(code: int) -> str:
    return load().pbd_strerror(code).decode()


def call(name: str, *args) -> None:
    rc = getattr(load(), name)(*args)
    if rc != PBD_OK:
        raise PbdError(name, rc, strerror(rc))


def query(name: str, *args) -> int:
    out = c_size_t(0)
    call(name, *args, ctypes.byref(out))
    return int(out.value)


def launch_count() -> int:
    n = ctypes.c_longlong(0)
    call("pbd_launch_count", ctypes.byref(n))
    return int(n.value)


def workspace_status(ws, stream=None) -> int:
    """Status of the last library call that used the device workspace tensor ``ws``:
    PBD_OK or PBD_ERR_TIMEOUT (synchronises the stream)."""
    st = c_int(0)
    call("pbd_workspace_status", ptr(ws), ws.numel(), ctypes.byref(st),
         stream if stream is not None else stream_handle(ws.device))
    return int(st.value)


def check_workspace(ws, fn: str, stream=None) -> None:
    """Raise PbdError(PBD_ERR_TIMEOUT) when the last call on ``ws`` ran out of a device wait."""
    st = workspace_status(ws, stream)
    if st != PBD_OK:
        raise PbdError(fn, st, strerror(st))


def test_hook(wait_limit_ns: int = 0, hold: bool = False) -> None:
    """Test hook of the timeout path (pbd_test_hook): per calling thread."""
    call("pbd_test_hook", int(wait_limit_ns), 1 if hold else 0)


def profile_begin() -> None:
    call("pbd_profile_begin")


def profile_end() -> dict:
    fm, am = c_double(0), c_double(0)
    fn, an = c_int(0), c_int(0)
    call("pbd_profile_end", ctypes.byref(fm), ctypes.byref(fn), ctypes.byref(am), ctypes.byref(an))
    return {"fwd_ms": fm.value, "n_fwd": fn.value, "adj_ms": am.value, "n_adj": an.value}


def same_device(a, b) -> bool:
    """Whether two torch devices name the same GPU ("cuda" means the current one)."""
    if a.type != b.type:
        return False
    if a.type != "cuda":
        return True
    import torch
    cur = torch.cuda.current_device()
    return (cur if a.index is None else a.index) == (cur if b.index is None else b.index)


def check_arg(t, name: str, numel: int, dtype, device):
    """A tensor the library reads or writes through a raw pointer: on ``device``, of ``dtype``,
    contiguous, ``numel`` elements -- anything else would be read or written out of bounds,
    so it is refused here, before any launch."""
    import torch
    if not torch.is_tensor(t):
        raise TypeError(f"{name} must be a torch tensor")
    if not same_device(t.device, device):
        raise ValueError(f"{name} is on {t.device}, expected {device}")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.numel() != numel:
        raise ValueError(f"{name} has {t.numel()} elements, expected {numel}")
    return t


def ptr(t) -> int | None:
    """Device address of a torch tensor (None for None)."""
    if t is None:
        return None
    return int(t.data_ptr())


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("a CUDA device is required: this engine has no CPU path")
    return torch


def stream_handle(device=None) -> int:
    torch = require_cuda()
    return int(torch.cuda.current_stream(device).cuda_stream)


def precision_code(p) -> int:
    if isinstance(p, int):
        return p
    try:
        return PREC[str(p).lower()]
    except KeyError:
        raise ValueError(f"unknown precision {p!r}; expected one of {sorted(PREC)}") from None
