"""Autotuner of the layer-to-CTA schedule.

The forward splits each depth slice's active layers into work items of C_f layers and
the adjoint groups C_a slices (FP32 path) or layers (tensor-core path) per item.  Small
items balance the persistent grid; large ones amortise per-item work (operand set-up,
the tensor-core pipeline drain, the partial-slice traffic).  The best pair depends on the
geometry (how many (layer, slice) pairs are active and how unevenly), so it is measured:
``tune(plan)`` times the plan's operation for each candidate pair with CUDA events,
keeps the fastest, and caches it per geometry and precision in a JSON file
(``$PBD_TUNING_CACHE`` or ``~/.cache/pbdose_b200/tuning.json``).  ``DosePlan`` applies a
cached choice automatically.
"""
from __future__ import annotations

import contextlib
import json
import os
import threading

from . import _lib

# 0 = the library's default: 20 forward layers per unit (split FP16), and for one job the
# adjoint's unit size derived on the device from the active pairs (ceil(T / grid) + 1); an
# explicit adjoint size switches that derivation off, so 0 stays a candidate.
CANDIDATES_FWD = (0, 12, 16, 24, 32)
CANDIDATES_ADJ = (0, 4, 8, 10)
_lock = threading.Lock()


def cache_path() -> str:
    return os.environ.get("PBD_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "pbdose_b200", "tuning.json"))


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(d: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass   # an unwritable cache only costs a re-tune


def geometry_key(plan, op: str) -> str:
    f = plan.field
    return (f"{op}|{f.nx}x{f.ny}x{f.nz}|{f.n_sx}x{f.n_sy}x{f.n_layers}|p{plan.precision}"
            f"|a{plan.active_pairs()}")


@contextlib.contextmanager
def schedule(fwd: int, adj: int):
    """Work-item sizes for the library calls made inside the block (this thread)."""
    _lib.call("pbd_set_schedule", int(fwd), int(adj))
    try:
        yield
    finally:
        _lib.call("pbd_set_schedule", 0, 0)


def lookup(plan, op: str):
    with _lock:
        v = _load().get(geometry_key(plan, op))
    return tuple(v["schedule"]) if v else None


def tune(plan, op: str = "loss_grad", mask=None, presc=None, fwd_candidates=CANDIDATES_FWD,
         adj_candidates=CANDIDATES_ADJ, reps: int = 5, store: bool = True):
    """Time ``op`` ("forward" or "loss_grad") for every candidate schedule and return
    (best (fwd, adj), {(fwd, adj): ms})."""
    torch = _lib.require_cuda()
    if op == "loss_grad" and (mask is None or presc is None):
        raise ValueError("loss_grad tuning needs mask and presc")
    adj_list = adj_candidates if op == "loss_grad" else (0,)
    outs = plan.alloc_outputs()
    timings = {}
    saved = plan.schedule
    plan.schedule = None
    plan._tuning_off = True
    try:
        for cf in fwd_candidates:
            for ca in adj_list:
                with schedule(cf, ca):
                    run = (lambda: plan.forward(out=outs["dose"])) if op == "forward" else \
                        (lambda: plan.loss_grad(mask, presc, outputs=outs))
                    run()   # warm-up (workspace, attributes)
                    torch.cuda.synchronize(plan.device)
                    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                    ev[0].record()
                    for _ in range(reps):
                        run()
                    ev[1].record()
                    torch.cuda.synchronize(plan.device)
                    timings[(cf, ca)] = ev[0].elapsed_time(ev[1]) / reps
    finally:
        plan.schedule = saved
        plan._tuning_off = False
        plan._tuned = False
    best = min(timings, key=timings.get)
    if store:
        with _lock:
            d = _load()
            d[geometry_key(plan, op)] = {"schedule": list(best), "ms": timings[best]}
            _store(d)
    return best, timings
