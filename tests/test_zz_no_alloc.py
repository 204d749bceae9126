"""The allocation-free forward entry point, pbd_forward_noalloc, through the C ABI.

Some callers cannot allocate device memory once they are running -- a real-time
adaptive-therapy loop that reserved everything at start-up, or a host that owns the GPU
through its own memory pool -- so they cannot provide the workspace the other entry
points take.  pbd_forward_noalloc keeps its scratch in a fixed array inside the library.
This test checks it against pbd_forward (the workspace version) on two calls in a row
with different fields, so the second call also shows that the shared array's leftovers
from the first call do not leak into its result.  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden, has_gpu, load_pkg

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

DOSE_TOL = 1e-6   # the dose tolerance of the other GPU parity tests


def _inputs(pb, torch, prob):
    L = prob.lattice
    w = torch.as_tensor(np.ascontiguousarray(L.ensure_weights(), dtype=np.float32), device="cuda")
    idd = torch.as_tensor(np.ascontiguousarray(prob.idd, dtype=np.float64), device="cuda")
    sig = torch.as_tensor(np.ascontiguousarray(prob.sigma, dtype=np.float64), device="cuda")
    return w, idd, sig


def _with_workspace(pb, torch, lib, prob, prec):
    f = pb._lib.field_of(prob)
    w, idd, sig = _inputs(pb, torch, prob)
    out = torch.empty(prob.grid.shape, dtype=torch.float32, device="cuda")
    n = ctypes.c_size_t(0)
    assert lib.pbd_forward_workspace(ctypes.byref(f), prec, ctypes.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device="cuda")
    rc = lib.pbd_forward(ctypes.byref(f), w.data_ptr(), idd.data_ptr(), sig.data_ptr(),
                         out.data_ptr(), prec, ws.data_ptr(), n.value,
                         torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.pbd_strerror(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _without(pb, torch, lib, prob, prec):
    f = pb._lib.field_of(prob)
    w, idd, sig = _inputs(pb, torch, prob)
    out = torch.full(prob.grid.shape, 7.0, dtype=torch.float32, device="cuda")   # stale bytes
    rc = lib.pbd_forward_noalloc(ctypes.byref(f), w.data_ptr(), idd.data_ptr(), sig.data_ptr(),
                                 out.data_ptr(), prec, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, lib.pbd_strerror(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _fields(pb):
    wl = pb.workloads.build_workload(0)
    lut = golden("luts_cfg0.npz")
    a = pb.model.problem_from_workload(wl, lut["energies"], lut["idd"], lut["sigma"])
    rng = np.random.default_rng(5)
    M = pb.model
    grid = M.DoseGrid(150, 70, 21, 0.15, 0.2, 0.3, -11.0, -6.9, 0.0)
    w = rng.uniform(0.1, 1.0, (5, 13, 61))
    lat = M.SpotLattice(61, 13, 5, 0.25, 0.3, x0=0.05, y0=-0.1, weights=w)
    idd = rng.uniform(0.0, 5.0, (5, 21))
    idd[rng.random((5, 21)) < 0.3] = 0.0
    b = M.PBProblem(grid, lat, idd, rng.uniform(0.2, 0.8, (5, 21)))
    return a, b


def _deep_field(pb):
    """64 layers (the entry point's limit: one item holds every layer of its slice) on a
    128 x 96 grid, with slices that no layer reaches (all-zero depth-dose columns)."""
    rng = np.random.default_rng(17)
    M = pb.model
    nl, nz = 64, 12
    grid = M.DoseGrid(128, 96, nz, 0.2, 0.2, 0.25, -12.7, -9.5, 0.0)
    w = rng.uniform(0.2, 1.2, (nl, 21, 25))
    lat = M.SpotLattice(25, 21, nl, 0.5, 0.5, x0=0.1, y0=-0.05, weights=w)
    idd = rng.uniform(0.1, 3.0, (nl, nz))
    idd[rng.random((nl, nz)) < 0.2] = 0.0
    idd[:, [3, 8]] = 0.0                        # slices no layer reaches
    return M.PBProblem(grid, lat, idd, rng.uniform(0.3, 0.9, (nl, nz)))


def _oracle(prob):
    from oracle import engine_ref as er
    g, L = prob.grid, prob.lattice
    return er.separable_f64(g.x, g.y, L.spot_x, L.spot_y, L.weights, prob.idd, prob.sigma)


@pytest.mark.parametrize("prec", [0, 1])   # FP32 and TF32x3
def test_noalloc_matches_workspace_forward_two_calls(prec):
    import torch
    pb = load_pkg()
    lib = pb._lib.load()
    first, second = _fields(pb)
    got1 = _without(pb, torch, lib, first, prec)
    got2 = _without(pb, torch, lib, second, prec)
    for prob, got in ((first, got1), (second, got2)):
        ref = _with_workspace(pb, torch, lib, prob, prec)
        err = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
        assert err <= DOSE_TOL, err
    # the ragged second field against the float64 oracle directly
    ref64 = _oracle(second)
    assert float(np.max(np.abs(got2 - ref64)) / np.max(np.abs(ref64))) <= DOSE_TOL


# FP32 on the CUDA cores sums a slice's 64 layers in one register chain here and in 4-layer
# chunks in pbd_forward: two float32 summation orders, each ~1e-6 of max from float64 on this
# 64-layer field, so the FP32 case states 2e-6; the tensor-core split form keeps 1e-6.
DEEP_TOL = {0: 2e-6, 1: DOSE_TOL}


@pytest.mark.parametrize("prec", [0, 1])   # FP32 and TF32x3
def test_noalloc_64_layers_and_empty_slices(prec):
    import torch
    pb = load_pkg()
    lib = pb._lib.load()
    prob = _deep_field(pb)
    got = _without(pb, torch, lib, prob, prec)
    got_again = _without(pb, torch, lib, prob, prec)
    ref = _with_workspace(pb, torch, lib, prob, prec)
    ref64 = _oracle(prob)
    for g in (got, got_again):
        assert float(np.max(np.abs(g - ref)) / np.max(np.abs(ref))) <= DEEP_TOL[prec]
        assert float(np.max(np.abs(g - ref64)) / np.max(np.abs(ref64))) <= DEEP_TOL[prec]
        assert np.all(g[[3, 8]] == 0.0)          # stale bytes overwritten with zeros


def test_noalloc_rejects_what_does_not_fit():
    pb = load_pkg()
    lib = pb._lib.load()
    fake = 0x1000
    big_l = pb._lib.Field(nx=32, ny=32, nz=8, dx=0.2, dy=0.2, dz=0.2, ox=0, oy=0, oz=0, n_sx=3,
                          n_sy=3, n_layers=65, dx_spot=0.5, dy_spot=0.5, x0=0, y0=0)
    assert lib.pbd_forward_noalloc(ctypes.byref(big_l), fake, fake, fake, fake, 0, None) == -5
    many = pb._lib.Field(nx=1024, ny=1024, nz=1000, dx=0.2, dy=0.2, dz=0.2, ox=0, oy=0, oz=0,
                         n_sx=3, n_sy=3, n_layers=4, dx_spot=0.5, dy_spot=0.5, x0=0, y0=0)
    assert lib.pbd_forward_noalloc(ctypes.byref(many), fake, fake, fake, fake, 0, None) == -7
