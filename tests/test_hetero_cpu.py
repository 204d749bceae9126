"""Heterogeneous media, host side (no GPU): the oracle's WED against fixtures made with the
reference's own wed_from_density_path (bit for bit per voxel path, 1e-13 cumulated), the
package's host copy of that helper, and argument validation of the C ABI."""
import ctypes
import os

import numpy as np
import pytest

from conftest import golden, load_pkg
from oracle import hetero_ref as hr


@pytest.mark.parametrize("case", [0, 1, 2])
def test_oracle_wed_matches_reference_fixture(case):
    z = golden("hetero.npz")
    rho, want = z[f"rho{case}"].astype(np.float64), z[f"wed{case}"]
    oz, dz = z[f"grid{case}"]
    for y in range(rho.shape[1]):
        for x in range(rho.shape[2]):
            for k in range(rho.shape[0]):
                dens, lens = hr.wed_path(rho[:, y, x], oz, dz, k)
                assert float(np.sum(dens * lens)) == want[k, y, x]
    got = hr.wed_ref(rho, oz, dz)
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


def test_package_helper_equals_reference_definition():
    pb = load_pkg()
    d, l = [1.0, 1.6, 0.25], [0.1, 0.2, 0.1]
    assert pb.hetero.wed_from_density_path(d, l) == float(np.sum(np.asarray(d) * np.asarray(l)))


def test_wed_entry_points_validate_before_device_work():
    pb = load_pkg()
    if not os.path.exists(pb._lib.LIB_PATH):
        pytest.skip("library not built")
    lib = pb._lib.load()
    fake = ctypes.c_void_p(0x1000)
    assert lib.pbd_wed_raytrace(4, 4, 4, 0.0, 0.2, None, fake, None) == -1
    assert lib.pbd_wed_raytrace(0, 4, 4, 0.0, 0.2, fake, fake, None) == -2
    assert lib.pbd_wed_raytrace(4, 4, 4, 0.0, 0.0, fake, fake, None) == -10
    assert lib.pbd_wed_raytrace(4, 4, 4, float("nan"), 0.2, fake, fake, None) == -10
    f = pb._lib.Field(nx=32, ny=32, nz=64, dx=0.2, dy=0.2, dz=0.2, ox=-3.1, oy=-3.1, oz=0.0,
                      n_sx=11, n_sy=11, n_layers=8, dx_spot=0.5, dy_spot=0.5, x0=0.0, y0=0.0)
    spec = pb.physics.lut_spec(64, 0.0, 0.2)
    sz = ctypes.c_size_t(0)
    assert lib.pbd_forward_wed_workspace(ctypes.byref(f), ctypes.byref(spec), 1,
                                         ctypes.byref(sz)) == 0 and sz.value > 0
    assert lib.pbd_forward_wed_workspace(ctypes.byref(f), None, 1, ctypes.byref(sz)) == -1
    args = [ctypes.byref(f), ctypes.byref(spec), fake, None, fake, fake, fake, fake, 1]
    assert lib.pbd_forward_wed(*args, None, 0, None) == -7
    bad = list(args)
    bad[6] = None                                   # no WED map
    assert lib.pbd_forward_wed(*bad, fake, sz.value, None) == -1
    # the curve blob: size query, build and forward validate before any device work
    cb = ctypes.c_size_t(0)
    assert lib.pbd_wed_curves_workspace(ctypes.byref(spec), 8, ctypes.byref(cb)) == 0
    assert cb.value > 0
    assert lib.pbd_wed_curves_workspace(None, 8, ctypes.byref(cb)) == -1
    assert lib.pbd_wed_curves_workspace(ctypes.byref(spec), 0, ctypes.byref(cb)) < 0
    assert lib.pbd_build_wed_curves(ctypes.byref(spec), 8, None, None, fake, cb.value, None) == -1
    assert lib.pbd_build_wed_curves(ctypes.byref(spec), 8, fake, None, fake, 16, None) == -7
    cargs = [ctypes.byref(f), ctypes.byref(spec), fake, cb.value, fake, fake, fake, fake, 1]
    assert lib.pbd_forward_wed_curves(*cargs, None, 0, None) == -7
    short = list(cargs)
    short[3] = 16                                   # curve blob too small
    assert lib.pbd_forward_wed_curves(*short, fake, sz.value, None) == -7
    nul = list(cargs)
    nul[2] = None                                   # no curve blob
    assert lib.pbd_forward_wed_curves(*nul, fake, sz.value, None) == -1
    # dL/dW of the heterogeneous dose
    ab = ctypes.c_size_t(0)
    assert lib.pbd_adjoint_wed_workspace(ctypes.byref(f), ctypes.byref(spec), 1,
                                         ctypes.byref(ab)) == 0 and ab.value > 0
    assert lib.pbd_adjoint_wed_workspace(ctypes.byref(f), None, 1, ctypes.byref(ab)) == -1
    aargs = [ctypes.byref(f), ctypes.byref(spec), fake, cb.value, fake, fake, fake, fake, fake, 1]
    assert lib.pbd_adjoint_wed(*aargs, None, 0, None) == -7
    nog = list(aargs)
    nog[7] = None                                   # no dL/dD
    assert lib.pbd_adjoint_wed(*nog, fake, ab.value, None) == -1
    # dL/dW and dL/d(range shift) of the heterogeneous dose
    rb = ctypes.c_size_t(0)
    assert lib.pbd_adjoint_wed_range_workspace(ctypes.byref(f), ctypes.byref(spec), 1,
                                               ctypes.byref(rb)) == 0 and rb.value > ab.value
    assert lib.pbd_adjoint_wed_range_workspace(ctypes.byref(f), None, 1, ctypes.byref(rb)) == -1
    rargs = [ctypes.byref(f), ctypes.byref(spec), fake, cb.value, fake, fake, 0.005, fake, fake,
             fake, fake, fake, fake, fake, 1]
    assert lib.pbd_adjoint_wed_range(*rargs, None, 0, None) == -7
    bad_h = list(rargs)
    bad_h[6] = 0.0                                  # no central-difference step
    assert lib.pbd_adjoint_wed_range(*bad_h, fake, rb.value, None) == -10
    nor = list(rargs)
    nor[13] = None                                  # no dL/dR output
    assert lib.pbd_adjoint_wed_range(*nor, fake, rb.value, None) == -1


def test_oracle_dose_in_water_equals_reference_dose():
    """In water the oracle's whole heterogeneous chain -- the WED ray trace of rho = 1, then
    the depth dose at that WED times each layer's lateral dose -- gives the reference's own
    float64 dose of the 32 x 32 x 64 workload (tests/golden/dose_cfg0.npz, made by the
    reference's separable_numpy with its own tables)."""
    wl = load_pkg().workloads.build_workload(0)
    lut = golden("luts_cfg0.npz")
    ref = golden("dose_cfg0.npz")
    gr = wl["grid"]
    rho = np.ones((gr["nz"], gr["ny"], gr["nx"]))
    wed = hr.wed_ref(rho, gr["oz"], gr["dz"])
    assert np.max(np.abs(wed[:, 0, 0] - lut["z"])) <= 1e-13
    xv = gr["ox"] + np.arange(gr["nx"]) * gr["dx"]
    yv = gr["oy"] + np.arange(gr["ny"]) * gr["dy"]
    xs = wl["x0"] + (np.arange(wl["n_sx"]) - (wl["n_sx"] - 1) / 2.0) * wl["spot_pitch"]
    ys = wl["y0"] + (np.arange(wl["n_sy"]) - (wl["n_sy"] - 1) / 2.0) * wl["spot_pitch"]
    d = hr.dose_ref(xv, yv, xs, ys, wl["weights"], lut["energies"], lut["sigma"], wed)
    err = np.max(np.abs(d - ref["dose"])) / np.max(np.abs(ref["dose"]))
    assert err < 1e-11, err


def test_oracle_gradient_is_the_dose_derivative():
    """The oracle's dL/dW of L = <g, D(W)> equals L(W + e_k) - L(W) (D is linear in W) on a
    small field in a slab medium."""
    rng = np.random.default_rng(5)
    nz, ny, nx, nl = 12, 7, 9, 3
    dz = 0.25
    xv = (np.arange(nx) - (nx - 1) / 2) * 0.2
    yv = (np.arange(ny) - (ny - 1) / 2) * 0.2
    xs = (np.arange(4) - 1.5) * 0.4
    ys = (np.arange(3) - 1.0) * 0.4
    en = np.array([45.0, 55.0, 62.0])
    rho = np.ones((nz, ny, nx))
    rho[4:7] = 1.7
    wed = hr.wed_ref(rho, 0.0, dz)
    z = np.arange(nz) * dz
    sig = np.stack([np.linspace(0.3, 0.5, nz) + 0.02 * l for l in range(nl)])
    w = rng.uniform(0.5, 1.5, (nl, 3, 4))
    g = rng.standard_normal((nz, ny, nx))
    gw = hr.grad_w_ref(xv, yv, xs, ys, w, en, sig, wed, g)
    base = float(np.sum(g * hr.dose_ref(xv, yv, xs, ys, w, en, sig, wed)))
    scale = np.max(np.abs(gw))
    for k in [(0, 0, 0), (1, 2, 3), (2, 1, 2)]:
        w1 = w.copy()
        w1[k] += 1.0
        diff = float(np.sum(g * hr.dose_ref(xv, yv, xs, ys, w1, en, sig, wed))) - base
        assert abs(diff - gw[k]) <= 1e-10 * scale, k
    assert z.size == nz


def test_oracle_nan_and_out_of_range_semantics():
    """The oracle's dose at a WED follows np.interp: NaN in, NaN out at that voxel only;
    beyond every layer's curve, or at a negative WED, exactly 0 -- the behaviour the device
    test checks against."""
    nz, ny, nx = 6, 5, 4
    xv = (np.arange(nx) - 1.5) * 0.3
    yv = (np.arange(ny) - 2.0) * 0.3
    xs = np.array([-0.2, 0.2])
    ys = np.array([-0.2, 0.0, 0.2])
    en = np.array([60.0, 70.0])
    sig = np.full((2, nz), 0.35)
    w = np.ones((2, 3, 2))
    wed = np.tile((np.arange(nz) * 0.5)[:, None, None], (1, ny, nx))
    base = hr.dose_ref(xv, yv, xs, ys, w, en, sig, wed)
    wn = wed.copy()
    wn[2, 1, 3] = np.nan
    d = hr.dose_ref(xv, yv, xs, ys, w, en, sig, wn)
    nan = np.isnan(d)
    assert nan.sum() == 1 and nan[2, 1, 3]
    assert np.array_equal(d[~nan], base[~nan])
    for fill in (1e3, -1.0):
        assert np.count_nonzero(hr.dose_ref(xv, yv, xs, ys, w, en, sig,
                                            np.full_like(wed, fill))) == 0


def test_oracle_range_gradient_matches_its_central_difference():
    """The oracle's heterogeneous dL/d(range shift) (the chain rule through the +-h central
    differences of the depth curves and widths, what the device computes) against the central
    difference of the oracle's own loss L(dR) = sum(g D(dR)) on the 32 x 32 x 64 field in a
    slab phantom, layers 0, 3 and 7.  The two differ at second order in the secants, which the
    tables' non-smoothness in range (CSDA binning, the Fermi-Eyges grid) makes ~1e-3 of max."""
    from oracle import physics_ref as pr
    pb = load_pkg()
    wl = pb.workloads.build_workload(0)
    gd = wl["grid"]
    grid = pb.model.DoseGrid(gd["nx"], gd["ny"], gd["nz"], gd["dx"], gd["dy"], gd["dz"], gd["ox"],
                             gd["oy"], gd["oz"])
    lat = pb.model.SpotLattice(wl["n_sx"], wl["n_sy"], wl["n_layers"], wl["spot_pitch"],
                               wl["spot_pitch"], x0=wl["x0"], y0=wl["y0"], weights=wl["weights"])
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    zc = grid.oz + np.arange(grid.nz) * grid.dz
    rho = np.ones((grid.nz, grid.ny, grid.nx))
    rho[(zc >= 2.0) & (zc < 3.0)] = 1.6
    rho[(zc >= 4.0) & (zc < 5.4), :, : grid.nx // 2] = 0.25
    wed = hr.wed_ref(rho, grid.oz, grid.dz)
    g = np.random.default_rng(5).standard_normal(wed.shape)
    h = 0.005
    got = hr.grad_range_ref(grid.x, grid.y, lat.spot_x, lat.spot_y, wl["weights"], en, zc, wed,
                            g, h)

    def loss(shift):
        _, sig = pr.layer_luts(zc, en, range_shift=shift)
        e2 = pr.energy_from_range(pr.csda_range(en) + shift)
        d = hr.dose_ref(grid.x, grid.y, lat.spot_x, lat.spot_y, wl["weights"], e2, sig, wed)
        return float(np.sum(g * d))

    scale = np.max(np.abs(got))
    for l in (0, 3, 7):
        s = np.zeros(len(en))
        s[l] = h
        fd = (loss(s) - loss(-s)) / (2.0 * h)
        assert abs(fd - got[l]) <= 1e-2 * scale, (l, fd, got[l])
