"""Synthetic workloads of the named shapes (host-side, NumPy only).

The reference quotes its numbers on a synthetic water phantom (run_benchmark.py:34-39);
these builders produce the grids, lattices and seeded spot weights of the five
benchmark workloads, plus the plan loss of the gradient workload and the robust
scenario list of the batched workload.  Depth tables are not built here: they come
from the device LUT builder (``physics.layer_luts``) or, in tests, from the oracle.

This module has no package-relative imports so that fixture scripts can load it
by file path.

Workloads
---------
0  32x32x64 voxels of 2 mm, 11x11 spots at 5 mm, 8 layers, ranges 40-90 mm,
   weights U[0.5,1.5] (seed 0)
1  128^3 voxels of 2 mm, 41x41 spots at 2.5 mm, 40 layers, ranges 60-160 mm,
   weights 0.3 (proximal) .. 1.0 (distal) linear x U[0.9,1.1] (seed 1)
2  workload 1 + masked quadratic loss (60 mm target cube at 110 mm depth, 20 mm shell)
3  4 fields 21x21x16, 33x33x28, 41x41x40, 51x41x48 (nsx x nsy x layers) on 128^3 / 2 mm,
   ranges 50-170 mm, weights U[0.5,1.5] (seed 2); 25 robust scenarios each
4  200x200x256 voxels of 1 mm, 61x61 spots at 2.5 mm, 60 layers, ranges 40-220 mm,
   weights lognormal(0, 0.3) (seed 3)
"""
from __future__ import annotations

import numpy as np


def centered_grid(nx, ny, nz, dx, dy, dz):
    """Grid centred laterally with the entrance plane at z = 0 (DoseGrid.centered, model.py:73-79)."""
    return {"nx": nx, "ny": ny, "nz": nz, "dx": dx, "dy": dy, "dz": dz,
            "ox": -(nx - 1) * dx / 2.0, "oy": -(ny - 1) * dy / 2.0, "oz": 0.0}


def _base(grid, nsx, nsy, n_layers, pitch, r_min, r_max, weights, name):
    return {"name": name, "grid": grid, "n_sx": nsx, "n_sy": nsy, "n_layers": n_layers,
            "spot_pitch": pitch, "x0": 0.0, "y0": 0.0, "r_min": r_min, "r_max": r_max,
            "weights": np.ascontiguousarray(weights, dtype=np.float32)}


def build_workload(cfg: int) -> dict:
    """Geometry and weights of workload ``cfg`` (0, 1, 2 or 4; see ``robust_fields`` for 3)."""
    if cfg == 0:
        rng = np.random.default_rng(0)
        w = rng.uniform(0.5, 1.5, (8, 11, 11))
        return _base(centered_grid(32, 32, 64, 0.2, 0.2, 0.2), 11, 11, 8, 0.5, 4.0, 9.0, w,
                     "32x32x64 / 11x11x8")
    if cfg in (1, 2):
        rng = np.random.default_rng(1)
        n_layers = 40
        sobp = 0.3 + 0.7 * np.arange(n_layers) / (n_layers - 1)
        w = sobp[:, None, None] * rng.uniform(0.9, 1.1, (n_layers, 41, 41))
        wl = _base(centered_grid(128, 128, 128, 0.2, 0.2, 0.2), 41, 41, n_layers, 0.25, 6.0, 16.0,
                   w, "128^3 / 41x41x40")
        if cfg == 2:
            wl["mask"], wl["presc"] = target_loss_arrays(wl["grid"])
            wl["name"] = "128^3 / 41x41x40 fwd+adjoint"
        return wl
    if cfg == 4:
        rng = np.random.default_rng(3)
        w = rng.lognormal(0.0, 0.3, (60, 61, 61))
        return _base(centered_grid(200, 200, 256, 0.1, 0.1, 0.1), 61, 61, 60, 0.25, 4.0, 22.0, w,
                     "200x200x256 / 61x61x60")
    raise ValueError(f"unknown workload {cfg}")


def target_loss_arrays(grid, half=3.0, shell=2.0, depth=11.0, presc_value=2.0):
    """Mask m and prescription P of the gradient workload.

    m = 1 inside the box |x|,|y| <= 3 cm, |z - 11| <= 3 cm (voxel centres), 0.2 in the
    2 cm shell around it, 0 elsewhere; P = 2 inside the box, 0 elsewhere."""
    eps = 1e-9
    x = grid["ox"] + np.arange(grid["nx"]) * grid["dx"]
    y = grid["oy"] + np.arange(grid["ny"]) * grid["dy"]
    z = grid["oz"] + np.arange(grid["nz"]) * grid["dz"]
    ax, ay, az = np.abs(x), np.abs(y), np.abs(z - depth)
    inner = ((az[:, None, None] <= half + eps) & (ay[None, :, None] <= half + eps)
             & (ax[None, None, :] <= half + eps))
    outer = ((az[:, None, None] <= half + shell + eps) & (ay[None, :, None] <= half + shell + eps)
             & (ax[None, None, :] <= half + shell + eps))
    mask = np.where(inner, 1.0, np.where(outer, 0.2, 0.0)).astype(np.float32)
    presc = np.where(inner, presc_value, 0.0).astype(np.float32)
    return mask, presc


def fd_sample(cfg_w: dict, n_spots=64, n_layers=8, seed=12):
    """Indices (l, j, i) of the finite-difference spot sample and the FD layer sample."""
    rng = np.random.default_rng(seed)
    nl, nsy, nsx = cfg_w["weights"].shape
    flat = rng.choice(nl * nsy * nsx, size=n_spots, replace=False)
    spots = np.stack(np.unravel_index(flat, (nl, nsy, nsx)), axis=1)
    layers = np.sort(rng.choice(nl, size=n_layers, replace=False))
    return spots, layers


ROBUST_LATTICES = ((21, 21, 16), (33, 33, 28), (41, 41, 40), (51, 41, 48))


def robust_fields():
    """The four uneven fields of the batched workload (nsx, nsy, layers as listed)."""
    rng = np.random.default_rng(2)
    grid = centered_grid(128, 128, 128, 0.2, 0.2, 0.2)
    out = []
    for nsx, nsy, nl in ROBUST_LATTICES:
        w = rng.uniform(0.5, 1.5, (nl, nsy, nsx))
        out.append(_base(grid, nsx, nsy, nl, 0.25, 5.0, 17.0, w, f"{nsx}x{nsy}x{nl}"))
    return out


def robust_scenarios(shift=0.3, scales=(0.965, 1.0, 1.035)):
    """25 scenarios (dx, dy, dz in cm, depth scale s).

    Nominal plus +-shift along x, y and z (7 setups) at each of the three range scalings
    (21), plus four combined corners.  x/y shifts move the spot lattice (sub-voxel lattice
    offsets); a z shift moves the water surface (depth d = z - dz); the range scaling
    multiplies the water-equivalent depth (d = s (z - dz)), i.e. a stopping-power scaling."""
    setups = [(0.0, 0.0, 0.0)]
    for ax in range(3):
        for sgn in (1.0, -1.0):
            v = [0.0, 0.0, 0.0]
            v[ax] = sgn * shift
            setups.append(tuple(v))
    out = [(sx, sy, sz, s) for s in scales for (sx, sy, sz) in setups]
    lo, hi = scales[0], scales[-1]
    out += [(shift, shift, shift, hi), (-shift, -shift, -shift, lo),
            (shift, -shift, shift, lo), (-shift, shift, -shift, hi)]
    return out
