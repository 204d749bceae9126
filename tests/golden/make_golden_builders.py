"""Generate tests/golden/builders.npz with the REFERENCE's own model builders.

Run in a container where the reference checkout is available (read-only):

    python tests/golden/make_golden_builders.py /root/reference

Host parts of the reference's model.py: DoseGrid axes (centred with z from 0, centred in all
three axes, and an anisotropic off-centre grid), SpotLattice spot positions, the flat spot
table with the default seeded weights (ensure_weights), and flat_field_weights for several
argument sets.  The GPU box never needs the reference.
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def import_model(ref_dir):
    tmp = tempfile.mkdtemp(prefix="pbdose_ref_")
    os.symlink(os.path.abspath(ref_dir), os.path.join(tmp, "pbdose"))
    sys.path.insert(0, tmp)
    return importlib.import_module("pbdose.model")


def main(ref_dir):
    M = import_model(ref_dir)
    out = {}
    grids = {"centered_z": M.DoseGrid.centered(64, 0.25),
             "centered_xyz": M.DoseGrid.centered(33, 0.3, axis="xyz"),
             "aniso": M.DoseGrid(20, 30, 40, 0.15, 0.2, 0.3, -1.4, -2.9, 0.5)}
    for name, g in grids.items():
        out[f"{name}__x"], out[f"{name}__y"], out[f"{name}__z"] = g.x, g.y, g.z
        out[f"{name}__dims"] = np.array([g.nx, g.ny, g.nz, g.n_vox])
    lat = M.SpotLattice(7, 5, 3, 0.4, 0.6, x0=0.07, y0=-0.11)
    out["lat__spot_x"], out["lat__spot_y"] = lat.spot_x, lat.spot_y
    x, y, layer, w = lat.flat_spot_table()
    out["lat__table_x"], out["lat__table_y"] = x, y
    out["lat__table_l"], out["lat__table_w"] = layer, w
    out["flat_default"] = M.flat_field_weights(41, 41, 4)
    out["flat_args"] = M.flat_field_weights(21, 21, 3, field_half_width=3.0, spot_spacing=0.4,
                                            edge=0.5, radial_falloff=0.1, layer_jitter=0.3,
                                            seed=7)
    out["flat_nojitter"] = M.flat_field_weights(15, 15, 2, layer_jitter=0.0)
    path = os.path.join(HERE, "builders.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
