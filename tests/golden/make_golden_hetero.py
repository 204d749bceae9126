"""Generate tests/golden/hetero.npz with the REFERENCE's own WED helper.

    python tests/golden/make_golden_hetero.py /root/reference

The reference's ``physics.wed_from_density_path(densities, lengths)`` is applied to the path
of every voxel of small seeded relative stopping-power maps (the path lists of
``oracle.hetero_ref.wed_path``: water above the first voxel, full voxels, half the voxel
itself).  The GPU box never needs the reference.
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main(ref_dir):
    tmp = tempfile.mkdtemp(prefix="pbdose_ref_")
    os.symlink(os.path.abspath(ref_dir), os.path.join(tmp, "pbdose"))
    sys.path.insert(0, tmp)
    sys.path.insert(0, REPO)
    ph = importlib.import_module("pbdose.physics")
    from oracle.hetero_ref import wed_path
    rng = np.random.default_rng(11)
    out = {}
    for case, (oz, dz) in enumerate(((0.0, 0.2), (0.05, 0.2), (0.37, 0.25))):
        rho = rng.choice([0.25, 1.0, 1.05, 1.6], size=(12, 3, 4)).astype(np.float32)
        wed = np.zeros(rho.shape)
        for y in range(rho.shape[1]):
            for x in range(rho.shape[2]):
                for k in range(rho.shape[0]):
                    dens, lens = wed_path(rho[:, y, x].astype(np.float64), oz, dz, k)
                    wed[k, y, x] = ph.wed_from_density_path(dens, lens)
        out[f"rho{case}"] = rho
        out[f"wed{case}"] = wed
        out[f"grid{case}"] = np.array([oz, dz])
    np.savez_compressed(os.path.join(HERE, "hetero.npz"), **out)
    print("wrote hetero.npz")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
