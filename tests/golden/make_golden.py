"""Generate the golden fixtures in this directory by running the REFERENCE itself.

Run in a container where the reference checkout is available (read-only):

    python tests/golden/make_golden.py /root/reference

The reference is a flat Python repo whose modules import each other as the
package ``pbdose``; a temporary directory with a ``pbdose`` symlink makes that
import work without touching the checkout.  The fixtures are small NumPy
archives; the GPU box never needs the reference.

Fixtures (all float64 unless noted):
  physics.npz   range table, range/energy lookups, Bohr straggling, sigma_R,
                Fermi-Eyges moments and IDDs at a few energies
  luts_cfg{0,1,4}.npz  per-layer (idd, sigma) tables of the workload configs,
                as filled by model.py:225-233
  dose_cfg0.npz  separable_numpy(per_layer=True) dose of config 0, plus the
                reference's torch float32 CPU result
  dose_cfg1_slices.npz  selected depth slices + checksums of config 1's dose
  engine_check.npz  the reference's engine_check.py small case: naive triple
                loop and separable dose
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def import_reference(ref_dir):
    tmp = tempfile.mkdtemp(prefix="pbdose_ref_")
    os.symlink(os.path.abspath(ref_dir), os.path.join(tmp, "pbdose"))
    sys.path.insert(0, tmp)
    ph = importlib.import_module("pbdose.physics")
    md = importlib.import_module("pbdose.model")
    en = importlib.import_module("pbdose.engines")
    return ph, md, en


def load_workloads():
    import importlib.util
    pkg_dir = os.path.join(REPO, "gpu-proton-dose-engine_b200")
    spec = importlib.util.spec_from_file_location("_wl", os.path.join(pkg_dir, "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def ref_luts(ph, z, energies):
    idd = np.stack([ph.idd_pristine(z, e, normalize=False)[0] for e in energies])
    sig = np.stack([ph.fermi_eyges_moments(z, e, sigma_x0=0.30)["sigma_x"] for e in energies])
    return idd, sig


def main(ref_dir):
    ph, md, en = import_reference(ref_dir)
    wl = load_workloads()
    out = {}

    # --- physics pieces -----------------------------------------------------------
    E_tab, R_tab = ph._range_table()
    e_q = np.array([0.7, 3.0, 15.0, 50.0, 100.0, 150.0, 200.0, 250.0, 399.0])
    r_q = np.array([0.0, 0.01, 0.5, 3.0, 10.0, 25.0, 40.0, 80.0])
    strag_e = np.array([40.0, 70.0, 120.0, 200.0])
    fe_z = np.linspace(0.0, 25.0, 51)
    fe_e = np.array([100.0, 150.0, 200.0])
    fe = [ph.fermi_eyges_moments(fe_z, e, sigma_x0=0.3) for e in fe_e]
    idd_z = np.arange(0.0, 34.0, 0.02)
    idd_e = np.array([100.0, 200.0])
    idd = [ph.idd_pristine(idd_z, e, return_components=True, normalize=False) for e in idd_e]
    np.savez_compressed(
        os.path.join(HERE, "physics.npz"),
        E_tab=E_tab, R_tab=R_tab, e_q=e_q, csda_q=ph.csda_range(e_q), r_q=r_q,
        efr_q=ph.energy_from_range(r_q), strag_e=strag_e,
        bohr=np.array([ph.range_straggling_bohr(e) for e in strag_e]),
        sigma_R=np.array([ph.DEFAULT_IDD.sigma_range(e)[0] for e in strag_e]),
        stopping=ph.bethe_bloch_water(e_q), highland=ph.scattering_power(e_q),
        fe_z=fe_z, fe_e=fe_e, fe_sigma=np.stack([m["sigma_x"] for m in fe]),
        fe_B=np.stack([m["B"] for m in fe]), fe_A2=np.stack([m["A2"] for m in fe]),
        idd_z=idd_z, idd_e=idd_e, idd=np.stack([o["idd"] for o in idd]),
        idd_sigma_R=np.array([o["sigma_R"] for o in idd]),
        idd_R0=np.array([o["R0"] for o in idd]))
    out["physics"] = True

    # --- workload LUTs --------------------------------------------------------------
    for cfg in (0, 1, 4):
        w = wl.build_workload(cfg)
        z = w["grid"]["oz"] + np.arange(w["grid"]["nz"]) * w["grid"]["dz"]
        energies = ph.energy_from_range(np.linspace(w["r_min"], w["r_max"], w["n_layers"]))
        idd_t, sig_t = ref_luts(ph, z, energies)
        np.savez_compressed(os.path.join(HERE, f"luts_cfg{cfg}.npz"), z=z, energies=energies,
                            idd=idd_t, sigma=sig_t)
        if cfg == 0:
            prob = wl_to_ref_problem(md, w, idd_t, sig_t, energies)
            d64 = en.separable_numpy(prob, per_layer=True)
            d32 = en.torch_separable(prob, "cpu", dtype=__import__("torch").float32).numpy()
            np.savez_compressed(os.path.join(HERE, "dose_cfg0.npz"), dose=d64, dose_torch_f32=d32)
        if cfg == 1:
            prob = wl_to_ref_problem(md, w, idd_t, sig_t, energies)
            d64 = en.separable_numpy(prob, per_layer=True)
            ks = np.array([0, 20, 45, 60, 75])
            np.savez_compressed(os.path.join(HERE, "dose_cfg1_slices.npz"), k=ks, slices=d64[ks],
                                dmax=d64.max(), dsum=d64.sum(),
                                zsum=d64.sum(axis=(1, 2)))
        print("cfg", cfg, "done", flush=True)

    # --- engine_check.py small case (engine_check.py:15-24) --------------------------
    grid = md.DoseGrid(24, 24, 32, 0.25, 0.25, 0.25, -3.0, -3.0, 0.0)
    energies = np.array([80.0, 130.0, 180.0])
    rng = np.random.default_rng(7)
    w = rng.random((3, 3, 3))
    lat = md.SpotLattice(3, 3, 3, 0.5, 0.5, energies=energies, weights=w)
    z = grid.z
    idd_s = np.stack([ph.idd_pristine(z, e)[0] for e in energies])
    sig_s = np.stack([ph.fermi_eyges_moments(z, e, sigma_x0=0.3)["sigma_x"] for e in energies])
    prob = md.PBProblem(grid, lat, idd_s, sig_s)
    d_naive = en.naive_python_triple_loop(prob)
    d_sep = en.separable_numpy(prob, per_layer=True)
    np.savez_compressed(os.path.join(HERE, "engine_check.npz"), w=w, energies=energies,
                        idd=idd_s, sigma=sig_s, dose_naive=d_naive, dose_sep=d_sep)
    print("engine_check done")


def wl_to_ref_problem(md, w, idd, sig, energies):
    g = w["grid"]
    grid = md.DoseGrid(g["nx"], g["ny"], g["nz"], g["dx"], g["dy"], g["dz"],
                       g["ox"], g["oy"], g["oz"])
    lat = md.SpotLattice(w["n_sx"], w["n_sy"], w["n_layers"], w["spot_pitch"], w["spot_pitch"],
                         energies=energies, weights=w["weights"].astype(np.float64))
    return md.PBProblem(grid, lat, idd, sig)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
