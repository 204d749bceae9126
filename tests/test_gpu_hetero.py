"""Heterogeneous media on the device: the WED ray trace against fixtures made with the
reference's own wed_from_density_path and against the oracle; in water the heterogeneous
dose reproduces the homogeneous engine; in a slab phantom (bone and lung slabs) it matches
the float64 oracle (depth dose evaluated at the WED, lateral widths of water).

Tolerances: WED 1e-13 of max; doses 1e-6 of max (FP32 and TF32x3, like the homogeneous
engine)."""
import numpy as np
import pytest

from conftest import golden, has_gpu, load_pkg
from oracle import hetero_ref as hr
from oracle import physics_ref as pr

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def pb():
    return load_pkg()


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("case", [0, 1, 2])
def test_wed_raytrace_matches_reference_fixture(pb, case):
    z = golden("hetero.npz")
    rho, want = z[f"rho{case}"], z[f"wed{case}"]
    oz, dz = z[f"grid{case}"]
    grid = {"nz": rho.shape[0], "ny": rho.shape[1], "nx": rho.shape[2], "oz": oz, "dz": dz}
    got = pb.hetero.wed_raytrace(rho, grid).cpu().numpy()
    assert rel(got, want) <= 1e-13


def _cfg0(pb):
    wl = pb.workloads.build_workload(0)
    en = pr.layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    return wl, en, pb.model.problem_from_workload(wl, energies=en)


def test_water_reproduces_homogeneous_dose(pb):
    import torch
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    wed = pb.hetero.wed_raytrace(rho, g)
    zc = np.maximum(g.oz + np.arange(g.nz) * g.dz, 0.0)[:, None, None]
    assert np.max(np.abs(wed.cpu().numpy() - zc)) <= 1e-12
    for prec in ("fp32", "tf32x3"):
        d_wed = pb.hetero.WedPlan(prob, precision=prec).forward(wed)
        d_ref = pb.engines.DosePlan(prob, tables="device", precision=prec).forward()
        torch.cuda.synchronize()
        assert rel(d_wed.cpu().numpy(), d_ref.cpu().numpy()) < 1e-6, prec


def test_slab_phantom_vs_oracle(pb):
    """Bone (1.6) from 2 to 3 cm and lung (0.25) from 4 to 5.4 cm; with a lateral edge."""
    wl, en, prob = _cfg0(pb)
    g = prob.grid
    zc = g.oz + np.arange(g.nz) * g.dz
    rho = np.ones((g.nz, g.ny, g.nx), dtype=np.float32)
    rho[(zc >= 2.0) & (zc < 3.0)] = 1.6
    lung = (zc >= 4.0) & (zc < 5.4)
    rho[lung, :, : g.nx // 2] = 0.25                    # lung only on one side
    wed_ref = hr.wed_ref(rho, g.oz, g.dz)
    sig = pr.layer_luts(zc, en)[1]
    want = hr.dose_ref(g.x, g.y, prob.lattice.spot_x, prob.lattice.spot_y, wl["weights"], en, sig,
                       wed_ref)
    wed = pb.hetero.wed_raytrace(rho, g)
    assert rel(wed.cpu().numpy(), wed_ref) <= 1e-13
    for prec in ("fp32", "tf32x3"):
        d = pb.hetero.WedPlan(prob, precision=prec).forward(wed).cpu().numpy()
        err = rel(d, want)
        print(f"{prec}: heterogeneous dose max rel err {err:.2e}")
        assert err < 1e-6, prec
    # the slabs move the dose: not the water result
    d_water = pb.engines.DosePlan(prob, tables="device", precision="fp32").forward().cpu().numpy()
    assert rel(d, d_water) > 1e-2
