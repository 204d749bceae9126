"""Dose grid, spot lattice and problem types (the reference's API, model.py:27-344).

Same classes, fields, properties and builders as the reference so that code written
against ``pbdose.model`` runs unchanged.  The difference is where the per-layer depth
tables come from: the builders call the device LUT builder (``physics.layer_luts``)
instead of looping over layers on the host.

Conventions (model.py:5-11): lengths in cm, energies in MeV, dose (nz, ny, nx) indexed
``dose[k_z, k_y, k_x]``, voxel centre x = ox + k_x dx, spots on a lattice centred on
(x0, y0), weights (L, nsy, nsx).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from . import physics as ph


@dataclass
class DoseGrid:
    """Regular voxel grid (model.py:27-79)."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    ox: float = 0.0
    oy: float = 0.0
    oz: float = 0.0

    @property
    def shape(self) -> tuple:
        return (self.nz, self.ny, self.nx)

    @property
    def n_vox(self) -> int:
        return self.nx * self.ny * self.nz

    def axis(self, name: str) -> np.ndarray:
        n, d, o = {"x": (self.nx, self.dx, self.ox), "y": (self.ny, self.dy, self.oy),
                   "z": (self.nz, self.dz, self.oz)}[name]
        return o + np.arange(n) * d

    @property
    def x(self) -> np.ndarray:
        return self.axis("x")

    @property
    def y(self) -> np.ndarray:
        return self.axis("y")

    @property
    def z(self) -> np.ndarray:
        return self.axis("z")

    def voxel_volume(self) -> float:
        return self.dx * self.dy * self.dz

    def as_dict(self) -> dict:
        return dict(nx=self.nx, ny=self.ny, nz=self.nz, dx=self.dx, dy=self.dy, dz=self.dz,
                    ox=self.ox, oy=self.oy, oz=self.oz)

    @staticmethod
    def centered(n: int, d: float, axis: str = "z") -> "DoseGrid":
        """Cube centred on the origin; with axis="z" the entrance plane is z = 0."""
        half = (n - 1) * d / 2.0
        if axis == "z":
            return DoseGrid(n, n, n, d, d, d, -half, -half, 0.0)
        return DoseGrid(n, n, n, d, d, d, -half, -half, -half)


@dataclass
class SpotLattice:
    """IMPT spot lattice (model.py:85-131); weights[l, j, i] of layer l at spot (i, j)."""
    n_sx: int
    n_sy: int
    n_layers: int
    dx_spot: float
    dy_spot: float
    x0: float = 0.0
    y0: float = 0.0
    energies: Optional[np.ndarray] = None
    weights: Optional[np.ndarray] = None

    @property
    def n_spots(self) -> int:
        return self.n_sx * self.n_sy * self.n_layers

    @property
    def spot_x(self) -> np.ndarray:
        return self.x0 + (np.arange(self.n_sx) - (self.n_sx - 1) / 2.0) * self.dx_spot

    @property
    def spot_y(self) -> np.ndarray:
        return self.y0 + (np.arange(self.n_sy) - (self.n_sy - 1) / 2.0) * self.dy_spot

    def ensure_weights(self, rng: np.random.Generator | None = None) -> np.ndarray:
        if self.weights is None:
            rng = rng or np.random.default_rng(0)
            self.weights = rng.random((self.n_layers, self.n_sy, self.n_sx))
        return self.weights

    def flat_spot_table(self) -> tuple:
        """(x, y, layer, weight) flattened over (L, nsy, nsx)."""
        w = self.ensure_weights()
        X, Y = np.meshgrid(self.spot_x, self.spot_y)
        X = np.broadcast_to(X, (self.n_layers, self.n_sy, self.n_sx))
        Y = np.broadcast_to(Y, (self.n_layers, self.n_sy, self.n_sx))
        L = np.broadcast_to(np.arange(self.n_layers)[:, None, None], w.shape)
        return (X.ravel().copy(), Y.ravel().copy(), L.ravel().copy(), w.ravel().copy())


@dataclass
class PBProblem:
    """Grid + lattice + per-layer depth tables idd[l, k], sigma[l, k] (model.py:137-187)."""
    grid: DoseGrid
    lattice: SpotLattice
    idd: np.ndarray
    sigma: np.ndarray
    meta: dict = field(default_factory=dict)
    fluence_normalized: bool = True

    @property
    def n_layers(self) -> int:
        return self.lattice.n_layers

    @property
    def nz(self) -> int:
        return self.grid.nz

    def field_descriptor(self) -> _lib.Field:
        """The C ABI's pbd_field for this problem (``_lib.field_of``, which the engines use so
        that the reference's own PBProblem, which has no such method, works too)."""
        return _lib.field_of(self)

    def summary(self) -> str:
        g, L = self.grid, self.lattice
        lines = ["=" * 74, "Pencil-beam dose problem", "=" * 74,
                 f"  voxel grid    : {g.nx} x {g.ny} x {g.nz}  ({g.n_vox/1e6:.2f} M voxels, "
                 f"{g.dx*10:.1f} mm)",
                 f"  spot lattice  : {L.n_sx} x {L.n_sy} at {L.dx_spot*10:.1f} mm",
                 f"  energy layers : {L.n_layers}",
                 f"  pencil beams  : {L.n_spots:,}"]
        if L.energies is not None:
            lines.append(f"  energies      : {np.min(L.energies):.1f} - {np.max(L.energies):.1f} MeV")
        for k, v in self.meta.items():
            lines.append(f"  {k:<14}: {v}")
        lines.append("=" * 74)
        return "\n".join(lines)


def _tables(grid: DoseGrid, energies, idd_model, beam_sigma_x0, beam_sigma_theta0,
            fluence_normalized):
    idd, sig = ph.layer_luts(grid.z, energies, idd_model=idd_model, sigma_x0=beam_sigma_x0,
                             sigma_theta0=beam_sigma_theta0)
    if not fluence_normalized:   # peak-normalised curves (physics.py:378-379)
        peak = idd.max(axis=1, keepdims=True)
        idd = idd / np.where(peak > 0, peak, 1.0)
    return idd, sig


def gaussian_impt_field(energies: np.ndarray, grid: DoseGrid | None = None, *, n_spot: int = 41,
                        spot_spacing: float = 0.5, spot_sigma: float = 0.28, seed: int = 0,
                        idd_model: ph.IDDModel = ph.DEFAULT_IDD, beam_sigma_x0: float = 0.30,
                        beam_sigma_theta0: float = 0.0,
                        fluence_normalized: bool = True) -> PBProblem:
    """Gaussian-envelope field with 25 % per-layer weight noise (model.py:193-245)."""
    grid = grid or DoseGrid.centered(128, 0.2)
    n_layers = len(energies)
    rng = np.random.default_rng(seed)
    sx = np.arange(n_spot) - (n_spot - 1) / 2.0
    X, Y = np.meshgrid(sx * spot_spacing, sx * spot_spacing)
    env = np.exp(-(X**2 + Y**2) / (2.0 * spot_sigma**2))
    env /= env.max()
    w = env[None, :, :] * (1.0 + 0.25 * rng.standard_normal((n_layers, n_spot, n_spot)))
    w = np.clip(w, 0.0, None)
    lat = SpotLattice(n_spot, n_spot, n_layers, spot_spacing, spot_spacing,
                      energies=np.asarray(energies, dtype=np.float64), weights=w)
    idd, sig = _tables(grid, lat.energies, idd_model, beam_sigma_x0, beam_sigma_theta0,
                       fluence_normalized)
    meta = {"spot envelope": f"Gaussian sigma={spot_sigma*10:.1f} mm",
            "beam sigma_x0": f"{beam_sigma_x0*10:.1f} mm"}
    return PBProblem(grid=grid, lattice=lat, idd=idd, sigma=sig, meta=meta,
                     fluence_normalized=fluence_normalized)


def clinical_layer_energies(n_layers: int = 40, r_min: float = 3.0, r_max: float = 25.5) -> np.ndarray:
    """Energies of layers evenly spaced in CSDA range (model.py:248-255), on the device."""
    return np.asarray(ph.energy_from_range(np.linspace(r_min, r_max, n_layers)))


def flat_field_weights(n_sx: int, n_sy: int, n_layers: int, *, field_half_width: float = 5.0,
                       spot_spacing: float = 0.5, edge: float = 0.8, radial_falloff: float = 0.06,
                       layer_jitter: float = 0.15, seed: int = 0) -> np.ndarray:
    """Flat-top lateral weights with a tanh edge and per-layer jitter (model.py:258-287)."""
    rng = np.random.default_rng(seed)
    sx = (np.arange(n_sx) - (n_sx - 1) / 2.0) * spot_spacing
    X, Y = np.meshgrid(sx, sx)
    R = np.hypot(X, Y)
    w2 = 0.5 * (1.0 - np.tanh((R - field_half_width) / max(edge, 1e-6)))
    w2 = w2 * np.exp(-np.clip(R - field_half_width, 0, None) / max(radial_falloff, 1e-6))
    w = np.broadcast_to(w2, (n_layers, n_sy, n_sx)).copy()
    if layer_jitter > 0:
        w *= 1.0 + layer_jitter * rng.standard_normal(w.shape)
    return np.clip(w, 0.0, None)


def flat_impt_field(energies: np.ndarray, grid: DoseGrid | None = None, *, n_spot: int = 41,
                    spot_spacing: float = 0.5, field_half_width: float = 5.0, seed: int = 0,
                    idd_model: ph.IDDModel = ph.DEFAULT_IDD, beam_sigma_x0: float = 0.30,
                    beam_sigma_theta0: float = 0.0, fluence_normalized: bool = True) -> PBProblem:
    """Flat-top IMPT field (model.py:290-330)."""
    grid = grid or DoseGrid.centered(128, 0.2)
    energies = np.asarray(energies, dtype=np.float64)
    n_layers = len(energies)
    w = flat_field_weights(n_spot, n_spot, n_layers, field_half_width=field_half_width,
                           spot_spacing=spot_spacing, seed=seed)
    lat = SpotLattice(n_spot, n_spot, n_layers, spot_spacing, spot_spacing, energies=energies,
                      weights=w)
    idd, sig = _tables(grid, energies, idd_model, beam_sigma_x0, beam_sigma_theta0,
                       fluence_normalized)
    meta = {"cross-section": f"flat {2*field_half_width:.1f} x {2*field_half_width:.1f} cm"}
    return PBProblem(grid=grid, lattice=lat, idd=idd, sigma=sig, meta=meta,
                     fluence_normalized=fluence_normalized)


def single_spot_problem(E0: float = 200.0, grid: DoseGrid | None = None, n_spot: int = 1,
                        spot_spacing: float = 0.5, beam_sigma_x0: float = 0.30) -> PBProblem:
    """Single spot (or small lattice) at one energy (model.py:333-344).

    Like the reference, the depth dose here is peak-normalised (idd_pristine's default)."""
    grid = grid or DoseGrid(256, 256, 300, 0.1, 0.1, 0.1, -12.8, -12.8, 0.0)
    lat = SpotLattice(n_spot, n_spot, 1, spot_spacing, spot_spacing, energies=np.array([E0]),
                      weights=np.ones((1, n_spot, n_spot)))
    idd, sig = _tables(grid, lat.energies, ph.DEFAULT_IDD, beam_sigma_x0, 0.0, False)
    return PBProblem(grid, lat, idd, sig, meta={"E0": f"{E0} MeV"})


def problem_from_workload(wl: dict, energies=None, idd=None, sigma=None) -> PBProblem:
    """PBProblem of a synthetic workload (``workloads.build_workload``).  Tables are built
    on the device unless given."""
    g = wl["grid"]
    grid = DoseGrid(g["nx"], g["ny"], g["nz"], g["dx"], g["dy"], g["dz"], g["ox"], g["oy"], g["oz"])
    if energies is None:
        energies = clinical_layer_energies(wl["n_layers"], wl["r_min"], wl["r_max"])
    lat = SpotLattice(wl["n_sx"], wl["n_sy"], wl["n_layers"], wl["spot_pitch"], wl["spot_pitch"],
                      wl.get("x0", 0.0), wl.get("y0", 0.0), energies=np.asarray(energies),
                      weights=wl["weights"])
    if idd is None or sigma is None:
        idd, sigma = ph.layer_luts(grid.z, energies)
    return PBProblem(grid, lat, np.asarray(idd), np.asarray(sigma), meta={"workload": wl["name"]})
