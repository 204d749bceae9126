"""CPU float64 restatement of the reference's depth-LUT physics (TEST INFRASTRUCTURE ONLY).

This module is the oracle for the device LUT builder.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it;
the product path (the package and its CUDA library) never does.

Every function restates one function of the reference's ``physics.py`` in
plain NumPy float64 and cites the lines it follows.  Parity of this oracle with
the reference itself is pinned by ``tests/test_oracle_golden.py`` against the
fixtures in ``tests/golden/`` (generated by importing the reference in the
build container, see ``tests/golden/make_golden.py``).

Units: cm, MeV, rad.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np

# Physical constants, physics.py:42-66
PROTON_MC2 = 938.27208816       # MeV
ELECTRON_MC2 = 0.51099895000    # MeV
K_BETHE = 0.307075              # MeV cm^2 / mol
WATER_ZA = 10.0 / 18.01528
WATER_I = 75.0e-6               # MeV
WATER_RHO = 1.0
WATER_X0 = 36.08                # cm
POWER_LAW_P = 1.77              # exponent of R = a E^p, physics.py:57-58
HIGHLAND_E = 13.6               # MeV
E_TABLE_LO = 0.5
E_TABLE_HI = 400.0
BOHR_K = K_BETHE * WATER_ZA * WATER_RHO * ELECTRON_MC2   # physics.py:151


def kinematics(e_kin):
    """(beta, gamma, beta^2) of a proton of kinetic energy ``e_kin``; physics.py:72-77."""
    e = np.asarray(e_kin, dtype=np.float64)
    gam = 1.0 + e / PROTON_MC2
    b2 = np.clip(1.0 - 1.0 / gam**2, 1e-14, 1.0)
    return np.sqrt(b2), gam, b2


def stopping_power(e_kin):
    """Bethe-Bloch electronic stopping power of water, MeV/cm; physics.py:80-100."""
    e = np.asarray(e_kin, dtype=np.float64)
    _, gam, b2 = kinematics(e)
    ratio = ELECTRON_MC2 / PROTON_MC2
    tmax = 2.0 * ELECTRON_MC2 * b2 * gam**2 / (1.0 + 2.0 * gam * ratio + ratio**2)
    log_arg = 2.0 * ELECTRON_MC2 * b2 * gam**2 * tmax / (WATER_I**2)
    log_arg = np.clip(log_arg, 1.0 + 1e-12, None)
    return K_BETHE * WATER_ZA * WATER_RHO / b2 * (0.5 * np.log(log_arg) - b2)


@lru_cache(maxsize=1)
def range_table():
    """(E, R) CSDA range table by trapezoid integration of 1/S; physics.py:111-127.

    The energy grid is four linspace pieces joined with duplicates removed
    (3797 points, 0.5-400 MeV)."""
    pieces = [np.linspace(E_TABLE_LO, 2.0, 800), np.linspace(2.0, 20.0, 900),
              np.linspace(20.0, 60.0, 900), np.linspace(60.0, E_TABLE_HI, 1200)]
    e = np.unique(np.concatenate(pieces))
    inv_s = 1.0 / stopping_power(e)
    steps = 0.5 * (inv_s[1:] + inv_s[:-1]) * np.diff(e)
    r = np.concatenate([[0.0], np.cumsum(steps)])
    return e, r


def csda_range(e_kin):
    """R(E) by linear interpolation in the range table; physics.py:130-133."""
    e, r = range_table()
    return np.interp(np.asarray(e_kin, dtype=np.float64), e, r)


def energy_from_range(r_cm):
    """E(R), the inverse table lookup with R clipped to [0, R_max]; physics.py:136-139."""
    e, r = range_table()
    return np.interp(np.clip(np.asarray(r_cm, dtype=np.float64), 0.0, r[-1]), r, e)


def bohr_straggling(e0, n: int = 4000) -> float:
    """Bohr range straggling sigma_R(E0) = sqrt(int BOHR_K / (beta^2 S^3) dE); physics.py:154-174."""
    e = np.linspace(E_TABLE_LO, float(e0), n)
    if e[-1] <= e[0]:
        return 0.0
    s = stopping_power(e)
    _, _, b2 = kinematics(e)
    f = BOHR_K / (np.clip(b2, 1e-12, None) * s**3)
    return float(np.sqrt(np.trapezoid(f, e)))


def sigma_range(e0, energy_spread: float = 0.0033, model: str = "bohr",
                coef: float = 0.012, expo: float = 0.935):
    """Total range spread (sigma_R, straggling part, energy-spread part); physics.py:310-322."""
    r0 = float(csda_range(e0))
    if model == "bohr":
        strag = bohr_straggling(e0)
    elif model == "icru49":
        strag = coef * r0 ** expo
    elif model == "none":
        strag = 0.0
    else:
        raise ValueError(model)
    espr = POWER_LAW_P * energy_spread * r0
    return float(np.hypot(strag, espr)), float(strag), float(espr)


def highland_local_power(e_kin):
    """Local Highland scattering power T(E) at L = 1 (ln L = 0), rad^2/cm; physics.py:185-218."""
    beta, gam, _ = kinematics(e_kin)
    pc = np.sqrt(np.clip(gam**2 - 1.0, 0.0, None)) * PROTON_MC2
    bpc = np.clip(beta * pc, 1e-9, None)
    base = (HIGHLAND_E / bpc) ** 2 / WATER_X0
    lnl = np.log(1.0)
    return base * (1.0 + 0.038 * lnl) * (1.076 + 0.038 * lnl)


def fine_depth_count(z0: float, z1: float, nz: int, n_sub: int = 4,
                     max_step: float = 0.02) -> int:
    """Size of the Fermi-Eyges integration grid; physics.py:256-258."""
    span = float(z1 - z0)
    need = int(np.ceil(span / max(max_step, 1e-6))) + 1 if span > 0 else 2
    return max((nz - 1) * n_sub + 1, need, 2)


def fermi_eyges_sigma(z, e0, sigma_x0=0.0, sigma_theta0=0.0, rho0=0.0,
                      n_sub: int = 4, max_step: float = 0.02, return_all: bool = False):
    """Lateral sigma_x(z) from the direct scattering integral B(z); physics.py:221-286.

    B(z_i) = sum_{j: z_i > z_j} (z_i - z_j)^2 T_j h_j on a fine grid of at most
    ``max_step`` cm, with h = np.gradient(zf) and T = 0 beyond the CSDA range,
    then linearly interpolated back to ``z``; sigma^2 = sigma_x0^2 + ... + B."""
    z = np.asarray(z, dtype=np.float64)
    single = z.size == 1
    if single:
        z = np.array([0.0, z[0]]) if z[0] > 0 else np.array([0.0, 1e-6])
    nf = fine_depth_count(z[0], z[-1], len(z), n_sub, max_step)
    zf = np.linspace(z[0], z[-1], nf)
    hf = np.gradient(zf)
    r0 = float(csda_range(e0))
    inside = zf < r0
    e_loc = np.where(inside, energy_from_range(np.clip(r0 - zf, 0.0, None)), 0.0)
    t_loc = np.where(inside, highland_local_power(np.clip(e_loc, 1e-3, None)), 0.0)
    a0 = np.cumsum(t_loc * hf)
    a1 = np.cumsum(a0 * hf)
    a2 = np.cumsum(a1 * hf)
    lag = zf[:, None] - zf[None, :]
    b_f = np.where(lag > 0, lag**2 * t_loc[None, :] * hf[None, :], 0.0).sum(axis=1)
    b = np.interp(z, zf, b_f)
    var = (sigma_x0**2 + 2.0 * rho0 * sigma_x0 * sigma_theta0 * z
           + sigma_theta0**2 * z**2 + b)
    sig = np.sqrt(np.clip(var, 0.0, None))
    if single:
        sig, b = sig[-1:], b[-1:]
    if return_all:
        return {"sigma_x": sig, "B": b, "A0": np.interp(z, zf, a0),
                "A1": np.interp(z, zf, a1), "A2": np.interp(z, zf, a2), "n_fine": nf}
    return sig


def idd_fluence(z, e0, energy_spread: float = 0.0033, atten_len: float = 150.0,
                n_fine: int = 6000, model: str = "bohr", return_all: bool = False):
    """Un-normalised integral depth dose per unit fluence, MeV/cm; physics.py:328-387.

    Energy-conserving CSDA binning on ``n_fine`` bins up to R0 + 8 sigma_R + 0.2,
    times exp(-z/atten_len), convolved with a Gaussian of sigma_R through a
    zero-padded FFT, then interpolated to ``z`` with zero outside the fine grid."""
    z = np.asarray(z, dtype=np.float64)
    r0 = float(csda_range(e0))
    s_r, _, _ = sigma_range(e0, energy_spread, model)
    zmax = r0 + 8.0 * s_r + 0.2
    zf = np.linspace(0.0, zmax, n_fine)
    h = zf[1] - zf[0]
    edges = np.linspace(0.0, zmax, n_fine + 1)
    e_edge = np.where(edges < r0, energy_from_range(np.clip(r0 - edges, 0.0, None)), 0.0)
    binned = np.exp(-zf / atten_len) * (e_edge[:-1] - e_edge[1:]) / h
    nfft = int(2 ** np.ceil(np.log2(2 * n_fine)))
    freq = np.fft.rfftfreq(nfft, d=h)
    gauss_ft = np.exp(-2.0 * (np.pi * freq * s_r) ** 2)
    smooth = np.fft.irfft(np.fft.rfft(binned, nfft) * gauss_ft, nfft)[:n_fine]
    out = np.interp(z, zf, smooth, left=0.0, right=0.0)
    if return_all:
        return {"idd": out, "sigma_R": s_r, "R0": r0, "z_fine": zf, "binned": binned,
                "smooth": smooth}
    return out


def layer_luts(z, energies, sigma_x0: float = 0.30, range_shift=None):
    """(idd, sigma) tables of shape (L, nz) as filled by model.py:225-233.

    ``range_shift`` (cm, per layer, optional) moves each layer's CSDA range to
    R0_l + dR_l before the build; the energy is recovered through the table
    inverse.  dR = 0 gives exactly the reference's tables."""
    energies = np.asarray(energies, dtype=np.float64)
    if range_shift is not None:
        r = csda_range(energies) + np.asarray(range_shift, dtype=np.float64)
        energies = energy_from_range(r)
    idd = np.stack([idd_fluence(z, e) for e in energies])
    sig = np.stack([fermi_eyges_sigma(z, e, sigma_x0=sigma_x0) for e in energies])
    return idd, sig


def scenario_luts(z0, dz, nz, energies, depth_scale=1.0, sigma_x0=0.30):
    """Tables of a robust scenario (no counterpart in the reference).

    Water-equivalent depths d_k = s (z0 + k dz); the scattering integral starts at the
    water surface (depth 0): the Fermi-Eyges depth list is [0] + {d_k > 0}; depths <= 0
    get B = 0 and IDD = 0; the lateral variance is sigma_x0^2 + B(d) / s^2.  With s = 1
    and z0 = 0 this is exactly ``layer_luts``."""
    d = depth_scale * (z0 + np.arange(nz) * dz)
    pos = d[d > 0]
    zl = np.concatenate([[0.0], pos]) if pos.size else np.array([0.0, 1e-6])
    idd = np.stack([idd_fluence(d, e) for e in energies])
    sig = []
    for e in energies:
        m = fermi_eyges_sigma(zl, e, sigma_x0=0.0, return_all=True)
        b = np.where(d > 0, np.interp(d, zl, m["B"]), 0.0)
        sig.append(np.sqrt(np.clip(sigma_x0**2 + b / depth_scale**2, 0.0, None)))
    return idd, np.stack(sig)


def layer_energies(n_layers: int, r_min: float, r_max: float):
    """Energies of layers evenly spaced in CSDA range; model.py:248-255."""
    return energy_from_range(np.linspace(r_min, r_max, n_layers))
