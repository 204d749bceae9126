"""CPU restatement of the water-equivalent depth and the heterogeneous dose (TEST
INFRASTRUCTURE ONLY).

Oracle for ``pbd_wed_raytrace``, ``pbd_forward_wed`` and ``pbd_adjoint_wed``.  Only
``tests/`` and ``bench.py``'s CPU-baseline leg may import it; the product path never does.

* ``wed_path``  the (densities, lengths) of the path from depth 0 to voxel k of a column:
  water above the first voxel, voxels i < k in full, half of voxel k, each voxel filling
  [z_i - dz/2, z_i + dz/2], lengths clipped at depth 0.  Its WED is the reference's
  ``wed_from_density_path`` (physics.py:421-423): ``np.sum(densities * lengths)``.
* ``wed_ref``   the same per voxel for a whole map, cumulated along z (float64).
* ``dose_ref``  sum over layers of IDD_l(WED) (``physics_ref.idd_fluence`` evaluated at the
  WED) times the layer's separable lateral dose with unit depth dose (``engine_ref``).
* ``grad_w_ref`` its dL/dW for a given dL/dD, by float64 autograd.
* ``grad_range_ref`` its dL/d(range shift) per layer: the chain rule through the central
  differences at range shifts +-h of the depth curve (at the WED) and of the widths (at the
  geometric depth), float64, the widths' part by torch autograd.
Pinned: ``wed_path`` + the reference's helper reproduce tests/golden/hetero.npz, made by the
reference itself.
"""
from __future__ import annotations

import numpy as np

from . import engine_ref as er
from . import physics_ref as pr


def wed_path(rho_col, oz, dz, k):
    z = oz + np.arange(k + 1) * dz
    dens = [1.0]
    lens = [max(0.0, z[0] - 0.5 * dz)]
    for i in range(k):
        dens.append(float(rho_col[i]))
        lens.append(max(0.0, z[i] + 0.5 * dz) - max(0.0, z[i] - 0.5 * dz))
    dens.append(float(rho_col[k]))
    lens.append(max(0.0, z[k]) - max(0.0, z[k] - 0.5 * dz))
    return np.array(dens), np.array(lens)


def wed_ref(rho, oz, dz):
    rho = np.asarray(rho, dtype=np.float64)
    nz = rho.shape[0]
    z = oz + np.arange(nz) * dz
    lo = np.maximum(z - 0.5 * dz, 0.0)
    mid = np.maximum(z, 0.0)
    hi = np.maximum(z + 0.5 * dz, 0.0)
    full = rho * (hi - lo)[:, None, None]
    before = np.concatenate([np.zeros((1,) + rho.shape[1:]), np.cumsum(full, axis=0)[:-1]])
    return max(0.0, z[0] - 0.5 * dz) + before + rho * (mid - lo)[:, None, None]


def dose_ref(xv, yv, xs, ys, w, energies, sigma, wed):
    w = np.asarray(w, dtype=np.float64)
    nz = sigma.shape[1]
    d = np.zeros(wed.shape)
    for l, e in enumerate(energies):
        lat = er.separable_f64(xv, yv, xs, ys, w[l:l + 1], np.ones((1, nz)), sigma[l:l + 1])
        d += pr.idd_fluence(wed.ravel(), e).reshape(wed.shape) * lat
    return d


def grad_w_ref(xv, yv, xs, ys, w, energies, sigma, wed, grad_dose):
    """dL/dW of L = sum(grad_dose * D(W)) for the heterogeneous dose of ``dose_ref`` (linear
    in W), by float64 torch autograd through ``engine_ref.separable_torch``."""
    import torch
    wt = torch.tensor(np.asarray(w, dtype=np.float64), requires_grad=True)
    nz = sigma.shape[1]
    d = torch.zeros(wed.shape, dtype=torch.float64)
    for l, e in enumerate(energies):
        lat = er.separable_torch(xv, yv, xs, ys, wt[l:l + 1], np.ones((1, nz)), sigma[l:l + 1])
        idd = torch.as_tensor(pr.idd_fluence(wed.ravel(), e).reshape(wed.shape))
        d = d + idd * lat
    (d * torch.as_tensor(np.asarray(grad_dose, dtype=np.float64))).sum().backward()
    return wt.grad.numpy()


def grad_range_ref(xv, yv, xs, ys, w, energies, z, wed, grad_dose, h, sigma_x0: float = 0.30):
    """dL/dR_l of L = sum(grad_dose * D) for ``dose_ref``'s heterogeneous dose, D = sum_l
    IDD_l(WED) Lat_l(sigma_l): sum_v g (IDD+_l - IDD-_l)(WED) / (2 h) Lat_l + sum_z dL/dsigma_lz
    (sigma+_lz - sigma-_lz) / (2 h), the +-h curves and widths built at the shifted ranges
    (``physics_ref.layer_luts`` with ``range_shift``), dL/dsigma by float64 torch autograd."""
    import torch
    w = np.asarray(w, dtype=np.float64)
    g = np.asarray(grad_dose, dtype=np.float64)
    nz = len(z)
    n = len(energies)
    _, sig0 = pr.layer_luts(z, energies, sigma_x0=sigma_x0)
    idd_p = [pr.idd_fluence(wed.ravel(), e).reshape(wed.shape)
             for e in pr.energy_from_range(pr.csda_range(energies) + h)]
    idd_m = [pr.idd_fluence(wed.ravel(), e).reshape(wed.shape)
             for e in pr.energy_from_range(pr.csda_range(energies) - h)]
    _, sig_p = pr.layer_luts(z, energies, sigma_x0=sigma_x0, range_shift=np.full(n, h))
    _, sig_m = pr.layer_luts(z, energies, sigma_x0=sigma_x0, range_shift=np.full(n, -h))
    out = np.zeros(n)
    gt = torch.as_tensor(g)
    for l, e in enumerate(energies):
        st = torch.tensor(sig0[l:l + 1], dtype=torch.float64, requires_grad=True)
        lat = er.separable_torch(xv, yv, xs, ys, w[l:l + 1], np.ones((1, nz)), st)
        idd = torch.as_tensor(pr.idd_fluence(wed.ravel(), e).reshape(wed.shape))
        (gt * idd * lat).sum().backward()
        dsig = (sig_p[l] - sig_m[l]) / (2.0 * h)
        t2 = float(np.sum(st.grad.numpy()[0] * dsig))
        t1 = float(np.sum(g * (idd_p[l] - idd_m[l]) / (2.0 * h) * lat.detach().numpy()))
        out[l] = t1 + t2
    return out
