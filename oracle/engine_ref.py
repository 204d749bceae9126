"""CPU restatements of the reference's separable dose engine (TEST INFRASTRUCTURE ONLY).

Oracle for the CUDA forward and adjoint kernels.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may import it; the
product path never does.

* ``separable_f64``     NumPy float64, the reference's per-layer separable
                        engine (engines.py:172-202, ``per_layer=True``).
* ``separable_torch``   the same contraction as two batched matmuls in torch on
                        the CPU (engines.py:208-283, ``per_layer=True``), any
                        dtype, differentiable with autograd.  In float64 this is
                        the gradient oracle; it is also the CPU baseline that
                        ``bench.py`` times.
* ``masked_quadratic_loss`` the plan loss L = sum m (D - P)^2.
* ``relative_error``    the reference's parity metric (engines.py:364-378).

Inputs are plain arrays, so the oracle does not depend on the package's types:
voxel axes ``xv, yv`` (cm), spot axes ``xs, ys`` (cm), weights ``w`` of shape
(L, nsy, nsx), tables ``idd, sigma`` of shape (L, nz).
"""
from __future__ import annotations

import numpy as np

INV_SQRT_2PI = 1.0 / np.sqrt(2.0 * np.pi)


def lateral_kernel(vox, spots, sigma):
    """G[..., v, s] = exp(-(vox_v - spot_s)^2 / (2 sigma^2)) / (sqrt(2 pi) sigma); engines.py:49-61.

    sigma is clipped at 1e-9 and broadcast over leading dims."""
    d2 = (np.asarray(vox, np.float64)[:, None] - np.asarray(spots, np.float64)[None, :]) ** 2
    s = np.clip(np.asarray(sigma, dtype=np.float64), 1e-9, None)
    return np.exp(-d2 / (2.0 * s[..., None, None] ** 2)) * (INV_SQRT_2PI / s)[..., None, None]


def separable_f64(xv, yv, xs, ys, w, idd, sigma, layer_block: int | None = None):
    """D (nz, ny, nx) = sum_l IDD_l(z) Gx_l(z) W_l Gy_l(z)^T in float64; engines.py:191-197.

    Same two einsums as the reference; ``layer_block`` bounds memory by summing
    blocks of layers (the sum over layers is linear, so the result is the same
    up to float64 summation order)."""
    w = np.asarray(w, np.float64)
    idd = np.asarray(idd, np.float64)
    sigma = np.asarray(sigma, np.float64)
    n_layers, nz = idd.shape
    step = layer_block or n_layers
    out = np.zeros((nz, len(yv), len(xv)))
    for l0 in range(0, n_layers, step):
        sl = slice(l0, min(l0 + step, n_layers))
        amp = idd[sl, :, None, None] * w[sl, None, :, :]           # (l, z, j, i)
        gx = lateral_kernel(xv, xs, sigma[sl])                     # (l, z, x, i)
        gy = lateral_kernel(yv, ys, sigma[sl])                     # (l, z, y, j)
        t = np.einsum("zkji,zkvj->zkiv", amp, gy)                  # (l, z, i, y)
        dl = np.einsum("zkai,zkiy->zkay", gx, t)                   # (l, z, x, y)
        out += dl.sum(axis=0).transpose(0, 2, 1)
    return out


def separable_torch(xv, yv, xs, ys, w, idd, sigma, dtype=None, layer_chunk=None):
    """Torch CPU form of the per-layer batched-matmul engine; engines.py:256-274.

    ``w``, ``idd`` and ``sigma`` may be torch tensors that require grad; the
    result is differentiable with respect to each of them."""
    import torch

    dtype = dtype or torch.float64

    def as_t(a):
        return a.to(dtype) if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a), dtype=dtype)

    xv_t, yv_t, xs_t, ys_t = (as_t(a) for a in (xv, yv, xs, ys))
    w_t, idd_t, sig_t = as_t(w), as_t(idd), as_t(sigma)
    n_layers, nz = idd_t.shape
    nx, ny, nsx, nsy = len(xv_t), len(yv_t), len(xs_t), len(ys_t)
    dx2 = (xv_t.view(1, 1, -1, 1) - xs_t.view(1, 1, 1, -1)) ** 2
    dy2 = (yv_t.view(1, 1, -1, 1) - ys_t.view(1, 1, 1, -1)) ** 2
    step = layer_chunk or n_layers
    out = torch.zeros((nz, ny, nx), dtype=dtype)
    for l0 in range(0, n_layers, step):
        l1 = min(l0 + step, n_layers)
        nl = l1 - l0
        s4 = sig_t[l0:l1].clamp_min(1e-9).reshape(nl, nz, 1, 1)
        norm = INV_SQRT_2PI / s4
        gx = (norm * torch.exp(-dx2 / (2.0 * s4**2))).reshape(nl * nz, nx, nsx)
        gy = (norm * torch.exp(-dy2 / (2.0 * s4**2))).reshape(nl * nz, ny, nsy)
        amp = (idd_t[l0:l1, :, None, None] * w_t[l0:l1, None, :, :]).reshape(nl * nz, nsy, nsx)
        t = torch.bmm(amp.transpose(1, 2), gy.transpose(1, 2))
        dl = torch.bmm(gx, t)
        out = out + dl.reshape(nl, nz, nx, ny).sum(0).transpose(1, 2)
    return out


def masked_quadratic_loss(dose, mask, presc):
    """L = sum_v m_v (D_v - P_v)^2 (works for numpy arrays and torch tensors)."""
    r = dose - presc
    return (mask * r * r).sum()


def relative_error(a, b, mask=None) -> dict:
    """Error of ``a`` against reference ``b``; engines.py:364-378."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if mask is None:
        mask = np.ones_like(b, dtype=bool)
    d = (a - b)[mask]
    ref = float(np.max(np.abs(b))) or 1.0
    if d.size == 0:
        return {"max_abs_err": 0.0, "max_rel_err_global": 0.0, "rms_err": 0.0,
                "rms_rel_global": 0.0, "n_vox": 0}
    return {"max_abs_err": float(np.abs(d).max()),
            "max_rel_err_global": float(np.abs(d).max() / ref),
            "rms_err": float(np.sqrt((d**2).mean())),
            "rms_rel_global": float(np.sqrt((d**2).mean()) / ref),
            "n_vox": int(mask.sum())}


def naive_dose(xv, yv, zlen, xs, ys, w, idd, sigma):
    """O(M N) per-beam sum, the textbook definition (engines.py:142-166); small cases only."""
    w = np.asarray(w, np.float64)
    n_layers, nsy, nsx = w.shape
    out = np.zeros((zlen, len(yv), len(xv)))
    X = np.asarray(xv)[None, None, :]
    Y = np.asarray(yv)[None, :, None]
    for l in range(n_layers):
        s = np.clip(np.asarray(sigma[l], np.float64), 1e-9, None)[:, None, None]
        for j in range(nsy):
            for i in range(nsx):
                g = np.exp(-((X - xs[i]) ** 2 + (Y - ys[j]) ** 2) / (2.0 * s**2))
                out += w[l, j, i] * np.asarray(idd[l])[:, None, None] * g / (2.0 * np.pi * s**2)
    return out
