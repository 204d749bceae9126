"""CPU restatement of the plan-optimisation steps (TEST INFRASTRUCTURE ONLY).

Oracle for ``pbd_adam_step`` and ``pbd_scenario_combine``.  Only ``tests/`` may import
it; the product path never does.

The reference computes dose only and has no optimiser, so there is no reference source to
follow.  The restated algorithm is Adam as published (Kingma & Ba, "Adam: A Method for
Stochastic Optimization", ICLR 2015, Algorithm 1) with a projection onto a box, in FP32
with every operation rounded separately -- the order of operations the CUDA kernel uses,
so the two agree bit for bit:

    g' = g * grad_scale
    m  = b1*m + (1-b1)*g'            v  = b2*v + (1-b2)*(g'*g')
    mh = m / float32(1 - b1^t)       vh = v / float32(1 - b2^t)      (1 - b^t in float64)
    x  = clip(x - lr * (mh / (sqrt(vh) + eps)), lo, hi)

``optimize_ref`` runs the same loop with the float64 gradient of the oracle's separable
engine (autograd through ``engine_ref.separable_torch``), for trajectory checks.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def adam_step(x, m, v, g, t, *, lr, beta1=0.9, beta2=0.999, eps=1e-8, lo=-np.inf, hi=np.inf,
              grad_scale=1.0):
    """One projected Adam step at step number ``t`` (1-based); returns new (x, m, v), float32."""
    x, m, v, g = (np.asarray(a, dtype=f32) for a in (x, m, v, g))
    b1, b2 = f32(beta1), f32(beta2)
    bc1 = f32(1.0 - np.float64(b1) ** t)
    bc2 = f32(1.0 - np.float64(b2) ** t)
    gs = g * f32(grad_scale)
    m1 = b1 * m + (f32(1) - b1) * gs
    v1 = b2 * v + (f32(1) - b2) * (gs * gs)
    mh = m1 / bc1
    vh = v1 / bc2
    upd = mh / (np.sqrt(vh) + f32(eps))
    x1 = x - f32(lr) * upd
    x1 = np.minimum(np.maximum(x1, f32(lo)), f32(hi)).astype(f32)
    return x1, m1.astype(f32), v1.astype(f32)


def scenario_combine(mode, grads, losses):
    """Robust objective over scenarios: ``mode`` "mean" or "max" (first index on ties).
    grads (S, n) float32, losses (S,) float64 -> (grad (n,) float32, loss float)."""
    grads = np.asarray(grads, dtype=f32)
    losses = np.asarray(losses, dtype=np.float64)
    if mode == "max":
        s = int(np.argmax(losses))            # argmax returns the first maximum
        return grads[s].copy(), float(losses[s])
    acc = np.zeros(grads.shape[1], dtype=f32)
    for s in range(grads.shape[0]):
        acc = acc + grads[s]
    return (acc / f32(grads.shape[0])).astype(f32), float(losses.sum() / grads.shape[0])


def loss_and_grad_f64(xv, yv, xs, ys, w, idd, sigma, mask, presc):
    """L = sum m (D - P)^2 and dL/dw in float64 (autograd through the oracle engine)."""
    import torch
    from .engine_ref import separable_torch
    wt = torch.tensor(np.asarray(w, dtype=np.float64), requires_grad=True)
    d = separable_torch(xv, yv, xs, ys, wt, idd, sigma, dtype=torch.float64)
    m = torch.as_tensor(np.asarray(mask, dtype=np.float64))
    p = torch.as_tensor(np.asarray(presc, dtype=np.float64))
    loss = (m * (d - p) ** 2).sum()
    loss.backward()
    return float(loss.detach()), wt.grad.numpy()


def optimize_ref(xv, yv, xs, ys, w0, idd, sigma, mask, presc, n_iter, **adam):
    """``n_iter`` projected Adam steps on the spot weights with float64 gradients;
    returns (w, losses) where losses[t] is the loss at the start of step t+1."""
    w = np.asarray(w0, dtype=f32).copy()
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    losses = []
    for t in range(1, n_iter + 1):
        loss, g = loss_and_grad_f64(xv, yv, xs, ys, w, idd, sigma, mask, presc)
        losses.append(loss)
        w, m, v = adam_step(w, m, v, g.astype(f32), t, **adam)
    return w, np.array(losses)
