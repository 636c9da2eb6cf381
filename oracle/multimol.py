"""FP64 restatement of the reference's multi-molecule L-BFGS optimizer.

TEST INFRASTRUCTURE ONLY (the checker of ``mmff_optimize_metal_multi_mol``):
imported by the tests, never by the product path.

It follows mlxmolkit/mmff_metal_optimizer.py step by step: ``_lbfgs_direction_batch``
(:47-74), the main loop with the per-atom step cap, the curvature gate
EPS_CURV = 1e-10, the best-seen guard and the convergence record every
``eval_freq`` iterations (:346-410), the return to the best-seen positions
(:412-428), the polish pass of ``max_iters // 4`` iterations (:430-483) and the
final result fields (:485-533).  Each conformer's energy and gradient come
from the FP64 C oracle with the mega-kernel term constants (``MODE_MEGA``).
The reference advances all conformers in lockstep; so does this.
"""
from __future__ import annotations

import numpy as np

from . import oracle

EPS_CURV = 1e-10


def _two_loop(g, s_hist, y_hist, rho_hist):
    m = len(s_hist)
    q = g.copy()
    alphas = []
    for i in range(m - 1, -1, -1):
        a = rho_hist[i] * np.sum(s_hist[i] * q, axis=1, keepdims=True)
        q = q - a * y_hist[i]
        alphas.append(a)
    if m:
        sy = np.sum(s_hist[-1] * y_hist[-1], axis=1, keepdims=True)
        yy = np.sum(y_hist[-1] * y_hist[-1], axis=1, keepdims=True) + 1e-30
        gamma = sy / yy
    else:
        gamma = 1.0
    r = gamma * q
    for i in range(m):
        beta = rho_hist[i] * np.sum(y_hist[i] * r, axis=1, keepdims=True)
        r = r + s_hist[i] * (alphas[m - 1 - i] - beta)
    return -r


def multi_mol(params_list, conf_counts, x_flat, *, max_iters=200, eval_freq=10, max_step_per_atom=0.3,
              lbfgs_m=10, grad_scale=0.1, grad_tol=1e-4, mode=oracle.MODE_MEGA):
    """Returns dict(positions (C, max_dim), energies, grad_norms, n_iters, per_conf_iters, converged)."""
    conf_p = [p for p, k in zip(params_list, conf_counts) for _ in range(k)]
    dims = [3 * p.n_atoms for p in conf_p]
    C, D = len(conf_p), max(dims)
    A = D // 3
    x = np.zeros((C, D))
    o = 0
    for c, d in enumerate(dims):
        x[c, :d] = x_flat[o: o + d]
        o += d

    def eg(X):
        e = np.empty(C)
        g = np.zeros((C, D))
        for c, (p, d) in enumerate(zip(conf_p, dims)):
            e[c], gc, _ = oracle.energy_grad(p, X[c, :d], mode=mode)
            g[c, :d] = gc
        return e, g

    def max_norm(g):
        return np.sqrt((g.reshape(C, A, 3) ** 2).sum(-1)).max(axis=1)

    def capped(d):
        d3 = d.reshape(C, A, 3)
        disp = np.sqrt((d3 * d3).sum(-1, keepdims=True) + 1e-30)
        return (d3 * np.minimum(max_step_per_atom / disp, 1.0)).reshape(C, D)

    def push(hist, s, y):
        sy = np.sum(s * y, axis=1, keepdims=True)
        rho = np.where(sy > EPS_CURV, 1.0 / (sy + 1e-30), 0.0)
        for h, v in zip(hist, (s, y, rho)):
            if len(h) >= lbfgs_m:
                h.pop(0)
            h.append(v)

    e, g = eg(x)
    g = g * grad_scale
    best_e, best_x = e.copy(), x.copy()
    per_conf = np.full(C, max_iters, dtype=np.int32)
    conv = np.zeros(C, dtype=bool)
    iters_used = max_iters
    hist = ([], [], [])
    for it in range(max_iters):
        xn = x + capped(_two_loop(g, *hist))
        en, gn = eg(xn)
        gn = gn * grad_scale
        push(hist, xn - x, gn - g)
        x, g = xn, gn
        if (it + 1) % eval_freq == 0:
            better = en < best_e
            best_x[better] = x[better]
            best_e = np.minimum(en, best_e)
            newly = (~conv) & (max_norm(g) <= grad_tol)
            per_conf[newly] = it + 1
            conv[newly] = True
            if conv.all():
                iters_used = it + 1
                break
    x = best_x.copy()
    _, g = eg(x)
    g = g * grad_scale
    hist = ([], [], [])
    for it in range(max_iters // 4):
        xn = x + capped(_two_loop(g, *hist))
        en, gn = eg(xn)
        gn = gn * grad_scale
        push(hist, xn - x, gn - g)
        x, g = xn, gn
        if (it + 1) % eval_freq == 0:
            better = en < best_e
            best_x[better] = x[better]
            best_e = np.minimum(en, best_e)
            if (max_norm(g) <= grad_tol).all():
                break
    final_e, _ = eg(best_x)
    return dict(positions=best_x, energies=final_e, grad_norms=max_norm(g), n_iters=iters_used,
                per_conf_iters=per_conf, converged=conv, dims=dims)
