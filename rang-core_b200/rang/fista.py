"""FISTA through the B200 gridder (the reference's `prox_solver::solve` and
`power_iteration`, core/src/prox_solver.rs:302-445 and :888-911).

The problem is the reference's: minimise
    0.5 x^T G x - d^T x + lambda ||x||_1,  x >= 0 unless `signed`,
with G = A^H W A (`DevicePlan.gram`) and d the dirty image A^H W v. Every
iteration applies G once (to the extrapolated point y); G x for the
objective comes from linearity, G x = (G y + beta G x_prev) / (1 + beta),
as the reference does. The gridder runs in this library's CUDA kernels; the
few vector updates per iteration are PyTorch tensor arithmetic on the GPU.
"""

import math

import torch


def power_iteration(gram, shape, device, seed=1, tolerance=1e-3, max_iterations=30, dtype=torch.float32):
    """The largest eigenvalue of `gram` from a seeded start (prox_solver.rs:888-911):
    returns (estimate, applies used)."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    v = torch.rand(shape, generator=g, device=device, dtype=torch.float64) - 0.5
    v = v / v.norm()
    value = 0.0
    for k in range(1, max_iterations + 1):
        gv = gram(v.to(dtype)).double()
        nxt = float(gv.norm())
        v = gv / max(nxt, 1e-300)
        if k > 1 and abs(nxt - value) <= tolerance * nxt:
            return nxt, k
        value = nxt
    return value, max_iterations


def soft_threshold(z, tau, signed):
    """L1Prior::prox (prox_solver.rs:80-105)."""
    if signed:
        return torch.sign(z) * torch.clamp(z.abs() - tau, min=0.0)
    return torch.clamp(z - tau, min=0.0)


def solve(gram, dirty, lam, step, max_iterations, q0=0.0, x0=None, momentum=True, restart=True, signed=False,
          observer=None, stop=None, gx0=None):
    """FISTA with gradient restart from `x0` (zero by default). `observer(k, x,
    gx, misfit)` sees every iterate; `stop(k, misfit)` returning True ends the
    run early; `gx0`, when given, is G x0 (it saves the first apply of G).
    Returns (x, G x, iterations, restarts)."""
    x = torch.zeros_like(dirty) if x0 is None else x0.clone()
    x_prev = x.clone()
    y = x.clone()
    g_x_prev = torch.zeros_like(dirty)
    t = 1.0
    beta = 0.0
    restarts = 0
    for k in range(max_iterations + 1):
        g_y = gx0 if (k == 0 and gx0 is not None) else gram(y)
        g_x = g_y if beta == 0.0 else (g_y + beta * g_x_prev) / (1.0 + beta)
        misfit = q0 - float(torch.dot(dirty.double().ravel(), x.double().ravel())) + 0.5 * float(
            torch.dot(x.double().ravel(), g_x.double().ravel()))
        if observer is not None:
            observer(k, x, g_x, misfit)
        if k == max_iterations or (stop is not None and stop(k, misfit)):
            return x, g_x, k, restarts
        z = y + step * (dirty - g_y)
        x_next = soft_threshold(z, step * lam, signed)
        next_beta = 0.0
        if momentum:
            inner = float(torch.sum((y - x_next) * (x_next - x)))
            if restart and inner > 0.0:
                t = 1.0
                restarts += 1
            else:
                t_next = 0.5 * (1.0 + math.sqrt(1.0 + 4.0 * t * t))
                next_beta = (t - 1.0) / t_next
                t = t_next
        g_x_prev = g_x
        x_prev, x = x, x_next
        y = x + next_beta * (x - x_prev)
        beta = next_beta
    return x, g_x_prev, max_iterations, restarts
