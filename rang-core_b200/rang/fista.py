"""FISTA through the B200 gridder (the reference's `prox_solver::solve` and
`power_iteration`, core/src/prox_solver.rs:302-445 and :888-911).

The problem is the reference's: minimise
    0.5 x^T G x - d^T x + lambda ||x||_1,  x >= 0 unless `signed`,
with G = A^H W A (`DevicePlan.gram`) and d the dirty image A^H W v. Every
iteration applies G once (to the extrapolated point y); G x for the
objective comes from linearity, G x = (G y + beta G x_prev) / (1 + beta),
as the reference does. The gridder and the iteration's vector steps run in
this library's CUDA kernels (`include/rang_solver.h`): the prox step, the
inner products, the misfit, the restart test and the momentum keep their
scalars on the device, so an iteration never waits for it. A stop test
reads the recorded misfits every `check_every` iterations (one wait each).
"""

import ctypes
import math

import torch

from . import core

_lib = None
_STATE = 16


def _library():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(core.library_path())
        P, I, D, S = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_size_t
        lib.rang_b200_fista_init.argtypes = [P, P, D, D, D, I, D, P]
        lib.rang_b200_fista_step.argtypes = [I, S, P, P, P, P, P, P, P, P, P, P, I, I, I, I, P, P]
        lib.rang_b200_fista_partials.restype = S
        lib.rang_b200_dot.argtypes = [I, S, P, P, P, P, P]
        lib.rang_b200_gaussian_lowpass.argtypes = [S, S, P, P, D, P]
        for f in (lib.rang_b200_fista_init, lib.rang_b200_fista_step, lib.rang_b200_dot,
                  lib.rang_b200_gaussian_lowpass):
            f.restype = ctypes.c_int32
        _lib = lib
    return _lib


def _check(status, what):
    if status != 0:
        msg = core.extension().wgridder_last_error()
        raise (ValueError if status == 1 else RuntimeError)(f"{what} failed with status {status}: {msg}")


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _single(t):
    if t.dtype == torch.float32:
        return 1
    if t.dtype == torch.float64:
        return 0
    raise TypeError("images must be float32 or float64")


class Workspace:
    """Device scratch of the library's reductions (FP64 block partials)."""

    def __init__(self, device):
        self.partials = torch.empty(int(_library().rang_b200_fista_partials()), dtype=torch.float64, device=device)


def dot(a, b, out=None, ws=None):
    """<a, b> summed in FP64 in a fixed order, into a 0-dimensional float64
    CUDA tensor (no wait)."""
    if out is None:
        out = torch.empty((), dtype=torch.float64, device=a.device)
    ws = ws or Workspace(a.device)
    a, b = a.contiguous(), b.contiguous()
    _check(_library().rang_b200_dot(_single(a), a.numel(), a.data_ptr(), b.data_ptr(), out.data_ptr(),
                                    ws.partials.data_ptr(), _stream(a.device)), "dot")
    return out


def gaussian_lowpass(img, sigma, out=None):
    """The periodic Gaussian blur of a float32 image, standard deviation
    `sigma` pixels, through cuFFT (R2C, the Gaussian's transfer function,
    C2R)."""
    img = img.contiguous()
    if img.dtype != torch.float32 or img.dim() != 2:
        raise TypeError("a 2-D float32 image is required")
    if out is None:
        out = torch.empty_like(img)
    _check(_library().rang_b200_gaussian_lowpass(img.shape[0], img.shape[1], img.data_ptr(), out.data_ptr(),
                                                 float(sigma), _stream(img.device)), "low-pass")
    return out


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


class Solve:
    """The outcome of `solve`: the iterate `x` and `gx` = G x of the last
    iteration `k`, the restarts, the misfit of every iteration (`misfits`, a
    float64 CUDA tensor), the first iteration whose misfit reached the
    target (`first`, None if none) and, with `events`, a CUDA event recorded
    after each iteration's vector steps."""

    def __init__(self, x, gx, k, restarts, misfits, first, events, snapshots):
        self.x, self.gx, self.k, self.restarts = x, gx, k, restarts
        self.misfits, self.first, self.events, self.snapshots = misfits, first, events, snapshots

    def __iter__(self):  # (x, G x, iterations, restarts), as the earlier tuple
        return iter((self.x, self.gx, self.k, self.restarts))


def solve(gram, dirty, lam, step, max_iterations, q0=0.0, x0=None, momentum=True, restart=True, signed=False,
          observer=None, stop=None, gx0=None, target_misfit=None, check_every=20, events=False, keep=()):
    """FISTA with gradient restart from `x0` (zero by default), for
    iterations k = 0 .. max_iterations (the reference's loop, which applies G
    max_iterations + 1 times). `q0` (a float or a 0-dimensional CUDA tensor)
    is |W^(1/2) v|^2 / 2, so that the recorded misfit is the data misfit.

    The run ends at max_iterations, or at the first check (every
    `check_every` iterations; each check waits for the device) after the
    misfit reached `target_misfit` or `stop(k, misfit)` returned True for a
    recorded iteration; `first` says which iteration that was. `observer(k,
    x, gx, misfit)` sees every iterate, which waits for the device every
    iteration. `keep`: iterations whose (x, G x) are copied into
    `snapshots` without waiting. `gx0`, when given, is G x0 (it saves the
    first apply of G). Returns a `Solve` (which unpacks as (x, G x,
    iterations, restarts))."""
    lib = _library()
    dev = dirty.device
    single = _single(dirty)
    n = dirty.numel()
    s = _stream(dev)
    x = torch.zeros_like(dirty) if x0 is None else x0.clone()
    y = x.clone()
    g_x_prev = torch.zeros_like(dirty)
    g_x = torch.empty_like(dirty)
    x_next = torch.empty_like(dirty)
    y_next = torch.empty_like(dirty)
    state = torch.empty(_STATE, dtype=torch.float64, device=dev)
    misfits = torch.full((max_iterations + 1,), float("nan"), dtype=torch.float64, device=dev)
    ws = Workspace(dev)
    q0_dev = q0 if torch.is_tensor(q0) else None
    if q0_dev is not None:
        q0_dev = q0_dev.to(dev, torch.float64).reshape(())
    has_target = target_misfit is not None
    _check(lib.rang_b200_fista_init(state.data_ptr(), None if q0_dev is None else q0_dev.data_ptr(),
                                    0.0 if q0_dev is not None else float(q0), float(step), float(lam),
                                    int(has_target), float(target_misfit) if has_target else 0.0, s), "fista init")
    keep = set(keep)
    snapshots = {}
    evs = []
    first = None
    checked = -1
    k = 0
    for k in range(max_iterations + 1):
        g_y = gx0 if (k == 0 and gx0 is not None) else gram(y)
        _check(lib.rang_b200_fista_step(single, n, dirty.data_ptr(), x.data_ptr(), y.data_ptr(), g_y.data_ptr(),
                                        g_x_prev.data_ptr(), g_x.data_ptr(), x_next.data_ptr(), y_next.data_ptr(),
                                        state.data_ptr(), misfits.data_ptr(), k, int(bool(signed)),
                                        int(bool(momentum)), int(bool(restart)), ws.partials.data_ptr(), s),
               "fista step")
        if events:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            evs.append(e)
        if k in keep:
            snapshots[k] = (x.clone(), g_x.clone())
        if observer is not None:
            observer(k, x, g_x, float(misfits[k]))
        done = k == max_iterations
        if not done and (has_target or stop is not None) and (k + 1 - (checked + 1)) >= check_every:
            if has_target:
                f = float(state[7])
                if f >= 0.0:
                    first = int(f)
                    done = True
            if stop is not None and first is None:
                vals = misfits[checked + 1:k + 1].tolist()
                for j, m in enumerate(vals):
                    if stop(checked + 1 + j, m):
                        first = checked + 1 + j
                        done = True
                        break
            checked = k
        if done:
            break
        # x_prev is not kept: the step reads x, and x_next - x is all the momentum needs.
        x, x_next = x_next, x
        g_x_prev, g_x = g_x, g_x_prev
        y, y_next = y_next, y
    if has_target and first is None:
        f = float(state[7])
        first = int(f) if f >= 0.0 else None
    if stop is not None and first is None:
        vals = misfits[checked + 1:k + 1].tolist()
        for j, m in enumerate(vals):
            if stop(checked + 1 + j, m):
                first = checked + 1 + j
                break
    restarts = int(float(state[5]))
    return Solve(x, g_x, k, restarts, misfits[:k + 1], first, evs, snapshots)


def misfit_of(dirty, x, gx, q0, ws=None):
    """q0 - <dirty, x> + <x, G x> / 2 as a 0-dimensional float64 CUDA tensor."""
    ws = ws or Workspace(dirty.device)
    return q0 - dot(dirty, x, ws=ws) + 0.5 * dot(x, gx, ws=ws)


def momentum_of(t):
    """(t', beta') of the accelerated step from t (prox_solver.rs:425-428)."""
    t_next = 0.5 * (1.0 + math.sqrt(1.0 + 4.0 * t * t))
    return t_next, (t - 1.0) / t_next
