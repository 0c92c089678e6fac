"""The consumers of the path on the GPU: the persistent plan's residual, the
differentiable degridder (autograd forward = degridding, backward =
gridding) and FISTA, checked against the CPU oracle and against themselves
(adjointness, finite differences)."""

import numpy as np
import pytest

import oracle
from cases import meerkat_like, rel_linf

pytestmark = pytest.mark.gpu


def _problem(single, npix=128, seed=0, nant=32, ntime=6, nchan=12):
    import torch

    from rang import synth, wgrid_torch

    uvw, freq = meerkat_like(nant=nant, ntime=ntime, nchan=nchan, seed=seed)
    rng = np.random.default_rng(seed)
    shape = (uvw.shape[0], freq.size)
    wgt = rng.uniform(0.5, 1.5, shape)
    wgt.ravel()[::11] = 0.0
    cell = 3.0 * synth.ARCSEC
    kw = dict(npix_x=npix, npix_y=npix, pixsize_x=cell, pixsize_y=cell, epsilon=1e-5 if single else 1e-10)
    dev = torch.device("cuda", 0)
    rt = torch.float32 if single else torch.float64
    t_wgt = torch.from_numpy(wgt).to(dev, rt)
    plan = wgrid_torch.DevicePlan(torch.from_numpy(uvw).to(dev), freq, wgt=t_wgt, single=single, **kw)
    return plan, uvw, freq, wgt, t_wgt, kw, dev


@pytest.mark.parametrize("single", [True, False])
def test_adjoint_dot_product(single):
    """<A x, y> = <x, A^H y> for the weighted degridder A and the gridder."""
    import torch

    plan, uvw, freq, wgt, t_wgt, kw, dev = _problem(single)
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    x = torch.randn(plan.shape, generator=g, device=dev, dtype=plan.real)
    y = torch.randn((plan.nrow, plan.nchan), generator=g, device=dev, dtype=plan.cplx)
    ax = plan.degrid(x, t_wgt)
    aty = plan.grid(y, t_wgt)
    lhs = torch.sum((ax.conj() * y).real.double())
    rhs = torch.sum(x.double() * aty.double())
    rel = abs(float(lhs - rhs)) / (float(ax.abs().double().norm()) * float(y.abs().double().norm()))
    assert rel < (1e-6 if single else 1e-12)


def test_autograd_gradient_matches_oracle_adjoint_and_finite_differences():
    """L(x) = 0.5 ||A x - d||^2: the autograd gradient equals the CPU
    oracle's gridding of the residual (the reference gridder's adjoint), and
    central finite differences on 32 random directions."""
    import torch

    from rang import wgrid_torch

    plan, uvw, freq, wgt, t_wgt, kw, dev = _problem(False, npix=96)
    rng = np.random.default_rng(4)
    d = rng.standard_normal((plan.nrow, plan.nchan)) + 1j * rng.standard_normal((plan.nrow, plan.nchan))
    d = d * (wgt != 0)
    x0 = rng.standard_normal(plan.shape)
    td = torch.from_numpy(d).to(dev)
    x = torch.from_numpy(x0).to(dev).requires_grad_(True)

    def loss(img):
        r = wgrid_torch.degrid(img, plan, t_wgt) - td
        return 0.5 * torch.sum(r.real**2 + r.imag**2)

    L = loss(x)
    L.backward()
    grad = x.grad.detach().cpu().numpy()
    okw = dict(uvw=uvw, freq=freq, pixsize_x=kw["pixsize_x"], pixsize_y=kw["pixsize_y"], epsilon=kw["epsilon"])
    ax = oracle.dirty2vis(dirty=x0, wgt=wgt, **okw)
    ref = oracle.vis2dirty(vis=ax - d, wgt=wgt, npix_x=kw["npix_x"], npix_y=kw["npix_y"], **okw)
    assert rel_linf(grad, ref) < 1e-8
    h = 1e-4
    g = torch.Generator(device=dev)
    g.manual_seed(9)
    with torch.no_grad():
        for _ in range(32):
            v = torch.randn(plan.shape, generator=g, device=dev, dtype=torch.float64)
            fd = (float(loss(x + h * v)) - float(loss(x - h * v))) / (2 * h)
            an = float(torch.sum(x.grad * v))
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


@pytest.mark.parametrize("single", [True, False])
def test_residual_matches_the_composition_and_the_oracle(single):
    import torch

    plan, uvw, freq, wgt, t_wgt, kw, dev = _problem(single)
    rng = np.random.default_rng(6)
    d = rng.standard_normal((plan.nrow, plan.nchan)) + 1j * rng.standard_normal((plan.nrow, plan.nchan))
    model = np.zeros(plan.shape)
    model[40, 70] = 2.0
    model[90, 20] = -1.0
    td = torch.from_numpy(d).to(dev, plan.cplx)
    tm = torch.from_numpy(model).to(dev, plan.real)
    img, q = plan.residual(td, t_wgt, tm)
    okw = dict(uvw=uvw, freq=freq, pixsize_x=kw["pixsize_x"], pixsize_y=kw["pixsize_y"], epsilon=kw["epsilon"])
    dd = d.astype(np.complex64) if single else d
    mm = model.astype(np.float32) if single else model
    ww = wgt.astype(np.float32) if single else wgt
    pred = oracle.dirty2vis(dirty=mm, wgt=(ww != 0).astype(ww.dtype), **okw)
    r = dd - pred
    ref = oracle.vis2dirty(vis=r, wgt=ww, npix_x=kw["npix_x"], npix_y=kw["npix_y"], **okw)
    assert rel_linf(img.cpu().numpy(), ref) < (1e-4 if single else 1e-9)
    qref = float(np.sum(wgt * np.abs(r.astype(np.complex128)) ** 2))
    assert abs(float(q) - qref) / qref < (1e-5 if single else 1e-12)


def _numpy_fista(gram, dirty, lam, step, iters):
    """The same iteration as rang.fista.solve, in NumPy on the CPU oracle."""
    x = np.zeros_like(dirty)
    y = x.copy()
    x_prev = x.copy()
    t, beta = 1.0, 0.0
    for _ in range(iters):
        g_y = gram(y)
        z = y + step * (dirty - g_y)
        xn = np.maximum(z - step * lam, 0.0)
        nb = 0.0
        if np.sum((y - xn) * (xn - x)) > 0.0:
            t = 1.0
        else:
            tn = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t * t))
            nb = (t - 1.0) / tn
            t = tn
        x_prev, x = x, xn
        y = x + nb * (x - x_prev)
        beta = nb
    return x


def test_fista_and_power_iteration_match_a_cpu_run():
    """Ten FISTA iterations and the step size from power iteration on the GPU
    equal the same iteration on the CPU oracle (float64, to rounding)."""
    import torch

    from rang import fista

    plan, uvw, freq, wgt, t_wgt, kw, dev = _problem(False, npix=64, nchan=8)
    okw = dict(uvw=uvw, freq=freq, pixsize_x=kw["pixsize_x"], pixsize_y=kw["pixsize_y"], epsilon=kw["epsilon"])
    sky = np.zeros(plan.shape)
    sky[20, 30], sky[40, 10], sky[33, 33] = 1.0, 0.5, 0.25
    vis = oracle.dirty2vis(dirty=sky, **okw)
    dirty = oracle.vis2dirty(vis=vis, wgt=wgt, npix_x=kw["npix_x"], npix_y=kw["npix_y"], **okw)

    def gram_cpu(x):
        return oracle.vis2dirty(vis=oracle.dirty2vis(dirty=x, **okw), wgt=wgt, npix_x=kw["npix_x"],
                                npix_y=kw["npix_y"], **okw)

    def gram_gpu(x):
        return plan.gram(x, t_wgt)

    lmax, _ = fista.power_iteration(gram_gpu, plan.shape, dev, max_iterations=30, dtype=torch.float64)
    v = np.random.default_rng(1).standard_normal(plan.shape)
    for _ in range(30):
        v = gram_cpu(v)
        v /= np.linalg.norm(v)
    lcpu = float(np.sum(v * gram_cpu(v)))
    assert abs(lmax - lcpu) / lcpu < 1e-2
    step = 1.0 / lmax
    lam = 1e-3 * float(np.abs(dirty).max())
    x, gx, k, _ = fista.solve(gram_gpu, torch.from_numpy(dirty).to(dev), lam, step, 10)
    xref = _numpy_fista(gram_cpu, dirty, lam, step, 10)
    assert rel_linf(x.cpu().numpy(), xref) < 1e-8


def test_fista_reaches_the_noise():
    """Plain FISTA on point sources plus noise drives the visibility residual
    RMS down to the noise level."""
    import torch

    from rang import fista

    plan, uvw, freq, wgt, t_wgt, kw, dev = _problem(True, npix=128, nant=48, ntime=8, nchan=16)
    okw = dict(uvw=uvw, freq=freq, pixsize_x=kw["pixsize_x"], pixsize_y=kw["pixsize_y"], epsilon=1e-6)
    sky = np.zeros(plan.shape, np.float32)
    rng = np.random.default_rng(2)
    for _ in range(12):
        sky[rng.integers(10, 118), rng.integers(10, 118)] += rng.uniform(0.1, 1.0)
    sigma = 0.05
    vis = oracle.dirty2vis(dirty=sky, **okw)
    vis = vis + sigma * (rng.standard_normal(vis.shape) + 1j * rng.standard_normal(vis.shape))
    tv = torch.from_numpy(vis.astype(np.complex64)).to(dev)
    act = torch.from_numpy(wgt != 0).to(dev)
    tw = torch.where(act, 1.0, 0.0).to(torch.float32)
    dirty, q0 = plan.residual(tv, tw)
    lmax, _ = fista.power_iteration(lambda x: plan.gram(x, tw), plan.shape, dev)
    nvis = int(act.sum())

    def rms(misfit):
        return np.sqrt(max(2.0 * misfit, 0.0) / (2 * nvis))

    x, gx, k, _ = fista.solve(lambda x: plan.gram(x, tw), dirty, 1e-4 * float(dirty.max()), 1.0 / lmax, 200,
                              q0=0.5 * q0, stop=lambda k, m: rms(m) <= 1.2 * sigma)
    _, q = plan.residual(tv, tw, x)
    q = float(q)
    assert np.sqrt(q / (2 * nvis)) <= 1.25 * sigma, (k, np.sqrt(q / (2 * nvis)))
