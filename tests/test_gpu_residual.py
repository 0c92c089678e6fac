"""The plan's fused residual and Gram passes on the GPU (the reference's
Prepared::residual, residual_sorted, sorted, memory and release_grids,
core/src/wgridder.rs:3232-3440, and gram_apply), the plan and footprint
queries, and the solver's library kernels (include/rang_solver.h), against
the oracle, NumPy and the separate degrid / grid calls."""

import numpy as np
import pytest

import oracle
from cases import meerkat_like, rel_linf

pytestmark = pytest.mark.gpu


def _problem(single, method=None, npix=128, seed=0, nant=32, ntime=6, nchan=12):
    import torch

    from rang import core, synth, wgrid_torch

    if method is not None:
        core.extension().wgridder_set_method(method)
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
    d = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    model = np.zeros(plan.shape)
    n = npix
    model[5 * n // 16, 9 * n // 16], model[11 * n // 16, n // 8], model[n // 2, n // 2] = 2.0, -1.0, 0.5
    return plan, uvw, freq, wgt, t_wgt, kw, dev, d, model


@pytest.fixture(autouse=True)
def _default_method():
    from rang import core

    yield
    core.extension().wgridder_set_method(3)


# 3: integer tensor cores (the stored-values path in single precision); 0:
# FP32 CUDA cores (the visibility-indexed work space).
@pytest.mark.parametrize("single,method", [(True, 3), (True, 0), (False, None)])
def test_residual_against_the_oracle_sorted_and_dense(single, method):
    import torch

    plan, uvw, freq, wgt, t_wgt, kw, dev, d, model = _problem(single, method)
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
    # residual_sorted: the same values read from the sorted arrays give the same bits.
    img2, q2 = plan.residual(plan.sorted_values(td), plan.sorted_values(t_wgt), tm, sorted=True)
    assert torch.equal(img, img2) and torch.equal(q, q2)
    # Reproducible bit for bit, the misfit included.
    img3, q3 = plan.residual(td, t_wgt, tm)
    assert torch.equal(img, img3) and torch.equal(q, q3)
    # No model: the data alone, against plain gridding with the weights.
    img0, q0 = plan.residual(td, t_wgt)
    ref0 = plan.grid(td, t_wgt)
    assert rel_linf(img0.cpu().numpy(), ref0.cpu().numpy()) < (1e-6 if single else 1e-12)
    qd = float(np.sum(wgt * np.abs(dd.astype(np.complex128)) ** 2))
    assert abs(float(q0) - qd) / qd < (1e-6 if single else 1e-13)
    plan.close()


@pytest.mark.parametrize("single,method", [(True, 3), (True, 0), (False, None)])
def test_gram_matches_degrid_then_grid(single, method):
    import torch

    plan, uvw, freq, wgt, t_wgt, kw, dev, d, model = _problem(single, method)
    tm = torch.from_numpy(model).to(dev, plan.real)
    xgx = torch.empty((), dtype=torch.float64, device=dev)
    g = plan.gram(tm, t_wgt, xgx=xgx)
    pred = plan.degrid(tm)  # unweighted
    ref = plan.grid((pred * t_wgt).to(plan.cplx), None)
    assert rel_linf(g.cpu().numpy(), ref.cpu().numpy()) < (2e-6 if single else 1e-12)
    p = pred.cpu().numpy().astype(np.complex128)
    want = float(np.sum(wgt * np.abs(p) ** 2))
    assert abs(float(xgx) - want) / want < (1e-6 if single else 1e-12)
    # x^T G x from the image side agrees.
    side = float(torch.dot(tm.double().ravel(), g.double().ravel()))
    assert abs(side - want) / want < (1e-4 if single else 1e-9)
    assert torch.equal(g, plan.gram(tm, t_wgt))
    plan.close()


def test_memory_report_and_release():
    import torch

    plan, uvw, freq, wgt, t_wgt, kw, dev, d, model = _problem(True)
    before = plan.memory()
    assert len(before) == 8 and before["gridder: stored sorted values"] == 0
    assert before["gridder: sorted visibility index"] == 4 * plan.active
    plan.residual(torch.from_numpy(d).to(dev, plan.cplx), t_wgt, torch.from_numpy(model).to(dev, plan.real))
    torch.cuda.synchronize()
    assert plan.memory()["gridder: stored sorted values"] == 8 * plan.active
    plan.release_work()
    assert plan.memory()["gridder: stored sorted values"] == 0
    plan.close()


def test_sorted_values_follow_the_binning_order():
    import torch

    plan, uvw, freq, wgt, t_wgt, kw, dev, d, model = _problem(True)
    idx = torch.arange(plan.nrow * plan.nchan, device=dev, dtype=torch.int32).reshape(plan.nrow, plan.nchan)
    got = plan.sorted_values(idx).cpu().numpy()
    assert got.size == plan.active == int((wgt != 0).sum())
    assert np.array_equal(np.sort(got), np.flatnonzero(wgt.ravel() != 0))
    plan.close()


@pytest.mark.parametrize("single", [True, False])
def test_plan_and_footprint_equal_the_binning_plan(single):
    from rang import gridder

    uvw, freq = meerkat_like(nant=24, ntime=4, nchan=8, seed=3)
    rng = np.random.default_rng(2)
    wgt = rng.uniform(0.5, 1.5, (uvw.shape[0], freq.size))
    wgt.ravel()[::5] = 0.0
    kw = dict(uvw=uvw, freq=freq, npix_x=256, npix_y=192, pixsize_x=1e-5, pixsize_y=1.2e-5,
              epsilon=1e-5 if single else 1e-9)
    info = gridder.plan(wgt=wgt, single=single, **kw)
    ref = oracle.binning(wgt=wgt, single=single, with_vis=False, **kw)["info"]
    assert info == ref
    info2, fp = gridder.gridding_footprint(wgt=wgt, single=single, nout=2, **kw)
    assert info2 == ref
    cell = 16 if single else 32  # the fixed-point cell, complex
    assert fp >= 2 * info["nu"] * info["nv"] * cell


def test_library_dot_and_lowpass_against_numpy():
    import torch

    from rang import fista

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(4)
    a = rng.standard_normal((300, 257)).astype(np.float32)
    b = rng.standard_normal((300, 257)).astype(np.float32)
    got = float(fista.dot(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)))
    want = float(np.dot(a.astype(np.float64).ravel(), b.astype(np.float64).ravel()))
    assert abs(got - want) <= 1e-12 * np.abs(a.astype(np.float64) * b).sum()
    sigma = 3.5
    low = fista.gaussian_lowpass(torch.from_numpy(a).to(dev), sigma).cpu().numpy()
    f0 = np.fft.fftfreq(300)[:, None]
    f1 = np.fft.rfftfreq(257)[None, :]
    ref = np.fft.irfft2(np.fft.rfft2(a.astype(np.float64)) * np.exp(-2 * np.pi**2 * sigma**2 * (f0**2 + f1**2)),
                        s=a.shape)
    assert np.abs(low - ref).max() < 1e-5 * np.abs(ref).max()


def test_device_fista_matches_a_numpy_run_with_its_misfits():
    """Twelve iterations of the library's step kernels equal the same FISTA in
    NumPy on the GPU's own Gram operator (float64), iterate and misfits."""
    import torch

    from rang import fista

    plan, uvw, freq, wgt, t_wgt, kw, dev, d, model = _problem(False, npix=64, nchan=6)
    td = torch.from_numpy(d).to(dev, plan.cplx)
    dirty, q = plan.residual(td, t_wgt)
    q0 = 0.5 * float(q)

    def gram(x):
        return plan.gram(x, t_wgt)

    lam = 1e-3 * float(dirty.abs().max())
    step = 1.0 / fista.power_iteration(gram, plan.shape, dev, dtype=torch.float64)[0]
    res = fista.solve(gram, dirty, lam, step, 12, q0=0.5 * q)
    dn = dirty.cpu().numpy()
    x = np.zeros_like(dn)
    xp = x.copy()
    y, t, beta, gxp = x.copy(), 1.0, 0.0, np.zeros_like(dn)
    misfits = []
    for k in range(13):
        gy = gram(torch.from_numpy(y).to(dev)).cpu().numpy()
        gx = gy if beta == 0.0 else (gy + beta * gxp) / (1.0 + beta)
        misfits.append(q0 - np.sum(dn * x) + 0.5 * np.sum(x * gx))
        if k == 12:
            break
        xn = np.maximum(y + step * (dn - gy) - step * lam, 0.0)
        nb = 0.0
        if np.sum((y - xn) * (xn - x)) > 0.0:
            t = 1.0
        else:
            tn = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t * t))
            nb, t = (t - 1.0) / tn, tn
        gxp = gx
        xp, x = x, xn
        y = x + nb * (x - xp)
        beta = nb
    assert res.k == 12
    assert rel_linf(res.x.cpu().numpy(), x) < 1e-10
    assert np.allclose(res.misfits.cpu().numpy(), misfits, rtol=1e-10, atol=1e-12 * abs(q0))
    plan.close()


@pytest.mark.parametrize("single", [True, False])
def test_grid_of_the_scanned_data_skips_its_bound_pass_with_the_same_bits(single):
    """A plan made with the visibilities grids them with the scan's value bound
    (`scanned=True`) to the same bits as with the bound pass over the data."""
    import torch

    from rang import wgrid_torch

    uvw, freq = meerkat_like(nant=24, ntime=6, nchan=10, seed=4)
    rng = np.random.default_rng(8)
    shape = (uvw.shape[0], freq.size)
    vis = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    dev = torch.device("cuda", 0)
    tv = torch.from_numpy(vis).to(dev, torch.complex64 if single else torch.complex128)
    kw = dict(npix_x=128, npix_y=96, pixsize_x=2e-5, pixsize_y=2e-5, epsilon=1e-5 if single else 1e-9)
    plan = wgrid_torch.DevicePlan(torch.from_numpy(uvw).to(dev), freq, vis=tv, single=single, **kw)
    a = plan.grid(tv)
    b = plan.grid(tv, scanned=True)
    assert torch.equal(a, b)
    plan.close()


@pytest.mark.parametrize("single", [True, False])
def test_residual_and_gram_of_a_plan_with_nothing_active(single):
    """All weights zero: the plan is empty, the residual and Gram images are
    zero, the misfit and x^T G x are zero, and nothing is stored."""
    import torch

    from rang import wgrid_torch

    uvw, freq = meerkat_like(nant=8, ntime=2, nchan=4, seed=2)
    dev = torch.device("cuda", 0)
    rt = torch.float32 if single else torch.float64
    w = torch.zeros((uvw.shape[0], freq.size), dtype=rt, device=dev)
    plan = wgrid_torch.DevicePlan(torch.from_numpy(uvw).to(dev), freq, wgt=w, single=single, npix_x=64, npix_y=64,
                                  pixsize_x=2e-5, pixsize_y=2e-5, epsilon=1e-5 if single else 1e-9)
    assert plan.active == 0
    d = torch.ones((uvw.shape[0], freq.size), dtype=plan.cplx, device=dev)
    img, q = plan.residual(d, w, torch.ones(plan.shape, dtype=rt, device=dev))
    assert float(img.abs().max()) == 0.0 and float(q) == 0.0
    xgx = torch.full((), 7.0, dtype=torch.float64, device=dev)
    g = plan.gram(torch.ones(plan.shape, dtype=rt, device=dev), w, xgx=xgx)
    assert float(g.abs().max()) == 0.0 and float(xgx) == 0.0
    assert plan.memory()["gridder: stored sorted values"] == 0
    plan.close()


def test_cached_buffers_are_reused_and_released():
    """Buffers of 64 MB or more stay cached for the next call of the same
    shape (no allocation then), and release_cached gives them back to the
    device, so that other allocators in the process can use the memory."""
    import torch

    from rang import core, gridder as cw

    ext = core.extension()
    uvw, freq = meerkat_like(nant=64, ntime=32, nchan=64, seed=3)  # 4.1 M visibilities: 132 MB of records
    rng = np.random.default_rng(3)
    vis = (rng.standard_normal((uvw.shape[0], freq.size)) + 1j).astype(np.complex64)
    kw = dict(uvw=uvw, freq=freq, npix_x=256, npix_y=256, pixsize_x=3e-5, pixsize_y=3e-5, epsilon=1e-5)
    assert ext.wgridder_release_cached() == 0  # the earlier tests' buffers
    first = cw.vis2dirty(vis=vis, **kw)
    held = ext.wgridder_cached_bytes()
    assert held >= 64 << 20
    again = cw.vis2dirty(vis=vis, **kw)
    assert np.array_equal(first, again)
    assert ext.wgridder_cached_bytes() == held  # the same buffers, taken and returned
    free_before, _ = torch.cuda.mem_get_info(0)
    assert ext.wgridder_release_cached() == 0
    assert ext.wgridder_cached_bytes() == 0
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after >= free_before + held - (256 << 20)  # allocation granularity aside
