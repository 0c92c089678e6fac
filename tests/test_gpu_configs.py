"""The CUDA path at the benchmark configurations' own sizes, against the CPU
oracle (the restatement of the reference's wgridder.rs, pinned to the
reference's known answers and recorded DF1 errors by test_oracle.py).

* Configuration 1: the 64-antenna MeerKAT-shaped array, 128 integrations of
  8 s, 64 channels over 856-1712 MHz (16,515,072 visibilities, 50 seeded
  point sources plus complex noise of sigma 0.1, unit weights, no flags),
  1024^2 at 1.5 arcsec; single precision at epsilon 1e-5 and double at
  1e-7. The plan (`info`) and every visibility's binning integers equal the
  oracle's bit for bit, the active visibilities come out in the reference's
  layout order, and images and visibilities are compared with the oracle at
  the same precision and epsilon and with the oracle's FP64 run at epsilon
  1e-7 (the error of the single-precision path against FP64), as L-inf over
  the reference's peak with the border (outer two pixels) apart from the
  interior (eight pixels in), the protocol of the reference's edge study
  (research/df2-wgridder-speed.md:446-487).
* Configuration 3: the differentiable degridder on 2048^2 float32 images
  with 64 antennas x 256 integrations x 256 channels (132,120,576
  visibilities): the adjoint dot-product test to 1e-6, central finite
  differences along 32 random image directions, and the autograd gradient
  against the oracle's gridding of the residual (the reference gridder's
  adjoint).

Both run the oracle on the host's cores (tens of seconds).
"""

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def border_interior(x, ref):
    """(border, interior) L-inf of x - ref over max |ref|: the outer two
    pixels of the image, and the pixels eight or more in from the edge."""
    err = np.abs(np.asarray(x, np.float64) - ref)
    peak = float(np.abs(ref).max())
    inner = np.zeros(err.shape, bool)
    inner[8:-8, 8:-8] = True
    outer = np.ones(err.shape, bool)
    outer[2:-2, 2:-2] = False
    return float(err[outer].max() / peak), float(err[inner].max() / peak)


def rel_linf(x, ref):
    return float(np.abs(np.asarray(x) - ref).max() / np.abs(ref).max())


@pytest.fixture(scope="module")
def config1():
    from rang import gridder, synth

    uvw = synth.uvw_tracks(nant=64, ntime=128, tint=8.0, dec_deg=-30.0, seed=7)
    freq = synth.channels(64)
    npix, cell = 1024, 1.5 * synth.ARCSEC
    sky = synth.point_sky(npix, nsrc=50, seed=11)
    kw = dict(uvw=uvw, freq=freq, pixsize_x=cell, pixsize_y=cell)
    # The sky's visibilities, predicted in double precision at epsilon 1e-9
    # (the data for both sides; made on the GPU, which is fast), plus seeded
    # complex noise of sigma 0.1.
    model = gridder.dirty2vis(dirty=sky, epsilon=1e-9, **kw)
    rng = np.random.default_rng(101)
    vis = model + 0.1 * (rng.standard_normal(model.shape) + 1j * rng.standard_normal(model.shape))
    assert vis.size == 16_515_072
    fp64 = oracle.vis2dirty(vis=vis, npix_x=npix, npix_y=npix, epsilon=1e-7, **kw)
    return dict(kw=kw, npix=npix, vis=vis, sky=sky, fp64=fp64)


@pytest.mark.parametrize("single,eps", [(True, 1e-5), (False, 1e-7)])
def test_config1_plan_and_binning_equal_the_oracle(config1, single, eps):
    from rang import gridder

    c = config1
    n = c["npix"]
    common = dict(npix_x=n, npix_y=n, epsilon=eps, **c["kw"])
    vis = c["vis"].astype(np.complex64) if single else c["vis"]
    g = gridder.binning(vis=vis, single=single, with_vis=True, **common)
    o = oracle.binning(vis=vis, single=single, with_vis=True, **common)
    assert g["info"] == o["info"]
    nb = max(o["info"]["nplanes"], 1)
    act = o["tile"] >= 0
    assert np.array_equal(g["iu0"][act], o["iu0"][act]) and np.array_equal(g["iv0"][act], o["iv0"][act])
    okey = np.where(act, o["tile"] * nb + o["minplane"], 0xFFFFFFFF).astype(np.uint32)
    assert np.array_equal(g["key"], okey)
    assert np.array_equal(g["sorted"], o["sorted"])


@pytest.mark.parametrize("single,eps", [(True, 1e-5), (False, 1e-7)])
def test_config1_images_against_the_oracle_and_fp64(config1, single, eps):
    from rang import gridder

    c = config1
    n = c["npix"]
    vis = c["vis"].astype(np.complex64) if single else c["vis"]
    d, info = gridder.vis2dirty(vis=vis, npix_x=n, npix_y=n, epsilon=eps, return_info=True, **c["kw"])
    od, oinfo = oracle.vis2dirty(vis=vis, npix_x=n, npix_y=n, epsilon=eps, return_info=True, **c["kw"])
    assert info == oinfo and info["nvis"] == vis.size
    # Against the oracle at the same precision and epsilon (summation order, FFT).
    b, i = border_interior(d, od)
    assert max(b, i) < (2e-6 if single else 1e-11), (b, i)
    # Against FP64 at epsilon 1e-7: the error of this precision and epsilon.
    b, i = border_interior(d, c["fp64"])
    assert max(b, i) < (10 * eps if single else 1e-9), (b, i)
    # Reproducible bit for bit.
    assert np.array_equal(d, gridder.vis2dirty(vis=vis, npix_x=n, npix_y=n, epsilon=eps, **c["kw"]))


@pytest.mark.parametrize("single,eps", [(True, 1e-5), (False, 1e-7)])
def test_config1_visibilities_against_the_oracle_and_fp64(config1, single, eps):
    from rang import gridder

    c = config1
    img = c["sky"].astype(np.float32) if single else c["sky"]
    v = gridder.dirty2vis(dirty=img, epsilon=eps, **c["kw"])
    ov = oracle.dirty2vis(dirty=img, epsilon=eps, **c["kw"])
    assert rel_linf(v, ov) < (2e-6 if single else 1e-11)
    fp64 = oracle.dirty2vis(dirty=c["sky"], epsilon=1e-7, **c["kw"])
    assert rel_linf(v, fp64) < (10 * eps if single else 1e-9)
    assert np.array_equal(v, gridder.dirty2vis(dirty=img, epsilon=eps, **c["kw"]))


def test_config3_differentiable_degridder_at_full_size():
    """2048^2 float32, 132,120,576 visibilities: adjointness, 32 central
    finite differences and the gradient against the oracle's adjoint."""
    import torch

    from rang import synth, wgrid_torch

    uvw_np = synth.uvw_tracks(nant=64, ntime=256, tint=8.0, dec_deg=-30.0, seed=7)
    freq = synth.channels(256)
    n, cell = 2048, 1.5 * synth.ARCSEC
    dev = torch.device("cuda", 0)
    kw = dict(npix_x=n, npix_y=n, pixsize_x=cell, pixsize_y=cell, epsilon=1e-5)
    plan = wgrid_torch.DevicePlan(torch.from_numpy(uvw_np).to(dev), freq, single=True, **kw)
    assert plan.nrow * plan.nchan == 132_120_576
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    # Adjointness <A x, y> = <x, A^H y>.
    x = torch.randn(plan.shape, generator=g, device=dev, dtype=torch.float32)
    y = torch.randn((plan.nrow, plan.nchan), generator=g, device=dev, dtype=torch.complex64)
    ax = plan.degrid(x)
    aty = plan.grid(y)
    lhs = torch.sum((ax.conj() * y).real.double())
    rhs = torch.sum(x.double() * aty.double())
    rel = abs(float(lhs - rhs)) / (float(ax.abs().double().norm()) * float(y.abs().double().norm()))
    assert rel < 1e-6, rel
    del ax, aty, y
    # L(x) = 0.5 ||A x - d||^2 with data d = A x_true.
    xt = torch.randn(plan.shape, generator=g, device=dev, dtype=torch.float32)
    d = plan.degrid(xt)
    x = torch.randn(plan.shape, generator=g, device=dev, dtype=torch.float32).requires_grad_(True)

    def loss(img):
        r = wgrid_torch.degrid(img, plan) - d
        return 0.5 * torch.sum(r.real.double() ** 2 + r.imag.double() ** 2)

    L = loss(x)
    L.backward()
    grad = x.grad.detach()
    # Central differences along 32 random directions. L is quadratic in x, so
    # a central difference is the exact directional derivative at any step;
    # a unit step keeps the float32 rounding of L small beside it.
    h = 1.0
    with torch.no_grad():
        for _ in range(32):
            v = torch.randn(plan.shape, generator=g, device=dev, dtype=torch.float32)
            fd = (float(loss(x + h * v)) - float(loss(x - h * v))) / (2 * h)
            an = float(torch.sum(grad.double() * v.double()))
            assert abs(fd - an) <= 1e-3 * abs(an), (fd, an)
    # The gradient is A^H (A x - d): against the oracle gridding the residual.
    with torch.no_grad():
        r = (plan.degrid(x.detach()) - d).cpu().numpy()
    ref = oracle.vis2dirty(uvw=uvw_np, freq=freq, vis=r.astype(np.complex64), **kw)
    assert rel_linf(grad.cpu().numpy(), ref) < 1e-5
