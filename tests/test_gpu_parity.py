"""Parity of the CUDA path (through `rang._core`, the C ABI) with the CPU
oracle and the FP64 DFT.

Tolerances: the integer binning (iu0, iv0, tile, first plane, plan) must be
bit-identical to the oracle's; images and visibilities agree with the
oracle's to 1e-9 (f64) and 2e-5 (f32) relative L-inf (the two differ only in
accumulation order and FFT rounding, which the wide-field correction factors
amplify up to ~1e5 at the image corners of the 0.3 rad cases), and with the
DFT to the reference's own gates (10 eps, research/df1-wgridder.md:179-203)."""

from pathlib import Path

import numpy as np
import pytest

import oracle
from cases import DF1_RECORDED, df1_cases, df1_record, df1_worst, lcg_case, meerkat_like, rel_linf, small_case

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = {True: 2e-5, False: 1e-9}


@pytest.fixture(scope="module")
def cw():
    from rang import gridder

    return gridder


def _info_equal(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert a[k] == b[k], (k, a[k], b[k])


def test_vis2dirty_matches_dft_both_precisions(cw):
    # reference tests/test_core_wgridder.py:75-95
    uvw, freq, vis, wgt, nx, ny, dx = small_case()
    ref = oracle.dft_dirty(uvw, freq, vis * wgt, nx, ny, dx, dx)
    common = dict(uvw=uvw, freq=freq, npix_x=nx, npix_y=ny, pixsize_x=dx, pixsize_y=dx)
    d64, info = cw.vis2dirty(vis=vis, wgt=wgt, epsilon=1e-9, return_info=True, **common)
    assert rel_linf(d64, ref) < 1e-8
    assert info["nvis"] == vis.size and info["nplanes"] > info["supp"]
    _, oinfo = oracle.vis2dirty(vis=vis, wgt=wgt, epsilon=1e-9, return_info=True, **common)
    _info_equal(info, oinfo)
    d32 = cw.vis2dirty(vis=vis.astype(np.complex64), wgt=wgt.astype(np.float32), epsilon=1e-4, **common)
    assert d32.dtype == np.float32 and rel_linf(d32, ref) < 1e-3


def test_lcg_cases_match_dft(cw):
    # core/src/wgridder.rs:4667-4686
    for nx, ny, field, wmax in [(32, 32, 0.2, 500.0), (32, 16, 0.05, 50.0)]:
        uvw, freq, vis, wgt, dx = lcg_case(nx, ny, field, wmax, 60, 7)
        d = cw.vis2dirty(uvw=uvw, freq=freq, vis=vis, wgt=wgt, npix_x=nx, npix_y=ny, pixsize_x=dx,
                         pixsize_y=dx, epsilon=1e-9)
        assert rel_linf(d, oracle.dft_dirty(uvw, freq, vis * wgt, nx, ny, dx, dx)) < 1e-8


def test_adjoint_and_dirty2vis(cw):
    # reference tests/test_core_wgridder.py:98-125
    uvw, freq, vis, wgt, nx, ny, dx = small_case(seed=8)
    x = np.random.default_rng(1).standard_normal((nx, ny))
    common = dict(uvw=uvw, freq=freq, wgt=wgt, pixsize_x=dx, pixsize_y=dx, epsilon=1e-9)
    ax = cw.dirty2vis(dirty=x, **common)
    aty = cw.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, **common)
    lhs = np.real(np.vdot(ax, vis))
    assert abs(lhs - np.sum(x * aty)) / (np.linalg.norm(ax) * np.linalg.norm(vis)) < 1e-12
    img = np.zeros((nx, ny))
    img[5, 20] = 2.0
    got = cw.dirty2vis(dirty=img, **common)
    assert rel_linf(got, oracle.dft_vis(uvw, freq, img, dx, dx) * wgt) < 1e-8


def test_zero_weights_and_bad_input(cw):
    # reference tests/test_core_wgridder.py:128-147
    uvw, freq, vis, wgt, nx, ny, dx = small_case(nrow=6)
    common = dict(uvw=uvw, freq=freq, npix_x=nx, npix_y=ny, pixsize_x=dx, pixsize_y=dx)
    empty, info = cw.vis2dirty(vis=vis, wgt=np.zeros_like(wgt), epsilon=1e-6, return_info=True, **common)
    assert not empty.any() and info["nvis"] == 0
    with pytest.raises(ValueError, match="ascending"):
        cw.vis2dirty(vis=vis, wgt=wgt, epsilon=1e-6, **{**common, "freq": freq[::-1]})
    with pytest.raises(ValueError, match="kernel"):
        cw.vis2dirty(vis=vis, wgt=wgt, epsilon=1e-14, **common)
    with pytest.raises(ValueError, match="even"):
        cw.vis2dirty(vis=vis, wgt=wgt, epsilon=1e-6, **{**common, "npix_x": 31})
    v = cw.dirty2vis(dirty=np.ones((nx, ny)), uvw=uvw, freq=freq, wgt=np.zeros_like(wgt), pixsize_x=dx,
                     pixsize_y=dx, epsilon=1e-6)
    assert not v.any()


@pytest.fixture(scope="module")
def df1():
    return df1_cases(GOLDEN)


@pytest.mark.parametrize("single,eps", DF1_RECORDED)
def test_df1_errors_within_the_references_record(cw, df1, single, eps):
    """The GPU's worst error against the DFT over the four DF1 cases (made by
    the reference's own generator) is within 1.5 times the reference
    gridder's own recorded worst for the same precision, epsilon and
    direction (research/results/df1-wgridder.json "worst")."""
    wd, wv = df1_worst(df1, single, eps, cw.vis2dirty, cw.dirty2vis)
    assert wd <= 1.5 * df1_record(GOLDEN, single, eps, "vis2dirty")
    assert wv <= 1.5 * df1_record(GOLDEN, single, eps, "dirty2vis")


@pytest.mark.parametrize("eps,single", [(1e-5, True), (1e-5, False), (1e-7, False), (1e-9, False)])
def test_golden_df1_cases(cw, df1, eps, single):
    """Within 10 eps of the golden FP64 DFT, and equal to the oracle to
    rounding, in both directions."""
    for name, c in df1.items():
        nx, ny, dx, dy = int(c["nx"]), int(c["ny"]), float(c["dx"]), float(c["dy"])
        vis = c["vis"].astype(np.complex64) if single else c["vis"]
        wgt = c["wgt"].astype(np.float32) if single else c["wgt"]
        kw = dict(uvw=c["uvw"], freq=c["freq"], wgt=wgt, pixsize_x=dx, pixsize_y=dy, epsilon=eps)
        d, info = cw.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, return_info=True, **kw)
        od, oinfo = oracle.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, return_info=True, **kw)
        _info_equal(info, oinfo)
        assert rel_linf(d, c["dft_dirty"]) < 10 * eps, name
        assert rel_linf(d, od) < TOL[single], name
        img = c["image"].astype(np.float32) if single else c["image"]
        v = cw.dirty2vis(dirty=img, **kw)
        assert rel_linf(v, c["dft_vis"]) < 10 * eps, name
        assert rel_linf(v, oracle.dirty2vis(dirty=img, **kw)) < TOL[single], name


OPTION_SETS = [
    {},
    {"flip_u": True, "flip_v": True},
    {"flip_w": True},
    {"center_x": 0.01, "center_y": -0.02},
    {"center_x": -0.005, "flip_u": True, "allow_nshift": False},
    {"divide_by_n": True},
    {"do_wgridding": False},
    {"sigma_min": 1.5, "sigma_max": 2.0},
]


@pytest.mark.parametrize("single", [True, False])
@pytest.mark.parametrize("opts", OPTION_SETS, ids=lambda o: ",".join(o) or "default")
def test_options_match_oracle(cw, opts, single):
    uvw, freq = meerkat_like(nant=16, ntime=6, nchan=8, seed=3)
    rng = np.random.default_rng(11)
    shape = (uvw.shape[0], freq.size)
    vis = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    wgt = rng.uniform(0.5, 1.5, shape)
    mask = (rng.uniform(size=shape) > 0.2).astype(np.uint8)
    if single:
        vis, wgt = vis.astype(np.complex64), wgt.astype(np.float32)
    nx, ny, dx = 96, 64, 2.0e-4
    eps = 1e-5 if single else 1e-10
    kw = dict(uvw=uvw, freq=freq, wgt=wgt, mask=mask, pixsize_x=dx, pixsize_y=dx * 1.1, epsilon=eps, **opts)
    d, info = cw.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, return_info=True, **kw)
    od, oinfo = oracle.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, return_info=True, **kw)
    _info_equal(info, oinfo)
    assert rel_linf(d, od) < TOL[single]
    x = rng.standard_normal((nx, ny)).astype(np.float32 if single else np.float64)
    v = cw.dirty2vis(dirty=x, **kw)
    ov = oracle.dirty2vis(dirty=x, **kw)
    assert rel_linf(v, ov) < TOL[single]
    assert not v[mask == 0].any()


@pytest.mark.parametrize("single", [True, False])
@pytest.mark.parametrize("opts", [{}, {"center_x": 0.01, "center_y": -0.02}, {"flip_u": True, "center_x": -0.005}],
                         ids=["centred", "shifted", "flipped-shifted"])
def test_touched_row_pruning_matches_oracle(cw, opts, single):
    """Small pixels (0.5 arcsec, 256^2) against baselines up to 41 k
    wavelengths: the footprints reach a tenth of the grid's width on either
    side of the centre, so the v transforms run on about two thirds of the
    rows (with the recentring term |r_l| |w| in the bound). Both directions
    equal the oracle, which transforms every row."""
    uvw, freq = meerkat_like(nant=32, ntime=16, nchan=16, seed=4)
    rng = np.random.default_rng(21)
    shape = (uvw.shape[0], freq.size)
    vis = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    mask = (rng.uniform(size=shape) > 0.1).astype(np.uint8)
    if single:
        vis = vis.astype(np.complex64)
    nx = ny = 256
    dx = 0.5 * np.pi / 648000.0
    eps = 1e-5 if single else 1e-10
    kw = dict(uvw=uvw, freq=freq, mask=mask, pixsize_x=dx, pixsize_y=dx, epsilon=eps, **opts)
    d, info = cw.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, return_info=True, **kw)
    od, oinfo = oracle.vis2dirty(vis=vis, npix_x=nx, npix_y=ny, return_info=True, **kw)
    _info_equal(info, oinfo)
    assert rel_linf(d, od) < TOL[single]
    x = rng.standard_normal((nx, ny)).astype(np.float32 if single else np.float64)
    assert rel_linf(cw.dirty2vis(dirty=x, **kw), oracle.dirty2vis(dirty=x, **kw)) < TOL[single]


@pytest.mark.parametrize("single", [True, False])
def test_binning_is_bit_exact(cw, single):
    """iu0, iv0, tile and first plane of every visibility equal the oracle's
    (the reference's index arithmetic), and the GPU's order is the oracle's
    up to the order inside a (tile, plane) bin."""
    uvw, freq = meerkat_like(nant=24, ntime=8, nchan=32, seed=5)
    rng = np.random.default_rng(2)
    shape = (uvw.shape[0], freq.size)
    vis = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    vis.ravel()[::17] = 0.0
    wgt = rng.uniform(0.5, 1.5, shape)
    wgt.ravel()[::13] = 0.0
    for opts in ({}, {"center_x": 0.003, "flip_v": True}, {"do_wgridding": False}):
        for with_vis in (True, False):
            kw = dict(uvw=uvw, freq=freq, vis=vis, wgt=wgt, npix_x=512, npix_y=384, pixsize_x=1.5e-5,
                      pixsize_y=1.5e-5, epsilon=1e-5 if single else 1e-7, single=single, with_vis=with_vis,
                      **opts)
            g = cw.binning(**kw)
            o = oracle.binning(**kw)
            _info_equal(g["info"], o["info"])
            nb = max(o["info"]["nplanes"], 1)
            act = o["tile"] >= 0
            okey = np.where(act, o["tile"] * nb + o["minplane"], 0xFFFFFFFF).astype(np.uint32)
            assert np.array_equal(g["key"], okey)
            assert np.array_equal(g["iu0"][act], o["iu0"][act])
            assert np.array_equal(g["iv0"][act], o["iv0"][act])
            assert np.array_equal(g["sorted"], o["sorted"])


def test_psf_mode_and_weight_kinds(cw):
    # reference tests/test_core_wgridder.py:215-261, bit for bit: the grid
    # sums exact fixed-point terms, so the one-pass PSF, the two weights and
    # the separate calls give the same bits
    uvw, freq, vis, wgt, nx, ny, dx = small_case(seed=21, nrow=50)
    vis64 = vis.astype(np.complex64)
    wgt32 = wgt.astype(np.float32)
    wgt32[3, 1] = 0.0
    common = dict(uvw=uvw, freq=freq, npix_x=nx, npix_y=ny, pixsize_x=dx, pixsize_y=dx, epsilon=1e-7)
    dirty, psf = cw.dirty_psf(vis=vis64, wgt=wgt32, **common)
    odirty, opsf = oracle.dirty_psf(vis=vis64, wgt=wgt32, **common)
    assert rel_linf(dirty, odirty) < 1e-10 and rel_linf(psf, opsf) < 1e-10
    sep = cw.vis2dirty(vis=vis64.astype(np.complex128), wgt=wgt32.astype(np.float64), **common)
    assert np.array_equal(dirty, sep)
    b = np.random.default_rng(99).uniform(0.1, 1.1, wgt32.shape).astype(np.float32)
    one = cw.dirty_psf(vis=vis64, wgt=wgt32 * b, single=True, **{**common, "epsilon": 1e-5})
    two = cw.dirty_psf(vis=vis64, wgt=wgt32, wgt2=b, single=True, **{**common, "epsilon": 1e-5})
    assert np.array_equal(one[0], two[0]) and np.array_equal(one[1], two[1])
    x = np.random.default_rng(2).standard_normal((nx, ny))
    kw = {k: common[k] for k in ("uvw", "freq", "pixsize_x", "pixsize_y", "epsilon")}
    assert np.array_equal(cw.dirty2vis(dirty=x, wgt=wgt32, **kw),
                          cw.dirty2vis(dirty=x, wgt=wgt32.astype(np.float64), **kw))


def test_larger_case_matches_oracle(cw):
    """A MeerKAT-shaped case with flags at eps 1e-5 (single) and 1e-7
    (double), against the oracle and, on a few pixels, the DFT."""
    uvw, freq = meerkat_like(nant=64, ntime=8, nchan=16, seed=1)
    rng = np.random.default_rng(5)
    shape = (uvw.shape[0], freq.size)
    vis = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    mask = (rng.uniform(size=shape) > 0.2).astype(np.uint8)
    nx = ny = 256
    dx = 1.5 * np.pi / 648000.0
    for single, eps in ((True, 1e-5), (False, 1e-7)):
        v = vis.astype(np.complex64) if single else vis
        kw = dict(uvw=uvw, freq=freq, mask=mask, pixsize_x=dx, pixsize_y=dx, epsilon=eps)
        d = cw.vis2dirty(vis=v, npix_x=nx, npix_y=ny, **kw)
        od = oracle.vis2dirty(vis=v, npix_x=nx, npix_y=ny, **kw)
        assert rel_linf(d, od) < TOL[single] * 5
        x = rng.standard_normal((nx, ny)).astype(np.float32 if single else np.float64)
        assert rel_linf(cw.dirty2vis(dirty=x, **kw), oracle.dirty2vis(dirty=x, **kw)) < TOL[single] * 5


@pytest.fixture
def method():
    """Runs a test under one single-precision gridding method and restores
    the default afterwards."""
    ext = __import__("rang._core", fromlist=["_core"])
    old = ext.wgridder_set_method(1)
    yield ext
    ext.wgridder_set_method(old)


@pytest.mark.parametrize("which", [0, 1, 2], ids=["fp32-cuda-cores", "3xtf32-tensor-cores", "3xbf16-tensor-cores"])
def test_single_precision_methods_match_oracle(cw, method, df1, which):
    """Every single-precision gridding path, the plain FP32 CUDA-core one and
    the split-precision 3 x TF32 and 3 x BF16 tensor-core ones, stays within
    the f32 tolerance of the oracle (2e-5 of the peak) and within 1e-4 of the
    FP64 DFT."""
    method.wgridder_set_method(which)
    for name, c in df1.items():
        nx, ny, dx, dy = int(c["nx"]), int(c["ny"]), float(c["dx"]), float(c["dy"])
        kw = dict(uvw=c["uvw"], freq=c["freq"], wgt=c["wgt"].astype(np.float32), npix_x=nx, npix_y=ny,
                  pixsize_x=dx, pixsize_y=dy, epsilon=1e-5)
        vis = c["vis"].astype(np.complex64)
        d = cw.vis2dirty(vis=vis, **kw)
        assert rel_linf(d, c["dft_dirty"]) < 1e-4, name
        assert rel_linf(d, oracle.vis2dirty(vis=vis, **kw)) < TOL[True], name
    uvw, freq = meerkat_like(nant=64, ntime=8, nchan=16, seed=1)
    rng = np.random.default_rng(5)
    shape = (uvw.shape[0], freq.size)
    vis = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    kw = dict(uvw=uvw, freq=freq, mask=(rng.uniform(size=shape) > 0.2).astype(np.uint8), npix_x=256, npix_y=192,
              pixsize_x=7e-6, pixsize_y=7e-6, epsilon=1e-5)
    for opts in ({}, {"do_wgridding": False}, {"center_x": 1e-4}):
        d, psf = cw.dirty_psf(vis=vis, single=True, **kw, **opts)
        od, opsf = oracle.dirty_psf(vis=vis, single=True, **kw, **opts)
        assert rel_linf(d, od) < TOL[True] and rel_linf(psf, opsf) < TOL[True]


def test_split_precision_error_on_a_single_visibility(cw, method):
    """One visibility, where no averaging hides the error of its footprint:
    3 x TF32 (about 21 bits of each factor) stays at epsilon against the
    float64 result, as plain FP32 does; 3 x BF16 (about 16 bits) does not,
    measured at 3-4 epsilon, and stays below 10 epsilon (the DFT gate). This
    is why 3 x TF32 is the default."""
    rng = np.random.default_rng(11)
    uvw = rng.uniform(-2000.0, 2000.0, size=(1, 3)) * np.array([1.0, 1.0, 0.2])
    vis = rng.standard_normal((1, 1)) + 1j * rng.standard_normal((1, 1))
    kw = dict(uvw=uvw, freq=np.array([1.0e9]), npix_x=256, npix_y=256, pixsize_x=4.0 * np.pi / 648000.0,
              pixsize_y=4.0 * np.pi / 648000.0)
    ref = cw.vis2dirty(vis=vis, epsilon=1e-12, **kw)
    for eps in (1e-5, 1e-6):
        err = {}
        for code in (0, 1, 2):
            method.wgridder_set_method(code)
            err[code] = rel_linf(cw.vis2dirty(vis=vis.astype(np.complex64), epsilon=eps, **kw), ref)
        assert err[0] < eps and err[1] < eps, (eps, err)
        assert err[1] < 2.0 * err[0] + 1e-7, (eps, err)
        assert err[1] < err[2] < 10.0 * eps, (eps, err)
