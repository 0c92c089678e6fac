"""Imaging weights and Stokes I on the GPU (rang.weighting over the C ABI
of include/rang_weights.h) against the CPU oracle's restatement of the
reference's weights.rs.

Bar: the imaging weights, the finished grid and the Stokes I values and
weights bit for bit (per-sample arithmetic is the reference's; the cell sums
of float weights are exact in double, so their order does not matter); the
header sums' double totals to 1e-12 relative, as the reference's own test
allows between its core and NumPy."""

import numpy as np
import pytest

import oracle
from cases import meerkat_like

pytestmark = pytest.mark.gpu

SCALE = 8.0 * np.pi / (180.0 * 60.0 * 60.0)


def _case(seed, nant=40, ntime=20, nchan=32, flagged=0.1):
    uvw, freq = meerkat_like(nant=nant, ntime=ntime, nchan=nchan, seed=seed)
    rng = np.random.default_rng(seed)
    shape = (uvw.shape[0], freq.size)
    # Float weights with few distinct binary exponents, as visibility weights are.
    w = rng.uniform(0.5, 2.0, shape).astype(np.float32)
    w[rng.uniform(size=shape) < flagged] = 0.0
    sel = (rng.uniform(size=uvw.shape[0]) > 0.05).astype(np.uint8)
    from rang import weighting

    return uvw, weighting.wavelengths(freq), w, sel


def _gpu(uvw, wl, w, sel, width, height, pixel_scale, rank_filter=(3.0, 16), with_grid=True, **kw):
    from rang import weighting

    return weighting.ImagingWeights(width, height, pixel_scale, rank_filter=rank_filter, **kw)(
        uvw, wl, w, sel, with_grid=with_grid)


def _compare(got, ref):
    assert np.array_equal(got.weights.view(np.uint32), ref["weights"].view(np.uint32))
    assert np.array_equal(got.grid.view(np.uint64), ref["grid"].view(np.uint64))
    r = ref["sums"]
    assert got.count == int(r[3])
    assert got.max_gridded_weight == r[2]
    assert got.visibility_weight_sum == pytest.approx(r[0], rel=1e-12)
    assert got.total_weight == pytest.approx(r[1], rel=1e-12)


@pytest.mark.parametrize("mode,robust", [("briggs", 0.5), ("briggs", -1.0), ("briggs", 2.0), ("uniform", 0.0),
                                         ("natural", 0.0)])
@pytest.mark.parametrize("rank", [(3.0, 16), None])
def test_imaging_weights_match_the_oracle(mode, robust, rank):
    uvw, wl, w, sel = _case(3)
    kw = dict(mode=mode, robust=robust, width=616, height=616, pixel_scale=SCALE * 4, rank_filter=rank)
    _compare(_gpu(uvw, wl, w, sel, **kw), oracle.imaging_weights(uvw, wl, w, sel, **kw))


def test_super_weight_and_odd_geometry():
    uvw, wl, w, sel = _case(4, ntime=12, nchan=48)
    kw = dict(mode="briggs", robust=0.0, width=1000, height=904, pixel_scale=SCALE * 3, super_weight=2.5,
              rank_filter=(2.0, 7))
    _compare(_gpu(uvw, wl, w, sel, **kw), oracle.imaging_weights(uvw, wl, w, sel, **kw))


def test_reference_known_answers_on_the_gpu():
    # tests/test_core_weights.py:42-82 of the reference, through the GPU
    from rang import weighting

    geom = dict(width=weighting.padded_size(512), height=weighting.padded_size(512), pixel_scale=SCALE)
    uvw = np.array([[100.0, 50.0, 0.0], [-100.0, -50.0, 0.0], [100.0, 50.0, 0.0]])
    wavelength = np.array([0.2, 0.25])
    weights = np.ones((3, 2), np.float32)
    weights[0, 1] = 3.0
    r = _gpu(uvw, wavelength, weights, [True, True, False], mode="briggs", robust=0.5, **geom)
    out = r.weights
    assert np.all(out[2] == 0) and np.array_equal(out[0], out[1])
    assert r.grid.shape == (308, 616) and np.count_nonzero(r.grid) == 2
    avg_w = (2.0**2 + 4.0**2) / 6.0
    f = 5.0 * 10.0**-0.5
    expected = 1.0 / (1.0 + np.array([2.0, 4.0]) * f * f / avg_w)
    np.testing.assert_array_equal(np.sort(out[0]), np.sort(expected.astype(np.float32)))
    assert r.count == 4 and r.visibility_weight_sum == 6.0
    total = float(np.sum((weights * out).astype(np.float64)))
    assert total == pytest.approx(r.total_weight, rel=1e-12)
    uvw2 = np.array([[100.0, 50.0, 0.0], [100.0, 50.0, 0.0]])
    w2 = np.array([[2.0], [3.0]], np.float32)
    assert np.all(_gpu(uvw2, [0.2], w2, [1, 1], mode="uniform", with_grid=False, **geom).weights == np.float32(0.2))
    assert np.all(_gpu(uvw2, [0.2], w2, [1, 1], mode="natural", rank_filter=None, **geom).weights == 1.0)


def test_invalid_arguments_give_status_1():
    with pytest.raises(RuntimeError, match="code 1"):
        _gpu(np.zeros((1, 3)), [1.0], np.ones((1, 1)), [1], width=616, height=616, pixel_scale=-1.0)
    with pytest.raises(ValueError):
        _gpu(np.zeros((1, 3)), [1.0], np.ones((1, 1)), [1], width=616, height=616, pixel_scale=SCALE, mode="robust")


def test_stokes_i_bit_identical():
    from rang import weighting

    rng = np.random.default_rng(8)
    shape = (37, 19, 4)
    data = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    data.ravel()[::97] = np.nan
    weights = rng.uniform(0, 3, shape).astype(np.float32)
    flags = rng.uniform(size=shape) < 0.2
    vis, w = weighting.stokes_i(data, weights, flags)
    ovis, ow = oracle.stokes_i(data, weights, flags)
    assert np.array_equal(vis.view(np.uint32), ovis.view(np.uint32))
    assert np.array_equal(w.view(np.uint32), ow.view(np.uint32))
