"""Imaging weights and Stokes I on the GPU (rang.core_weights over the C ABI
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
    from rang import core_weights

    return uvw, core_weights.wsclean_wavelengths(freq), w, sel


def _compare(got, ref):
    assert np.array_equal(got["weights"].view(np.uint32), ref["weights"].view(np.uint32))
    assert np.array_equal(got["grid"].view(np.uint64), ref["grid"].view(np.uint64))
    s = got["sums"]
    r = ref["sums"]
    assert s["count"] == int(r[3])
    assert s["max_gridded_weight"] == r[2]
    assert s["visibility_weight_sum"] == pytest.approx(r[0], rel=1e-12)
    assert s["total_weight"] == pytest.approx(r[1], rel=1e-12)


@pytest.mark.parametrize("mode,robust", [("briggs", 0.5), ("briggs", -1.0), ("briggs", 2.0), ("uniform", 0.0),
                                         ("natural", 0.0)])
@pytest.mark.parametrize("rank", [(3.0, 16), None])
def test_imaging_weights_match_the_oracle(mode, robust, rank):
    from rang import core_weights

    uvw, wl, w, sel = _case(3)
    kw = dict(mode=mode, robust=robust, width=616, height=616, pixel_scale=SCALE * 4, rank_filter=rank)
    _compare(core_weights.imaging_weights(uvw, wl, w, sel, **kw), oracle.imaging_weights(uvw, wl, w, sel, **kw))


def test_super_weight_and_odd_geometry():
    from rang import core_weights

    uvw, wl, w, sel = _case(4, ntime=12, nchan=48)
    kw = dict(mode="briggs", robust=0.0, width=1000, height=904, pixel_scale=SCALE * 3, super_weight=2.5,
              rank_filter=(2.0, 7))
    _compare(core_weights.imaging_weights(uvw, wl, w, sel, **kw), oracle.imaging_weights(uvw, wl, w, sel, **kw))


def test_reference_known_answers_on_the_gpu():
    # tests/test_core_weights.py:42-82 of the reference, through the GPU
    from rang import core_weights

    uvw = np.array([[100.0, 50.0, 0.0], [-100.0, -50.0, 0.0], [100.0, 50.0, 0.0]])
    wavelength = np.array([0.2, 0.25])
    weights = np.ones((3, 2), np.float32)
    weights[0, 1] = 3.0
    r = core_weights.imaging_weights(uvw, wavelength, weights, [True, True, False], mode="briggs", robust=0.5)
    out = r["weights"]
    assert np.all(out[2] == 0) and np.array_equal(out[0], out[1])
    assert r["grid"].shape == (308, 616) and np.count_nonzero(r["grid"]) == 2
    avg_w = (2.0**2 + 4.0**2) / 6.0
    f = 5.0 * 10.0**-0.5
    expected = 1.0 / (1.0 + np.array([2.0, 4.0]) * f * f / avg_w)
    np.testing.assert_array_equal(np.sort(out[0]), np.sort(expected.astype(np.float32)))
    assert r["sums"]["count"] == 4 and r["sums"]["visibility_weight_sum"] == 6.0
    numpy_sums = core_weights.weight_sums(weights, out)
    assert numpy_sums["total_weight"] == pytest.approx(r["sums"]["total_weight"], rel=1e-12)
    uvw2 = np.array([[100.0, 50.0, 0.0], [100.0, 50.0, 0.0]])
    w2 = np.array([[2.0], [3.0]], np.float32)
    assert np.all(core_weights.imaging_weights(uvw2, [0.2], w2, [1, 1], mode="uniform",
                                               return_grid=False)["weights"] == np.float32(0.2))
    assert np.all(core_weights.imaging_weights(uvw2, [0.2], w2, [1, 1], mode="natural",
                                               rank_filter=None)["weights"] == 1.0)


def test_invalid_arguments_give_status_1():
    from rang import core_weights

    with pytest.raises(RuntimeError, match="code 1"):
        core_weights.imaging_weights(np.zeros((1, 3)), [1.0], np.ones((1, 1)), [1], pixel_scale=-1.0)
    with pytest.raises(ValueError):
        core_weights.imaging_weights(np.zeros((1, 3)), [1.0], np.ones((1, 1)), [1], mode="robust")


def test_stokes_i_bit_identical():
    from rang import core_weights

    rng = np.random.default_rng(8)
    shape = (37, 19, 4)
    data = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    data.ravel()[::97] = np.nan
    weights = rng.uniform(0, 3, shape).astype(np.float32)
    flags = rng.uniform(size=shape) < 0.2
    vis, w = core_weights.stokes_i(data, weights, flags)
    ovis, ow = oracle.stokes_i(data, weights, flags)
    assert np.array_equal(vis.view(np.uint32), ovis.view(np.uint32))
    assert np.array_equal(w.view(np.uint32), ow.view(np.uint32))
