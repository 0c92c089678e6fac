"""Pins of the CPU oracle's imaging-weight restatement (oracle/weights_oracle.cpp)
against the reference's own known answers for `core/src/weights.rs`
(its unit tests, weights.rs:598-700, and tests/test_core_weights.py)."""

import numpy as np
import pytest

import oracle

SCALE = 8.0 * np.pi / (180.0 * 60.0 * 60.0)


def _cell_uv(x, y, width, height, scale):
    """(u, v) in wavelengths of the centre of weight-grid cell (x, y)."""
    return (x - width // 2 + 0.5) / (width * scale), (y + 0.5) / (height * scale)


def test_padded_size_and_grid_shape():
    # weights.rs:588-611, tests/test_core_weights.py:9-13
    assert oracle.padded_size(512) == 616
    assert oracle.padded_size(1024) == 1232
    for trimmed in range(2, 4097, 2):
        expected = int(np.ceil(trimmed * 1.2))
        expected += (4 - expected % 4) % 4
        assert oracle.padded_size(trimmed) == expected
    assert oracle.weight_grid_shape(616, 616) == (616, 616)
    assert oracle.weight_grid_shape(616, 616, 3.0) == (206, 206)
    assert oracle.weight_grid_shape(610, 610, 4.0) == (154, 154)  # 152.5 rounds up
    assert oracle.weight_grid_shape(614, 614, 4.0) == (154, 154)


def test_briggs_uniform_natural_match_the_formulas():
    # weights.rs:612-637: two samples (2 + 3) in one cell and one off the grid
    u, v = 120.5, 33.25
    uvw = np.array([[u, v, 0.0], [u, v, 0.0], [u + 1e6, v, 0.0]])
    wl = np.array([1.0])
    w = np.array([[2.0], [3.0], [1.0]], np.float32)
    r = oracle.imaging_weights(uvw, wl, w, [1, 1, 1], mode="briggs", robust=0.5, pixel_scale=SCALE,
                               rank_filter=None)
    avg_w = 25.0 / 5.0
    f = 5.0 * np.exp(-np.log(10.0) * 0.5)
    expected = 1.0 / (1.0 + 5.0 * (f * f / avg_w))
    assert r["weights"][0, 0] == np.float32(expected) and r["weights"][1, 0] == np.float32(expected)
    assert r["weights"][2, 0] == 0.0
    conj = oracle.imaging_weights(-uvw, wl, w, [1, 1, 1], mode="briggs", robust=0.5, pixel_scale=SCALE,
                                  rank_filter=None)
    assert conj["weights"][0, 0] == np.float32(expected)
    assert oracle.imaging_weights(uvw, wl, w, [1, 1, 1], mode="uniform", pixel_scale=SCALE,
                                  rank_filter=None)["weights"][0, 0] == np.float32(0.2)
    nat = oracle.imaging_weights(uvw, wl, w, [1, 1, 1], mode="natural", pixel_scale=SCALE, rank_filter=None)
    assert nat["weights"][0, 0] == 1.0 and np.count_nonzero(nat["grid"]) == 1


def test_reference_python_cases():
    # tests/test_core_weights.py:42-82
    uvw = np.array([[100.0, 50.0, 0.0], [-100.0, -50.0, 0.0], [100.0, 50.0, 0.0]])
    wavelength = np.array([0.2, 0.25])
    weights = np.ones((3, 2), np.float32)
    weights[0, 1] = 3.0
    r = oracle.imaging_weights(uvw, wavelength, weights, [1, 1, 0], mode="briggs", robust=0.5)
    out = r["weights"]
    assert np.all(out[2] == 0) and np.array_equal(out[0], out[1])
    assert r["grid"].shape == (308, 616) and np.count_nonzero(r["grid"]) == 2
    avg_w = (2.0**2 + 4.0**2) / 6.0
    f = 5.0 * 10.0**-0.5
    expected = 1.0 / (1.0 + np.array([2.0, 4.0]) * f * f / avg_w)
    np.testing.assert_array_equal(np.sort(out[0]), np.sort(expected.astype(np.float32)))
    assert r["sums"][3] == 4 and r["sums"][0] == 6.0
    uvw2 = np.array([[100.0, 50.0, 0.0], [100.0, 50.0, 0.0]])
    w2 = np.array([[2.0], [3.0]], np.float32)
    assert np.all(oracle.imaging_weights(uvw2, [0.2], w2, [1, 1], mode="uniform")["weights"] == np.float32(0.2))
    assert np.all(oracle.imaging_weights(uvw2, [0.2], w2, [1, 1], mode="natural", rank_filter=None)["weights"] == 1.0)


def test_rank_filter_clips_to_window_mean():
    # weights.rs:639-652, the cells set through uniform weighting (1 / sum)
    width = height = 32
    cells = [((5, 5), 0.01), ((6, 5), 1.0), ((5, 6), 1.0), ((4, 5), 1.0), ((5, 4), 1.0), ((9, 9), 1.0)]
    uvw = np.array([[*_cell_uv(x, y, width, height, SCALE), 0.0] for (x, y), _ in cells])
    w = np.array([[s] for _, s in cells], np.float32)
    r = oracle.imaging_weights(uvw, [1.0], w, [1] * len(cells), mode="uniform", width=width, height=height,
                               pixel_scale=SCALE, rank_filter=(3.0, 16))
    g = r["grid"]
    cell = float(np.float32(0.01))
    mean = (1.0 / cell + 5.0) / 6.0
    assert g[5, 5] == mean * 3.0
    assert g[5, 6] == 1.0 and g[9, 9] == 1.0


def test_stokes_i_rules():
    # weights.rs:654-678
    nan = np.nan
    data = np.array([
        1.0, 2.0, 9.0, 9.0, 9.0, 9.0, 3.0, -2.0,
        1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0,
        nan, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0,
        2.0, 0.0, 0.0, 0.0, 0.0, 0.0, 4.0, 0.0], np.float32).view(np.complex64).reshape(4, 4)
    weights = np.array([2, 7, 7, 3, 1, 1, 1, 1, 1, 1, 1, 1, 5, 1, 1, 0.5], np.float32).reshape(4, 4)
    flags = np.zeros((4, 4), bool)
    flags[1, 3] = True
    vis, w = oracle.stokes_i(data, weights, flags)
    assert vis[0] == 2.0 and vis[1] == 1.0 and vis[2] == 0.0 and vis[3] == 3.0
    np.testing.assert_array_equal(w, np.array([8.0, 0.0, 0.0, 2.0], np.float32))


def test_weight_sums_follow_apply_weights():
    # weights.rs:680-689: the sums of one selected row of four channels
    uvw = np.array([[100.0, 50.0, 0.0]])
    wl = np.array([0.2, 0.21, 0.22, 0.23])
    w = np.array([[1.0, 2.0, 3.0, 4.0]], np.float32)
    r = oracle.imaging_weights(uvw, wl, w, [1], mode="natural", rank_filter=None)
    img = r["weights"].ravel()
    cum = w.ravel() * img
    assert r["sums"][3] == np.count_nonzero(cum)
    assert r["sums"][0] == float(w.ravel()[cum != 0].astype(np.float64).sum())
    assert r["sums"][2] == float(cum.max())


def test_rejects_bad_arguments():
    with pytest.raises(ValueError):
        oracle.imaging_weights(np.zeros((1, 3)), [1.0], np.ones((1, 1), np.float32), [1], super_weight=0.0)
