"""Imaging weights and Stokes I of the B200 library, on host arrays.

The CUDA kernels sit behind the reference's weights C ABI
(`include/rang_weights.h`, `core/src/ffi_weights.rs`) and its Python-level
functions in `rang._core` (`stokes_i`, `imaging_weights`, `padded_size`,
`weight_grid_shape`), so the reference's own `python/rang/core_weights.py`
runs on it unchanged. This module is this library's own layer: an
`ImagingWeights` object fixes one image geometry and weighting, and calling
it on a set of samples returns a `WeightsResult`.
"""

from dataclasses import dataclass

import numpy as np

from .core import extension

_MODE = {"natural": 0, "uniform": 1, "briggs": 2}


def wavelengths(freq_hz):
    """Channel wavelengths (metres) as WSClean computes them: the speed of
    light over the frequency in extended precision, rounded to float64."""
    return (np.longdouble(299792458) / np.asarray(freq_hz, dtype=np.longdouble)).astype(np.float64)


def padded_size(trimmed, padding=1.2):
    """The padded image size WSClean uses for a trimmed size."""
    return int(extension().padded_size(int(trimmed), float(padding)))


def _fail(what, code):
    raise RuntimeError(f"{what} failed with code {code}: {extension().wgridder_last_error()}")


def stokes_i(data, weights, flags):
    """Stokes I of cells of four linear correlations (XX, XY, YX, YY last):
    complex64 visibilities and float32 weights of shape data.shape[:-1]."""
    d = np.ascontiguousarray(data, dtype=np.complex64)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    f = np.ascontiguousarray(flags, dtype=np.uint8)
    if d.shape[-1:] != (4,) or w.shape != d.shape or f.shape != d.shape:
        raise ValueError("data, weights and flags must share one shape ending in 4 correlations")
    cells = d.shape[:-1]
    vis = np.zeros(cells, dtype=np.complex64)
    weight = np.zeros(cells, dtype=np.float32)
    code = extension().stokes_i(int(np.prod(cells, dtype=np.int64)), d.view(np.float32), w, f, vis.view(np.float32),
                                weight)
    if code:
        _fail("Stokes I", code)
    return vis, weight


@dataclass
class WeightsResult:
    """Imaging weights (nrow, nchan) float32, WSClean's header sums, and the
    finished half-plane weight grid (rows, columns) float64 when asked for."""

    weights: np.ndarray
    visibility_weight_sum: float
    total_weight: float
    max_gridded_weight: float
    count: int
    grid: np.ndarray | None = None


@dataclass
class ImagingWeights:
    """WSClean imaging weights for one padded image (width x height pixels of
    `pixel_scale` radians): `mode` natural, uniform or briggs (`robust`),
    `super_weight`, and the rank filter (level, cells) or None."""

    width: int
    height: int
    pixel_scale: float
    mode: str = "briggs"
    robust: float = 0.5
    super_weight: float = 1.0
    rank_filter: tuple | None = (3.0, 16)

    def grid_shape(self):
        """The weight grid's (width, height) after the super weight."""
        st, w, h = extension().weight_grid_shape(int(self.width), int(self.height), float(self.super_weight))
        if st:
            raise ValueError("the super weight must be positive")
        return int(w), int(h)

    def __call__(self, uvw, wavelength, weights, row_selected, with_grid=False):
        """The weights of samples with `uvw` (nrow, 3) metres, `wavelength`
        (nchan,) metres, visibility weights (nrow, nchan) (zero where
        flagged) and rows selected by `row_selected` (nrow,)."""
        if self.mode not in _MODE:
            raise ValueError(f"mode {self.mode!r} is not one of {sorted(_MODE)}")
        w = np.ascontiguousarray(weights, dtype=np.float32)
        if w.ndim != 2:
            raise ValueError("weights must be (nrow, nchan)")
        nrow, nchan = w.shape
        u = np.ascontiguousarray(uvw, dtype=np.float64)
        lam = np.ascontiguousarray(wavelength, dtype=np.float64)
        sel = np.ascontiguousarray(row_selected, dtype=np.uint8)
        if u.shape != (nrow, 3) or lam.shape != (nchan,) or sel.shape != (nrow,):
            raise ValueError("uvw must be (nrow, 3), wavelength (nchan,) and row_selected (nrow,)")
        level, cells = self.rank_filter if self.rank_filter is not None else (0.0, 0)
        out = np.zeros((nrow, nchan), dtype=np.float32)
        sums = np.zeros(4, dtype=np.float64)
        grid = None
        if with_grid:
            gw, gh = self.grid_shape()
            grid = np.zeros((gh // 2, gw), dtype=np.float64)
        code = extension().imaging_weights(nrow, nchan, u, lam, w, sel, _MODE[self.mode], float(self.robust),
                                           int(self.width), int(self.height), float(self.pixel_scale),
                                           float(self.pixel_scale), float(self.super_weight), float(level), int(cells),
                                           out, grid, sums)
        if code:
            _fail("imaging weights", code)
        return WeightsResult(out, float(sums[0]), float(sums[1]), float(sums[2]), int(sums[3]), grid)
