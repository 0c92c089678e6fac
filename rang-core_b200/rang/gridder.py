"""Host-array calls of the B200 w-gridder through `rang._core`.

`rang._core` carries the reference's Python-level gridder functions
(`wgridder_vis2dirty_f64(opts, uvw, freq, vis, wgt, wgt2, mask, dirty, psf,
info)` and the rest, `core/py/src/lib.rs:1053-1446`), so the reference's own
`python/rang/core_wgridder.py` runs on it unchanged. This module is this
library's own small layer over the same functions, used by its tests, its
benchmark and its device-side modules: arrays are checked and given the
dtypes the extension reads in place, the 18 options are packed in the field
order of `WgridderOptions` (`include/rang_wgridder.h`), and a non-zero status
becomes an exception (ValueError for invalid arguments, status 1;
RuntimeError otherwise) carrying the library's message.

Keywords name the options as the C struct does (`do_wgridding`,
`divide_by_n`, `flip_u`, `flip_v`, `flip_w`, `center_x`, `center_y`,
`allow_nshift`, `sigma_min`, `sigma_max`), plus `kernel=(index, nu, nv)` to
force a kernel row and grid. The image is `(npix_x, npix_y)`, first axis l.
"""

from dataclasses import dataclass, fields

import numpy as np

from .core import extension

# The 14 doubles of a call's plan report, in the order of `info`.
INFO_NAMES = ("kernel_index", "supp", "nu", "nv", "nplanes", "nvis", "wmin_d", "wmax_d", "nm1min", "nm1max",
              "nshift", "dw", "wmin", "ofactor")
_INT_INFO = frozenset(INFO_NAMES[:6])

# Data kind codes of the `_ex` entry points.
_VIS_DTYPES = (np.dtype(np.complex64), np.dtype(np.complex128))
_WGT_DTYPES = (np.dtype(np.float32), np.dtype(np.float64))


@dataclass
class Options:
    """`WgridderOptions` field for field; `packed()` is the extension's list."""

    nx: int
    ny: int
    pixsize_x: float
    pixsize_y: float
    epsilon: float
    center_x: float = 0.0
    center_y: float = 0.0
    sigma_min: float = 1.1
    sigma_max: float = 2.6
    do_wgridding: bool = True
    divide_by_n: bool = False
    flip_u: bool = False
    flip_v: bool = False
    flip_w: bool = False
    allow_nshift: bool = True
    kernel_index: int = -1
    nu: int = 0
    nv: int = 0

    @classmethod
    def make(cls, nx, ny, pixsize_x, pixsize_y, epsilon, extra):
        """Options from the image geometry and keyword options; `extra` is
        consumed and an unknown keyword raises TypeError."""
        kw = dict(extra)
        forced = kw.pop("kernel", None)
        names = {f.name for f in fields(cls)} - {"nx", "ny", "pixsize_x", "pixsize_y", "epsilon", "kernel_index",
                                                  "nu", "nv"}
        unknown = sorted(set(kw) - names)
        if unknown:
            raise TypeError(f"unexpected options {unknown}")
        opts = cls(int(nx), int(ny), float(pixsize_x), float(pixsize_y), float(epsilon), **kw)
        if forced is not None:
            opts.kernel_index, opts.nu, opts.nv = (int(v) for v in forced)
        return opts

    def packed(self):
        return [float(getattr(self, f.name)) for f in fields(self)]


def options_list(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, kw):
    """The 18 options as the extension takes them (see `Options`)."""
    return Options.make(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, kw).packed()


def info_dict(info):
    """The plan report as a dict, counts as ints."""
    return {k: (int(v) if k in _INT_INFO else float(v)) for k, v in zip(INFO_NAMES, info, strict=True)}


def _raise_on(status):
    if status == 0:
        return
    message = extension().wgridder_last_error()
    if status == 1:
        raise ValueError(message)
    raise RuntimeError(f"gridder status {status}: {message}")


class _Call:
    """One call's host arrays: uvw (nrow, 3) and freq (nchan,) as float64,
    the per-visibility arrays checked against (nrow, nchan)."""

    def __init__(self, uvw, freq):
        self.uvw = np.ascontiguousarray(uvw, dtype=np.float64)
        self.freq = np.ascontiguousarray(freq, dtype=np.float64)
        if self.uvw.ndim != 2 or self.uvw.shape[1] != 3 or self.freq.ndim != 1:
            raise ValueError("uvw must be (nrow, 3) and freq (nchan,)")
        self.shape = (self.uvw.shape[0], self.freq.shape[0])

    def _sized(self, a, what):
        if a.shape != self.shape:
            raise ValueError(f"{what} must be (nrow, nchan) = {self.shape}, not {a.shape}")
        return a

    def vis(self, vis):
        if vis is None:
            return None
        a = np.asarray(vis)
        return self._sized(np.ascontiguousarray(a if a.dtype in _VIS_DTYPES else a.astype(np.complex128)), "vis")

    def weights(self, wgt, wgt2=None):
        """(wgt, wgt2): two float32 arrays go to the library, which multiplies
        them per visibility; any other pair is multiplied here in NumPy."""
        if wgt is None:
            if wgt2 is not None:
                raise ValueError("wgt2 needs wgt")
            return None, None
        a = np.asarray(wgt)
        if wgt2 is not None:
            b = np.asarray(wgt2)
            if a.dtype == np.float32 and b.dtype == np.float32:
                return (self._sized(np.ascontiguousarray(a), "wgt"), self._sized(np.ascontiguousarray(b), "wgt2"))
            a = a * b
        a = np.ascontiguousarray(a if a.dtype in _WGT_DTYPES else a.astype(np.float64))
        return self._sized(a, "wgt"), None

    def mask(self, mask):
        return None if mask is None else self._sized(np.ascontiguousarray(mask, dtype=np.uint8), "mask")


def _grid_images(call, vis, wgt, wgt2, mask, opts, single, want_psf):
    real = np.float32 if single else np.float64
    dirty = np.empty((opts.nx, opts.ny), real)
    psf = np.empty((opts.nx, opts.ny), real) if want_psf else None
    info = np.empty(len(INFO_NAMES), np.float64)
    fn = extension().wgridder_vis2dirty_f32 if single else extension().wgridder_vis2dirty_f64
    _raise_on(fn(opts.packed(), call.uvw, call.freq, vis, wgt, wgt2, mask, dirty, psf, info))
    return dirty, psf, info_dict(info)


def vis2dirty(*, uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, wgt=None, mask=None,
              return_info=False, **kw):
    """Dirty image (npix_x, npix_y) of `vis` (nrow, nchan): single precision
    for complex64 data, double otherwise."""
    call = _Call(uvw, freq)
    v = call.vis(vis)
    w, _ = call.weights(wgt)
    opts = Options.make(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, kw)
    dirty, _, info = _grid_images(call, v, w, None, call.mask(mask), opts, v.dtype == np.complex64, False)
    return (dirty, info) if return_info else dirty


def dirty_psf(*, uvw, freq, vis, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, wgt=None, wgt2=None, mask=None,
              single=False, return_info=False, **kw):
    """Dirty image and PSF in one pass (one plan, that of the visibilities
    with weight times mask non-zero)."""
    call = _Call(uvw, freq)
    w, w2 = call.weights(wgt, wgt2)
    opts = Options.make(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, kw)
    dirty, psf, info = _grid_images(call, call.vis(vis), w, w2, call.mask(mask), opts, bool(single), True)
    return (dirty, psf, info) if return_info else (dirty, psf)


def dirty2vis(*, uvw, freq, dirty, pixsize_x, pixsize_y, epsilon, wgt=None, mask=None, return_info=False, **kw):
    """Visibilities (nrow, nchan) of the image `dirty`: single precision for a
    float32 image, double otherwise."""
    call = _Call(uvw, freq)
    img = np.asarray(dirty)
    single = img.dtype == np.float32
    real = np.float32 if single else np.float64
    img = np.ascontiguousarray(img, dtype=real)
    w, _ = call.weights(wgt)
    opts = Options.make(img.shape[0], img.shape[1], pixsize_x, pixsize_y, epsilon, kw)
    out = np.empty(call.shape, np.complex64 if single else np.complex128)
    info = np.empty(len(INFO_NAMES), np.float64)
    fn = extension().wgridder_dirty2vis_f32 if single else extension().wgridder_dirty2vis_f64
    _raise_on(fn(opts.packed(), call.uvw, call.freq, img, w, call.mask(mask), out.view(real), info))
    return (out, info_dict(info)) if return_info else out


def binning(*, uvw, freq, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, single, with_vis, vis=None, wgt=None,
            wgt2=None, mask=None, **kw):
    """The device binning of one call, for parity tests: per visibility iu0,
    iv0 and the key tile * max(nplanes, 1) + first plane, the active
    visibilities in the reference's (tile, first plane, row, channel) order,
    and the plan report."""
    call = _Call(uvw, freq)
    v = call.vis(vis)
    if wgt2 is not None:
        w, w2 = (np.ascontiguousarray(a, dtype=np.float32) for a in (wgt, wgt2))
    else:
        w, w2 = call.weights(wgt)
    opts = Options.make(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, kw)
    st, iu0, iv0, key, srt, ns, info = extension().wgridder_binning(
        opts.packed(), call.uvw, call.freq, v, w, w2, call.mask(mask), int(bool(with_vis)), int(bool(single)))
    _raise_on(st)
    return {"iu0": iu0, "iv0": iv0, "key": key, "sorted": srt[:ns].copy(), "info": info_dict(info)}


def kernel_row(index):
    """Kernel table row `index` as (support, oversampling, epsilon, beta, e0,
    ndim, single precision), or None past the end of the table."""
    out = np.empty(7, np.float64)
    if extension().wgridder_kernel_row(int(index), out):
        return None
    return (int(out[0]), float(out[1]), float(out[2]), float(out[3]), float(out[4]), int(out[5]), bool(out[6]))


def kernel_table():
    """Every row of the kernel table."""
    table = []
    row = kernel_row(0)
    while row is not None:
        table.append(row)
        row = kernel_row(len(table))
    return table


def plan(*, uvw, freq, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, vis=None, wgt=None, wgt2=None, mask=None,
         single=False, **kw):
    """The kernel and grid a call would choose, without binning or gridding
    (the reference's `plan`, core/src/wgridder.rs:3527-3551): the plan
    report of `vis2dirty` on these arrays (the activity |vis|^2 wgt mask != 0
    with `vis`, else wgt mask != 0)."""
    info, _ = _plan_only(uvw, freq, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, vis, wgt, wgt2, mask, single, 1,
                         kw)
    return info


def gridding_footprint(*, uvw, freq, wgt, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, nout=1, single=False,
                       **kw):
    """The plan a gridding pass would choose on the weights `wgt` (a
    visibility is active where its weight is non-zero) and the device bytes
    of its work space for `nout` images, without gridding (the reference's
    `gridding_footprint`, core/src/wgridder.rs:3553-3588). Returns
    (plan report, bytes)."""
    return _plan_only(uvw, freq, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, None, wgt, None, None, single, nout,
                      kw)


def _plan_only(uvw, freq, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, vis, wgt, wgt2, mask, single, nout, kw):
    call = _Call(uvw, freq)
    v = call.vis(vis)
    if wgt2 is not None:
        w, w2 = (call._sized(np.ascontiguousarray(a, dtype=np.float32), n) for a, n in ((wgt, "wgt"), (wgt2, "wgt2")))
    else:
        w, w2 = call.weights(wgt)
    opts = Options.make(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, kw)
    st, info, footprint = extension().wgridder_plan_only(opts.packed(), call.uvw, call.freq, v, w, w2, call.mask(mask),
                                                         int(bool(single)), int(nout))
    _raise_on(st)
    return info_dict(info), int(footprint)
