"""Exact w-gridder and degridder on the B200: the keyword API of the
reference's `python/rang/core_wgridder.py` over the CUDA extension.

Same functions, arguments, conventions and errors as the reference:
`vis2dirty` (visibilities to a dirty image), `dirty_psf` (dirty image and PSF
in one pass), `dirty2vis` (an image to visibilities), `kernel_row` /
`kernel_table` (the ES-kernel table), `info_dict` and `fits_image` (WSClean
orientation and PSF normalisation). The image is `(nx, ny)` with the first
axis l, pixel `(i, j)` at `l = (i - nx/2) dx`, `m = (j - ny/2) dy`;
`dirty = sum wgt Re[V exp(+2 pi i (u l + v m + w (n-1)))]` and
`V = wgt sum I exp(-2 pi i (...))` (ducc0 with `flip_w=True`).

Status 1 from the extension raises ValueError with the library's message,
any other failure RuntimeError (reference `core_wgridder.py:106-112`).
"""

import numpy as np

from . import core

N_INFO = 14
INFO_NAMES = (
    "kernel_index",
    "supp",
    "nu",
    "nv",
    "nplanes",
    "nvis",
    "wmin_d",
    "wmax_d",
    "nm1min",
    "nm1max",
    "nshift",
    "dw",
    "wmin",
    "ofactor",
)
ARCSEC = np.pi / (180.0 * 3600.0)
VIS_KIND = {np.dtype(np.complex64): 1, np.dtype(np.complex128): 2}
WGT_KIND = {np.dtype(np.float32): 1, np.dtype(np.float64): 2}

_OPTION_DEFAULTS = (
    ("center_x", 0.0),
    ("center_y", 0.0),
    ("sigma_min", 1.1),
    ("sigma_max", 2.6),
)
_FLAG_DEFAULTS = (
    ("do_wgridding", True),
    ("divide_by_n", False),
    ("flip_u", False),
    ("flip_v", False),
    ("flip_w", False),
    ("allow_nshift", True),
)


def extension():
    """The extension module that runs the gridder (`rang._core`)."""
    return core.extension()


def backend():
    """The name of the implementation: the CUDA extension."""
    return "extension"


def library_path():
    return core.library_path()


def options_list(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, kw):
    """The 18 `WgridderOptions` fields as floats in declaration order; `kw`
    is consumed (unknown keys raise TypeError)."""
    kernel = kw.pop("kernel", None)
    head = [int(npix_x), int(npix_y), float(pixsize_x), float(pixsize_y), float(epsilon)]
    reals = [float(kw.pop(k, d)) for k, d in _OPTION_DEFAULTS]
    flags = [int(bool(kw.pop(k, d))) for k, d in _FLAG_DEFAULTS]
    tail = [-1, 0, 0] if kernel is None else [int(kernel[0]), int(kernel[1]), int(kernel[2])]
    if kw:
        raise TypeError(f"unexpected options {sorted(kw)}")
    return [float(v) for v in head + reals + flags + tail]


def _check(status):
    if status == 0:
        return
    if status == 1:
        raise ValueError(extension().wgridder_last_error())
    raise RuntimeError(f"gridder failed with status {status}: {extension().wgridder_last_error()}")


def _coords(uvw, freq):
    uvw = np.ascontiguousarray(uvw, np.float64)
    freq = np.ascontiguousarray(freq, np.float64)
    if uvw.ndim != 2 or uvw.shape[1] != 3 or freq.ndim != 1:
        raise ValueError("uvw must be (nrow, 3) and freq (nchan,)")
    return uvw, freq, (uvw.shape[0], freq.shape[0])


def _weights(wgt, mask, shape):
    if wgt is not None:
        wgt = np.asarray(wgt)
        if wgt.dtype not in WGT_KIND:
            wgt = wgt.astype(np.float64)
        wgt = np.ascontiguousarray(wgt)
        if wgt.shape != shape:
            raise ValueError("wgt must be (nrow, nchan)")
    if mask is not None:
        mask = np.ascontiguousarray(mask, np.uint8)
        if mask.shape != shape:
            raise ValueError("mask must be (nrow, nchan)")
    return wgt, mask


def _vis(vis, shape):
    vis = np.asarray(vis)
    if vis.dtype not in VIS_KIND:
        vis = vis.astype(np.complex128)
    vis = np.ascontiguousarray(vis)
    if vis.shape != shape:
        raise ValueError("visibility arrays must be (nrow, nchan)")
    return vis


def _second_weight(wgt, wgt2, shape):
    """A float32 imaging weight beside a float32 reader weight is multiplied in
    the library; any other pair is multiplied here (the same float32 value
    for float32 inputs)."""
    if wgt2 is None:
        return wgt, None
    wgt2 = np.asarray(wgt2)
    if wgt is None:
        raise ValueError("wgt2 needs wgt")
    if wgt.dtype == np.float32 and wgt2.dtype == np.float32:
        wgt2 = np.ascontiguousarray(wgt2)
        if wgt2.shape != shape:
            raise ValueError("wgt2 must be (nrow, nchan)")
        return wgt, wgt2
    return np.ascontiguousarray(wgt * wgt2), None


def _grid(uvw, freq, vis, wgt, mask, npix, pix, epsilon, single, outputs, kw, wgt2=None):
    uvw, freq, shape = _coords(uvw, freq)
    vis = _vis(vis, shape)
    wgt, mask = _weights(wgt, mask, shape)
    wgt, wgt2 = _second_weight(wgt, wgt2, shape)
    opts = options_list(npix[0], npix[1], pix[0], pix[1], epsilon, dict(kw))
    real = np.float32 if single else np.float64
    images = {name: np.empty((int(npix[0]), int(npix[1])), real) for name in outputs}
    info = np.empty(N_INFO, np.float64)
    fn = getattr(extension(), "wgridder_vis2dirty_f32" if single else "wgridder_vis2dirty_f64")
    _check(fn(opts, uvw, freq, vis, wgt, wgt2, mask, images.get("dirty"), images.get("psf"), info))
    return images, info_dict(info)


def vis2dirty(*, uvw, freq, vis, wgt=None, mask=None, npix_x, npix_y, pixsize_x, pixsize_y, epsilon,
              return_info=False, **kw):
    """The dirty image `(npix_x, npix_y)` of `vis` `(nrow, nchan)`; single
    precision for complex64 data, else double. Keywords as ducc0's
    (`do_wgridding`, `divide_by_n`, `flip_u/v/w`, `center_x/y`,
    `allow_nshift`, `sigma_min/max`) plus `kernel=(row, nu, nv)`."""
    single = np.asarray(vis).dtype == np.complex64
    images, info = _grid(uvw, freq, vis, wgt, mask, (npix_x, npix_y), (pixsize_x, pixsize_y), epsilon, single,
                         ("dirty",), kw)
    return (images["dirty"], info) if return_info else images["dirty"]


def dirty_psf(*, uvw, freq, vis, wgt=None, mask=None, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, single=False,
              return_info=False, wgt2=None, **kw):
    """Dirty image and PSF (unit visibilities, same weights and mask) with one
    plan, that of the visibilities with `wgt * mask != 0`."""
    images, info = _grid(uvw, freq, vis, wgt, mask, (npix_x, npix_y), (pixsize_x, pixsize_y), epsilon, single,
                         ("dirty", "psf"), kw, wgt2=wgt2)
    if return_info:
        return images["dirty"], images["psf"], info
    return images["dirty"], images["psf"]


def dirty2vis(*, uvw, freq, dirty, wgt=None, mask=None, pixsize_x, pixsize_y, epsilon, return_info=False, **kw):
    """Visibilities `(nrow, nchan)` of the image `dirty` `(nx, ny)`, single
    precision for a float32 image, else double."""
    dirty = np.asarray(dirty)
    single = dirty.dtype == np.float32
    real = np.float32 if single else np.float64
    dirty = np.ascontiguousarray(dirty, real)
    uvw, freq, shape = _coords(uvw, freq)
    wgt, mask = _weights(wgt, mask, shape)
    opts = options_list(dirty.shape[0], dirty.shape[1], pixsize_x, pixsize_y, epsilon, dict(kw))
    vis = np.empty(shape, np.complex64 if single else np.complex128)
    info = np.empty(N_INFO, np.float64)
    fn = getattr(extension(), "wgridder_dirty2vis_f32" if single else "wgridder_dirty2vis_f64")
    _check(fn(opts, uvw, freq, dirty, wgt, mask, vis.view(real), info))
    return (vis, info_dict(info)) if return_info else vis


def info_dict(info):
    rec = dict(zip(INFO_NAMES, (float(v) for v in info), strict=True))
    for key in ("kernel_index", "supp", "nu", "nv", "nplanes", "nvis"):
        rec[key] = int(rec[key])
    return rec


def kernel_row(index):
    """Row `index` of the kernel table: (W, ofactor, epsilon, beta, e0, ndim,
    singleprec), or None past its end."""
    out = np.empty(7, np.float64)
    if extension().wgridder_kernel_row(int(index), out):
        return None
    return (int(out[0]), *(float(v) for v in out[1:5]), int(out[5]), bool(out[6]))


def kernel_table():
    rows = []
    while (row := kernel_row(len(rows))) is not None:
        rows.append(row)
    return rows


def fits_image(uvw, freq, data, weights, width, height, scale_arcsec, epsilon=1e-6, single=False,
               imaging_weights=None, **kw):
    """Dirty image and PSF as `(height, width)` arrays in WSClean's FITS pixel
    order (v and w flipped, transposed), both divided by the PSF centre."""
    dirty, psf, info = dirty_psf(uvw=uvw, freq=freq, vis=data, wgt=weights, wgt2=imaging_weights, **kw,
                                 npix_x=width, npix_y=height, pixsize_x=scale_arcsec * ARCSEC,
                                 pixsize_y=scale_arcsec * ARCSEC, epsilon=epsilon, single=single,
                                 return_info=True, flip_v=True, flip_w=True)
    norm = psf[width // 2, height // 2]
    return {
        "dirty": (dirty.T / norm).astype(np.float64),
        "psf": (psf.T / norm).astype(np.float64),
        "info": info,
        "info_psf": info,
        "psf_centre_raw": float(norm),
    }


def binning(*, uvw, freq, vis=None, wgt=None, mask=None, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, single,
            with_vis, wgt2=None, **kw):
    """The GPU's visibility binning, for parity tests: per visibility iu0,
    iv0 and bin key (tile * max(nplanes, 1) + first plane), the sorted
    order and the plan."""
    uvw, freq, shape = _coords(uvw, freq)
    if vis is not None:
        vis = _vis(vis, shape)
    wgt, mask = _weights(wgt, mask, shape)
    if wgt2 is not None:
        wgt = np.ascontiguousarray(wgt, np.float32)
        wgt2 = np.ascontiguousarray(wgt2, np.float32)
    opts = options_list(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, dict(kw))
    st, iu0, iv0, key, srt, ns, info = extension().wgridder_binning(opts, uvw, freq, vis, wgt, wgt2, mask,
                                                                    int(bool(with_vis)), int(bool(single)))
    _check(st)
    return {"iu0": iu0, "iv0": iv0, "key": key, "sorted": srt[:ns].copy(), "info": info_dict(info)}
