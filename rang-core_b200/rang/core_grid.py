"""The imaging driver over the B200 exact gridder: the reference's
`python/rang/core_grid.py` `invert(..., gridder="wgrid")` path, its WSClean
counters, WCS header and FITS output.

`invert` forms the dirty image and PSF with one double-precision pass of the
GPU gridder (`core_wgridder.fits_image`, the visibility weight and the
imaging weight multiplied in the gridder), in WSClean's FITS pixel order and
normalised by the PSF centre, with WSClean's counters of the gridded samples
(core_grid.py:324-407 of the reference). The reference's default gridder,
"wstack" (its WSClean w-stacking reproducer), is not part of this library.
"""

import math

import numpy as np

ARCSEC = math.pi / (180.0 * 3600.0)
GRIDDERS = ("wstack", "wgrid")
WGRID_EPSILON = 1e-6


def invert(uvw, frequencies, data, weights, imaging_weights, width=512, height=512, scale_arcsec=8.0, w_layers=64,
           kernel_size=7, oversampling=1023, padding=1.2, gridder="wstack", epsilon=WGRID_EPSILON, device=None,
           precision=None):
    """Dirty image and PSF, `(height, width)` in FITS pixel order, with
    WSClean's counters (the reference's `invert`). Only `gridder="wgrid"`
    exists here; it runs on the GPU, and `w_layers`, `kernel_size`,
    `oversampling`, `padding` and `precision` do not apply to it."""
    if gridder not in GRIDDERS:
        raise ValueError(f"gridder must be one of {GRIDDERS}, not {gridder!r}")
    if gridder != "wgrid":
        raise ValueError("this library has the exact gridder only: pass gridder='wgrid'")
    if device not in (None, "gpu"):
        raise RuntimeError("the exact gridder runs on the GPU here; there is no CPU path")
    return _invert_wgrid(uvw, frequencies, data, weights, imaging_weights, width, height, scale_arcsec, epsilon)


def _weight_counters(weights, imaging_weights, block=4096):
    """WSClean's counters of the gridded samples (`w * iw != 0`, the product
    in float32 as the gridder forms it), in row blocks: image weight, count,
    visibility weight sum and the largest gridded weight."""
    total = vsum = 0.0
    count = 0
    largest = 0.0
    for start in range(0, len(weights), block):
        w = weights[start:start + block]
        cum = w * imaging_weights[start:start + block]
        live = cum != 0
        total += float(cum.sum(dtype=np.float64))
        vsum += float(w[live].sum(dtype=np.float64))
        count += int(np.count_nonzero(live))
        if cum.size:
            largest = max(largest, float(cum.max()))
    return total, count, vsum, largest


def _invert_wgrid(uvw, frequencies, data, weights, imaging_weights, width, height, scale_arcsec, epsilon):
    from . import core_wgridder

    data = np.asarray(data)
    if data.dtype not in (np.complex64, np.complex128):
        data = data.astype(np.complex64)
    data = np.ascontiguousarray(data)
    weights = np.ascontiguousarray(weights, np.float32)
    imaging_weights = np.ascontiguousarray(imaging_weights, np.float32)
    nrow, nchan = data.shape
    if np.shape(uvw) != (nrow, 3) or np.shape(frequencies) != (nchan,):
        raise ValueError("uvw must be (nrow, 3) and frequencies (nchan,)")
    if weights.shape != (nrow, nchan) or imaging_weights.shape != (nrow, nchan):
        raise ValueError("weights must match data")
    image_weight, count, vsum, largest = _weight_counters(weights, imaging_weights)
    if image_weight == 0.0:
        raise RuntimeError("core gridder failed: no visibility carries weight")
    out = core_wgridder.fits_image(uvw, frequencies, data, weights, width, height, scale_arcsec, epsilon=epsilon,
                                   imaging_weights=imaging_weights)
    info = out["info"]
    centre = out["psf_centre_raw"]
    stats = {
        "image_weight": image_weight,
        "gridded_count": count,
        "visibility_weight_sum": vsum,
        "max_gridded_weight": largest,
        "min_w": info["wmin_d"],
        "max_w": info["wmax_d"],
        "psf_normalization": image_weight / centre if centre else 0.0,
        "n_w_layers": info["nplanes"],
    }
    return {"dirty": out["dirty"], "psf": out["psf"], "stats": stats, "gridder": "wgrid",
            "wgridder": {"epsilon": float(epsilon), "backend": core_wgridder.backend(),
                         "psf_centre_raw": float(centre), **info}}


def wcs_header(phase_dir_rad, width, height, scale_arcsec, frequencies):
    """FITS keywords in WSClean's convention for a SIN image at the phase
    centre; the frequency axis spans the channel edges."""
    ra = math.degrees(phase_dir_rad[0])
    if ra > 180.0:
        ra -= 360.0
    dec = math.degrees(phase_dir_rad[1])
    frequencies = np.asarray(frequencies, float)
    step = frequencies[1] - frequencies[0] if len(frequencies) > 1 else 0.0
    low, high = frequencies[0] - step / 2, frequencies[-1] + step / 2
    scale = scale_arcsec / 3600.0
    return {
        "BUNIT": "JY/BEAM", "BTYPE": "Intensity", "EQUINOX": 2000.0, "LONPOLE": 180.0,
        "CTYPE1": "RA---SIN", "CRPIX1": width / 2 + 1, "CRVAL1": ra, "CDELT1": -scale, "CUNIT1": "deg",
        "CTYPE2": "DEC--SIN", "CRPIX2": height / 2 + 1, "CRVAL2": dec, "CDELT2": scale, "CUNIT2": "deg",
        "CTYPE3": "FREQ", "CRPIX3": 1.0, "CRVAL3": (low + high) / 2, "CDELT3": high - low, "CUNIT3": "Hz",
        "CTYPE4": "STOKES", "CRPIX4": 1.0, "CRVAL4": 1.0, "CDELT4": 1.0,
        "SPECSYS": "TOPOCENT",
    }


def _card(key, value):
    """One 80-character FITS header card (fixed format)."""
    key = key.upper()
    if len(key) > 8:
        raise ValueError(f"FITS keyword longer than 8 characters: {key}")
    if isinstance(value, (bool, np.bool_)):
        v = ("T" if value else "F").rjust(20)
    elif isinstance(value, (int, np.integer)):
        v = str(int(value)).rjust(20)
    elif isinstance(value, (float, np.floating)):
        text = repr(float(value)).upper()
        if "E" not in text and "." not in text:
            text += ".0"
        v = text.rjust(20)
    else:
        s = str(value).replace("'", "''")
        v = ("'" + s.ljust(8) + "'").ljust(20)
    card = f"{key:<8}= {v}"
    if len(card) > 80:
        raise ValueError(f"FITS card too long: {key}")
    return card.ljust(80)


def write_fits(path, image, header, extra=None):
    """Write a `(height, width)` image as a 4-axis float32 FITS file in the
    pixel order WSClean uses (row y, column x; no flip). An existing file is
    not overwritten."""
    image = np.asarray(image, np.float32)
    if image.ndim != 2:
        raise ValueError("a (height, width) image is required")
    h, w = image.shape
    cards = [_card("SIMPLE", True), _card("BITPIX", -32), _card("NAXIS", 4), _card("NAXIS1", w),
             _card("NAXIS2", h), _card("NAXIS3", 1), _card("NAXIS4", 1), _card("EXTEND", True)]
    cards += [_card(k, v) for k, v in header.items()]
    cards.append(_card("ORIGIN", "Rang core gridder"))
    cards += [_card(k, v) for k, v in (extra or {}).items()]
    cards.append("END".ljust(80))
    head = "".join(cards).encode("ascii")
    head += b" " * (-len(head) % 2880)
    data = image.astype(">f4").tobytes()
    data += b"\0" * (-len(data) % 2880)
    with open(path, "xb") as f:
        f.write(head)
        f.write(data)


def read_fits(path):
    """The header cards (as a dict) and the (height, width) image of a file
    written by `write_fits`, for checks without a FITS library."""
    raw = open(path, "rb").read()
    header, pos = {}, 0
    while True:
        card = raw[pos:pos + 80].decode("ascii")
        pos += 80
        if card.startswith("END"):
            break
        key, _, rest = card.partition("=")
        value = rest.strip()
        if value.startswith("'"):
            header[key.strip()] = value[1:value.rfind("'")].replace("''", "'").rstrip()
        elif value in ("T", "F"):
            header[key.strip()] = value == "T"
        else:
            header[key.strip()] = float(value) if any(c in value for c in ".E") else int(value)
    pos += -pos % 2880
    w, h = header["NAXIS1"], header["NAXIS2"]
    image = np.frombuffer(raw[pos:pos + 4 * w * h], ">f4").reshape(h, w).astype(np.float32)
    return header, image
