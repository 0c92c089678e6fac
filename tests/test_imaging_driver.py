"""The imaging driver (rang.core_grid): WCS header, FITS output and the
driver's argument checks on the CPU; `invert(gridder="wgrid")` on the GPU
against the reference's own checks (tests/test_df2b_wgrid.py:78-150 of the
reference), with one difference: the reference compares two runs bit for
bit, while the GPU's atomic accumulation makes runs agree to rounding."""

import math

import numpy as np
import pytest

C_LIGHT = 299792458.0


def _inputs(nrow=40, nchan=3, seed=5, scale_arcsec=120.0):
    from rang import core_grid

    rng = np.random.default_rng(seed)
    freq = np.array([1.0e9, 1.1e9, 1.3e9])[:nchan]
    dx = scale_arcsec * core_grid.ARCSEC
    lam = freq.max() / C_LIGHT
    uvw = np.stack([rng.uniform(-0.4, 0.4, nrow) / dx / lam, rng.uniform(-0.4, 0.4, nrow) / dx / lam,
                    rng.uniform(-300, 300, nrow) / lam], axis=1)
    data = (rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan))).astype(np.complex64)
    weights = rng.uniform(0.5, 1.5, (nrow, nchan)).astype(np.float32)
    weights[2] = 0.0
    imaging = rng.uniform(0.1, 3.0, (nrow, nchan)).astype(np.float32)
    imaging[5, 1] = 0.0
    settings = {"width": 32, "height": 32, "scale_arcsec": scale_arcsec, "w_layers": 8, "kernel_size": 7,
                "oversampling": 1023, "padding": 1.2}
    return uvw, freq, data, weights, imaging, settings


def test_wcs_header_follows_wsclean():
    from rang import core_grid

    h = core_grid.wcs_header((math.radians(200.0), math.radians(-30.0)), 512, 256, 8.0, [1.0e9, 1.1e9, 1.2e9])
    assert h["CRVAL1"] == pytest.approx(-160.0) and h["CRVAL2"] == pytest.approx(-30.0)
    assert h["CRPIX1"] == 257 and h["CRPIX2"] == 129
    assert h["CDELT1"] == -8.0 / 3600 and h["CDELT2"] == 8.0 / 3600
    assert h["CRVAL3"] == pytest.approx(1.1e9) and h["CDELT3"] == pytest.approx(0.3e9)


def test_fits_round_trip(tmp_path):
    from rang import core_grid

    img = np.arange(12 * 7, dtype=np.float32).reshape(12, 7) - 5.5
    header = core_grid.wcs_header((0.1, -0.5), 7, 12, 2.0, [1.4e9])
    path = tmp_path / "dirty.fits"
    core_grid.write_fits(path, img, header, extra={"WSCNVIS": 42, "WSCIMGWG": 3.5})
    raw = path.read_bytes()
    assert len(raw) % 2880 == 0 and raw[:30] == b"SIMPLE  =                    T"
    h, back = core_grid.read_fits(path)
    assert np.array_equal(back, img)
    assert h["BITPIX"] == -32 and h["NAXIS"] == 4 and h["NAXIS1"] == 7 and h["NAXIS2"] == 12
    assert h["CTYPE1"] == "RA---SIN" and h["ORIGIN"] == "Rang core gridder" and h["WSCNVIS"] == 42
    assert h["CDELT1"] == header["CDELT1"] and h["WSCIMGWG"] == 3.5
    with pytest.raises(FileExistsError):
        core_grid.write_fits(path, img, header)


def test_driver_argument_checks():
    from rang import core_grid

    uvw, freq, data, weights, imaging, s = _inputs()
    with pytest.raises(ValueError, match="gridder"):
        core_grid.invert(uvw, freq, data, weights, imaging, **s, gridder="idg")
    with pytest.raises(ValueError, match="wgrid"):
        core_grid.invert(uvw, freq, data, weights, imaging, **s)
    with pytest.raises(RuntimeError, match="GPU"):
        core_grid.invert(uvw, freq, data, weights, imaging, **s, gridder="wgrid", device="cpu")
    with pytest.raises(RuntimeError, match="no visibility"):
        core_grid.invert(uvw, freq, data, weights * 0, imaging, **s, gridder="wgrid")


@pytest.mark.gpu
def test_wgrid_invert_equals_fits_image_of_the_product():
    from rang import core_grid, core_wgridder

    uvw, freq, data, weights, imaging, s = _inputs()
    out = core_grid.invert(uvw, freq, data, weights, imaging, **s, gridder="wgrid")
    product = weights * imaging
    ref = core_wgridder.fits_image(uvw, freq, data, product, 32, 32, s["scale_arcsec"])
    # Grid cells are summed with atomics, so two GPU runs agree to rounding
    # (the reference's CPU code repeats bit for bit).
    for key in ("dirty", "psf"):
        assert np.abs(out[key] - ref[key]).max() <= 1e-12 * np.abs(ref[key]).max()
    assert out["gridder"] == "wgrid" and out["wgridder"]["epsilon"] == 1e-6
    assert out["psf"][16, 16] == 1.0
    st = out["stats"]
    live = product != 0
    assert st["gridded_count"] == int(live.sum()) == out["wgridder"]["nvis"]
    assert st["image_weight"] == pytest.approx(float(product.astype(np.float64).sum()), rel=1e-14)
    assert st["visibility_weight_sum"] == pytest.approx(float(weights[live].astype(np.float64).sum()), rel=1e-14)
    assert st["max_gridded_weight"] == float(product.max())
    assert st["n_w_layers"] == out["wgridder"]["nplanes"]
    assert st["psf_normalization"] == pytest.approx(st["image_weight"] / out["wgridder"]["psf_centre_raw"])


@pytest.mark.gpu
def test_imaging_weights_into_the_driver(tmp_path):
    # The caller's chain: Stokes I weights -> WSClean imaging weights -> invert -> FITS.
    from rang import core_grid, core_weights

    uvw, freq, data, weights, _, s = _inputs(nrow=60, seed=9)
    wl = core_weights.wsclean_wavelengths(freq)
    iw = core_weights.imaging_weights(uvw, wl, weights, np.ones(len(uvw), np.uint8), mode="briggs", robust=0.5,
                                      width=core_weights.padded_size(32), height=core_weights.padded_size(32),
                                      pixel_scale=s["scale_arcsec"] * core_grid.ARCSEC)["weights"]
    out = core_grid.invert(uvw, freq, data, weights, iw, **s, gridder="wgrid")
    assert out["psf"][16, 16] == 1.0 and np.isfinite(out["dirty"]).all()
    header = core_grid.wcs_header((0.0, -0.5), 32, 32, s["scale_arcsec"], freq)
    core_grid.write_fits(tmp_path / "dirty.fits", out["dirty"], header,
                         extra={"WSCNVIS": out["stats"]["gridded_count"]})
    h, img = core_grid.read_fits(tmp_path / "dirty.fits")
    assert np.array_equal(img, out["dirty"].astype(np.float32)) and h["WSCNVIS"] == out["stats"]["gridded_count"]
