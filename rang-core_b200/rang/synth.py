"""Seeded synthetic MeerKAT-shaped observations for benchmarks and tests.

The array: 64 antennas at seeded ENU positions, 48 in a 2-D Gaussian core
(sigma 500 m) and 16 uniform in a 4 km-radius disk (2016 baselines), at
latitude -30.7 deg. uvw come from Earth-rotation synthesis of the baseline
vectors (the projection of the reference's `examples/bench_df2.py:101-122`)
for integrations of `tint` seconds centred on transit at declination `dec`.
Channels are evenly spaced over [f0, f1]. No public dataset is used; these
stand in for one.
"""

import numpy as np

C_LIGHT = 299792458.0
OMEGA_EARTH = 7.2921159e-5
ARCSEC = np.pi / (180.0 * 3600.0)


def antennas(nant=64, seed=7, core_frac=0.75, core_sigma=500.0, disk_radius=4000.0):
    rng = np.random.default_rng(seed)
    ncore = int(round(nant * core_frac))
    core = rng.normal(0.0, core_sigma, (ncore, 2))
    r = disk_radius * np.sqrt(rng.uniform(0.0, 1.0, nant - ncore))
    th = rng.uniform(0.0, 2.0 * np.pi, nant - ncore)
    outer = np.stack([r * np.cos(th), r * np.sin(th)], axis=1)
    return np.concatenate([core, outer])


def uvw_tracks(nant=64, ntime=128, tint=8.0, dec_deg=-30.0, lat_deg=-30.7, seed=7, subset=None):
    """(ntime * nbaselines, 3) uvw in metres, time-major; `subset` (antenna
    indices) keeps those antennas of the array only."""
    en = antennas(nant, seed)
    if subset is not None:
        en = en[np.sort(np.asarray(subset))]
    lat = np.deg2rad(lat_deg)
    east, north, up = en[:, 0], en[:, 1], np.zeros(len(en))
    x = -np.sin(lat) * north + np.cos(lat) * up
    y = east
    z = np.cos(lat) * north + np.sin(lat) * up
    i1, i2 = np.triu_indices(len(en), 1)
    b = np.stack([x[i2] - x[i1], y[i2] - y[i1], z[i2] - z[i1]], axis=1)
    ha = (np.arange(ntime) - 0.5 * (ntime - 1)) * tint * OMEGA_EARTH
    dec = np.deg2rad(dec_deg)
    sh, ch = np.sin(ha)[:, None], np.cos(ha)[:, None]
    bx, by, bz = b[None, :, 0], b[None, :, 1], b[None, :, 2]
    uvw = np.stack(
        [
            sh * bx + ch * by,
            -np.sin(dec) * ch * bx + np.sin(dec) * sh * by + np.cos(dec) * bz,
            np.cos(dec) * ch * bx - np.cos(dec) * sh * by + np.sin(dec) * bz,
        ],
        axis=-1,
    )
    return np.ascontiguousarray(uvw.reshape(-1, 3))


def channels(nchan, f0=856e6, f1=1712e6):
    return np.linspace(f0, f1, nchan)


def point_sky(npix, nsrc=50, smin=1e-3, smax=1.0, index=-1.5, seed=11, margin=8):
    """An (npix, npix) image of `nsrc` point sources on pixel centres, uniform
    over the field, fluxes from the power law dN/dS ~ S^index on [smin, smax]."""
    rng = np.random.default_rng(seed)
    a = index + 1.0
    u = rng.uniform(0.0, 1.0, nsrc)
    flux = (smin**a + u * (smax**a - smin**a)) ** (1.0 / a)
    ix = rng.integers(margin, npix - margin, nsrc)
    iy = rng.integers(margin, npix - margin, nsrc)
    img = np.zeros((npix, npix))
    np.add.at(img, (ix, iy), flux)
    return img


def extended_sky(npix, npoint=300, ngauss=40, smin=1e-3, smax=1.0, index=-1.5, seed=21, margin=40):
    """An (npix, npix) float32 sky: `npoint` point sources and `ngauss`
    elliptical Gaussians (FWHM 3-30 pixels along each axis, random
    orientation), all inside `margin` pixels of the edge. Every source's
    integrated flux follows the power law of `point_sky`."""
    rng = np.random.default_rng(seed)
    img = point_sky(npix, nsrc=npoint, smin=smin, smax=smax, index=index, seed=seed + 1, margin=margin)
    a = index + 1.0
    yy, xx = np.mgrid[0:npix, 0:npix].astype(np.float32)
    for _ in range(ngauss):
        flux = (smin**a + rng.uniform() * (smax**a - smin**a)) ** (1.0 / a)
        fx, fy = rng.uniform(3.0, 30.0, 2)
        th = rng.uniform(0.0, np.pi)
        cx, cy = rng.uniform(margin, npix - margin, 2)
        sx, sy = fx / 2.3548, fy / 2.3548
        ct, st = np.cos(th), np.sin(th)
        h = int(4 * max(sx, sy)) + 1
        x0, x1 = int(max(cx - h, 0)), int(min(cx + h + 1, npix))
        y0, y1 = int(max(cy - h, 0)), int(min(cy + h + 1, npix))
        dx, dy = xx[y0:y1, x0:x1] - cx, yy[y0:y1, x0:x1] - cy
        u = (ct * dx + st * dy) / sx
        v = (-st * dx + ct * dy) / sy
        img[y0:y1, x0:x1] += flux / (2.0 * np.pi * sx * sy) * np.exp(-0.5 * (u * u + v * v))
    return img.astype(np.float32)


# The workloads of the benchmark configurations.
WORKLOADS = {
    # 64 antennas x 512 integrations x 1024 channels: 1,056,964,608 visibilities,
    # 20 % flagged, 4096^2 image at 1.0 arcsec.
    "ms2dirty+dirty2ms 1.06G vis 4096^2": dict(ntime=512, nchan=1024, npix=4096, cell_arcsec=1.0, flag=0.2),
    # 64 antennas x 128 integrations x 64 channels: 16.5 M visibilities, no flags,
    # 1024^2 image at 1.5 arcsec.
    "ms2dirty 16.5M vis 1024^2": dict(ntime=128, nchan=64, npix=1024, cell_arcsec=1.5, flag=0.0),
    # The round trip's field of view at a quarter of the pixels and an eighth of
    # the integrations (132 M visibilities, 2048^2 at 2.0 arcsec): a profiling
    # case a few GB in size.
    "ms2dirty+dirty2ms 132M vis 2048^2": dict(ntime=64, nchan=1024, npix=2048, cell_arcsec=2.0, flag=0.2),
}
