"""Seeded inputs shared by the tests."""

import numpy as np

C_LIGHT = 299792458.0


def small_case(nx=32, ny=32, field=0.2, wmax=600.0, nrow=40, seed=3):
    """The reference's `_case` (tests/test_core_wgridder.py:20-37)."""
    rng = np.random.default_rng(seed)
    freq = np.array([1.0e9, 1.3e9])
    dx = field / nx
    lam = freq.max() / C_LIGHT
    uvw = np.stack(
        [
            rng.uniform(-0.45, 0.45, nrow) / dx / lam,
            rng.uniform(-0.45, 0.45, nrow) / dx / lam,
            rng.uniform(-wmax, wmax, nrow) / lam,
        ],
        axis=1,
    )
    vis = rng.standard_normal((nrow, 2)) + 1j * rng.standard_normal((nrow, 2))
    wgt = rng.uniform(0.5, 1.5, (nrow, 2))
    return uvw, freq, vis, wgt, nx, ny, dx


def lcg_case(nx, ny, field, wmax, nrow, seed):
    """The reference's Rust test case (core/src/wgridder.rs:4547-4593): a
    64-bit LCG, three channels, weights in [0.5, 1.5)."""
    state = [seed]

    def lcg():
        state[0] = (state[0] * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        return (state[0] >> 11) / float(1 << 53)

    freq = np.array([1.0e9, 1.2e9, 1.4e9])
    dx = field / nx
    lam = 1.4e9 / C_LIGHT
    uvw = np.empty((nrow, 3))
    for r in range(nrow):
        uvw[r, 0] = (lcg() - 0.5) * 0.9 / dx / lam
        uvw[r, 1] = (lcg() - 0.5) * 0.9 / dx / lam
        uvw[r, 2] = (lcg() - 0.5) * 2.0 * wmax / lam
    n = nrow * 3
    vis = np.array([complex(lcg() - 0.5, lcg() - 0.5) for _ in range(n)]).reshape(nrow, 3)
    wgt = np.array([0.5 + lcg() for _ in range(n)]).reshape(nrow, 3)
    return uvw, freq, vis, wgt, dx


def meerkat_like(nant=64, ntime=16, nchan=16, dec_deg=-30.0, tint=8.0, f0=856e6, f1=1712e6, seed=7):
    """Earth-rotation uvw of a MeerKAT-shaped array: 48 antennas in a
    Gaussian core (sigma 500 m) and 16 uniform in a 4 km disk, ENU positions
    projected as `examples/bench_df2.py:101-122` does."""
    rng = np.random.default_rng(seed)
    ncore = nant * 3 // 4
    core = rng.normal(0.0, 500.0, (ncore, 2))
    r = 4000.0 * np.sqrt(rng.uniform(0, 1, nant - ncore))
    th = rng.uniform(0, 2 * np.pi, nant - ncore)
    outer = np.stack([r * np.cos(th), r * np.sin(th)], axis=1)
    en = np.concatenate([core, outer])
    lat = np.deg2rad(-30.7)
    east, north, up = en[:, 0], en[:, 1], np.zeros(nant)
    x = -np.sin(lat) * north + np.cos(lat) * up
    y = east
    z = np.cos(lat) * north + np.sin(lat) * up
    i1, i2 = np.triu_indices(nant, 1)
    b = np.stack([x[i2] - x[i1], y[i2] - y[i1], z[i2] - z[i1]], axis=1)
    ha = -0.5 * ntime * tint * 7.2921159e-5 + np.arange(ntime) * tint * 7.2921159e-5
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
    ).reshape(-1, 3)
    freq = np.linspace(f0, f1, nchan)
    return uvw, freq


def rel_linf(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def df1_cases(golden):
    """The four DF1 cases of `df1_cases.npz` (made by the reference's own
    generator), as {name: {field: array}}."""
    data = np.load(golden / "df1_cases.npz")
    names = sorted({k.split("/")[0] for k in data.files})
    return {n: {k.split("/")[1]: data[k] for k in data.files if k.startswith(n + "/")} for n in names}


# Precisions and epsilons the reference's DF1 run recorded errors for.
DF1_RECORDED = ((True, 1e-4), (True, 1e-5), (False, 1e-7), (False, 1e-9))


def df1_record(golden, single, eps, direction):
    """The reference gridder's worst error against the FP64 DFT for one
    precision, epsilon and direction ("vis2dirty" or "dirty2vis"), as its DF1
    run recorded it (research/results/df1-wgridder.json, "worst"): dirty2vis
    over the four synthetic cases, vis2dirty over them and the LUNO slice."""
    import json

    rec = json.loads((golden / "df1_reference_errors.json").read_text())
    return rec[f"{'f32' if single else 'f64'}_eps{eps:g} {direction} vs DFT"]


def df1_worst(df1, single, eps, vis2dirty, dirty2vis):
    """Worst L-inf error relative to the DFT's peak over the DF1 cases of the
    gridder calls given (keyword APIs of rang.gridder or the oracle)."""
    wd = wv = 0.0
    for c in df1.values():
        nx, ny, dx, dy = int(c["nx"]), int(c["ny"]), float(c["dx"]), float(c["dy"])
        vis = c["vis"].astype(np.complex64) if single else c["vis"]
        wgt = c["wgt"].astype(np.float32) if single else c["wgt"]
        kw = dict(uvw=c["uvw"], freq=c["freq"], wgt=wgt, pixsize_x=dx, pixsize_y=dy, epsilon=eps)
        wd = max(wd, rel_linf(vis2dirty(vis=vis, npix_x=nx, npix_y=ny, **kw), c["dft_dirty"]))
        img = c["image"].astype(np.float32) if single else c["image"]
        wv = max(wv, rel_linf(dirty2vis(dirty=img, **kw), c["dft_vis"]))
    return wd, wv
