"""Generate the golden fixtures of the gridder tests.

* `df1_cases.npz` — the four seeded synthetic cases of the reference's DF1
  protocol (generator `examples/oracle_ducc0.py:216-286`: seeds 101-104,
  uv up to 0.45 of the Nyquist extent, w of both signs, point sources on
  pixel centres plus noise, weights in [0.5, 1.5)) with their FP64
  direct-Fourier-transform dirty images and the FP64 DFT visibilities of a
  sparse 16-pixel image (the reference's `dft_dirty` / `dft_vis`,
  `examples/oracle_ducc0.py:85-120`).
* `kernel_rows.json` — the 939 rows of the kernel table as parsed from the
  reference, after checking the SHA256 its own test pins
  (`tests/test_core_wgridder.py:16`), so the table can be checked where the
  reference checkout is absent.

    python tests/golden/make_golden.py /path/to/reference

The DFT is independent of every gridder (oracle and CUDA path alike).
"""

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO / "rang-core_b200" / "csrc"))

import oracle  # noqa: E402

C_LIGHT = oracle.C_LIGHT

# name, npix, field (rad), w scale (wavelengths), rows, channels, seed
CASES = (
    ("small-8arcmin", 64, 8.0 / 60.0 * np.pi / 180.0, 1.0e3, 400, 4, 101),
    ("mid-2deg", 128, 2.0 * np.pi / 180.0, 3.0e3, 400, 4, 102),
    ("wide-0p3rad", 128, 0.3, 1.0e4, 400, 4, 103),
    ("wide-0p3rad-rect", 128, 0.3, 1.0e4, 300, 3, 104),
)


def make_case(name, npix, field, wscale, nrow, nchan, seed):
    rng = np.random.default_rng(seed)
    nx = npix
    ny = npix if not name.endswith("rect") else npix // 2
    dx = dy = field / nx
    freq = np.linspace(0.9e9, 1.6e9, nchan)
    lam_max = freq.max() / C_LIGHT
    umax = 0.45 / dx / lam_max
    vmax = 0.45 / dy / lam_max
    uvw = np.stack(
        [
            rng.uniform(-umax, umax, nrow),
            rng.uniform(-vmax, vmax, nrow),
            rng.uniform(-wscale, wscale, nrow) / lam_max,
        ],
        axis=1,
    )
    nsrc = 4
    ix = rng.integers(2, nx - 2, nsrc)
    iy = rng.integers(2, ny - 2, nsrc)
    ix[0], iy[0] = 3, ny - 4
    flux = rng.uniform(0.2, 1.0, nsrc)
    image = np.zeros((nx, ny))
    for a, b, f in zip(ix, iy, flux, strict=True):
        image[a, b] += f
    model = oracle.dft_vis(uvw, freq, image, dx, dy)
    noise = 0.05 * (rng.standard_normal((nrow, nchan)) + 1j * rng.standard_normal((nrow, nchan)))
    vis = model + noise
    wgt = rng.uniform(0.5, 1.5, (nrow, nchan))
    dirty = oracle.dft_dirty(uvw, freq, vis * wgt, nx, ny, dx, dy)
    img2 = np.zeros((nx, ny))
    pix = rng.integers(0, nx * ny, 16)
    img2.ravel()[pix] = rng.uniform(-1.0, 1.0, 16)
    img2.ravel()[pix[0]] = 2.0
    vis2 = oracle.dft_vis(uvw, freq, img2, dx, dy) * wgt
    return {
        "uvw": uvw, "freq": freq, "vis": vis, "wgt": wgt, "nx": nx, "ny": ny, "dx": dx, "dy": dy,
        "dft_dirty": dirty, "image": img2, "dft_vis": vis2,
    }


def main():
    reference = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    out = {}
    for case in CASES:
        rec = make_case(*case)
        for k, v in rec.items():
            out[f"{case[0]}/{k}"] = np.asarray(v)
    np.savez_compressed(HERE / "df1_cases.npz", **out)
    import gen_kernel_db

    rows, digest = gen_kernel_db.read_rows(reference)
    (HERE / "kernel_rows.json").write_text(json.dumps({"sha256": digest, "rows": rows}))
    print("wrote", HERE / "df1_cases.npz", "and", HERE / "kernel_rows.json")


if __name__ == "__main__":
    main()
