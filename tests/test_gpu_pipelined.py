"""The pipelined host calls: visibilities copied in row chunks that overlap
the gridding (vis2dirty) or the copy back (dirty2vis).

Calls whose visibilities take 256 MB or more are split into row chunks by
default; RANG_WGRIDDER_ROW_CHUNKS forces a chunk count, so small cases run
the same code here. The chunked degridder computes each visibility exactly
as the single pass does, so its output must be bit-identical. The chunked
gridder adds the same footprints in another order (float atomics), so its
image agrees to rounding, and with the oracle to the suite's tolerance; the
plan report must be identical. Visibilities that are exactly zero leave the
reference's active set, which the chunked gridder only learns after the
copy: such a call must fall back and still report the reference's plan."""

import numpy as np
import pytest

import oracle
from cases import meerkat_like, rel_linf

pytestmark = pytest.mark.gpu

TOL = {True: 2e-5, False: 1e-9}


@pytest.fixture
def chunks(monkeypatch):
    def set_chunks(k):
        monkeypatch.setenv("RANG_WGRIDDER_ROW_CHUNKS", str(k))

    return set_chunks


def _case(single, seed=5, zeros=False):
    uvw, freq = meerkat_like(nant=40, ntime=12, nchan=24, seed=seed)
    rng = np.random.default_rng(seed)
    shape = (uvw.shape[0], freq.size)
    vis = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    wgt = rng.uniform(0.5, 1.5, shape)
    mask = (rng.uniform(size=shape) > 0.15).astype(np.uint8)
    if zeros:
        # Zero the visibilities of the largest |w|: the active |w| range shrinks.
        w = np.abs(uvw[:, 2])[:, None] * freq[None, :]
        vis[w >= np.quantile(w, 0.97)] = 0.0
    if single:
        vis, wgt = vis.astype(np.complex64), wgt.astype(np.float32)
    kw = dict(uvw=uvw, freq=freq, npix_x=192, npix_y=160, pixsize_x=3e-5, pixsize_y=3e-5,
              epsilon=1e-5 if single else 1e-9)
    return vis, wgt, mask, kw


@pytest.mark.parametrize("single", [True, False])
@pytest.mark.parametrize("k", [3, 7])
def test_chunked_dirty2vis_is_bit_identical(chunks, single, k):
    from rang import gridder as cw

    vis, wgt, mask, kw = _case(single)
    kw = {key: v for key, v in kw.items() if key not in ("npix_x", "npix_y")}
    rng = np.random.default_rng(9)
    dirty = rng.standard_normal((192, 160)).astype(np.float32 if single else np.float64)
    chunks(1)
    ref, info1 = cw.dirty2vis(dirty=dirty, wgt=wgt, mask=mask, return_info=True, **kw)
    chunks(k)
    out, info2 = cw.dirty2vis(dirty=dirty, wgt=wgt, mask=mask, return_info=True, **kw)
    assert info1 == info2
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))


@pytest.mark.parametrize("single", [True, False])
@pytest.mark.parametrize("k", [3, 7])
def test_chunked_vis2dirty_is_bit_identical(chunks, single, k):
    """Gridding sums exact fixed-point terms, so a plan split into row chunks
    (a different sorted order and split of the work) gives the same bits."""
    from rang import gridder as cw

    vis, wgt, mask, kw = _case(single)
    chunks(1)
    ref, info1 = cw.vis2dirty(vis=vis, wgt=wgt, mask=mask, return_info=True, **kw)
    chunks(k)
    out, info2 = cw.vis2dirty(vis=vis, wgt=wgt, mask=mask, return_info=True, **kw)
    assert info1 == info2
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    oref = oracle.vis2dirty(vis=vis, wgt=wgt, mask=mask, **kw)
    assert rel_linf(out, oref) < TOL[single]


@pytest.mark.parametrize("single", [True, False])
def test_chunked_vis2dirty_with_zero_visibilities_falls_back(chunks, single):
    from rang import gridder as cw

    vis, wgt, mask, kw = _case(single, seed=6, zeros=True)
    _, oinfo = oracle.vis2dirty(vis=vis, wgt=wgt, mask=mask, return_info=True, **kw)
    chunks(4)
    out, info = cw.vis2dirty(vis=vis, wgt=wgt, mask=mask, return_info=True, **kw)
    assert info == oinfo
    oref = oracle.vis2dirty(vis=vis, wgt=wgt, mask=mask, **kw)
    assert rel_linf(out, oref) < TOL[single]


@pytest.mark.parametrize("k", [3, 7])
@pytest.mark.parametrize("change", ["later chunk larger", "first rows flagged", "later chunk smaller"])
def test_chunked_vis2dirty_regrids_when_the_bound_changes(chunks, k, change):
    """The chunked gridder grids each row chunk as it arrives, with the
    fixed-point scale of the values seen so far (the scale depends on their
    bound only through its exponent). A chunk that changes the exponent makes
    it clear the planes and grid the chunks before it again, so the image
    still equals the one-pass gridding's bit for bit."""
    from rang import gridder as cw

    vis, wgt, mask, kw = _case(True, seed=8)
    nrow = vis.shape[0]
    if change == "later chunk larger":
        vis[nrow * 2 // 3:] *= np.float32(1000.0)
    elif change == "first rows flagged":
        mask[: nrow // 2] = 0
    else:
        vis[nrow // 3:] *= np.float32(1e-4)
    chunks(1)
    ref, info1 = cw.vis2dirty(vis=vis, wgt=wgt, mask=mask, return_info=True, **kw)
    chunks(k)
    out, info2 = cw.vis2dirty(vis=vis, wgt=wgt, mask=mask, return_info=True, **kw)
    assert info1 == info2
    assert np.array_equal(out.view(np.uint8), ref.view(np.uint8))
    oref = oracle.vis2dirty(vis=vis, wgt=wgt, mask=mask, **kw)
    assert rel_linf(out, oref) < TOL[True]
