"""The binning entry point that allocates no device memory.

`rang_b200_wgridder_bin_noalloc` exists for callers that cannot call
cudaMalloc: an application that hands out all device memory through its own
allocator under a fixed budget, or a path that must not take the CUDA
allocator's locks or wait on it. It keeps every temporary in one fixed
16 MiB device array of the library instead. This test calls it through the C
ABI, twice in a row on different inputs (the second call must not see the
first call's counters), and checks each result against the ordinary binning
entry point: the per-visibility keys bit for bit, and the sorted order up to
the order inside a (tile, plane) bin, which the GPU's counting sort leaves
unspecified. It also checks the property the entry point exists for: once a
first call has loaded the library's kernels and its array, a further call
leaves the device's free memory unchanged. It runs last (file name) so that
a failure here does not stop the rest of the GPU suite.
"""

import ctypes

import numpy as np
import pytest

import oracle
from cases import meerkat_like

pytestmark = pytest.mark.gpu


def _lib():
    from rang import core

    lib = ctypes.CDLL(core.library_path())
    lib.rang_b200_wgridder_bin_noalloc.restype = ctypes.c_int32
    lib.rang_b200_wgridder_bin_noalloc.argtypes = [
        ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p]
    lib.rang_core_wgridder_last_error.restype = ctypes.c_size_t
    return lib


def _case(seed, nant, ntime, nchan, npix, single):
    uvw, freq = meerkat_like(nant=nant, ntime=ntime, nchan=nchan, seed=seed)
    rng = np.random.default_rng(seed)
    shape = (uvw.shape[0], freq.size)
    wgt = rng.uniform(0.5, 1.5, shape).astype(np.float32 if single else np.float64)
    wgt.ravel()[:: 7 + seed] = 0.0
    mask = (rng.uniform(size=shape) > 0.1).astype(np.uint8)
    kw = dict(npix_x=npix, npix_y=npix, pixsize_x=4e-5 / npix * 256, pixsize_y=4e-5 / npix * 256,
              epsilon=1e-5 if single else 1e-7)
    return uvw, freq, wgt, mask, kw


def _noalloc(lib, uvw, freq, wgt, mask, kw, single):
    import torch

    n = uvw.shape[0] * freq.size
    dev = torch.device("cuda", 0)
    d_uvw = torch.from_numpy(uvw).to(dev)
    d_wgt = torch.from_numpy(wgt).to(dev)
    d_mask = torch.from_numpy(mask).to(dev)
    key = torch.full((n,), 12345, dtype=torch.int32, device=dev)
    srt = torch.full((n,), 12345, dtype=torch.int32, device=dev)
    info = np.empty(14)
    ns = ctypes.c_size_t(0)
    o = oracle.options(kw["npix_x"], kw["npix_y"], kw["pixsize_x"], kw["pixsize_y"], kw["epsilon"])
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.rang_b200_wgridder_bin_noalloc(
        ctypes.byref(o), uvw.shape[0], freq.size, d_uvw.data_ptr(), freq.ctypes.data, d_wgt.data_ptr(),
        1 if single else 2, d_mask.data_ptr(), int(single), stream, key.data_ptr(), srt.data_ptr(),
        ctypes.byref(ns), info.ctypes.data)
    if st != 0:
        m = lib.rang_core_wgridder_last_error(None, 0)
        buf = ctypes.create_string_buffer(m)
        lib.rang_core_wgridder_last_error(buf, m)
        raise AssertionError(f"status {st}: {buf.raw.decode()}")
    keys = key.cpu().numpy().view(np.uint32)
    return keys, srt[: ns.value].cpu().numpy().view(np.uint32).astype(np.int64), info


@pytest.mark.parametrize("single", [True, False])
def test_no_alloc_binning_matches_the_allocating_entry_point(single):
    from rang import gridder as cw

    lib = _lib()
    cases = [_case(3, 32, 6, 24, 256, single), _case(4, 48, 4, 40, 384, single)]
    for uvw, freq, wgt, mask, kw in cases:  # two calls in a row on different inputs
        key, srt, info = _noalloc(lib, uvw, freq, wgt, mask, kw, single)
        ref = cw.binning(uvw=uvw, freq=freq, wgt=wgt, mask=mask, single=single, with_vis=False, **kw)
        assert np.array_equal(key, ref["key"])
        assert np.array_equal(info, np.array([ref["info"][k] for k in cw.INFO_NAMES], dtype=float))
        rs = ref["sorted"].astype(np.int64)
        assert srt.size == rs.size
        k = key[srt].astype(np.int64)
        assert np.all(np.diff(k) >= 0)
        assert np.array_equal(srt[np.lexsort((srt, k))], rs[np.lexsort((rs, key[rs].astype(np.int64)))])


def test_no_alloc_binning_takes_no_device_memory():
    import torch

    lib = _lib()
    uvw, freq, wgt, mask, kw = _case(5, 40, 6, 32, 256, True)
    _noalloc(lib, uvw, freq, wgt, mask, kw, True)  # loads the kernels and the array
    n = uvw.shape[0] * freq.size
    dev = torch.device("cuda", 0)
    d_uvw = torch.from_numpy(uvw).to(dev)
    d_wgt = torch.from_numpy(wgt).to(dev)
    d_mask = torch.from_numpy(mask).to(dev)
    key = torch.empty((n,), dtype=torch.int32, device=dev)
    srt = torch.empty((n,), dtype=torch.int32, device=dev)
    info = np.empty(14)
    ns = ctypes.c_size_t(0)
    o = oracle.options(kw["npix_x"], kw["npix_y"], kw["pixsize_x"], kw["pixsize_y"], kw["epsilon"])
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(dev)
    st = lib.rang_b200_wgridder_bin_noalloc(
        ctypes.byref(o), uvw.shape[0], freq.size, d_uvw.data_ptr(), freq.ctypes.data, d_wgt.data_ptr(), 1,
        d_mask.data_ptr(), 1, stream, key.data_ptr(), srt.data_ptr(), ctypes.byref(ns), info.ctypes.data)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info(dev)
    assert st == 0 and ns.value > 0
    assert free_after == free_before
