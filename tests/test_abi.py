"""The C ABI library and the `rang._core` binding without a GPU: the library
loads, exports every symbol include/rang_wgridder.h declares, serves the
kernel table, and refuses bad arguments with the reference's status codes
and messages before any device work."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from cases import small_case

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "rang_wgridder.h"


@pytest.fixture(scope="module")
def built():
    import importlib.util
    import sys

    spec = importlib.util.spec_from_file_location("rang_build", REPO / "rang-core_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()
    return mod


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(rang_(?:core|b200)_wgridder_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(str(built.LIB))
    names = declared_symbols()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name


def test_library_exports_every_weights_symbol(built):
    text = (REPO / "include" / "rang_weights.h").read_text()
    names = sorted(set(re.findall(r"^\w+\s+(rang_core_\w+)\s*\(", text, re.M)))
    assert names == ["rang_core_imaging_weights", "rang_core_padded_size", "rang_core_stokes_i",
                     "rang_core_weight_grid_shape"]
    lib = ctypes.CDLL(str(built.LIB))
    for name in names:
        assert hasattr(lib, name), name


def test_library_exports_every_solver_symbol(built):
    text = (REPO / "include" / "rang_solver.h").read_text()
    names = sorted(set(re.findall(r"^\w+\s+(rang_b200_\w+)\s*\(", text, re.M)))
    assert names == ["rang_b200_dot", "rang_b200_fista_init", "rang_b200_fista_partials", "rang_b200_fista_step",
                     "rang_b200_gaussian_lowpass"]
    lib = ctypes.CDLL(str(built.LIB))
    for name in names:
        assert hasattr(lib, name), name


def test_solver_entry_points_refuse_null_arrays(built):
    lib = ctypes.CDLL(str(built.LIB))
    P = ctypes.c_void_p
    lib.rang_b200_fista_step.argtypes = [ctypes.c_int32, ctypes.c_size_t] + [P] * 10 + [ctypes.c_int32] * 4 + [P, P]
    assert lib.rang_b200_fista_step(1, 16, *([None] * 10), 0, 0, 1, 1, None, None) == 1
    lib.rang_b200_gaussian_lowpass.argtypes = [ctypes.c_size_t, ctypes.c_size_t, P, P, ctypes.c_double, P]
    assert lib.rang_b200_gaussian_lowpass(8, 8, None, None, 1.0, None) == 1
    assert lib.rang_b200_fista_partials() > 0


def test_plan_extension_entry_points_refuse_null_plans(built):
    lib = ctypes.CDLL(str(built.LIB))
    P = ctypes.c_void_p
    lib.rang_b200_wgridder_plan_residual.argtypes = [P, P, ctypes.c_int32, P, P, ctypes.c_int32, P, ctypes.c_int32,
                                                     P, P, P]
    assert lib.rang_b200_wgridder_plan_residual(None, None, 1, None, None, 0, None, 0, None, None, None) == 1
    lib.rang_b200_wgridder_plan_gram.argtypes = [P, P, P, P, ctypes.c_int32, ctypes.c_int32, P, P, P]
    assert lib.rang_b200_wgridder_plan_gram(None, None, None, None, 0, 0, None, None, None) == 1
    lib.rang_b200_wgridder_plan_memory.argtypes = [P, P, ctypes.c_int32]
    assert lib.rang_b200_wgridder_plan_memory(None, None, 0) == -1
    lib.rang_b200_wgridder_plan_memory_name.restype = ctypes.c_char_p
    names = []
    while True:
        n = lib.rang_b200_wgridder_plan_memory_name(len(names))
        if n is None:
            break
        names.append(n.decode())
    assert len(names) == 8 and all(n.startswith("gridder: ") for n in names)


def test_library_exports_every_gram_symbol(built):
    text = (REPO / "include" / "rang_gram.h").read_text()
    names = sorted(set(re.findall(r"^\w+\s+(rang_b200_gram_\w+)\s*\(", text, re.M)))
    assert len(names) == 7
    lib = ctypes.CDLL(str(built.LIB))
    for name in names:
        assert hasattr(lib, name), name


def test_weight_geometry_without_a_gpu(built):
    # Host-side functions of the weights ABI against the oracle (weights.rs:38-42, :102-112).
    from rang import weighting

    for trimmed in (512, 1024, 2, 4096, 1000):
        assert weighting.padded_size(trimmed) == oracle.padded_size(trimmed)
    for args in [(616, 616, 1.0), (616, 616, 3.0), (610, 610, 4.0), (614, 614, 4.0), (1232, 900, 2.5)]:
        geometry = weighting.ImagingWeights(args[0], args[1], 1.0, super_weight=args[2])
        assert geometry.grid_shape() == oracle.weight_grid_shape(*args)
    with pytest.raises(ValueError):
        weighting.ImagingWeights(616, 616, 1.0, super_weight=0.0).grid_shape()


def test_kernel_table_through_the_extension(built):
    from rang import gridder

    assert gridder.kernel_table() == oracle.kernel_table()
    assert gridder.kernel_row(939) is None


def test_last_error_is_empty_then_set(built):
    from rang import gridder

    uvw, freq, vis, wgt, nx, ny, dx = small_case(nrow=6)
    common = dict(uvw=uvw, freq=freq, npix_x=nx, npix_y=ny, pixsize_x=dx, pixsize_y=dx)
    with pytest.raises(ValueError, match="ascending"):
        gridder.vis2dirty(vis=vis, wgt=wgt, epsilon=1e-6, **{**common, "freq": freq[::-1]})
    with pytest.raises(ValueError, match="epsilon must be positive"):
        gridder.vis2dirty(vis=vis, wgt=wgt, epsilon=0.0, **common)
    with pytest.raises(ValueError, match="pixel sizes must be positive"):
        gridder.vis2dirty(vis=vis, wgt=wgt, epsilon=1e-6, **{**common, "pixsize_x": -1.0})
    with pytest.raises(ValueError, match="positive"):
        gridder.dirty2vis(dirty=np.zeros((nx, ny)), uvw=uvw, freq=-freq, wgt=wgt, pixsize_x=dx,
                                pixsize_y=dx, epsilon=1e-6)


def test_binding_checks_like_the_reference(built):
    ext = __import__("rang._core", fromlist=["_core"])
    uvw, freq, vis, wgt, nx, ny, dx = small_case(nrow=6)
    info = np.empty(14)
    dirty = np.empty((nx, ny))
    with pytest.raises(ValueError, match="18 gridder options"):
        ext.wgridder_vis2dirty_f64([1.0] * 17, uvw, freq, vis, wgt, None, None, dirty, None, info)
    opts = [nx, ny, dx, dx, 1e-6, 0, 0, 1.1, 2.6, 1, 0, 0, 0, 0, 1, -1, 0, 0]
    with pytest.raises(ValueError, match="complex64 or complex128"):
        ext.wgridder_vis2dirty_f64(opts, uvw, freq, vis.real.copy(), wgt, None, None, dirty, None, info)
    with pytest.raises(ValueError, match="float32 or float64"):
        ext.wgridder_vis2dirty_f64(opts, uvw, freq, vis, wgt.astype(np.int32), None, None, dirty, None, info)
    with pytest.raises(ValueError, match="two weights must both be float32"):
        ext.wgridder_vis2dirty_f64(opts, uvw, freq, vis, wgt, wgt.astype(np.float32), None, dirty, None, info)
    with pytest.raises(ValueError, match="sizes disagree"):
        ext.wgridder_vis2dirty_f64(opts, uvw, freq, vis, wgt[:3], None, None, dirty, None, info)
    with pytest.raises(ValueError, match="C-contiguous"):
        ext.wgridder_vis2dirty_f64(opts, uvw, freq, np.asfortranarray(vis), wgt, None, None, dirty, None, info)


def test_c_abi_null_and_kind_checks(built):
    lib = ctypes.CDLL(str(built.LIB))
    lib.rang_core_wgridder_vis2dirty_ex2_f64.restype = ctypes.c_int32
    lib.rang_core_wgridder_last_error.restype = ctypes.c_size_t
    info = np.empty(14)

    def last():
        n = lib.rang_core_wgridder_last_error(None, ctypes.c_size_t(0))
        buf = ctypes.create_string_buffer(n)
        lib.rang_core_wgridder_last_error(buf, ctypes.c_size_t(n))
        return buf.raw.decode()

    st = lib.rang_core_wgridder_vis2dirty_ex2_f64(None, 0, 0, None, None, None, 0, None, None, 0, None, None, None,
                                                  info.ctypes.data_as(ctypes.c_void_p))
    assert st == 1 and last() == "null options"
    o = oracle.options(32, 32, 0.01, 0.01, 1e-6)
    uvw = np.zeros((2, 3))
    freq = np.array([1e9])
    st = lib.rang_core_wgridder_vis2dirty_ex2_f64(ctypes.byref(o), ctypes.c_size_t(2), ctypes.c_size_t(1),
                                                  uvw.ctypes.data_as(ctypes.c_void_p),
                                                  freq.ctypes.data_as(ctypes.c_void_p), None, 1, None, None, 0, None,
                                                  None, None, info.ctypes.data_as(ctypes.c_void_p))
    assert st == 1 and last() == "null array"
    dirty = np.empty(32 * 32)
    st = lib.rang_core_wgridder_vis2dirty_ex2_f64(ctypes.byref(o), ctypes.c_size_t(2), ctypes.c_size_t(1),
                                                  uvw.ctypes.data_as(ctypes.c_void_p),
                                                  freq.ctypes.data_as(ctypes.c_void_p), None, 1, None, None, 0, None,
                                                  dirty.ctypes.data_as(ctypes.c_void_p), None,
                                                  info.ctypes.data_as(ctypes.c_void_p))
    assert st == 1 and last() == "invalid visibility array or kind"
    st = lib.rang_core_wgridder_vis2dirty_ex2_f64(ctypes.byref(o), ctypes.c_size_t(2), ctypes.c_size_t(1),
                                                  uvw.ctypes.data_as(ctypes.c_void_p),
                                                  freq.ctypes.data_as(ctypes.c_void_p), None, 0, None, None, 3, None,
                                                  dirty.ctypes.data_as(ctypes.c_void_p), None,
                                                  info.ctypes.data_as(ctypes.c_void_p))
    assert st == 1 and last() == "invalid weight array or kind"
