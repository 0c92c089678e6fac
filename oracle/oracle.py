"""CPU ORACLE — test infrastructure only.

ctypes binding of `liboracle.so` (the C++ restatement of the reference's
`core/src/wgridder.rs`) and a NumPy FP64 direct Fourier transform (the
semantics of the reference's `examples/oracle_ducc0.py:80-120`). Only the
tests, `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py`
import this module; the product never does.

The Python-level calls mirror the reference's `python/rang/core_wgridder.py`
keyword interface (`vis2dirty`, `dirty_psf`, `dirty2vis`), so a parity test
can call the oracle and the CUDA path with the same arguments.
"""

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
C_LIGHT = 299792458.0
N_INFO = 14
INFO_NAMES = (
    "kernel_index", "supp", "nu", "nv", "nplanes", "nvis", "wmin_d", "wmax_d",
    "nm1min", "nm1max", "nshift", "dw", "wmin", "ofactor",
)


class Options(ctypes.Structure):
    """`WgridderOptions` (reference `core/src/ffi_wgridder.rs:24-42`)."""

    _fields_ = [
        ("nx", ctypes.c_size_t), ("ny", ctypes.c_size_t),
        ("pixsize_x", ctypes.c_double), ("pixsize_y", ctypes.c_double),
        ("epsilon", ctypes.c_double), ("center_x", ctypes.c_double),
        ("center_y", ctypes.c_double), ("sigma_min", ctypes.c_double),
        ("sigma_max", ctypes.c_double), ("do_wgridding", ctypes.c_int32),
        ("divide_by_n", ctypes.c_int32), ("flip_u", ctypes.c_int32),
        ("flip_v", ctypes.c_int32), ("flip_w", ctypes.c_int32),
        ("allow_nshift", ctypes.c_int32), ("kernel_index", ctypes.c_int64),
        ("nu", ctypes.c_size_t), ("nv", ctypes.c_size_t),
    ]


LIB_AVX512 = HERE / "liboracle_avx512.so"
# CPU flags the x86-64-v4 build may use.
_AVX512_FLAGS = ("avx512f", "avx512vl", "avx512bw", "avx512dq", "avx512cd")


def build():
    """Compile both libraries with the committed Makefile (idempotent)."""
    srcs = [HERE / "wgridder_oracle.cpp", HERE / "weights_oracle.cpp"]
    if any(not p.exists() or any(p.stat().st_mtime < s.stat().st_mtime for s in srcs) for p in (LIB, LIB_AVX512)):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def simd_level():
    """The instruction set of the library `lib()` loads, chosen as the
    reference chooses its gridding loops (`core/src/wgridder.rs:1592-1625`):
    "avx512" where the host has AVX-512 (the x86-64-v4 set), else "avx2";
    RANG_WGRIDDER_SIMD=avx2 caps it. The oracle has no variant below AVX2."""
    if os.environ.get("RANG_WGRIDDER_SIMD") in ("avx2", "baseline"):
        return "avx2"
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        return "avx2"
    return "avx512" if all(x in flags for x in _AVX512_FLAGS) else "avx2"


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB_AVX512 if simd_level() == "avx512" else LIB))
        P = ctypes.c_void_p
        S = ctypes.c_size_t
        I = ctypes.c_int
        _lib.oracle_vis2dirty.argtypes = [P, S, S, P, P, P, I, P, P, I, P, P, P, P, I]
        _lib.oracle_dirty2vis.argtypes = [P, S, S, P, P, P, P, I, P, P, P, I]
        _lib.oracle_binning.argtypes = [P, S, S, P, P, P, I, P, P, I, P, I, I, P, P, P, P, P, P, P]
        _lib.oracle_kernel_row.argtypes = [S, P]
        _lib.oracle_good_size.argtypes = [S]
        _lib.oracle_good_size.restype = S
        _lib.oracle_gauss_legendre.argtypes = [S, P, P]
        _lib.oracle_gauss_legendre.restype = S
        _lib.oracle_kernel_eval.argtypes = [S, I, S, P, P]
        _lib.oracle_coeff_even_odd.argtypes = [S, I, P]
        _lib.oracle_coeff_even_odd.restype = S
        _lib.oracle_fft.argtypes = [S, P, I]
        _lib.oracle_last_error.argtypes = [P, S]
        _lib.oracle_last_error.restype = S
        _lib.oracle_set_threads.argtypes = [I]
        _lib.oracle_padded_size.argtypes = [S, ctypes.c_double]
        _lib.oracle_padded_size.restype = S
        _lib.oracle_weight_grid_shape.argtypes = [S, S, ctypes.c_double, P]
        _lib.oracle_stokes_i.argtypes = [S, P, P, P, P, P]
        D = ctypes.c_double
        _lib.oracle_imaging_weights.argtypes = [S, S, P, P, P, P, ctypes.c_uint32, D, S, S, D, D, D, D, S, P, P, P]
        _lib.oracle_imaging_weights.restype = I
    return _lib


def set_threads(n):
    return lib().oracle_set_threads(int(n))


def _ptr(a):
    return None if a is None else a.ctypes.data


def _error():
    n = lib().oracle_last_error(None, 0)
    buf = ctypes.create_string_buffer(n)
    lib().oracle_last_error(buf, n)
    return buf.raw.decode()


def _check(status):
    if status == 1:
        raise ValueError(_error())
    if status != 0:
        raise RuntimeError(f"oracle failed with status {status}: {_error()}")


def options(nx, ny, pixsize_x, pixsize_y, epsilon, **kw):
    kernel = kw.pop("kernel", None)
    o = Options(
        nx=int(nx), ny=int(ny), pixsize_x=float(pixsize_x), pixsize_y=float(pixsize_y),
        epsilon=float(epsilon), center_x=float(kw.pop("center_x", 0.0)),
        center_y=float(kw.pop("center_y", 0.0)), sigma_min=float(kw.pop("sigma_min", 1.1)),
        sigma_max=float(kw.pop("sigma_max", 2.6)),
        do_wgridding=int(bool(kw.pop("do_wgridding", True))),
        divide_by_n=int(bool(kw.pop("divide_by_n", False))),
        flip_u=int(bool(kw.pop("flip_u", False))), flip_v=int(bool(kw.pop("flip_v", False))),
        flip_w=int(bool(kw.pop("flip_w", False))),
        allow_nshift=int(bool(kw.pop("allow_nshift", True))),
        kernel_index=-1 if kernel is None else int(kernel[0]),
        nu=0 if kernel is None else int(kernel[1]), nv=0 if kernel is None else int(kernel[2]),
    )
    if kw:
        raise TypeError(f"unexpected options {sorted(kw)}")
    return o


def info_dict(info):
    rec = dict(zip(INFO_NAMES, (float(v) for v in info)))
    for key in ("kernel_index", "supp", "nu", "nv", "nplanes", "nvis"):
        rec[key] = int(rec[key])
    return rec


_VIS_KIND = {np.dtype(np.complex64): 1, np.dtype(np.complex128): 2}
_WGT_KIND = {np.dtype(np.float32): 1, np.dtype(np.float64): 2}


def _weights(wgt, wgt2):
    if wgt is None:
        return None, None, 0
    wgt = np.ascontiguousarray(wgt)
    if wgt.dtype not in _WGT_KIND:
        wgt = wgt.astype(np.float64)
    if wgt2 is not None:
        wgt2 = np.ascontiguousarray(wgt2, np.float32)
        wgt = np.ascontiguousarray(wgt, np.float32)
        return wgt, wgt2, 3
    return wgt, None, _WGT_KIND[wgt.dtype]


def gridding(uvw, freq, vis, wgt=None, mask=None, *, npix_x, npix_y, pixsize_x, pixsize_y,
             epsilon, single, outputs=("dirty",), wgt2=None, **kw):
    """`vis2dirty_ex2` of the oracle; `outputs` a subset of ("dirty", "psf")."""
    uvw = np.ascontiguousarray(uvw, np.float64)
    freq = np.ascontiguousarray(freq, np.float64)
    nrow, nchan = uvw.shape[0], freq.shape[0]
    if vis is None:
        vkind = 0
    else:
        vis = np.ascontiguousarray(vis)
        if vis.dtype not in _VIS_KIND:
            vis = vis.astype(np.complex128)
        vkind = _VIS_KIND[vis.dtype]
    wgt, wgt2, wkind = _weights(wgt, wgt2)
    if mask is not None:
        mask = np.ascontiguousarray(mask, np.uint8)
    real = np.float32 if single else np.float64
    imgs = {o: np.empty((int(npix_x), int(npix_y)), real) for o in outputs}
    info = np.empty(N_INFO)
    o = options(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, **kw)
    _check(lib().oracle_vis2dirty(
        ctypes.byref(o), nrow, nchan, _ptr(uvw), _ptr(freq), _ptr(vis), vkind, _ptr(wgt),
        _ptr(wgt2), wkind, _ptr(mask), _ptr(imgs.get("dirty")), _ptr(imgs.get("psf")),
        _ptr(info), int(bool(single))))
    return imgs, info_dict(info)


def vis2dirty(*, uvw, freq, vis, wgt=None, mask=None, npix_x, npix_y, pixsize_x, pixsize_y,
              epsilon, return_info=False, single=None, **kw):
    if single is None:
        single = np.asarray(vis).dtype == np.complex64
    imgs, info = gridding(uvw, freq, vis, wgt, mask, npix_x=npix_x, npix_y=npix_y,
                          pixsize_x=pixsize_x, pixsize_y=pixsize_y, epsilon=epsilon,
                          single=single, **kw)
    return (imgs["dirty"], info) if return_info else imgs["dirty"]


def dirty_psf(*, uvw, freq, vis, wgt=None, mask=None, npix_x, npix_y, pixsize_x, pixsize_y,
              epsilon, single=False, return_info=False, wgt2=None, **kw):
    imgs, info = gridding(uvw, freq, vis, wgt, mask, npix_x=npix_x, npix_y=npix_y,
                          pixsize_x=pixsize_x, pixsize_y=pixsize_y, epsilon=epsilon,
                          single=single, outputs=("dirty", "psf"), wgt2=wgt2, **kw)
    if return_info:
        return imgs["dirty"], imgs["psf"], info
    return imgs["dirty"], imgs["psf"]


def dirty2vis(*, uvw, freq, dirty, wgt=None, mask=None, pixsize_x, pixsize_y, epsilon,
              return_info=False, **kw):
    dirty = np.asarray(dirty)
    single = dirty.dtype == np.float32
    real = np.float32 if single else np.float64
    dirty = np.ascontiguousarray(dirty, real)
    uvw = np.ascontiguousarray(uvw, np.float64)
    freq = np.ascontiguousarray(freq, np.float64)
    nrow, nchan = uvw.shape[0], freq.shape[0]
    wgt, _, wkind = _weights(wgt, None)
    if mask is not None:
        mask = np.ascontiguousarray(mask, np.uint8)
    vis = np.empty((nrow, nchan), np.complex64 if single else np.complex128)
    info = np.empty(N_INFO)
    o = options(dirty.shape[0], dirty.shape[1], pixsize_x, pixsize_y, epsilon, **kw)
    _check(lib().oracle_dirty2vis(
        ctypes.byref(o), nrow, nchan, _ptr(uvw), _ptr(freq), _ptr(dirty), _ptr(wgt), wkind,
        _ptr(mask), _ptr(vis), _ptr(info), int(single)))
    return (vis, info_dict(info)) if return_info else vis


def binning(*, uvw, freq, vis=None, wgt=None, mask=None, npix_x, npix_y, pixsize_x, pixsize_y,
            epsilon, single, with_vis, wgt2=None, **kw):
    """Per visibility iu0, iv0, tile and first plane (-1 inactive), the sorted
    order as linear indices, and the plan, as the reference's `layout`."""
    uvw = np.ascontiguousarray(uvw, np.float64)
    freq = np.ascontiguousarray(freq, np.float64)
    nrow, nchan = uvw.shape[0], freq.shape[0]
    n = nrow * nchan
    vkind = 0
    if vis is not None:
        vis = np.ascontiguousarray(vis)
        if vis.dtype not in _VIS_KIND:
            vis = vis.astype(np.complex128)
        vkind = _VIS_KIND[vis.dtype]
    wgt, wgt2, wkind = _weights(wgt, wgt2)
    if mask is not None:
        mask = np.ascontiguousarray(mask, np.uint8)
    out = {k: np.empty(n, np.int64) for k in ("iu0", "iv0", "tile", "minplane")}
    srt = np.empty(n, np.uint64)
    ns = ctypes.c_size_t(0)
    info = np.empty(N_INFO)
    o = options(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, **kw)
    _check(lib().oracle_binning(
        ctypes.byref(o), nrow, nchan, _ptr(uvw), _ptr(freq), _ptr(vis), vkind, _ptr(wgt),
        _ptr(wgt2), wkind, _ptr(mask), int(bool(with_vis)), int(bool(single)),
        _ptr(out["iu0"]), _ptr(out["iv0"]), _ptr(out["tile"]), _ptr(out["minplane"]),
        _ptr(srt), ctypes.byref(ns), _ptr(info)))
    out["sorted"] = srt[: ns.value].copy()
    out["info"] = info_dict(info)
    return out


def kernel_row(index):
    out = np.empty(7)
    if lib().oracle_kernel_row(int(index), _ptr(out)):
        return None
    return (int(out[0]), *(float(v) for v in out[1:5]), int(out[5]), bool(out[6]))


def kernel_table():
    rows = []
    while (row := kernel_row(len(rows))) is not None:
        rows.append(row)
    return rows


def good_size(n):
    return int(lib().oracle_good_size(int(n)))


def gauss_legendre(n):
    m = (n + 1) // 2
    x, w = np.empty(m), np.empty(m)
    lib().oracle_gauss_legendre(int(n), _ptr(x), _ptr(w))
    return x, w


def kernel_eval(index, what, v):
    v = np.ascontiguousarray(v, np.float64)
    out = np.empty_like(v)
    _check(lib().oracle_kernel_eval(int(index), {"phi": 0, "poly": 1, "corfunc": 2}[what],
                                    v.size, _ptr(v), _ptr(out)))
    return out


def coeff_even_odd(index, single):
    n = lib().oracle_coeff_even_odd(int(index), int(bool(single)), None)
    out = np.empty(n)
    lib().oracle_coeff_even_odd(int(index), int(bool(single)), _ptr(out))
    return out


def fft(x, inverse=False):
    a = np.ascontiguousarray(x, np.complex128).copy()
    lib().oracle_fft(a.size, _ptr(a), int(bool(inverse)))
    return a


# ------------------------------------------------------------ FP64 DFT


def lm_grid(nx, ny, dx, dy, center_x=0.0, center_y=0.0):
    l1 = center_x + (np.arange(nx) - nx // 2) * dx
    m1 = center_y + (np.arange(ny) - ny // 2) * dy
    return np.meshgrid(l1, m1, indexing="ij")


def nm1_of(L, M):
    r2 = L * L + M * M
    return np.where(r2 < 1.0, -r2 / (np.sqrt(np.maximum(1.0 - r2, 0.0)) + 1.0), 0.0)


def dft_dirty(uvw, freq, values, nx, ny, dx, dy, batch=64):
    """sum_k Re[values_k exp(+2 pi i (u l + v m + w (n-1)))] per pixel, FP64;
    `values` is (nrow, nchan) (data times weight)."""
    L, M = lm_grid(nx, ny, dx, dy)
    nm1 = nm1_of(L, M)
    lam = np.asarray(freq) / C_LIGHT
    u = (uvw[:, 0:1] * lam).ravel()
    v = (uvw[:, 1:2] * lam).ravel()
    w = (uvw[:, 2:3] * lam).ravel()
    vals = np.asarray(values).ravel()
    out = np.zeros(L.shape)
    for s in range(0, u.size, batch):
        ph = np.exp(2j * np.pi * (u[s:s + batch, None, None] * L + v[s:s + batch, None, None] * M
                                  + w[s:s + batch, None, None] * nm1))
        out += np.real(np.tensordot(vals[s:s + batch], ph, axes=(0, 0)))
    return out


def dft_vis(uvw, freq, image, dx, dy):
    """V_k = sum_lm I exp(-2 pi i (u l + v m + w (n-1))), FP64, over nonzero pixels."""
    nx, ny = image.shape
    L, M = lm_grid(nx, ny, dx, dy)
    nz = np.nonzero(image)
    lv, mv, iv = L[nz], M[nz], image[nz]
    nv = nm1_of(lv, mv)
    lam = np.asarray(freq) / C_LIGHT
    u = (uvw[:, 0:1] * lam).ravel()
    v = (uvw[:, 1:2] * lam).ravel()
    w = (uvw[:, 2:3] * lam).ravel()
    out = np.zeros(u.size, np.complex128)
    for s in range(0, lv.size, 64):
        ph = np.exp(-2j * np.pi * (u[:, None] * lv[None, s:s + 64] + v[:, None] * mv[None, s:s + 64]
                                   + w[:, None] * nv[None, s:s + 64]))
        out += ph @ iv[s:s + 64]
    return out.reshape(uvw.shape[0], len(freq))


if os.environ.get("RANG_ORACLE_THREADS"):
    set_threads(int(os.environ["RANG_ORACLE_THREADS"]))


# ------------------------------------------------------------------ imaging weights (core/src/weights.rs)

WEIGHT_CLASSES = {"natural": 0, "uniform": 1, "briggs": 2}


def padded_size(trimmed, padding=1.2):
    return int(lib().oracle_padded_size(int(trimmed), float(padding)))


def weight_grid_shape(width, height, super_weight=1.0):
    out = np.zeros(2, np.uint64)
    lib().oracle_weight_grid_shape(int(width), int(height), float(super_weight), out.ctypes.data)
    return int(out[0]), int(out[1])


def stokes_i(data, weights, flags):
    """`data` complex64 (..., 4), `weights` float32 and `flags` bool alike:
    Stokes I complex64 values and float32 weights."""
    data = np.ascontiguousarray(data, np.complex64)
    weights = np.ascontiguousarray(weights, np.float32)
    flags = np.ascontiguousarray(flags, np.uint8)
    shape = data.shape[:-1]
    n = int(np.prod(shape, dtype=np.int64))
    vis = np.zeros(shape, np.complex64)
    w = np.zeros(shape, np.float32)
    lib().oracle_stokes_i(n, data.ctypes.data, weights.ctypes.data, flags.ctypes.data, vis.ctypes.data, w.ctypes.data)
    return vis, w


def imaging_weights(uvw, wavelength, weights, row_selected, mode="briggs", robust=0.5, width=616, height=616,
                    pixel_scale=8.0 * np.pi / (180.0 * 3600.0), super_weight=1.0, rank_filter=(3.0, 16)):
    """The reference's imaging_weights (weights.rs:465-520) on host arrays:
    {"weights", "grid" (height // 2, width), "sums" (four values)}."""
    uvw = np.ascontiguousarray(uvw, np.float64)
    wavelength = np.ascontiguousarray(wavelength, np.float64)
    weights = np.ascontiguousarray(weights, np.float32)
    sel = np.ascontiguousarray(row_selected, np.uint8)
    nrow, nchan = weights.shape
    level, size = rank_filter if rank_filter is not None else (0.0, 0)
    gw, gh = weight_grid_shape(width, height, super_weight)
    out = np.zeros((nrow, nchan), np.float32)
    grid = np.zeros((gh // 2, gw), np.float64)
    sums = np.zeros(4, np.float64)
    st = lib().oracle_imaging_weights(nrow, nchan, uvw.ctypes.data, wavelength.ctypes.data, weights.ctypes.data,
                                      sel.ctypes.data, WEIGHT_CLASSES[mode], float(robust), int(width), int(height),
                                      float(pixel_scale), float(pixel_scale), float(super_weight), float(level),
                                      int(size), out.ctypes.data, grid.ctypes.data, sums.ctypes.data)
    if st:
        raise ValueError("invalid imaging-weight arguments")
    return {"weights": out, "grid": grid, "sums": sums}


# ------------------------------------------------------------------ Gram operator (core/src/gridder_gram.rs)


def w_expansion(stencil, theta, ridge):
    """WExpansion::new (gridder_gram.rs:88-163) in NumPy: the (8193, stencil)
    coefficient table, the sampled sup error and the Lebesgue constant."""
    s = int(stencil)
    t = np.arange(s) - (s - 1) / 2.0
    m = 64 * s
    xi = np.cos(np.pi * (np.arange(m) + 0.5) / m)

    def kern(d):
        return np.cos(theta * np.multiply.outer(np.asarray(d, float), xi)).sum(-1) / m

    normal = kern(t[:, None] - t[None, :])
    normal[np.diag_indices(s)] *= 1.0 + ridge
    bins = 8192
    sv = -0.5 + np.arange(bins + 1) / bins
    rhs = kern(sv[:, None] - t[None, :])
    table = np.linalg.solve(normal, rhs.T).T
    lebesgue = float(np.abs(table).sum(1).max())

    def coeff(sval):
        f = (sval + 0.5) * bins
        b = min(int(f), bins - 1)
        a = f - b
        return table[b] + a * (table[b + 1] - table[b])

    sup = 0.0
    xs = np.arange(513) / 512.0
    for sb in range(257):
        sval = -0.5 + sb / 256.0 + (0.5 / 8192.0 if sb < 256 else 0.0)
        c = coeff(sval)
        re = np.cos(theta * xs * sval) - (c[None, :] * np.cos(theta * xs[:, None] * t[None, :])).sum(1)
        im = np.sin(theta * xs * sval) - (c[None, :] * np.sin(theta * xs[:, None] * t[None, :])).sum(1)
        sup = max(sup, float(np.hypot(re, im).max()))
    return table, sup, lebesgue


def gram_direct(uvw, freq, wgt, m, cell, flip_v=False, flip_w=False):
    """The direct sum of the Gram matrix in the gridder's conventions
    (the reference's test oracle, gridder_gram.rs:765-803): for an n x n
    model m, sum_p W_p sum_l' m(l') cos 2 pi (u (l - l') + v (m - m') + w (x - x'))."""
    n = m.shape[0]
    half = n / 2
    fv = -1.0 if flip_v else 1.0
    fw = -1.0 if flip_w else 1.0
    idx = np.arange(n)
    L = (idx[:, None] - half) * cell * np.ones((1, n))
    M = (idx[None, :] - half) * cell * np.ones((n, 1))
    r2 = L * L + M * M
    X = -r2 / (np.sqrt(np.maximum(1.0 - r2, 0.0)) + 1.0)
    nz = np.nonzero(m)
    lp, mp, xp, vals = L[nz], M[nz], X[nz], m[nz]
    out = np.zeros((n, n))
    foc = np.asarray(freq) / 299792458.0
    for row in range(uvw.shape[0]):
        for ch in range(len(freq)):
            u, v, w = uvw[row, 0] * foc[ch], fv * uvw[row, 1] * foc[ch], fw * uvw[row, 2] * foc[ch]
            wt = wgt[row, ch]
            ph = 2.0 * np.pi * (u * (L[..., None] - lp) + v * (M[..., None] - mp) + w * (X[..., None] - xp))
            out += wt * (np.cos(ph) * vals).sum(-1)
    return out


def gram_case(n, nrow, wmax, flip):
    """The reference's test case (gridder_gram.rs:727-763): xorshift uvw,
    two channels at c and 1.05 c, weights normalised to sum 1, cell 8e-3."""
    state = 77
    mask = (1 << 64) - 1

    def nxt():
        nonlocal state
        state ^= (state << 13) & mask
        state ^= state >> 7
        state ^= (state << 17) & mask
        return (state >> 11) / float(1 << 53) - 0.5

    freq = np.array([299792458.0, 1.05 * 299792458.0])
    cell = 8e-3
    umax = 0.45 / cell
    uvw = np.array([nxt() * 2.0 * (wmax if i % 3 == 2 else umax / 1.05) for i in range(3 * nrow)]).reshape(nrow, 3)
    raw = np.array([0.2 + abs(nxt()) for _ in range(2 * nrow)])
    wgt = (raw / raw.sum()).reshape(nrow, 2)
    return uvw, freq, wgt, cell


def gram_test_model(n):
    m = np.zeros((n, n))
    m.flat[0] = 1.0
    m.flat[n * n - 1] = -0.5
    m.flat[(n // 2) * n + n // 2] = 0.75
    m.flat[5 * n + (n - 3)] = 0.25
    return m
