"""The visibility-free w-aware normal operator on the B200 (the reference's
`GramOperator` and `GramMeasurement`, core/src/gridder_gram.rs), over the C
ABI of include/rang_gram.h on PyTorch CUDA tensors.

`GramOperator(...)` approximates G = A^H W A of the measurement by a sum of
Toeplitz operators, one per w-node, each applied with 2-D FFTs on the 2n
grid; `GramOperator.no_w(...)` is its one-node, translation-invariant form
(the PSF convolution); `inverse_filter(rho)` the circulant preconditioner of
a one-node operator. An operator is callable on an (n, n) float64 CUDA tensor
and can stand for `DevicePlan.gram` in `rang.fista.solve`.
"""

import ctypes

import numpy as np
import torch

from . import core
from .gridder import options_list

N_STATS = 14
STAT_NAMES = ("planes", "stencil", "theta", "wmin", "wmax", "x_range", "sup_error", "lebesgue", "active_pairs",
              "cube_bytes", "setup_grid_seconds", "setup_fft_seconds", "spectral_sparsity", "hermitian_check")
TABLE_BINS = 8192


class _Options(ctypes.Structure):  # WgridderOptions (include/rang_wgridder.h)
    _fields_ = [("nx", ctypes.c_size_t), ("ny", ctypes.c_size_t), ("pixsize_x", ctypes.c_double),
                ("pixsize_y", ctypes.c_double), ("epsilon", ctypes.c_double), ("center_x", ctypes.c_double),
                ("center_y", ctypes.c_double), ("sigma_min", ctypes.c_double), ("sigma_max", ctypes.c_double),
                ("do_wgridding", ctypes.c_int32), ("divide_by_n", ctypes.c_int32), ("flip_u", ctypes.c_int32),
                ("flip_v", ctypes.c_int32), ("flip_w", ctypes.c_int32), ("allow_nshift", ctypes.c_int32),
                ("kernel_index", ctypes.c_int64), ("nu", ctypes.c_size_t), ("nv", ctypes.c_size_t)]


_lib = None


def _library():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(core.library_path())
        P, S, D, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_int32
        lib.rang_b200_gram_expansion.argtypes = [S, D, D, P, P, P]
        lib.rang_b200_gram_expansion.restype = I
        lib.rang_b200_gram_create.argtypes = [P, S, S, P, P, P, S, D, D, D, I, I, P, P, P]
        lib.rang_b200_gram_create.restype = I
        lib.rang_b200_gram_apply.argtypes = [P, P, P, P]
        lib.rang_b200_gram_apply.restype = I
        lib.rang_b200_gram_inverse_filter.argtypes = [P, D, P, P]
        lib.rang_b200_gram_inverse_filter.restype = I
        lib.rang_b200_gram_psf_no_w.argtypes = [P, P, P]
        lib.rang_b200_gram_psf_no_w.restype = I
        lib.rang_b200_gram_planes.argtypes = [P]
        lib.rang_b200_gram_planes.restype = I
        lib.rang_b200_gram_destroy.argtypes = [P]
        lib.rang_b200_gram_destroy.restype = None
        _lib = lib
    return _lib


def _check(status):
    if status == 0:
        return
    msg = core.extension().wgridder_last_error()
    if status == 1:
        raise ValueError(msg)
    raise RuntimeError(f"Gram operator failed with status {status}: {msg}")


def _options(n, pixsize_x, pixsize_y, epsilon, kw):
    o = options_list(n, n, pixsize_x, pixsize_y, epsilon, dict(kw))
    return _Options(int(o[0]), int(o[1]), *o[2:9], *(int(v) for v in o[9:15]), int(o[15]), int(o[16]), int(o[17]))


class WExpansion:
    """The compact w-expansion (gridder_gram.rs:42-175): `stencil` (even)
    nodes spaced theta / (2 pi X) apart, fitted with ridge `ridge`."""

    def __init__(self, stencil, theta, ridge):
        self.stencil, self.theta, self.ridge = int(stencil), float(theta), float(ridge)
        table = np.empty((TABLE_BINS + 1, self.stencil))
        sup, leb = ctypes.c_double(), ctypes.c_double()
        _check(_library().rang_b200_gram_expansion(self.stencil, self.theta, self.ridge, table.ctypes.data,
                                                   ctypes.byref(sup), ctypes.byref(leb)))
        self.table, self.sup_error, self.lebesgue = table, sup.value, leb.value

    def coefficient(self, s, j):
        f = (s + 0.5) * TABLE_BINS
        b = min(int(f), TABLE_BINS - 1)
        a = f - b
        return self.table[b, j] + a * (self.table[b + 1, j] - self.table[b, j])


class GramOperator:
    """G~ on the GPU for coordinates `uvw` ((nrow, 3) CUDA tensor, metres),
    channel frequencies `freq` and weights `wgt` ((nrow, nchan) CUDA
    tensor), imaging an n x n field (`npix`, pixel sizes, and the
    gridder's flips as keywords). `single` keeps float32 spectra."""

    def __init__(self, uvw, freq, wgt, *, npix, pixsize_x, pixsize_y, expansion=None, epsilon=1e-7, single=False,
                 no_w=False, _handle=None, **kw):
        self.n = int(npix)
        self._handle = None
        if _handle is not None:
            self._handle, self.stats = _handle
            return
        if not no_w and expansion is None:
            raise ValueError("an expansion is required (or no_w=True)")
        self.device = uvw.device
        uvw = uvw.to(torch.float64).contiguous()
        wgt = wgt.to(torch.float64).contiguous()
        freq = np.ascontiguousarray(np.asarray(freq, np.float64))
        nrow, nchan = int(uvw.shape[0]), int(freq.size)
        if tuple(wgt.shape) != (nrow, nchan):
            raise ValueError("wgt must be (nrow, nchan)")
        opts = _options(self.n, pixsize_x, pixsize_y, epsilon, kw)
        handle = ctypes.c_void_p()
        stats = np.zeros(N_STATS)
        st = 0 if no_w else expansion.stencil
        th = 0.0 if no_w else expansion.theta
        rg = 0.0 if no_w else expansion.ridge
        _check(_library().rang_b200_gram_create(ctypes.byref(opts), nrow, nchan, uvw.data_ptr(), freq.ctypes.data,
                                                wgt.data_ptr(), st, th, rg, float(epsilon), int(bool(single)),
                                                int(bool(no_w)), torch.cuda.current_stream(self.device).cuda_stream,
                                                ctypes.byref(handle), stats.ctypes.data))
        self._handle = handle
        self.stats = dict(zip(STAT_NAMES, stats.tolist()))

    @classmethod
    def no_w(cls, uvw, freq, wgt, *, npix, pixsize_x, pixsize_y, epsilon=1e-7, single=False, **kw):
        """The operator without the w-term (gridder_gram.rs:415-486): one node,
        G~ m = K * m with K the PSF on the 2n grid."""
        return cls(uvw, freq, wgt, npix=npix, pixsize_x=pixsize_x, pixsize_y=pixsize_y, epsilon=epsilon,
                   single=single, no_w=True, **kw)

    def planes(self):
        return int(_library().rang_b200_gram_planes(self._handle))

    def apply(self, m, out=None):
        """G~ m for an (n, n) model (float64 CUDA tensor)."""
        m = m.to(torch.float64).contiguous()
        if tuple(m.shape) != (self.n, self.n):
            raise ValueError("model size")
        if out is None:
            out = torch.empty_like(m)
        _check(_library().rang_b200_gram_apply(self._handle, m.data_ptr(), out.data_ptr(),
                                               torch.cuda.current_stream(m.device).cuda_stream))
        return out

    __call__ = apply

    def inverse_filter(self, rho):
        """The circulant preconditioner of a one-node operator (gridder_gram.rs:488-511)."""
        h = ctypes.c_void_p()
        _check(_library().rang_b200_gram_inverse_filter(self._handle, float(rho),
                                                        torch.cuda.current_stream().cuda_stream, ctypes.byref(h)))
        return GramOperator(None, None, None, npix=self.n, pixsize_x=0, pixsize_y=0, _handle=(h, dict(self.stats)))

    def psf_no_w(self):
        """Sum over nodes of Re K_k on the 2n grid, centred on (n, n)."""
        out = torch.empty((2 * self.n, 2 * self.n), dtype=torch.float64, device="cuda")
        _check(_library().rang_b200_gram_psf_no_w(self._handle, out.data_ptr(), torch.cuda.current_stream().cuda_stream))
        return out

    def close(self):
        if getattr(self, "_handle", None):
            torch.cuda.synchronize()
            _library().rang_b200_gram_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GramMeasurement:
    """A measurement on the operator (gridder_gram.rs:685-719): the dirty
    image and Q(0) from the data once, then every residual d - G~ m and the
    misfit Q(0) - d.m + m.G~m / 2 without visibilities."""

    def __init__(self, operator, dirty, q0):
        self.operator, self.dirty, self.q0 = operator, dirty.to(torch.float64), float(q0)

    def residual(self, model):
        model = model.to(torch.float64)
        if not bool((model != 0).any()):
            return self.dirty.clone(), self.q0
        g = self.operator.apply(model)
        misfit = self.q0 - float((self.dirty * model).sum()) + 0.5 * float((g * model).sum())
        return self.dirty - g, misfit

    def gram_apply(self, x):
        return self.operator.apply(x)
