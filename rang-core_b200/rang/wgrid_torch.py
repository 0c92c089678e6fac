"""The gridder on PyTorch CUDA tensors.

`DevicePlan` is the reference's `Prepared` (core/src/wgridder.rs:3170-3499)
on device memory: the scan, kernel choice and visibility binning of a fixed
set of coordinates, weights and mask, kept on the GPU, after which
`grid` (vis2dirty) and `degrid` (dirty2vis) run entirely on the device on
torch's current stream. `Degrid` is a `torch.autograd.Function` whose forward
is the degridder and whose hand-written backward is the gridder (its
adjoint): for a real image x and complex visibilities y = A x,
d L / d x = Re(A^H g) with g the gradient of L with respect to y (PyTorch's
conjugate-Wirtinger convention for a real input). PyTorch supplies only the
memory, the stream and autograd; all arithmetic runs in this library's CUDA
kernels.
"""

import numpy as np
import torch

from . import core
from .gridder import options_list

_VIS_KIND = {torch.complex64: 1, torch.complex128: 2}
_WGT_KIND = {torch.float32: 1, torch.float64: 2}


def _check(status):
    if status == 0:
        return
    msg = core.extension().wgridder_last_error()
    if status == 1:
        raise ValueError(msg)
    raise RuntimeError(f"gridder failed with status {status}: {msg}")


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


def _ptr(t):
    return 0 if t is None else t.data_ptr()


def _wgt(wgt, wgt2=None):
    if wgt is None:
        return None, None, 0
    if wgt2 is not None:
        return wgt, wgt2, 3
    return wgt, None, _WGT_KIND[wgt.dtype]


class DevicePlan:
    """The plan of one set of visibilities on the GPU.

    `uvw` (nrow, 3) float64 and the optional `wgt` / `mask` (nrow, nchan) are
    CUDA tensors (weights float32 or float64, mask uint8); `freq` is a
    sequence of channel frequencies. The active set is `wgt * mask != 0`, or
    `|vis|^2 wgt mask != 0` when `vis` is given (a dirty image alone, as the
    reference's `vis2dirty`). `single` selects float32 working precision.
    """

    def __init__(self, uvw, freq, *, npix_x, npix_y, pixsize_x, pixsize_y, epsilon, wgt=None, wgt2=None,
                 mask=None, vis=None, single=True, **kw):
        ext = core.extension()
        self.device = uvw.device
        self.single = bool(single)
        self.real = torch.float32 if single else torch.float64
        self.cplx = torch.complex64 if single else torch.complex128
        self.nrow, self.nchan = int(uvw.shape[0]), int(len(freq))
        self.shape = (int(npix_x), int(npix_y))
        uvw = uvw.to(torch.float64).contiguous()
        freq = np.ascontiguousarray(np.asarray(freq, np.float64))
        w, w2, wk = _wgt(wgt, wgt2)
        vk = 0 if vis is None else _VIS_KIND[vis.dtype]
        self._keep = (w, w2, mask)
        opts = options_list(npix_x, npix_y, pixsize_x, pixsize_y, epsilon, dict(kw))
        status, handle, info = ext.wgridder_plan_create(
            opts, self.nrow, self.nchan, uvw.data_ptr(), freq, _ptr(vis), vk, _ptr(w), _ptr(w2), wk, _ptr(mask),
            int(vis is not None), int(self.single), _stream(self.device))
        _check(status)
        self._handle = handle
        self._stream = torch.cuda.current_stream(self.device)
        from .gridder import info_dict

        self.info = info_dict(info)

    def close(self):
        """Releases the plan. Its device memory is freed in order on the
        stream it was made on, so no wait is needed while the current stream
        is that one; otherwise the device is synchronised first."""
        if getattr(self, "_handle", 0):
            if torch.cuda.current_stream(self.device) != getattr(self, "_stream", None):
                torch.cuda.synchronize(self.device)
            core.extension().wgridder_plan_destroy(self._handle)
            self._handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grid(self, vis=None, wgt=None, wgt2=None, out=None, scanned=False):
        """vis2dirty of `vis` (complex CUDA tensor (nrow, nchan); None: unit
        visibilities, the PSF) with weights `wgt` into a new or given image.
        `scanned`: `vis` (and the weights) are the tensors this plan was made
        with, unchanged since, so the plan's scan bounds their values and the
        pass over the data that would find the bound is skipped (as in the
        reference's stateless call, which plans and grids one set of data)."""
        if out is None:
            out = torch.empty(self.shape, dtype=self.real, device=self.device)
        w, w2, wk = _wgt(wgt, wgt2)
        vk = 0 if vis is None else _VIS_KIND[vis.dtype]
        flags = (1 if vis is None else 0) | (2 if scanned else 0)
        _check(core.extension().wgridder_plan_grid(self._handle, _ptr(vis), vk, _ptr(w), _ptr(w2), wk, flags,
                                                   out.data_ptr(), _stream(self.device)))
        return out

    def degrid(self, image, wgt=None, out=None):
        """dirty2vis of `image` times the weights `wgt` (complex (nrow, nchan)
        CUDA tensor; inactive visibilities zero)."""
        image = image.to(self.real).contiguous()
        if out is None:
            out = torch.empty((self.nrow, self.nchan), dtype=self.cplx, device=self.device)
        w, _, wk = _wgt(wgt)
        _check(core.extension().wgridder_plan_degrid(self._handle, image.data_ptr(), _ptr(w), wk, out.data_ptr(),
                                                     _stream(self.device)))
        return out

    def residual(self, data, wgt=None, model=None, out=None, misfit=None, sorted=False):
        """The residual image of `data` against the image `model` (None: the
        data alone), gridded with weights `wgt`, and the misfit
        sum w |data - A model|^2 over the active visibilities (the
        reference's Prepared::residual, core/src/wgridder.rs:3232-3395: the
        prediction is degridded without weights, the residual gridded with
        them). The values pass through the plan's stored work space in the
        sorted order; no visibility-sized tensor is made and nothing waits for
        the device. `sorted`: `data` and `wgt` hold the active visibilities in
        the plan's sorted order (`sorted_values`, the reference's
        residual_sorted). Returns (image, misfit as a 0-dimensional float64
        CUDA tensor)."""
        if out is None:
            out = torch.empty(self.shape, dtype=self.real, device=self.device)
        q = torch.empty((), dtype=torch.float64, device=self.device) if misfit is None else misfit
        data = data.contiguous()
        w, w2, wk = _wgt(None if wgt is None else wgt.contiguous())
        m = None if model is None else model.to(self.real).contiguous()
        _check(core.extension().wgridder_plan_residual(self._handle, data.data_ptr(), _VIS_KIND[data.dtype], _ptr(w),
                                                       _ptr(w2), wk, _ptr(m), int(bool(sorted)), out.data_ptr(),
                                                       q.data_ptr(), _stream(self.device)))
        return out, q

    def gram(self, x, wgt=None, out=None, xgx=None, sorted=False):
        """A^H W A x: the image of the unweighted prediction of `x`, weighted
        and gridded (the reference's gram_apply,
        core/src/clean_certified.rs:233-236), through the plan's stored work
        space; with `xgx` (a 0-dimensional float64 CUDA tensor) also
        x^T A^H W A x = sum w |A x|^2."""
        if out is None:
            out = torch.empty(self.shape, dtype=self.real, device=self.device)
        x = x.to(self.real).contiguous()
        w, w2, wk = _wgt(None if wgt is None else wgt.contiguous())
        _check(core.extension().wgridder_plan_gram(self._handle, x.data_ptr(), _ptr(w), _ptr(w2), wk,
                                                   int(bool(sorted)), out.data_ptr(), _ptr(xgx),
                                                   _stream(self.device)))
        return out

    @property
    def active(self):
        """The number of active visibilities (the sorted layout's length)."""
        st, n = core.extension().wgridder_plan_active(self._handle)
        _check(st)
        return int(n)

    def sorted_values(self, dense):
        """`dense` ((nrow, nchan) CUDA tensor) at the active visibilities in
        the plan's sorted order (the reference's Prepared::sorted)."""
        dense = dense.contiguous()
        if tuple(dense.shape[:2]) != (self.nrow, self.nchan):
            raise ValueError(f"expected ({self.nrow}, {self.nchan}), got {tuple(dense.shape)}")
        out = torch.empty((self.active,), dtype=dense.dtype, device=self.device)
        _check(core.extension().wgridder_plan_sorted(self._handle, dense.data_ptr(), dense.element_size(),
                                                     out.data_ptr(), _stream(self.device)))
        return out

    def memory(self):
        """Device bytes held by the plan, per buffer (the reference's
        Prepared::memory)."""
        return dict(core.extension().wgridder_plan_memory(self._handle))

    def release_work(self):
        """Frees the stored values that residual and Gram passes keep (the
        reference's Prepared::release_grids)."""
        core.extension().wgridder_plan_release_work(self._handle)

    def status(self):
        """Waits for the stream; raises if a kernel flagged an inconsistency."""
        _check(core.extension().wgridder_plan_status(self._handle, _stream(self.device)))


class Degrid(torch.autograd.Function):
    """y = A x: forward degrids the real image x with `plan` (weights
    `wgt`), backward grids the incoming visibility gradient (A^H)."""

    @staticmethod
    def forward(ctx, image, plan, wgt):
        ctx.plan = plan
        ctx.has_wgt = wgt is not None
        if wgt is not None:
            ctx.save_for_backward(wgt)
        return plan.degrid(image, wgt)

    @staticmethod
    def backward(ctx, grad):
        wgt = ctx.saved_tensors[0] if ctx.has_wgt else None
        g = grad.to(ctx.plan.cplx).contiguous()
        return ctx.plan.grid(g, wgt), None, None


def degrid(image, plan, wgt=None):
    """Differentiable dirty2vis: see `Degrid`."""
    return Degrid.apply(image, plan, wgt)
