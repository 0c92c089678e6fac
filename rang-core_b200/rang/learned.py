"""Learned-preconditioned FISTA on the B200: a U-Net proposes model updates
from the residual image and the PSF, trained and run by this library's own
bfloat16 kernels (the C ABI of include/rang_nn.h), and every proposal is
accepted only if the exact gridder's residual decreases.

The reference has no learned solver on its imaging path. Its solver is
`prox_solver::solve` (core/src/prox_solver.rs:302-445, `rang.fista` here);
its nearest learned relatives are the learned-stage interpreter
(core/src/learned_interp.rs:1-22) and the learned deconvolution trial
(examples/dl4b_train.py:51-72). The network and the acceptance rule here are
new:

* `UNet`: 4 levels of 32/64/128/256 channels, two 3x3 convolutions with
  ReLU per level, 2x2 average pooling down, nearest 2x upsampling up, skip
  connections by concatenation ([upsampled | encoder] channels), a 1x1 head
  to one float32 channel. Input: a 256 x 256 residual patch in units of the
  PSF peak and the PSF patch (peak 1) as two of 32 input channels. Output: a
  model update in sky units. Weights bfloat16 with float32 masters; Adam.
* `make_training_set`: patches of (residual, sky - model) pairs from seeded
  random skies (300 point sources and 40 Gaussians on 2048^2, the FISTA
  measurement's distribution) predicted onto random antenna subsets by the
  GPU gridder, with models from plain FISTA snapshots.
* `solve`: FISTA whose cycles begin with a proposal: the network's update d,
  projected onto the positive orthant, scaled by the exact minimiser of the
  quadratic misfit along it (one apply of G = A^H A by the exact gridder),
  and kept only when the misfit decreases; `cycle` plain FISTA iterations
  follow from the accepted point.
"""

import ctypes
import math

import numpy as np
import torch

from . import core, fista, synth

LEVELS = (32, 64, 128, 256)
IN_CHANNELS = 32
PATCH = 256


def layers(levels=LEVELS):
    """The 3x3 convolutions in order: (name, cin, cout)."""
    c1, c2, c3, c4 = levels
    return [("enc1a", IN_CHANNELS, c1), ("enc1b", c1, c1), ("enc2a", c1, c2), ("enc2b", c2, c2),
            ("enc3a", c2, c3), ("enc3b", c3, c3), ("mid_a", c3, c4), ("mid_b", c4, c4),
            ("dec3a", c4 + c3, c3), ("dec3b", c3, c3), ("dec2a", c3 + c2, c2), ("dec2b", c2, c2),
            ("dec1a", c2 + c1, c1), ("dec1b", c1, c1)]


def initial_parameters(levels=LEVELS, seed=0, live_inputs=2):
    """He-normal convolution weights (fan-in 9 cin; the first layer counts
    its `live_inputs` live channels), zero biases, a head of variance 1/32."""
    rng = np.random.default_rng(seed)
    p = {}
    for i, (name, cin, cout) in enumerate(layers(levels)):
        fan = 9 * (live_inputs if i == 0 else cin)
        p[name + ".w"] = rng.standard_normal((cout, 9, cin)) * np.sqrt(2.0 / fan)
        p[name + ".b"] = np.zeros(cout)
    p["head.w"] = rng.standard_normal(levels[0]) * np.sqrt(1.0 / levels[0])
    p["head.b"] = np.zeros(1)
    return p


def flops(height=PATCH, width=PATCH, levels=LEVELS, training=False):
    """Floating-point operations of the convolutions for one height x width
    input: the forward pass, or a training step (forward, input gradients
    except the first layer's, weight gradients)."""
    f = 0
    for name, cin, cout in layers(levels):
        level = {"enc1": 0, "enc2": 1, "enc3": 2, "mid_": 3, "dec3": 2, "dec2": 1, "dec1": 0}[name[:4]]
        f += 2 * 9 * cin * cout * (height >> level) * (width >> level)
    if not training:
        return f
    return 3 * f - 2 * 9 * IN_CHANNELS * levels[0] * height * width


_lib = None
_SIGNATURES = {
    "conv3": "PLPPPLPLLIIIIIIP",
    "conv3_weight_grad": "PLPLPPLIIIIP",
    "conv3_flip": "PPIIP",
    "pool": "PLPLLIIIP",
    "pool_backward": "PLPLPLLIIIP",
    "upsample": "PLPLLIIIP",
    "upsample_backward": "PLPLLIIIP",
    "pack": "PPLPLFFPLIIP",
    "head": "PLPPPLP",
    "head_backward": "PLPPPLPPLP",
    "mse": "PPPLPPLIIP",
    "unpack": "PPPLFPLIIP",
    "adam": "PPPPPLFFFFIP",
    "to_bf16": "PPLP",
    "set_conv_path": "I",
    "device_status": "P",
    "wait_probe": "LP",
}


def _library():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(core.library_path())
        kinds = {"P": ctypes.c_void_p, "L": ctypes.c_int64, "I": ctypes.c_int32, "F": ctypes.c_float}
        for name, sig in _SIGNATURES.items():
            f = getattr(lib, "rang_b200_nn_" + name)
            f.argtypes = [kinds[k] for k in sig]
            f.restype = ctypes.c_int32
        _lib = lib
    return _lib


def _call(name, *args):
    status = getattr(_library(), "rang_b200_nn_" + name)(*args)
    if status != 0:
        kind = ValueError if status == 1 else RuntimeError
        raise kind(f"rang_b200_nn_{name} failed with status {status}")


def _p(t, c0=0):
    """Device pointer of channel c0 of an (pixels, channels) tensor."""
    return t.data_ptr() + c0 * t.element_size()


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


class Workspace:
    """The activations (and, for training, the gradients) of `batch`
    height x width inputs: (pixels, channels) bfloat16 tensors, the
    concatenation buffers `catN` holding [upsampled | encoder] channels."""

    def __init__(self, net, batch, height, width, training=False):
        if height % 8 or width % 8:
            raise ValueError("height and width must be multiples of 8")
        self.batch, self.height, self.width, self.training = int(batch), int(height), int(width), training
        c1, c2, c3, c4 = net.levels
        dev = net.device
        P = [self.batch * (self.height >> k) * (self.width >> k) for k in range(4)]

        def bf(n, c):
            return torch.empty((n, c), dtype=torch.bfloat16, device=dev)

        self.x, self.c1a, self.cat1, self.p1 = bf(P[0], IN_CHANNELS), bf(P[0], c1), bf(P[0], c2 + c1), bf(P[1], c1)
        self.c2a, self.cat2, self.p2 = bf(P[1], c2), bf(P[1], c3 + c2), bf(P[2], c2)
        self.c3a, self.cat3, self.p3 = bf(P[2], c3), bf(P[2], c4 + c3), bf(P[3], c3)
        self.ma, self.mb = bf(P[3], c4), bf(P[3], c4)
        self.d3a, self.d3b, self.d2a, self.d2b = bf(P[2], c3), bf(P[2], c3), bf(P[1], c2), bf(P[1], c2)
        self.d1a, self.d1b = bf(P[0], c1), bf(P[0], c1)
        self.y = torch.empty(P[0], dtype=torch.float32, device=dev)
        self.offsets = torch.zeros(self.batch, dtype=torch.int64, device=dev)
        if training:
            self.dy = torch.empty(P[0], dtype=torch.float32, device=dev)
            self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
            self.g_d1b, self.g_d1a, self.g_cat1 = bf(P[0], c1), bf(P[0], c1), bf(P[0], c2 + c1)
            self.g_d2b, self.g_d2a, self.g_cat2 = bf(P[1], c2), bf(P[1], c2), bf(P[1], c3 + c2)
            self.g_d3b, self.g_d3a, self.g_cat3 = bf(P[2], c3), bf(P[2], c3), bf(P[2], c4 + c3)
            self.g_mb, self.g_ma, self.g_p3 = bf(P[3], c4), bf(P[3], c4), bf(P[3], c3)
            self.g_c3a, self.g_p2, self.g_c2a = bf(P[2], c3), bf(P[2], c2), bf(P[1], c2)
            self.g_p1, self.g_c1a = bf(P[1], c1), bf(P[0], c1)

    def launches(self):
        """Kernel launches of one use: a training step (pack, forward, loss,
        backward, Adam, weight flips) or a proposal (pack, forward, unpack)."""
        forward = 14 + 3 + 3 + 1  # convolutions, pools, upsamplings, head
        if not self.training:
            return 1 + forward + 1
        backward = 1 + 14 * 2 + 13 + 3 + 3  # head, weight+bias gradients, input gradients, upsample, pool
        return 1 + forward + 1 + backward + 1 + 14


class UNet:
    """The proposal network on `device`: float32 master parameters, their
    bfloat16 copy, gradients and Adam moments in flat buffers (every tensor
    at a multiple of 8 elements), and the flipped weights of the
    input-gradient convolutions."""

    def __init__(self, device="cuda", seed=0, levels=LEVELS, params=None):
        self.device = torch.device(device)
        self.levels = tuple(int(c) for c in levels)
        if any(c % 32 for c in self.levels):
            raise ValueError("channel counts must be multiples of 32")
        self.table = layers(self.levels)
        self.dims = {name: (cin, cout) for name, cin, cout in self.table}
        self.slots = {}
        off = 0
        shapes = [s for name, cin, cout in self.table for s in ((name + ".w", (cout, 9, cin)), (name + ".b", (cout,)))]
        shapes += [("head.w", (self.levels[0],)), ("head.b", (1,))]
        for key, shape in shapes:
            self.slots[key] = (off, shape)
            off += (int(np.prod(shape)) + 7) // 8 * 8
        self.size = off
        f32 = dict(dtype=torch.float32, device=self.device)
        self.master = torch.zeros(off, **f32)
        self.grad = torch.zeros(off, **f32)
        self.m = torch.zeros(off, **f32)
        self.v = torch.zeros(off, **f32)
        self.wb = torch.zeros(off, dtype=torch.bfloat16, device=self.device)
        self.flipped = {name: torch.empty(cin * 9 * cout, dtype=torch.bfloat16, device=self.device)
                        for name, cin, cout in self.table}
        self.step = 0
        self.load(initial_parameters(self.levels, seed) if params is None else params)

    def _ptr(self, key, buf):
        return buf.data_ptr() + self.slots[key][0] * buf.element_size()

    def parameters(self):
        """The float32 master parameters as float64 NumPy arrays."""
        host = self.master.double().cpu().numpy()
        return {k: host[o:o + int(np.prod(s))].reshape(s).copy() for k, (o, s) in self.slots.items()}

    def gradients(self):
        """The accumulated parameter gradients as float64 NumPy arrays."""
        host = self.grad.double().cpu().numpy()
        return {k: host[o:o + int(np.prod(s))].reshape(s).copy() for k, (o, s) in self.slots.items()}

    def zero_grad(self):
        self.grad.zero_()

    def load(self, params):
        host = np.zeros(self.size, np.float32)
        for k, (o, s) in self.slots.items():
            a = np.asarray(params[k], np.float64)
            if a.shape != s:
                raise ValueError(f"{k}: shape {a.shape}, expected {s}")
            host[o:o + a.size] = a.ravel()
        self.master.copy_(torch.from_numpy(host))
        self.refresh()

    def refresh(self):
        """The bfloat16 copy and the flipped weights from the masters."""
        s = _stream(self.device)
        _call("to_bf16", self.master.data_ptr(), self.wb.data_ptr(), self.size, s)
        self._flip()

    def _flip(self):
        s = _stream(self.device)
        for name, cin, cout in self.table:
            _call("conv3_flip", self._ptr(name + ".w", self.wb), self.flipped[name].data_ptr(), cin, cout, s)

    # ---------------------------------------------------------------- layers

    def _conv(self, ws, name, src, s0, dst, d0, level):
        cin, cout = self.dims[name]
        _call("conv3", _p(src, s0), src.shape[1], self._ptr(name + ".w", self.wb), self._ptr(name + ".b", self.master),
              _p(dst, d0), dst.shape[1], None, 0, ws.batch, ws.height >> level, ws.width >> level, cin, cout, 1, 0,
              _stream(self.device))

    def _wgrad(self, ws, name, src, s0, dz, z0, level):
        cin, cout = self.dims[name]
        _call("conv3_weight_grad", _p(src, s0), src.shape[1], _p(dz, z0), dz.shape[1], self._ptr(name + ".w", self.grad),
              self._ptr(name + ".b", self.grad), ws.batch, ws.height >> level, ws.width >> level, cin, cout,
              _stream(self.device))

    def _dgrad(self, ws, name, dz, z0, dst, mask, level):
        cin, cout = self.dims[name]
        _call("conv3", _p(dz, z0), dz.shape[1], self.flipped[name].data_ptr(), None, dst.data_ptr(), dst.shape[1],
              None if mask is None else mask.data_ptr(), 0 if mask is None else mask.shape[1], ws.batch,
              ws.height >> level, ws.width >> level, cout, cin, 0, 0, _stream(self.device))

    def _pool(self, ws, src, s0, dst, level, c):
        _call("pool", _p(src, s0), src.shape[1], dst.data_ptr(), dst.shape[1], ws.batch, ws.height >> level,
              ws.width >> level, c, _stream(self.device))

    def _up(self, ws, src, dst, level, c):
        _call("upsample", src.data_ptr(), src.shape[1], dst.data_ptr(), dst.shape[1], ws.batch, ws.height >> level,
              ws.width >> level, c, _stream(self.device))

    def forward(self, ws):
        """ws.y = the network applied to ws.x."""
        c1, c2, c3, c4 = self.levels
        self._conv(ws, "enc1a", ws.x, 0, ws.c1a, 0, 0)
        self._conv(ws, "enc1b", ws.c1a, 0, ws.cat1, c2, 0)
        self._pool(ws, ws.cat1, c2, ws.p1, 0, c1)
        self._conv(ws, "enc2a", ws.p1, 0, ws.c2a, 0, 1)
        self._conv(ws, "enc2b", ws.c2a, 0, ws.cat2, c3, 1)
        self._pool(ws, ws.cat2, c3, ws.p2, 1, c2)
        self._conv(ws, "enc3a", ws.p2, 0, ws.c3a, 0, 2)
        self._conv(ws, "enc3b", ws.c3a, 0, ws.cat3, c4, 2)
        self._pool(ws, ws.cat3, c4, ws.p3, 2, c3)
        self._conv(ws, "mid_a", ws.p3, 0, ws.ma, 0, 3)
        self._conv(ws, "mid_b", ws.ma, 0, ws.mb, 0, 3)
        self._up(ws, ws.mb, ws.cat3, 2, c4)
        self._conv(ws, "dec3a", ws.cat3, 0, ws.d3a, 0, 2)
        self._conv(ws, "dec3b", ws.d3a, 0, ws.d3b, 0, 2)
        self._up(ws, ws.d3b, ws.cat2, 1, c3)
        self._conv(ws, "dec2a", ws.cat2, 0, ws.d2a, 0, 1)
        self._conv(ws, "dec2b", ws.d2a, 0, ws.d2b, 0, 1)
        self._up(ws, ws.d2b, ws.cat1, 0, c2)
        self._conv(ws, "dec1a", ws.cat1, 0, ws.d1a, 0, 0)
        self._conv(ws, "dec1b", ws.d1a, 0, ws.d1b, 0, 0)
        _call("head", ws.d1b.data_ptr(), ws.d1b.shape[1], self._ptr("head.w", self.master),
              self._ptr("head.b", self.master), ws.y.data_ptr(), ws.y.numel(), _stream(self.device))
        return ws.y

    def backward(self, ws):
        """Adds the gradients of sum(ws.dy * ws.y) to self.grad (after `forward`)."""
        c1, c2, c3, c4 = self.levels
        s = _stream(self.device)
        B = ws.batch
        _call("head_backward", ws.d1b.data_ptr(), ws.d1b.shape[1], self._ptr("head.w", self.master), ws.dy.data_ptr(),
              ws.g_d1b.data_ptr(), ws.g_d1b.shape[1], self._ptr("head.w", self.grad), self._ptr("head.b", self.grad),
              ws.y.numel(), s)
        self._wgrad(ws, "dec1b", ws.d1a, 0, ws.g_d1b, 0, 0)
        self._dgrad(ws, "dec1b", ws.g_d1b, 0, ws.g_d1a, ws.d1a, 0)
        self._wgrad(ws, "dec1a", ws.cat1, 0, ws.g_d1a, 0, 0)
        self._dgrad(ws, "dec1a", ws.g_d1a, 0, ws.g_cat1, ws.cat1, 0)
        _call("upsample_backward", ws.g_cat1.data_ptr(), ws.g_cat1.shape[1], ws.g_d2b.data_ptr(), c2, B,
              ws.height >> 1, ws.width >> 1, c2, s)
        self._wgrad(ws, "dec2b", ws.d2a, 0, ws.g_d2b, 0, 1)
        self._dgrad(ws, "dec2b", ws.g_d2b, 0, ws.g_d2a, ws.d2a, 1)
        self._wgrad(ws, "dec2a", ws.cat2, 0, ws.g_d2a, 0, 1)
        self._dgrad(ws, "dec2a", ws.g_d2a, 0, ws.g_cat2, ws.cat2, 1)
        _call("upsample_backward", ws.g_cat2.data_ptr(), ws.g_cat2.shape[1], ws.g_d3b.data_ptr(), c3, B,
              ws.height >> 2, ws.width >> 2, c3, s)
        self._wgrad(ws, "dec3b", ws.d3a, 0, ws.g_d3b, 0, 2)
        self._dgrad(ws, "dec3b", ws.g_d3b, 0, ws.g_d3a, ws.d3a, 2)
        self._wgrad(ws, "dec3a", ws.cat3, 0, ws.g_d3a, 0, 2)
        self._dgrad(ws, "dec3a", ws.g_d3a, 0, ws.g_cat3, ws.cat3, 2)
        _call("upsample_backward", ws.g_cat3.data_ptr(), ws.g_cat3.shape[1], ws.g_mb.data_ptr(), c4, B,
              ws.height >> 3, ws.width >> 3, c4, s)
        self._wgrad(ws, "mid_b", ws.ma, 0, ws.g_mb, 0, 3)
        self._dgrad(ws, "mid_b", ws.g_mb, 0, ws.g_ma, ws.ma, 3)
        self._wgrad(ws, "mid_a", ws.p3, 0, ws.g_ma, 0, 3)
        self._dgrad(ws, "mid_a", ws.g_ma, 0, ws.g_p3, None, 3)
        for level, cat, gcat, prev, gprev, first, up_c, c, src, gsrc in (
                (2, ws.cat3, ws.g_cat3, ws.c3a, ws.g_c3a, "enc3", c4, c3, ws.p2, ws.g_p2),
                (1, ws.cat2, ws.g_cat2, ws.c2a, ws.g_c2a, "enc2", c3, c2, ws.p1, ws.g_p1),
                (0, ws.cat1, ws.g_cat1, ws.c1a, ws.g_c1a, "enc1", c2, c1, ws.x, None)):
            dpool = {2: ws.g_p3, 1: ws.g_p2, 0: ws.g_p1}[level]
            _call("pool_backward", _p(gcat, up_c), gcat.shape[1], dpool.data_ptr(), dpool.shape[1], _p(cat, up_c),
                  cat.shape[1], B, ws.height >> level, ws.width >> level, c, s)
            self._wgrad(ws, first + "b", prev, 0, gcat, up_c, level)
            self._dgrad(ws, first + "b", gcat, up_c, gprev, prev, level)
            self._wgrad(ws, first + "a", src, 0, gprev, 0, level)
            if gsrc is not None:
                self._dgrad(ws, first + "a", gprev, 0, gsrc, None, level)

    # ---------------------------------------------------------------- training

    def pack(self, ws, resid, offsets, ld_resid, psf, ld_psf, scale_resid=1.0, scale_psf=1.0):
        """ws.x from residual patches at `offsets` (device int64) of `resid`
        and the PSF patch `psf` (float32 device tensors)."""
        _call("pack", resid.data_ptr(), offsets.data_ptr(), ld_resid, psf.data_ptr(), ld_psf, float(scale_resid),
              float(scale_psf), ws.x.data_ptr(), ws.batch, ws.height, ws.width, _stream(self.device))

    def loss_and_grad(self, ws, target, offsets, ld_target):
        """ws.loss += the mean squared error of ws.y, ws.dy its gradient."""
        _call("mse", ws.y.data_ptr(), target.data_ptr(), offsets.data_ptr(), ld_target, ws.dy.data_ptr(),
              ws.loss.data_ptr(), ws.batch, ws.height, ws.width, _stream(self.device))

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        """One Adam step on all parameters; clears the gradients."""
        self.step += 1
        s = _stream(self.device)
        _call("adam", self.master.data_ptr(), self.wb.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
              self.v.data_ptr(), self.size, float(lr), float(beta1), float(beta2), float(eps), self.step, s)
        self._flip()

    def train_step(self, ws, resid, target, psf, offsets, lr):
        """One step on the patches at `offsets` of the (N, PATCH, PATCH)
        residual and target tensors with the PSF patch `psf`."""
        ws.loss.zero_()
        self.pack(ws, resid, offsets, ws.width, psf, ws.width)
        self.forward(ws)
        self.loss_and_grad(ws, target, offsets, ws.width)
        self.backward(ws)
        self.adam(lr)


# -------------------------------------------------------------------- data


class TrainingSet:
    """Patches on the GPU: residuals in units of the PSF peak and targets
    (true sky minus model) in sky units, (N, PATCH, PATCH) float32; the PSF
    patch (peak 1) of each coverage and the coverage of every patch."""

    def __init__(self, resid, target, psf, coverage, info):
        self.resid, self.target, self.psf, self.coverage, self.info = resid, target, psf, coverage, info

    def __len__(self):
        return int(self.resid.shape[0])


def psf_patch(psf, patch=PATCH):
    """The central patch of a PSF image, divided by its peak, and the peak."""
    n0, n1 = psf.shape
    peak = psf[n0 // 2, n1 // 2]
    crop = psf[n0 // 2 - patch // 2:n0 // 2 + patch // 2, n1 // 2 - patch // 2:n1 // 2 + patch // 2]
    return (crop / peak).contiguous().float(), float(peak)


def _patches(img, patch=PATCH):
    n0, n1 = img.shape
    return img.reshape(n0 // patch, patch, n1 // patch, patch).permute(0, 2, 1, 3).reshape(-1, patch, patch)


def make_training_set(device, n_patches=20000, n_coverages=8, nant=(32, 64), npix=2048, cell_arcsec=1.5, ntime=128,
                      nchan=64, snapshots=(0, 4, 12, 30), sigma=0.05, seed=1000, epsilon=1e-5, sky=None):
    """`n_patches` training patches from seeded random skies (by default the
    FISTA measurement's distribution: 300 point sources and 40 Gaussians on
    npix^2; `sky` overrides `synth.extended_sky`'s keywords) over
    `n_coverages` random subsets of 32-64 antennas of the 64-antenna array,
    each sky predicted by the GPU degridder with noise `sigma` and imaged by
    the gridder; the models are plain FISTA iterates at the `snapshots`
    iteration counts (0: the dirty image)."""
    from . import wgrid_torch

    dev = torch.device(device)
    sky_kw = dict(sky or {})
    cell = cell_arcsec * synth.ARCSEC
    per_sky = len(snapshots) * (npix // PATCH) ** 2
    skies = max(1, math.ceil(n_patches / (per_sky * n_coverages)))
    resid = torch.empty((n_patches, PATCH, PATCH), dtype=torch.float32, device=dev)
    target = torch.empty_like(resid)
    psfs = []
    coverage = np.zeros(n_patches, np.int64)
    filled = 0
    info = {"coverages": [], "skies": 0}
    for c in range(n_coverages):
        rng = np.random.default_rng(seed + c)
        na = int(rng.integers(nant[0], nant[1] + 1))
        subset = rng.choice(64, na, replace=False)
        uvw = torch.from_numpy(synth.uvw_tracks(nant=64, ntime=ntime, subset=subset)).to(dev)
        freq = synth.channels(nchan)
        plan = wgrid_torch.DevicePlan(uvw, freq, npix_x=npix, npix_y=npix, pixsize_x=cell, pixsize_y=cell,
                                      epsilon=epsilon, single=True)
        pp, peak = psf_patch(plan.grid(None))
        psfs.append(pp)
        lmax, _ = fista.power_iteration(plan.gram, plan.shape, dev, max_iterations=30)
        info["coverages"].append({"antennas": na, "visibilities": int(uvw.shape[0]) * nchan, "psf_peak": peak,
                                  "lmax": lmax})
        g = torch.Generator(device=dev)
        g.manual_seed(seed + 7919 * (c + 1))
        for k in range(skies):
            if filled >= n_patches:
                break
            truth = torch.from_numpy(synth.extended_sky(npix, seed=seed + 100 * c + k + 1, **sky_kw)).to(dev)
            vis = plan.degrid(truth)
            vis += sigma * math.sqrt(2.0) * torch.randn(vis.shape, dtype=vis.dtype, device=dev, generator=g)
            dirty, q = plan.residual(vis, None)
            del vis
            snaps = fista.solve(plan.gram, dirty, 1e-4 * float(dirty.max()), 1.0 / lmax, max(snapshots),
                                q0=0.5 * q, keep=snapshots).snapshots
            for it in snapshots:
                x, gx = snaps[it]
                r = _patches((dirty - gx) / peak)
                e = _patches(truth - x)
                n = min(r.shape[0], n_patches - filled)
                resid[filled:filled + n] = r[:n]
                target[filled:filled + n] = e[:n]
                coverage[filled:filled + n] = c
                filled += n
            info["skies"] += 1
        plan.close()
    if filled < n_patches:
        resid, target, coverage = resid[:filled], target[:filled], coverage[:filled]
    return TrainingSet(resid, target, torch.stack(psfs), coverage, info)


def train(net, data, steps, batch=16, lr=1e-3, lr_final=1e-5, warmup=50, seed=0, log_every=25):
    """`steps` Adam steps on random batches of one coverage at a time
    (cosine learning-rate decay after a linear warm-up). Returns the loss
    every `log_every` steps."""
    rng = np.random.default_rng(seed)
    ws = Workspace(net, batch, PATCH, PATCH, training=True)
    groups = [np.flatnonzero(data.coverage == c) for c in range(data.psf.shape[0])]
    sizes = np.array([len(gr) for gr in groups], np.float64)
    cov = rng.choice(len(groups), size=steps, p=sizes / sizes.sum())
    idx = np.stack([rng.choice(groups[c], batch, replace=len(groups[c]) < batch) for c in cov])
    offsets = torch.from_numpy(idx * PATCH * PATCH).to(net.device)
    losses = []
    for t in range(steps):
        if t < warmup:
            rate = lr * (t + 1) / warmup
        else:
            rate = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * (t - warmup) / max(1, steps - warmup)))
        net.train_step(ws, data.resid, data.target, data.psf[cov[t]], offsets[t], rate)
        if t % log_every == 0 or t == steps - 1:
            losses.append((t, float(ws.loss)))
    return losses


# -------------------------------------------------------------------- inference


def tiles(npix, patch=PATCH, margin=16):
    """Patch corners along one axis and the window of each patch (patch
    coordinates) such that the windows tile [0, npix) once: neighbouring
    patches overlap by at least 2 margin and split the overlap in half."""
    if npix < patch:
        raise ValueError("the image is smaller than a patch")
    step = patch - 2 * margin
    pos = list(range(0, npix - patch, step)) + [npix - patch]
    pos = sorted(set(pos))
    cuts = [0] + [(a + b + patch) // 2 for a, b in zip(pos[:-1], pos[1:])] + [npix]
    return [(p, cuts[i] - p, cuts[i + 1] - p) for i, p in enumerate(pos)]


class Proposer:
    """The network over an npix x npix residual image in overlapping
    patches (one batch): update = U(residual * scale, PSF patch)."""

    def __init__(self, net, npix, margin=16):
        self.net, self.npix = net, int(npix)
        ax = tiles(self.npix, PATCH, margin)
        corners = [(a, b) for a in ax for b in ax]
        self.batch = len(corners)
        self.ws = Workspace(net, self.batch, PATCH, PATCH, training=False)
        offs = np.array([a[0] * self.npix + b[0] for a, b in corners], np.int64)
        win = np.array([[a[1], a[2], b[1], b[2]] for a, b in corners], np.int32).ravel()
        self.ws.offsets.copy_(torch.from_numpy(offs))
        self.windows = torch.from_numpy(win).to(net.device)

    def __call__(self, resid, psf, scale, out=None):
        resid = resid.float().contiguous()
        if tuple(resid.shape) != (self.npix, self.npix):
            raise ValueError("residual image size")
        if out is None:
            out = torch.empty_like(resid)
        self.net.pack(self.ws, resid, self.ws.offsets, self.npix, psf, PATCH, scale, 1.0)
        self.net.forward(self.ws)
        _call("unpack", self.ws.y.data_ptr(), self.ws.offsets.data_ptr(), self.windows.data_ptr(), self.npix, 1.0,
              out.data_ptr(), self.batch, PATCH, PATCH, _stream(self.net.device))
        return out


def _blur(img, sigma):
    """The periodic Gaussian blur of standard deviation `sigma` pixels (the
    library's cuFFT low-pass)."""
    return fista.gaussian_lowpass(img.float(), sigma)


class LearnedSolve:
    """The outcome of `solve`: the iterate `x` and `gx` = G x, the applies of
    G made, the proposal statistics, the misfit after each apply (`misfits`,
    a float64 CUDA tensor, NaN where an apply was a proposal's) and, with
    `events`, a CUDA event recorded after each apply's iteration."""

    def __init__(self, x, gx, applies, stats, misfits, events):
        self.x, self.gx, self.applies, self.stats, self.misfits, self.events = x, gx, applies, stats, misfits, events

    def __iter__(self):  # (x, G x, applies, statistics), as the earlier tuple
        return iter((self.x, self.gx, self.applies, self.stats))


def solve(gram, dirty, lam, step, proposer, psf, peak, max_iterations, q0=0.0, cycle=40, bands=2, sigma=4.0,
          first=0, stop=None, observer=None, events=False, check_every=20):
    """Learned-preconditioned FISTA on the misfit Q(x) = Q(0) - <dirty, x> +
    <x, G x> / 2 with the L1 prior and positivity (the FISTA of `rang.fista`,
    with gradient restart), where at iteration `first` and every `cycle`
    iterations after it the network proposes an update from the residual:
    d = max(x + U(r / peak, psf), 0) - x. With `bands` 1 the step is alpha d,
    alpha = <d, r> / <d, G d> the exact minimiser of Q along d (one apply of
    the exact gridder's G); with `bands` 2, d is split into its Gaussian
    low-pass part (`sigma` pixels) and the rest, each scaled by the exact
    minimiser of Q over the pair (two applies). The step is kept only when
    Q decreases, and then shifts the iterate, the previous iterate and the
    extrapolated point alike, so that FISTA's momentum carries on.

    The plain iterations run on the library's step kernels with their
    scalars on the device; a proposal reads its inner products back (one
    wait per proposal). `stop(k, misfit)` is tested on the recorded misfits
    every `check_every` applies (k counts applies of G) and `observer(k, x,
    gx, misfit)` sees every iterate (a wait each). Returns a `LearnedSolve`
    (which unpacks as (x, G x, applies, proposal statistics))."""
    lib = fista._library()
    dev = dirty.device
    single = fista._single(dirty)
    n = dirty.numel()
    s = fista._stream(dev)
    ws = fista.Workspace(dev)
    x = torch.zeros_like(dirty)
    y = x.clone()
    g_x_prev = torch.zeros_like(dirty)
    g_x = torch.empty_like(dirty)
    x_next = torch.empty_like(dirty)
    y_next = torch.empty_like(dirty)
    state = torch.empty(fista._STATE, dtype=torch.float64, device=dev)
    q0_dev = q0.to(dev, torch.float64).reshape(()) if torch.is_tensor(q0) else None
    fista._check(lib.rang_b200_fista_init(state.data_ptr(), None if q0_dev is None else q0_dev.data_ptr(),
                                          0.0 if q0_dev is not None else float(q0), float(step), float(lam), 0, 0.0,
                                          s), "fista init")
    q0v = q0_dev if q0_dev is not None else torch.tensor(float(q0), dtype=torch.float64, device=dev)
    misfits = torch.full((max_iterations + 1,), float("nan"), dtype=torch.float64, device=dev)
    iters = torch.full((max_iterations + 1,), float("nan"), dtype=torch.float64, device=dev)
    evs = []
    applies = 0
    stats = {"proposals": 0, "accepted": 0, "steps": [], "misfit_drops": []}
    k = 0
    checked = 0

    def host_dot(a, b):
        return float(fista.dot(a, b, ws=ws))

    while True:
        g_y = gram(y)
        applies += 1
        if k >= first and (k - first) % cycle == 0 and applies + bands <= max_iterations:
            # G x and the misfit of the current iterate (beta from the device state).
            beta = state[1].to(dirty.dtype)
            gx_now = torch.where(beta == 0, g_y, (g_y + beta * g_x_prev) / (1.0 + beta))
            misfit = float(fista.misfit_of(dirty, x, gx_now, q0v, ws))
            r = dirty - gx_now
            d = torch.clamp(x + proposer(r, psf, 1.0 / peak), min=0.0) - x
            parts = [d] if bands == 1 else [_blur(d, sigma), None]
            if bands != 1:
                parts[1] = d - parts[0]
            gparts = [gram(p) for p in parts]
            applies += len(parts)
            stats["proposals"] += 1
            b = np.array([host_dot(p, r) for p in parts])
            m = np.array([[host_dot(p, q) for q in gparts] for p in parts])
            try:
                coef = np.linalg.solve(m, b)
            except np.linalg.LinAlgError:
                coef = np.zeros(len(parts))
            drop = float(coef @ b - 0.5 * coef @ m @ coef)
            if np.all(np.isfinite(coef)) and drop > 0.0:
                shift = sum(c * p for c, p in zip(coef, parts))
                gshift = sum(c * g for c, g in zip(coef, gparts))
                x_try, g_try = x + shift, gx_now + gshift
                m_try = float(fista.misfit_of(dirty, x_try, g_try, q0v, ws))
                if m_try < misfit:
                    stats["accepted"] += 1
                    stats["steps"].append([round(float(c), 4) for c in coef])
                    stats["misfit_drops"].append(misfit - m_try)
                    # The iterate, the previous iterate's G and the extrapolated
                    # point move alike; the step kernel forms G x from them.
                    x = x_try
                    g_x_prev = g_x_prev + gshift
                    y, g_y = y + shift, g_y + gshift
        fista._check(lib.rang_b200_fista_step(single, n, dirty.data_ptr(), x.data_ptr(), y.data_ptr(), g_y.data_ptr(),
                                              g_x_prev.data_ptr(), g_x.data_ptr(), x_next.data_ptr(),
                                              y_next.data_ptr(), state.data_ptr(), iters.data_ptr(), k, 0, 1, 1,
                                              ws.partials.data_ptr(), s), "fista step")
        misfits[applies:applies + 1].copy_(iters[k:k + 1])
        if events:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            evs.append((applies, e))
        if observer is not None:
            observer(applies, x, g_x, float(misfits[applies]))
        done = applies >= max_iterations
        if not done and stop is not None and applies - checked >= check_every:
            vals = misfits[checked + 1:applies + 1].tolist()
            done = any(stop(checked + 1 + j, v) for j, v in enumerate(vals) if v == v)
            checked = applies
        if done:
            return LearnedSolve(x, g_x, applies, stats, misfits[:applies + 1], evs)
        x, x_next = x_next, x
        g_x_prev, g_x = g_x, g_x_prev
        y, y_next = y_next, y
        k += 1
