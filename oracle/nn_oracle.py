"""CPU oracle of the learned proposal network (test infrastructure only:
imported by tests/ and the benchmark's checks, never by the library).

A float64 NumPy restatement of the U-Net that `rang.learned` runs on the GPU
through include/rang_nn.h, layer by layer, forward and backward, in the same
NHWC layout with weights [cout][9][cin]. The reference has no such network
(its learned-stage interpreter, core/src/learned_interp.rs:1-22, runs NCHW
f32 convolutions of a dilated CNN; examples/dl4b_train.py:51-72 trains one in
PyTorch): this oracle pins the network by its own mathematics — its
gradients are checked against central finite differences in float64 — and
then checks the GPU kernels. With `emulate=True` every tensor the GPU stores
in bfloat16 is rounded to bfloat16 (round to nearest even) at the same point,
so that the GPU and the oracle differ only by float32 summation order.
"""

import numpy as np

LEVELS = (32, 64, 128, 256)
IN_CHANNELS = 32


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(levels=LEVELS, in_channels=IN_CHANNELS):
    """The 3x3 convolutions in order: (name, cin, cout). The decoder input at
    level l is [upsampled level l+1 output | level l encoder output]."""
    c1, c2, c3, c4 = levels
    return [("enc1a", in_channels, c1), ("enc1b", c1, c1), ("enc2a", c1, c2), ("enc2b", c2, c2),
            ("enc3a", c2, c3), ("enc3b", c3, c3), ("mid_a", c3, c4), ("mid_b", c4, c4),
            ("dec3a", c4 + c3, c3), ("dec3b", c3, c3), ("dec2a", c3 + c2, c2), ("dec2b", c2, c2),
            ("dec1a", c2 + c1, c1), ("dec1b", c1, c1)]


def init(levels=LEVELS, in_channels=IN_CHANNELS, live_inputs=2, seed=0):
    """He-normal weights (fan-in 9 cin; the first layer counts its
    `live_inputs` channels), zero biases, a small head."""
    rng = np.random.default_rng(seed)
    p = {}
    for i, (name, cin, cout) in enumerate(layers(levels, in_channels)):
        fan = 9 * (live_inputs if i == 0 else cin)
        p[name + ".w"] = rng.standard_normal((cout, 9, cin)) * np.sqrt(2.0 / fan)
        p[name + ".b"] = np.zeros(cout)
    p["head.w"] = rng.standard_normal(levels[0]) * np.sqrt(1.0 / levels[0])
    p["head.b"] = np.zeros(1)
    return p


def _shift(x, dy, dx):
    """x[b, y + dy, x + dx, :] with zeros outside the image."""
    out = np.zeros_like(x)
    H, W = x.shape[1], x.shape[2]
    ys, yd = (slice(dy, H), slice(0, H - dy)) if dy >= 0 else (slice(0, H + dy), slice(-dy, H))
    xs, xd = (slice(dx, W), slice(0, W - dx)) if dx >= 0 else (slice(0, W + dx), slice(-dx, W))
    out[:, yd, xd, :] = x[:, ys, xs, :]
    return out


def conv3(x, w, b=None):
    """out[p, co] = b[co] + sum_{tap, ci} w[co, tap, ci] x[p + (ky - 1, kx - 1), ci]."""
    out = np.zeros(x.shape[:3] + (w.shape[0],))
    for tap in range(9):
        out += _shift(x, tap // 3 - 1, tap % 3 - 1) @ w[:, tap, :].T
    if b is not None:
        out += b
    return out


def conv3_input_grad(dz, w):
    """The gradient of conv3 with respect to its input."""
    out = np.zeros(dz.shape[:3] + (w.shape[2],))
    for tap in range(9):
        out += _shift(dz @ w[:, tap, :], -(tap // 3 - 1), -(tap % 3 - 1))
    return out


def conv3_weight_grad(x, dz):
    """dw[co, tap, ci] = sum_p dz[p, co] x[p + off(tap), ci]."""
    dw = np.zeros((dz.shape[3], 9, x.shape[3]))
    dzf = dz.reshape(-1, dz.shape[3])
    for tap in range(9):
        dw[:, tap, :] = dzf.T @ _shift(x, tap // 3 - 1, tap % 3 - 1).reshape(-1, x.shape[3])
    return dw


def pool(x):
    B, H, W, C = x.shape
    v = x.reshape(B, H // 2, 2, W // 2, 2, C)
    return 0.25 * (((v[:, :, 0, :, 0] + v[:, :, 0, :, 1]) + v[:, :, 1, :, 0]) + v[:, :, 1, :, 1])


def upsample(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def upsample_backward(g):
    B, H, W, C = g.shape
    v = g.reshape(B, H // 2, 2, W // 2, 2, C)
    return ((v[:, :, 0, :, 0] + v[:, :, 0, :, 1]) + v[:, :, 1, :, 0]) + v[:, :, 1, :, 1]


def pack(resid, psf, scale_resid=1.0, scale_psf=1.0, in_channels=IN_CHANNELS):
    """(B, H, W) residual patches and an (H, W) PSF patch -> the network input."""
    B, H, W = resid.shape
    x = np.zeros((B, H, W, in_channels))
    x[..., 0] = np.asarray(resid, np.float32) * np.float32(scale_resid)
    x[..., 1] = np.asarray(psf, np.float32)[None] * np.float32(scale_psf)
    return x


def forward(p, x, emulate=False, levels=LEVELS):
    """The network output (B, H, W) and the activations the backward needs."""
    r = bf16 if emulate else (lambda v: v)
    if emulate:
        x = bf16(x)
        p = {k: (bf16(v) if k.endswith(".w") and not k.startswith("head") else v) for k, v in p.items()}

    def c(name, inp):
        return r(np.maximum(conv3(inp, p[name + ".w"], p[name + ".b"]), 0.0))

    a = {"x": x}
    a["c1a"] = c("enc1a", x)
    a["e1"] = c("enc1b", a["c1a"])
    a["p1"] = r(pool(a["e1"]))
    a["c2a"] = c("enc2a", a["p1"])
    a["e2"] = c("enc2b", a["c2a"])
    a["p2"] = r(pool(a["e2"]))
    a["c3a"] = c("enc3a", a["p2"])
    a["e3"] = c("enc3b", a["c3a"])
    a["p3"] = r(pool(a["e3"]))
    a["ma"] = c("mid_a", a["p3"])
    a["mb"] = c("mid_b", a["ma"])
    a["cat3"] = np.concatenate([upsample(a["mb"]), a["e3"]], axis=3)
    a["d3a"] = c("dec3a", a["cat3"])
    a["d3b"] = c("dec3b", a["d3a"])
    a["cat2"] = np.concatenate([upsample(a["d3b"]), a["e2"]], axis=3)
    a["d2a"] = c("dec2a", a["cat2"])
    a["d2b"] = c("dec2b", a["d2a"])
    a["cat1"] = np.concatenate([upsample(a["d2b"]), a["e1"]], axis=3)
    a["d1a"] = c("dec1a", a["cat1"])
    a["d1b"] = c("dec1b", a["d1a"])
    y = a["d1b"] @ p["head.w"] + p["head.b"][0]
    if emulate:
        y = y.astype(np.float32).astype(np.float64)
    a["p"] = p
    return y, a


def mse(y, target):
    d = y - target
    return float(np.mean(d * d)), 2.0 * d / d.size


def backward(a, dy, emulate=False, levels=LEVELS):
    """Gradients of sum(dy * y) with respect to every parameter."""
    r = bf16 if emulate else (lambda v: v)
    p = a["p"]
    c1, c2, c3, c4 = levels
    g = {}

    def conv_back(name, inp, dz, mask=None, need_input=True):
        g[name + ".w"] = conv3_weight_grad(inp, dz)
        g[name + ".b"] = dz.sum(axis=(0, 1, 2))
        if not need_input:
            return None
        d = conv3_input_grad(dz, p[name + ".w"])
        if mask is not None:
            d = np.where(mask > 0, d, 0.0)
        return r(d)

    d1b = a["d1b"]
    g["head.w"] = np.einsum("bhw,bhwc->c", dy, d1b)
    g["head.b"] = np.array([dy.sum()])
    gz = r(np.where(d1b > 0, dy[..., None] * p["head.w"], 0.0))
    gz = conv_back("dec1b", a["d1a"], gz, a["d1a"])
    gcat1 = conv_back("dec1a", a["cat1"], gz, a["cat1"])
    gz = r(upsample_backward(gcat1[..., :c2]))
    gz = conv_back("dec2b", a["d2a"], gz, a["d2a"])
    gcat2 = conv_back("dec2a", a["cat2"], gz, a["cat2"])
    gz = r(upsample_backward(gcat2[..., :c3]))
    gz = conv_back("dec3b", a["d3a"], gz, a["d3a"])
    gcat3 = conv_back("dec3a", a["cat3"], gz, a["cat3"])
    gz = r(upsample_backward(gcat3[..., :c4]))
    gz = conv_back("mid_b", a["ma"], gz, a["ma"])
    gp = conv_back("mid_a", a["p3"], gz)
    ge = r(np.where(a["e3"] > 0, gcat3[..., c4:] + 0.25 * upsample(gp), 0.0))
    gz = conv_back("enc3b", a["c3a"], ge, a["c3a"])
    gp = conv_back("enc3a", a["p2"], gz)
    ge = r(np.where(a["e2"] > 0, gcat2[..., c3:] + 0.25 * upsample(gp), 0.0))
    gz = conv_back("enc2b", a["c2a"], ge, a["c2a"])
    gp = conv_back("enc2a", a["p1"], gz)
    ge = r(np.where(a["e1"] > 0, gcat1[..., c2:] + 0.25 * upsample(gp), 0.0))
    gz = conv_back("enc1b", a["c1a"], ge, a["c1a"])
    conv_back("enc1a", a["x"], gz, need_input=False)
    return g


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step with bias-corrected moments (in place on p, m, v)."""
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] ** 2
        p[k] = p[k] - lr * (m[k] / (1 - b1**step)) / (np.sqrt(v[k] / (1 - b2**step)) + eps)
