"""The learned proposal network (rang.learned over include/rang_nn.h): the
float64 oracle (oracle/nn_oracle.py) pinned by finite differences; every GPU
layer, the whole network's output and parameter gradients against the
oracle with bfloat16 rounding emulated at the GPU's storage points;
training through the library's kernels; and learned-preconditioned FISTA
against plain FISTA on the same measurement."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import nn_oracle as nno

REPO = Path(__file__).resolve().parents[1]


def _fd_case(seed=1):
    lv = (4, 6, 8, 10)
    p = nno.init(lv, in_channels=3, live_inputs=2, seed=seed)
    rng = np.random.default_rng(seed + 1)
    x = rng.standard_normal((2, 16, 16, 3))
    x[..., 2] = 0.0
    t = rng.standard_normal((2, 16, 16))
    return lv, p, x, t, rng


def test_oracle_gradients_match_finite_differences():
    lv, p, x, t, rng = _fd_case()

    def loss(q):
        return nno.mse(nno.forward(q, x, levels=lv)[0], t)[0]

    y, act = nno.forward(p, x, levels=lv)
    g = nno.backward(act, nno.mse(y, t)[1], levels=lv)
    eps = 1e-6
    for keys in (list(p), ["enc1a.w"], ["mid_b.b"], ["dec3a.w"], ["enc2b.w"], ["head.w"]):
        v = {k: (rng.standard_normal(p[k].shape) if k in keys else np.zeros_like(p[k])) for k in p}
        fd = (loss({k: p[k] + eps * v[k] for k in p}) - loss({k: p[k] - eps * v[k] for k in p})) / (2 * eps)
        an = sum(float((g[k] * v[k]).sum()) for k in keys)
        assert abs(fd - an) <= 1e-7 * abs(an) + 1e-12, (keys, fd, an)


def test_oracle_bf16_rounding():
    got = nno.bf16(np.array([1.0, 1.00390625, 1.005859375, -2.5, 1.0 + 2.0**-7, 3.0e-39]))
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0078125 and got[3] == -2.5
    assert got[4] == 1.0078125
    assert abs(got[5] - 3.0e-39) <= 2.0**-134  # subnormal: half a bfloat16 spacing


def test_oracle_emulation_is_a_small_perturbation():
    lv, p, x, t, _ = _fd_case(3)
    y, _ = nno.forward(p, x, levels=lv)
    ye, _ = nno.forward(p, x, emulate=True, levels=lv)
    assert 0 < np.abs(y - ye).max() <= 0.05 * np.abs(y).max()


def test_library_exports_every_nn_symbol():
    from rang import core

    text = (REPO / "include" / "rang_nn.h").read_text()
    names = sorted(set(re.findall(r"^\w+\s+(rang_b200_nn_\w+)\s*\(", text, re.M)))
    assert len(names) == 17
    lib = ctypes.CDLL(core.library_path())
    for name in names:
        assert hasattr(lib, name), name


def test_entry_points_refuse_bad_shapes_without_a_gpu():
    from rang import learned

    with pytest.raises(ValueError, match="conv3"):
        learned._call("conv3", 16, 32, 16, None, 16, 32, None, 0, 1, 8, 8, 30, 32, 1, 0, None)
    with pytest.raises(ValueError, match="conv3"):
        learned._call("conv3", 16, 36, 16, None, 16, 32, None, 0, 1, 8, 8, 32, 32, 1, 0, None)
    with pytest.raises(ValueError, match="pool"):
        learned._call("pool", 16, 8, 16, 8, 1, 7, 8, 8, None)
    with pytest.raises(ValueError, match="adam"):
        learned._call("adam", 16, None, 16, 16, 16, 8, 1e-3, 0.9, 0.999, 1e-8, 0, None)


@pytest.mark.parametrize("npix", [256, 300, 512, 2048])
def test_tiles_cover_the_image_once(npix):
    from rang import learned

    ax = learned.tiles(npix)
    cover = np.zeros(npix, int)
    for pos, lo, hi in ax:
        assert 0 <= lo < hi <= learned.PATCH and pos + learned.PATCH <= npix
        cover[pos + lo:pos + hi] += 1
        if pos > 0:
            assert lo >= 16
        if pos + learned.PATCH < npix:
            assert hi <= learned.PATCH - 16
    assert (cover == 1).all()


def test_initial_parameters_follow_the_oracle_definition():
    from rang import learned

    a = learned.initial_parameters(seed=5)
    b = nno.init(seed=5)
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


# ------------------------------------------------------------------ GPU


def _bf16_tensor(a, dev):
    import torch

    return torch.from_numpy(np.asarray(a, np.float32)).to(dev).to(torch.bfloat16)


def _close_bf16(got, ref):
    # equal up to one bfloat16 unit where float32 and float64 sums round differently
    return bool((np.abs(got - ref) <= 2.0**-7 * np.abs(ref)).all())


def _np(t):
    import torch

    return t.to(torch.float64).cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,relu,offset", [(32, 32, 1, 0), (64, 64, 0, 32), (96, 32, 1, 0), (32, 128, 1, 0)])
def test_conv3_matches_the_oracle(cin, cout, relu, offset):
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(cin + cout)
    B, H, W = 2, 24, 40
    wide = cin + offset
    x = nno.bf16(rng.standard_normal((B, H, W, wide)))
    w = nno.bf16(rng.standard_normal((cout, 9, cin)) / np.sqrt(9 * cin))
    b = rng.standard_normal(cout).astype(np.float32)
    xt = _bf16_tensor(x.reshape(-1, wide), dev)
    wt = _bf16_tensor(w, dev)
    bt = torch.from_numpy(b).to(dev)
    out = torch.zeros((B * H * W, cout + 8), dtype=torch.bfloat16, device=dev)
    learned._call("conv3", learned._p(xt, offset), wide, wt.data_ptr(), bt.data_ptr(), out.data_ptr(), cout + 8,
                  None, 0, B, H, W, cin, cout, relu, 0, torch.cuda.current_stream().cuda_stream)
    ref = nno.conv3(x[..., offset:], w, b.astype(np.float64))
    if relu:
        ref = np.maximum(ref, 0.0)
    got = _np(out)[:, :cout].reshape(ref.shape)
    assert np.abs(got - nno.bf16(ref)).max() <= 2.0**-7 * np.abs(ref).max()
    assert np.abs(got - ref).max() <= 2.0**-8 * np.abs(ref).max() + 2.0**-8 * np.abs(ref).max()
    assert (_np(out)[:, cout:] == 0).all()


@pytest.fixture
def conv_path():
    """The process-wide convolution kernel choice, restored afterwards."""
    from rang import learned

    lib = learned._library()
    old = lib.rang_b200_nn_set_conv_path(0)
    yield lib
    lib.rang_b200_nn_set_conv_path(old)


@pytest.mark.gpu
def test_a_tcgen05_wait_that_runs_out_reports_status_3_and_the_context_stays_usable(conv_path):
    """The convolutions' bounded wait, run out on purpose: one block holds TMEM
    and waits 20 ms on an mbarrier that nothing completes; the wait gives up,
    the block frees its TMEM, and the host reads status 3 once (the flag is
    then cleared). A tcgen05 convolution afterwards runs with status 0."""
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    assert conv_path.rang_b200_nn_device_status(s) == 0
    assert conv_path.rang_b200_nn_wait_probe(-1, s) == 1
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    assert conv_path.rang_b200_nn_wait_probe(20_000_000, s) == 0
    t1.record()
    assert conv_path.rang_b200_nn_device_status(s) == 3
    assert t0.elapsed_time(t1) >= 19.0
    assert conv_path.rang_b200_nn_device_status(s) == 0
    rng = np.random.default_rng(0)
    cin = cout = 64
    x = nno.bf16(rng.standard_normal((1, 8, 16, cin)))
    w = nno.bf16(rng.standard_normal((cout, 9, cin)) / np.sqrt(9 * cin))
    b = np.zeros(cout, np.float32)
    xt, wt, bt = _bf16_tensor(x.reshape(-1, cin), dev), _bf16_tensor(w, dev), torch.from_numpy(b).to(dev)
    out = torch.zeros((8 * 16, cout), dtype=torch.bfloat16, device=dev)
    learned._call("conv3", xt.data_ptr(), cin, wt.data_ptr(), bt.data_ptr(), out.data_ptr(), cout, None, 0, 1, 8, 16,
                  cin, cout, 0, 0, s)
    assert conv_path.rang_b200_nn_device_status(s) == 0
    ref = nno.conv3(x, w, b.astype(np.float64))
    assert np.abs(_np(out).reshape(1, 8, 16, cout) - ref).max() <= 2.0**-7 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,B,H,W", [(64, 64, 1, 8, 16), (32, 32, 1, 8, 16), (64, 128, 2, 16, 32),
                                            (96, 32, 2, 16, 16), (384, 128, 1, 16, 16), (128, 384, 1, 8, 16),
                                            (256, 256, 2, 32, 32), (32, 64, 1, 64, 64)],
                         ids=lambda v: str(v))
def test_conv3_tcgen05_matches_the_oracle_and_mma_sync(conv_path, cin, cout, B, H, W):
    """The tcgen05 kernel (TMA boxes with zero fill for the padding, TMEM
    accumulator) on shapes it takes: within one bfloat16 unit of the FP64
    oracle like the mma.sync kernel, within one unit of the mma.sync kernel's
    output, with no wait given up (device status 0)."""
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(cin * 3 + cout + H)
    x = nno.bf16(rng.standard_normal((B, H, W, cin)))
    w = nno.bf16(rng.standard_normal((cout, 9, cin)) / np.sqrt(9 * cin))
    b = rng.standard_normal(cout).astype(np.float32)
    xt, wt, bt = _bf16_tensor(x.reshape(-1, cin), dev), _bf16_tensor(w, dev), torch.from_numpy(b).to(dev)
    outs = []
    for path in (0, 1):
        conv_path.rang_b200_nn_set_conv_path(path)
        out = torch.zeros((B * H * W, cout), dtype=torch.bfloat16, device=dev)
        learned._call("conv3", xt.data_ptr(), cin, wt.data_ptr(), bt.data_ptr(), out.data_ptr(), cout, None, 0, B, H,
                      W, cin, cout, 1, 0, s)
        assert conv_path.rang_b200_nn_device_status(s) == 0
        outs.append(_np(out).reshape(B, H, W, cout))
    ref = np.maximum(nno.conv3(x, w, b.astype(np.float64)), 0.0)
    scale = np.abs(ref).max()
    assert np.abs(outs[0] - ref).max() <= 2.0**-7 * scale
    assert np.abs(outs[0] - outs[1]).max() <= 2.0**-7 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,B,H,W", [(64, 64, 1, 8, 16), (32, 32, 1, 8, 16), (64, 128, 2, 16, 32),
                                            (192, 64, 1, 16, 16), (96, 32, 1, 16, 16), (32, 64, 2, 16, 32),
                                            (64, 32, 1, 8, 16), (128, 384, 1, 8, 16), (256, 256, 2, 32, 32),
                                            (384, 128, 2, 64, 64)],
                         ids=lambda v: str(v))
def test_conv3_weight_grad_tcgen05_matches_the_oracle_and_mma_sync(conv_path, cin, cout, B, H, W):
    """The tcgen05 weight gradient (MN-major TMA operands, K = pixels, TMEM
    accumulator, vector atomics into dw) where cout is a multiple of 64, the
    mma.sync kernel for the 32-output-channel cases: within 1e-5 of the FP64
    oracle and of the mma.sync kernel, accumulating, with no wait given up."""
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(cin + 5 * cout + W)
    x = nno.bf16(np.maximum(rng.standard_normal((B, H, W, cin)), 0.0))
    dz = nno.bf16(rng.standard_normal((B, H, W, cout)))
    xt, dzt = _bf16_tensor(x.reshape(-1, cin), dev), _bf16_tensor(dz.reshape(-1, cout), dev)
    got = []
    for path in (0, 1):
        conv_path.rang_b200_nn_set_conv_path(path)
        dw = torch.zeros(cout * 9 * cin, dtype=torch.float32, device=dev)
        for _ in range(2):  # accumulates
            learned._call("conv3_weight_grad", xt.data_ptr(), cin, dzt.data_ptr(), cout, dw.data_ptr(), None, B, H,
                          W, cin, cout, s)
        assert conv_path.rang_b200_nn_device_status(s) == 0
        got.append(_np(dw).reshape(cout, 9, cin))
    ref = 2 * nno.conv3_weight_grad(x, dz)
    scale = np.abs(ref).max()
    assert np.abs(got[0] - ref).max() <= 1e-5 * scale
    assert np.abs(got[0] - got[1]).max() <= 1e-5 * scale


@pytest.mark.gpu
def test_conv3_epilogue_accumulate_and_mask():
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(9)
    B, H, W, C = 1, 16, 16, 32
    x = nno.bf16(rng.standard_normal((B, H, W, C)))
    w = nno.bf16(rng.standard_normal((C, 9, C)) / 16)
    old = nno.bf16(rng.standard_normal((B, H, W, C)))
    mask = nno.bf16(rng.standard_normal((B, H, W, C)))
    out = _bf16_tensor(old.reshape(-1, C), dev)
    mt = _bf16_tensor(mask.reshape(-1, C), dev)
    xt, wt = _bf16_tensor(x.reshape(-1, C), dev), _bf16_tensor(w, dev)  # kept alive until the kernel has run
    learned._call("conv3", xt.data_ptr(), C, wt.data_ptr(), None, out.data_ptr(), C, mt.data_ptr(), C, B, H, W, C, C, 0,
                  1, torch.cuda.current_stream().cuda_stream)
    ref = np.where(mask > 0, nno.conv3(x, w) + old, 0.0)
    got = _np(out).reshape(ref.shape)
    assert np.abs(got - ref).max() <= 2.0**-7 * np.abs(ref).max()
    assert (got[mask <= 0] == 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout", [(32, 32), (96, 32), (64, 128), (256, 256)])
def test_conv3_gradients_match_the_oracle(cin, cout):
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(cin * 7 + cout)
    B, H, W = 2, 16, 24
    x = nno.bf16(np.maximum(rng.standard_normal((B, H, W, cin)), 0.0))
    w = nno.bf16(rng.standard_normal((cout, 9, cin)) / np.sqrt(9 * cin))
    dz = nno.bf16(rng.standard_normal((B, H, W, cout)))
    xt, wt, dzt = _bf16_tensor(x.reshape(-1, cin), dev), _bf16_tensor(w, dev), _bf16_tensor(dz.reshape(-1, cout), dev)
    flip = torch.empty(cin * 9 * cout, dtype=torch.bfloat16, device=dev)
    learned._call("conv3_flip", wt.data_ptr(), flip.data_ptr(), cin, cout, s)
    ref_flip = w.transpose(2, 1, 0)[:, ::-1, :]
    assert np.array_equal(_np(flip).reshape(cin, 9, cout), ref_flip)
    dx = torch.empty((B * H * W, cin), dtype=torch.bfloat16, device=dev)
    learned._call("conv3", dzt.data_ptr(), cout, flip.data_ptr(), None, dx.data_ptr(), cin, xt.data_ptr(), cin, B, H,
                  W, cout, cin, 0, 0, s)
    ref_dx = np.where(x > 0, nno.conv3_input_grad(dz, w), 0.0)
    got_dx = _np(dx).reshape(ref_dx.shape)
    assert np.abs(got_dx - ref_dx).max() <= 2.0**-7 * np.abs(ref_dx).max()
    dw = torch.zeros(cout * 9 * cin, dtype=torch.float32, device=dev)
    db = torch.zeros(cout, dtype=torch.float32, device=dev)
    for _ in range(2):  # accumulates
        learned._call("conv3_weight_grad", xt.data_ptr(), cin, dzt.data_ptr(), cout, dw.data_ptr(), db.data_ptr(), B,
                      H, W, cin, cout, s)
    ref_dw = 2 * nno.conv3_weight_grad(x, dz)
    got_dw = _np(dw).reshape(ref_dw.shape)
    assert np.abs(got_dw - ref_dw).max() <= 1e-5 * np.abs(ref_dw).max()
    assert np.abs(_np(db) - 2 * dz.sum(axis=(0, 1, 2))).max() <= 1e-5 * np.abs(dz.sum(axis=(0, 1, 2))).max() + 1e-4


@pytest.mark.gpu
def test_pool_upsample_head_and_loss_match_the_oracle():
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(4)
    B, H, W, C, wide = 2, 16, 8, 32, 96
    a = nno.bf16(rng.standard_normal((B, H, W, wide)))
    at = _bf16_tensor(a.reshape(-1, wide), dev)
    pooled = torch.empty((B * H * W // 4, C), dtype=torch.bfloat16, device=dev)
    learned._call("pool", learned._p(at, 64), wide, pooled.data_ptr(), C, B, H, W, C, s)
    ref_pool = nno.bf16(nno.pool(a[..., 64:]))
    assert _close_bf16(_np(pooled).reshape(ref_pool.shape), ref_pool)
    # pool backward in place on the skip slice of a gradient tensor
    g = nno.bf16(rng.standard_normal((B, H, W, wide)))
    gt = _bf16_tensor(g.reshape(-1, wide), dev)
    dp = nno.bf16(rng.standard_normal((B, H // 2, W // 2, C)))
    dpt = _bf16_tensor(dp.reshape(-1, C), dev)
    learned._call("pool_backward", learned._p(gt, 64), wide, dpt.data_ptr(), C, learned._p(at, 64), wide, B, H, W, C, s)
    ref = nno.bf16(np.where(a[..., 64:] > 0, g[..., 64:] + 0.25 * nno.upsample(dp), 0.0))
    got = _np(gt).reshape(B, H, W, wide)
    assert _close_bf16(got[..., 64:], ref) and np.array_equal(got[..., :64], g[..., :64])
    # upsampling into a channel slice and its backward
    lo = nno.bf16(rng.standard_normal((B, H // 2, W // 2, 64)))
    cat = torch.zeros((B * H * W, wide), dtype=torch.bfloat16, device=dev)
    lot = _bf16_tensor(lo.reshape(-1, 64), dev)
    learned._call("upsample", lot.data_ptr(), 64, cat.data_ptr(), wide, B, H, W, 64, s)
    assert np.array_equal(_np(cat).reshape(B, H, W, wide)[..., :64], nno.upsample(lo))
    back = torch.empty((B * H * W // 4, 64), dtype=torch.bfloat16, device=dev)
    learned._call("upsample_backward", gt.data_ptr(), wide, back.data_ptr(), 64, B, H // 2, W // 2, 64, s)
    assert _close_bf16(_np(back).reshape(lo.shape), nno.bf16(nno.upsample_backward(g[..., :64])))
    # head, its backward and the loss
    hw = rng.standard_normal(C).astype(np.float32)
    hb = np.array([0.25], np.float32)
    hwt, hbt = torch.from_numpy(hw).to(dev), torch.from_numpy(hb).to(dev)
    act = nno.bf16(np.maximum(rng.standard_normal((B, H, W, C)), 0.0))
    actt = _bf16_tensor(act.reshape(-1, C), dev)
    y = torch.empty(B * H * W, dtype=torch.float32, device=dev)
    learned._call("head", actt.data_ptr(), C, hwt.data_ptr(), hbt.data_ptr(), y.data_ptr(), B * H * W, s)
    ref_y = act @ hw.astype(np.float64) + 0.25
    assert np.abs(_np(y).reshape(ref_y.shape) - ref_y).max() <= 1e-5 * np.abs(ref_y).max()
    target = rng.standard_normal((3, H, W)).astype(np.float32)
    offs = torch.tensor([2 * H * W, 0], dtype=torch.int64, device=dev)
    dy = torch.empty_like(y)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    tt = torch.from_numpy(target).to(dev)
    learned._call("mse", y.data_ptr(), tt.data_ptr(), offs.data_ptr(), W, dy.data_ptr(), loss.data_ptr(), B, H, W, s)
    tb = target[[2, 0]]
    ref_loss, ref_dy = nno.mse(ref_y, tb)
    assert float(loss) == pytest.approx(ref_loss, rel=1e-4)
    assert np.abs(_np(dy).reshape(ref_dy.shape) - ref_dy).max() <= 1e-4 * np.abs(ref_dy).max()
    dact = torch.empty((B * H * W, C), dtype=torch.bfloat16, device=dev)
    dhw = torch.zeros(C, dtype=torch.float32, device=dev)
    dhb = torch.zeros(1, dtype=torch.float32, device=dev)
    learned._call("head_backward", actt.data_ptr(), C, hwt.data_ptr(), dy.data_ptr(), dact.data_ptr(), C,
                  dhw.data_ptr(), dhb.data_ptr(), B * H * W, s)
    dyh = _np(dy).reshape(B, H, W)
    ref_dact = nno.bf16(np.where(act > 0, dyh[..., None] * hw, 0.0))
    assert np.abs(_np(dact).reshape(ref_dact.shape) - ref_dact).max() <= 2.0**-8 * np.abs(ref_dact).max()
    assert np.allclose(_np(dhw), np.einsum("bhw,bhwc->c", dyh, act), rtol=1e-4, atol=1e-7)
    assert float(dhb) == pytest.approx(dyh.sum(), rel=1e-4, abs=1e-7)


def _gpu_net_vs_oracle(seed, B, H, W):
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    net = learned.UNet(dev, seed=seed)
    p = net.parameters()
    rng = np.random.default_rng(seed + 10)
    resid = rng.standard_normal((B, H, W)).astype(np.float32)
    psf = rng.standard_normal((H, W)).astype(np.float32)
    target = rng.standard_normal((B, H, W)).astype(np.float32)
    ws = learned.Workspace(net, B, H, W, training=True)
    offs = torch.arange(B, dtype=torch.int64, device=dev) * (H * W)
    rt, tt = torch.from_numpy(resid).to(dev), torch.from_numpy(target).to(dev)
    pt = torch.from_numpy(psf).to(dev)
    net.pack(ws, rt, offs, W, pt, W, 0.5, 2.0)
    net.forward(ws)
    ws.loss.zero_()
    net.loss_and_grad(ws, tt, offs, W)
    net.backward(ws)
    torch.cuda.synchronize()
    x = nno.pack(resid, psf, 0.5, 2.0)
    y, act = nno.forward(p, x, emulate=True)
    loss, dy = nno.mse(y, target)
    g = nno.backward(act, dy, emulate=True)
    y64, act64 = nno.forward(p, x)
    g64 = nno.backward(act64, nno.mse(y64, target)[1])
    return net, ws, y, loss, g, g64


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.gpu
def test_network_output_and_gradients_match_the_oracle():
    # bfloat16 storage alone moves the float64 gradients by a few to ~15 %
    # (deep layers; ReLU masks flip where sums round differently): per
    # tensor the GPU must be closer to the emulating oracle than that
    # sensitivity, and as close to float64 as the emulating oracle is.
    net, ws, y, loss, g, g64 = _gpu_net_vs_oracle(3, 2, 32, 48)
    got_y = _np(ws.y).reshape(y.shape)
    assert np.linalg.norm(got_y - y) <= 1e-2 * np.linalg.norm(y)
    assert float(ws.loss) == pytest.approx(loss, rel=1e-2)
    grads = net.gradients()
    for k, ref in g.items():
        sens = _rel(ref, g64[k])
        assert _rel(grads[k], ref) <= 0.75 * sens + 1e-2, (k, _rel(grads[k], ref), sens)
        assert _rel(grads[k], g64[k]) <= 1.25 * sens + 1e-2, (k, _rel(grads[k], g64[k]), sens)
    flat = np.concatenate([grads[k].ravel() for k in g])
    ref = np.concatenate([g[k].ravel() for k in g])
    assert float(flat @ ref) / (np.linalg.norm(flat) * np.linalg.norm(ref)) > 0.99


@pytest.mark.gpu
def test_adam_step_matches_the_oracle():
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    net, ws, _, _, g, _ = _gpu_net_vs_oracle(4, 1, 16, 16)
    p = net.parameters()
    gpu_g = net.gradients()
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(x) for k, x in p.items()}
    nno.adam(p, gpu_g, m, v, 1, 1e-3)
    net.adam(1e-3)
    torch.cuda.synchronize()
    after = net.parameters()
    for k in p:
        assert np.abs(after[k] - p[k]).max() <= 1e-6 + 1e-5 * np.abs(p[k]).max(), k
    assert float(net.grad.abs().max()) == 0.0
    flip = net.flipped["dec1a"].to(torch.float64).cpu().numpy().reshape(96, 9, 32)
    w = net.wb[net.slots["dec1a.w"][0]:net.slots["dec1a.w"][0] + 32 * 9 * 96].to(torch.float64).cpu().numpy()
    assert np.array_equal(flip, w.reshape(32, 9, 96).transpose(2, 1, 0)[:, ::-1, :])


@pytest.mark.gpu
def test_training_reduces_the_loss_and_proposals_tile_the_image():
    import torch

    from rang import learned

    dev = torch.device("cuda", 0)
    data = learned.make_training_set(dev, n_patches=128, n_coverages=2, npix=512, ntime=32, nchan=8,
                                     snapshots=(0, 6), seed=500)
    assert len(data) == 128 and data.psf.shape == (2, 256, 256)
    assert float(data.psf[0, 128, 128]) == pytest.approx(1.0)
    net = learned.UNet(dev, seed=1)
    losses = learned.train(net, data, steps=120, batch=8, lr=1e-3, warmup=10, log_every=10)
    first = np.mean([l for _, l in losses[:2]])
    last = np.mean([l for _, l in losses[-2:]])
    assert np.isfinite(last) and last < 0.7 * first, losses
    prop = learned.Proposer(net, 512)
    resid = torch.randn((512, 512), device=dev)
    out = prop(resid, data.psf[0], 1.0)
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()
    # one patch at the origin reproduces the tiled result inside its window
    ws = learned.Workspace(net, 1, 256, 256)
    net.pack(ws, resid, ws.offsets, 512, data.psf[0], 256, 1.0, 1.0)
    one = net.forward(ws).reshape(256, 256)
    assert torch.equal(one[:240, :240], out[:240, :240])


@pytest.mark.gpu
def test_learned_fista_gains_over_plain_fista():
    # A 512^2 field at 1.5 arcsec (40 point sources and 6 Gaussians): the
    # network is trained on patches the gridder makes from other seeds and
    # antenna subsets, then both solvers get the same number of applies of
    # the exact gridder on a held-out sky with the full array. Every accepted
    # proposal lowers the misfit; the learned run ends with a lower misfit
    # and closer to the true sky.
    import torch

    from rang import fista, learned, synth, wgrid_torch

    dev = torch.device("cuda", 0)
    npix, cell, sky_kw = 512, 1.5 * synth.ARCSEC, dict(npoint=40, ngauss=6, margin=20)
    data = learned.make_training_set(dev, n_patches=1536, n_coverages=4, npix=npix, ntime=32, nchan=16,
                                     snapshots=(0, 4, 12), sky=sky_kw, seed=300)
    net = learned.UNet(dev, seed=0)
    learned.train(net, data, steps=600, batch=8, lr=1e-3, warmup=50)
    del data
    uvw = torch.from_numpy(synth.uvw_tracks(nant=64, ntime=32)).to(dev)
    freq = synth.channels(32)
    common = dict(npix_x=npix, npix_y=npix, pixsize_x=cell, pixsize_y=cell)
    truth = torch.from_numpy(synth.extended_sky(npix, seed=21, **sky_kw)).to(dev)
    plan = wgrid_torch.DevicePlan(uvw, freq, epsilon=1e-5, single=True, **common)
    vis = plan.degrid(truth)
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    vis += 0.05 * np.sqrt(2.0) * torch.randn(vis.shape, dtype=vis.dtype, device=dev, generator=g)
    dirty, q = plan.residual(vis, None)
    lmax, _ = fista.power_iteration(plan.gram, plan.shape, dev, max_iterations=30)
    lam = 1e-4 * float(dirty.max())
    x0, gx0, _, _ = fista.solve(plan.gram, dirty, lam, 1.0 / lmax, 60, q0=0.5 * q)
    psf, peak = learned.psf_patch(plan.grid(None))
    seen = []
    x1, gx1, applies, st = learned.solve(plan.gram, dirty, lam, 1.0 / lmax, learned.Proposer(net, npix), psf, peak,
                                         61, q0=0.5 * q, observer=lambda k, x, gx, m: seen.append(m))
    assert applies == 61 and st["proposals"] >= 1 and st["accepted"] >= 1
    assert all(d > 0 for d in st["misfit_drops"])

    def misfit(x, gx):
        return 0.5 * q - float(torch.dot(dirty.double().ravel(), x.double().ravel())) + 0.5 * float(
            torch.dot(x.double().ravel(), gx.double().ravel()))

    m0, m1 = misfit(x0, gx0), misfit(x1, gx1)
    e0, e1 = float((x0 - truth).norm() / truth.norm()), float((x1 - truth).norm() / truth.norm())
    assert m1 < m0 and e1 < e0, (m0, m1, e0, e1, st["steps"])
    plan.close()
