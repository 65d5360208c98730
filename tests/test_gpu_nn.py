"""The learned preconditioner's network kernels (include/stfwi_nn.h) on the
B200 against plain PyTorch FP32/FP64 references of the same ops.

Tolerances: the kernels read BF16 operands and accumulate in FP32; a single
op is compared with an FP64 evaluation on the same BF16 inputs, so only the
BF16 rounding of its output remains (rel-L2 <= 4e-3, 2^-8 = 3.9e-3 being
one BF16 ulp); the weight gradient (FP32 output) is held to 1e-4.  The whole
network is compared with the same host code running torch restatements of
every op that store BF16 at the same points (rel-L2 <= 1e-2), and with the
FP32 torch U-Net (see the test).
"""
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.double().cpu().flatten(); b = b.double().cpu().flatten()
    return float((a - b).norm() / max(float(b.norm()), 1e-300))


def _bf16(shape, seed, scale=1.0):
    import torch
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, generator=g) * scale).to(torch.bfloat16).cuda()


def _nchw(x):
    return x.double().cpu().permute(0, 3, 1, 2)


def _nhwc(x):
    return x.permute(0, 2, 3, 1)


@pytest.mark.parametrize("n,h,w,cin,cout", [
    (1, 2, 128, 16, 16),      # one box row, the smallest channel counts (32-byte swizzle)
    (2, 8, 128, 32, 32),      # 64-byte swizzle
    (1, 4, 64, 64, 64),       # 64-pixel rows: two rows per box
    (2, 6, 256, 96, 32),      # concatenated input, 96 = 3 x 32 channel blocks
    (1, 4, 64, 384, 128),     # the deepest decoder layer's channels
    (1, 2, 64, 128, 256),     # two 128-channel output tiles
])
def test_conv_forward_matches_torch(n, h, w, cin, cout):
    import torch
    from stfwi_b200 import _native as N
    from tests.unet_ref import conv
    x = _bf16((n, h, w, cin), 1)
    w9 = _bf16((9, cout, cin), 2, scale=0.1)
    b = torch.randn(cout, generator=torch.Generator().manual_seed(3)).cuda()
    y = torch.zeros((n, h, w, cout + 32), dtype=torch.bfloat16, device="cuda")
    L = N.load()
    rc = L.stfwi_nn_conv3x3(x.data_ptr(), n, h, w, cin, w9.data_ptr(), cout, b.data_ptr(), 1, y.data_ptr(),
                            cout + 32, 16, None)
    assert rc == 0, L.stfwi_nn_last_error()
    assert L.stfwi_nn_check(None) == 0, L.stfwi_nn_last_error()
    ref = conv(_nchw(x), w9.double().cpu(), b.double().cpu(), relu=True)
    got = y[..., 16:16 + cout].double().cpu().permute(0, 3, 1, 2)
    assert _rel(got, ref) < 4e-3
    # channels outside the output slice stay untouched
    assert float(y[..., :16].abs().max()) == 0.0 and float(y[..., 16 + cout:].abs().max()) == 0.0


@pytest.mark.parametrize("n,h,w,cin,cout", [(1, 4, 128, 32, 64), (2, 2, 64, 96, 32), (1, 4, 64, 16, 32)])
def test_conv_input_gradient_matches_torch(n, h, w, cin, cout):
    """dgrad with the tap-flipped transposed weights and the ReLU mask."""
    import torch
    from stfwi_b200 import _native as N
    from tests.unet_ref import conv
    L = N.load()
    dz = _bf16((n, h, w, cout), 4)
    w9 = _bf16((9, cout, cin), 5, scale=0.1)
    w32 = w9.float().contiguous()
    wf = torch.empty_like(w9)
    wt = torch.empty((9, cin, cout), dtype=torch.bfloat16, device="cuda")
    assert L.stfwi_nn_pack_weights(w32.data_ptr(), cout, cin, wf.data_ptr(), wt.data_ptr(), None) == 0
    mask = _bf16((n, h, w, cin + 16), 6)
    dx = torch.empty((n, h, w, cin), dtype=torch.bfloat16, device="cuda")
    rc = L.stfwi_nn_conv3x3_dgrad(dz.data_ptr(), n, h, w, cout, wt.data_ptr(), cin, mask.data_ptr(), cin + 16, 16,
                                  dx.data_ptr(), None)
    assert rc == 0, L.stfwi_nn_last_error()
    assert L.stfwi_nn_check(None) == 0
    assert torch.equal(wf, w9)
    xr = torch.zeros((n, cin, h, w), dtype=torch.float64, requires_grad=True)
    conv(xr, w9.double().cpu()).backward(_nchw(dz))
    ref = xr.grad * (_nchw(mask)[:, 16:] > 0)
    assert _rel(dx.double().cpu().permute(0, 3, 1, 2), ref) < 4e-3


@pytest.mark.parametrize("n,h,w,cin,cout", [
    (1, 4, 128, 16, 32), (2, 2, 64, 32, 32), (1, 2, 128, 96, 64), (1, 2, 64, 384, 128), (1, 2, 64, 128, 256),
])
def test_conv_weight_gradient_matches_torch(n, h, w, cin, cout):
    import torch
    from stfwi_b200 import _native as N
    from tests.unet_ref import conv
    L = N.load()
    x = _bf16((n, h, w, cin), 7)
    dz = _bf16((n, h, w, cout), 8)
    dw = torch.full((9, cout, cin), 0.5, dtype=torch.float32, device="cuda")   # accumulates into 0.5
    rc = L.stfwi_nn_conv3x3_wgrad(x.data_ptr(), dz.data_ptr(), n, h, w, cin, cout, dw.data_ptr(), None)
    assert rc == 0, L.stfwi_nn_last_error()
    assert L.stfwi_nn_check(None) == 0
    w9 = torch.zeros((9, cout, cin), dtype=torch.float64, requires_grad=True)
    conv(_nchw(x), w9).backward(_nchw(dz))
    assert _rel(dw.double().cpu() - 0.5, w9.grad) < 1e-4     # FP32 accumulation of exact BF16 products


def test_pool_upsample_skip_head_and_bias_kernels():
    import torch
    import torch.nn.functional as F
    from stfwi_b200 import _native as N
    L = N.load()
    n, h, w, c = 2, 8, 128, 32
    cat = _bf16((n, h, w, 96), 9)
    p = torch.empty((n, h // 2, w // 2, c), dtype=torch.bfloat16, device="cuda")
    assert L.stfwi_nn_avgpool2(cat.data_ptr(), n, h, w, c, 96, 64, p.data_ptr(), None) == 0
    assert _rel(_nchw(p), F.avg_pool2d(_nchw(cat)[:, 64:], 2)) < 4e-3
    low = _bf16((n, h // 2, w // 2, 64), 10)
    assert L.stfwi_nn_upsample2(low.data_ptr(), n, h // 2, w // 2, 64, 96, cat.data_ptr(), None) == 0
    assert torch.equal(cat[..., :64], _nhwc(F.interpolate(_nchw(low), scale_factor=2)).to(torch.bfloat16).cuda())
    dcat = _bf16((n, h, w, 96), 11)
    dz = torch.empty((n, h // 2, w // 2, 64), dtype=torch.bfloat16, device="cuda")
    assert L.stfwi_nn_upsample2_grad(dcat.data_ptr(), 96, low.data_ptr(), n, h // 2, w // 2, 64, dz.data_ptr(),
                                     None) == 0
    ref = F.avg_pool2d(_nchw(dcat)[:, :64], 2) * 4 * (_nchw(low) > 0)
    assert _rel(_nchw(dz), ref) < 4e-3
    dpool = _bf16((n, h // 2, w // 2, c), 12)
    ds = torch.empty((n, h, w, c), dtype=torch.bfloat16, device="cuda")
    assert L.stfwi_nn_skip_grad(dcat.data_ptr(), cat.data_ptr(), 96, 64, dpool.data_ptr(), n, h, w, c,
                                ds.data_ptr(), None) == 0
    ref = (_nchw(dcat)[:, 64:] + F.interpolate(_nchw(dpool), scale_factor=2) / 4) * (_nchw(cat)[:, 64:] > 0)
    assert _rel(_nchw(ds), ref) < 4e-3
    db = torch.full((c,), 1.0, device="cuda")
    assert L.stfwi_nn_bias_grad(ds.data_ptr(), n * h * w, c, db.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert _rel(db.double().cpu() - 1.0, ds.double().cpu().sum((0, 1, 2))) < 1e-5
    # head and its loss gradient
    y = _bf16((n, h, w, 32), 13)
    hw = torch.randn(32, generator=torch.Generator().manual_seed(14)).cuda()
    hb = torch.tensor([0.25], device="cuda")
    out = torch.empty((n, h, w), device="cuda")
    assert L.stfwi_nn_head(y.data_ptr(), n * h * w, 32, hw.data_ptr(), hb.data_ptr(), out.data_ptr(), None) == 0
    yr = _nchw(y)
    assert _rel(out, torch.einsum("bchw,c->bhw", yr, hw.double().cpu()) + 0.25) < 1e-6
    tgt = torch.randn((n, h, w), generator=torch.Generator().manual_seed(15)).cuda()
    wgt = (torch.rand((n, h, w), generator=torch.Generator().manual_seed(16)) > 0.3).float().cuda()
    dzh = torch.empty_like(y)
    dwt = torch.zeros(32, device="cuda")
    dbh = torch.zeros(1, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    inv = 1.0 / float(wgt.sum())
    assert L.stfwi_nn_head_loss_grad(y.data_ptr(), n * h * w, 32, hw.data_ptr(), out.data_ptr(), tgt.data_ptr(),
                                     wgt.data_ptr(), inv, dzh.data_ptr(), dwt.data_ptr(), dbh.data_ptr(),
                                     loss.data_ptr(), None) == 0
    o = out.double().cpu().requires_grad_(True)
    lref = (wgt.double().cpu() * (o - tgt.double().cpu()) ** 2).sum() * inv
    lref.backward()
    assert abs(float(loss) / float(lref.detach()) - 1) < 1e-5
    gout = o.grad
    assert _rel(dbh, gout.sum().reshape(1)) < 1e-5
    assert _rel(dwt, torch.einsum("bchw,bhw->c", yr, gout)) < 1e-5
    ref = gout[:, None] * hw.double().cpu()[None, :, None, None] * (yr > 0)
    assert _rel(_nchw(dzh), ref) < 4e-3


def _network_case(B=2, seed=0):
    import torch
    from stfwi_b200.learned import UNet
    net = UNet(32, 512, seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    feat = torch.randn((B, 4, 30, 500), generator=g).cuda()
    x = net.pack(feat, scale=(1.0, 0.5, 1.0, 1.0))
    tgt = torch.zeros((B, 32, 512), device="cuda")
    tgt[:, :30, :500] = torch.randn((B, 30, 500), generator=g).cuda()
    wgt = torch.zeros_like(tgt)
    wgt[:, :30, :500] = 1.0
    return net, feat, x, tgt, wgt


_FORWARD = ("a1", "cat1", "p1", "a2", "cat2", "p2", "a3", "cat3", "p3", "b1", "b2", "d3a", "d3b", "d2a", "d2b",
            "d1a", "d1b", "out")


def _emulated(net_gpu, x, tgt, wgt, inv, monkeypatch):
    """The same network run by the same host code on the CPU with every
    kernel replaced by its torch restatement (tests/fake_nn.py) storing BF16
    at the same points as the kernels.  Returns its forward output, then the
    loss and gradients of its backward pass run on the GPU's own forward
    activations, so that both backward passes see the same ReLU masks."""
    from stfwi_b200 import _native as N
    from stfwi_b200.learned import unet as U
    from tests.fake_nn import FakeNN
    with monkeypatch.context() as mp:
        mp.setattr(N, "load", lambda: FakeNN())
        mp.setattr(U, "_p", lambda t: t)
        net = U.UNet(net_gpu.h, net_gpu.w, device="cpu")
        net.params.copy_(net_gpu.params.cpu())
        net.pack_weights()
        xc = x.cpu()
        out = net.forward(xc, train=True).clone()
        b, bg = net.buffers(x.shape[0], True), net_gpu.buffers(x.shape[0], True)
        for k in _FORWARD:
            b[k].copy_(bg[k].cpu())
        loss = net.backward(xc, tgt.cpu(), wgt.cpu(), inv)
        return out, float(loss), net.grads.clone()


def test_unet_forward_and_gradients_match_torch(monkeypatch):
    """The whole network (14 tensor-core convolutions, pooling, upsampling,
    concatenation, head, masked MSE).  (1) Against the torch restatement of
    every op with the same BF16 storage points: forward output rel-L2 <=
    1e-2; backward pass on the same forward activations, every parameter
    gradient rel-L2 <= 1e-2.  (2) Against the FP32 torch U-Net with the same
    weights: output <= 3e-2; the gradients only within 0.2, because a loss
    with random targets makes each gradient a sum of many random-sign terms,
    so the few ReLU masks that BF16 activations flip move it by about
    sqrt(flipped fraction) (observed 2-12 %)."""
    import torch
    from stfwi_b200.learned.unet import LAYERS, param_layout
    from tests.unet_ref import masked_mse, unet_forward
    net, feat, x, tgt, wgt = _network_case()
    # the packed input is the scaled features in channels 0-3, zeros elsewhere
    xr = torch.zeros((2, 16, 32, 512), dtype=torch.float64)
    xr[:, :4, :30, :500] = feat.double().cpu() * torch.tensor([1.0, 0.5, 1.0, 1.0], dtype=torch.float64)[:, None, None]
    assert _rel(x.double().cpu().permute(0, 3, 1, 2), xr) < 4e-3
    out = net.forward(x, train=True).clone()
    inv = 1.0 / float(wgt.sum())
    loss = float(net.backward(x, tgt, wgt, inv))
    net.check()
    grads = net.grads.clone()
    lay, head, _ = param_layout()
    blocks = [(n, lay[n][0], lay[n][1], lay[n][1] + co) for n, _, co in LAYERS] + \
        [("head", head[0], head[1], head[1] + 1)]

    def per_block(g, ref):
        return {n: (_rel(g[wo:bo], ref[wo:bo]), _rel(g[bo:be], ref[bo:be])) for n, wo, bo, be in blocks}

    e_out, e_loss, e_grad = _emulated(net, x, tgt, wgt, inv, monkeypatch)
    emu = per_block(grads, e_grad)
    print("vs BF16-storage emulation: out", _rel(out, e_out), {k: (round(a, 5), round(b, 5)) for k, (a, b) in emu.items()})
    assert _rel(out, e_out) < 1e-2
    assert abs(loss / e_loss - 1) < 1e-4
    assert max(max(v) for v in emu.values()) < 1e-2, emu

    params = net.params.detach().double().cpu().requires_grad_(True)
    ref = unet_forward(params, x.double().cpu().permute(0, 3, 1, 2))
    lref = masked_mse(ref, tgt.double().cpu(), wgt.double().cpu(), inv)
    lref.backward()
    f32 = per_block(grads, params.grad)
    print("vs FP32 torch U-Net: out", _rel(out, ref.detach()), {k: (round(a, 5), round(b, 5)) for k, (a, b) in f32.items()})
    assert _rel(out, ref.detach()) < 3e-2
    assert abs(loss / float(lref.detach()) - 1) < 3e-2
    assert max(max(v) for v in f32.values()) < 0.2, f32


def test_unet_training_lowers_the_loss():
    """Adam on the tensor-core kernels fits a fixed batch: the loss falls by
    more than half in 60 steps."""
    import torch
    net, feat, x, _, wgt = _network_case(seed=3)
    tgt = torch.zeros((2, 32, 512), device="cuda")
    k = torch.ones((1, 1, 5, 5), device="cuda") / 25.0
    tgt[:, :30, :500] = torch.nn.functional.conv2d(feat[:, :1], k, padding=2)[:, 0]
    first = last = None
    for _ in range(60):
        loss = float(net.train_step(x, tgt, wgt, lr=2e-3))
        first = loss if first is None else first
        last = loss
    net.check()
    print("loss", first, "->", last)
    assert last < 0.5 * first, (first, last)
