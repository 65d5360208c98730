"""Host logic of the learned preconditioner on the CPU: the U-Net's wiring
(buffers, channel slices, masks, the order of the backward pass, the Adam
step) run against a torch stand-in of each C entry point, compared with
autograd of the plain torch U-Net."""
import numpy as np
import pytest


@pytest.fixture
def fake_net(monkeypatch):
    import torch
    from stfwi_b200 import _native as N
    from stfwi_b200.learned import unet as U
    from tests.fake_nn import FakeNN
    fake = FakeNN()
    monkeypatch.setattr(N, "load", lambda: fake)
    monkeypatch.setattr(U, "_p", lambda t: t)
    monkeypatch.setattr(U.UNet, "storage_dtype", torch.float64)
    return U.UNet(16, 512, seed=5, device="cpu")


def test_padded_shape_and_parameter_layout():
    from stfwi_b200.learned.unet import LAYERS, padded_shape, param_layout
    assert padded_shape(152, 500) == (160, 512)
    assert padded_shape(304, 1000) == (304, 1024)
    lay, head, total = param_layout()
    n = sum(9 * ci * co + co for _, ci, co in LAYERS)
    assert total == n + 32 + 16
    # every block starts on a 16-float boundary (the kernels want 16-byte aligned FP32 blocks)
    assert all(wo % 16 == 0 and bo % 16 == 0 for wo, bo in lay.values()) and head[0] % 16 == 0
    # the decoder inputs are the concatenations [upsampled, skip]
    ch = {nm: (ci, co) for nm, ci, co in LAYERS}
    assert ch["dec3a"][0] == ch["botb"][1] + ch["enc3b"][1]
    assert ch["dec2a"][0] == ch["dec3b"][1] + ch["enc2b"][1]
    assert ch["dec1a"][0] == ch["dec2b"][1] + ch["enc1b"][1]


def test_unet_rejects_unpadded_images():
    from stfwi_b200.learned import UNet
    with pytest.raises(ValueError):
        UNet(152, 500, device="cpu")


def test_unet_wiring_matches_autograd(fake_net):
    import torch
    from tests.unet_ref import masked_mse, unet_forward
    from stfwi_b200.learned.unet import LAYERS
    net = fake_net
    g = torch.Generator().manual_seed(0)
    feat = torch.randn((2, 4, 14, 500), generator=g)
    x = net.pack(feat, scale=(1.0, 2.0, 0.5, 1.0))
    tgt = torch.randn((2, 16, 512), generator=g)
    wgt = torch.zeros_like(tgt)
    wgt[:, :14, :500] = 1.0
    inv = 1.0 / float(wgt.sum())
    out = net.forward(x, train=True).clone()
    loss = net.backward(x, tgt, wgt, inv)
    params = net.params.detach().double().requires_grad_(True)
    ref = unet_forward(params, x.permute(0, 3, 1, 2).double())
    lref = masked_mse(ref, tgt.double(), wgt.double(), inv)
    lref.backward()
    assert float((out.double() - ref.detach()).norm() / ref.detach().norm()) < 1e-6
    assert abs(float(loss) / float(lref.detach()) - 1) < 1e-6   # the head output is FP32
    e = float((net.grads.double() - params.grad).norm() / params.grad.norm())
    assert e < 1e-6, e
    # every block of the parameters receives a gradient
    for name, _, _ in LAYERS:
        gw, gb = net.grad(name)
        assert float(gw.abs().max()) > 0 and float(gb.abs().max()) > 0, name


def test_adam_step_matches_the_efficient_form(fake_net):
    """Adam in the efficient form of Kingma and Ba (2015, section 2): the
    bias corrections folded into the step size, eps added to sqrt(v)."""
    import torch
    net = fake_net
    rng = np.random.default_rng(1)
    p = net.params.clone().double()
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    lr, b1, b2, eps = 1e-3, 0.9, 0.999, 1e-8
    for t in range(1, 4):
        g = torch.from_numpy(rng.standard_normal(net.nparam).astype(np.float32))
        net.grads.copy_(g)
        net.adam_step(lr)
        m = b1 * m + (1 - b1) * g.double()
        v = b2 * v + (1 - b2) * g.double() ** 2
        p = p - lr * np.sqrt(1 - b2 ** t) / (1 - b1 ** t) * m / (v.sqrt() + eps)
    assert float(net.grads.abs().max()) == 0.0          # cleared after the step
    assert float((net.params.double() - p).abs().max()) < 1e-6
    w, _ = net.weight("dec2a")
    assert torch.equal(net.wf["dec2a"], w.double())
    assert torch.equal(net.wt["dec2a"], w.double().flip(0).transpose(1, 2))


def test_compact_weights_keep_what_the_kernels_read(tmp_path):
    """The stored network: convolution weights as their BF16 values, biases
    and head exact; the shipped file loads into a full parameter vector."""
    import os
    import torch
    from stfwi_b200.learned.unet import load_weights, param_layout, save_weights
    lay, head, total = param_layout()
    rng = np.random.default_rng(3)
    p = rng.standard_normal(total).astype(np.float32)
    save_weights(tmp_path / "w.npz", p)
    q = load_weights(tmp_path / "w.npz")
    wo, bo = lay["dec2a"]
    assert np.array_equal(q[wo:bo], torch.from_numpy(p[wo:bo]).to(torch.bfloat16).float().numpy())
    assert np.array_equal(q[bo:bo + 64], p[bo:bo + 64])
    assert np.array_equal(q[head[0]:head[1] + 1], p[head[0]:head[1] + 1])
    shipped = os.path.join(os.path.dirname(__file__), "..", "stfwi_b200", "learned", "weights", "unet_152x500_3hz.npz")
    w = load_weights(shipped)
    assert w.shape == (total,) and np.isfinite(w).all() and float(np.abs(w).max()) > 0


def test_training_loop_keeps_the_best_validation_weights(monkeypatch):
    """experiment.train on the CPU stand-in of the kernels: mirror-image
    augmentation, the cosine schedule, and the weights of the epoch with
    the lowest validation loss restored at the end."""
    import torch
    from stfwi_b200 import _native as N
    from stfwi_b200.learned import experiment as E
    from stfwi_b200.learned import unet as U
    from tests.fake_nn import FakeNN
    monkeypatch.setattr(N, "load", lambda: FakeNN())
    monkeypatch.setattr(U, "_p", lambda t: t)
    monkeypatch.setattr(U.UNet, "storage_dtype", torch.float64)
    rng = np.random.default_rng(7)
    X = rng.standard_normal((6, 4, 14, 500)).astype(np.float32)
    Y = (0.5 * X[:, 0] + 0.1).astype(np.float32)
    logs = []
    net, hist, best = E.train(X, Y, epochs=2, batch=4, lr=1e-3, n_val=2, log=logs.append, device="cpu")
    assert len(hist) == 2 and len(logs) == 2 and 1 <= best <= 2
    vals = [v for _, v in hist]
    assert abs(E.validation_loss(net, X[4:], Y[4:], batch=4) - min(vals)) < 1e-9 * max(min(vals), 1.0)
    assert net.step_count == 2 * ((2 * 4) // 4)          # steps per epoch over the data and its mirror images
