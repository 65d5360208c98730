"""Plain PyTorch FP32 restatement of the learned preconditioner's U-Net
(stfwi_b200/learned/unet.py): the numerics reference of its CUDA kernels.
Test infrastructure only."""
import torch
import torch.nn.functional as F

from stfwi_b200.learned.unet import LAYERS, param_layout


def torch_weight(w9):
    """[9][cout][cin] with tap = 3 (dy + 1) + (dx + 1) -> conv2d's [cout][cin][3][3]."""
    _, cout, cin = w9.shape
    return w9.permute(1, 2, 0).reshape(cout, cin, 3, 3)


def conv(x, w9, b=None, relu=False):
    y = F.conv2d(x, torch_weight(w9), b, padding=1)
    return F.relu(y) if relu else y


def unet_forward(params, x):
    """params: flat tensor (param_layout); x: [B, 16, h, w] -> [B, h, w]."""
    lay, head, _ = param_layout()
    shapes = {n: (ci, co) for n, ci, co in LAYERS}

    def c(name, t):
        wo, bo = lay[name]
        ci, co = shapes[name]
        return conv(t, params[wo:bo].view(9, co, ci), params[bo:bo + co], relu=True)

    a1 = c("enc1a", x)
    s1 = c("enc1b", a1)
    a2 = c("enc2a", F.avg_pool2d(s1, 2))
    s2 = c("enc2b", a2)
    a3 = c("enc3a", F.avg_pool2d(s2, 2))
    s3 = c("enc3b", a3)
    b1 = c("bota", F.avg_pool2d(s3, 2))
    b2 = c("botb", b1)
    up = F.interpolate(b2, scale_factor=2, mode="nearest")
    d3 = c("dec3b", c("dec3a", torch.cat([up, s3], 1)))
    up = F.interpolate(d3, scale_factor=2, mode="nearest")
    d2 = c("dec2b", c("dec2a", torch.cat([up, s2], 1)))
    up = F.interpolate(d2, scale_factor=2, mode="nearest")
    d1 = c("dec1b", c("dec1a", torch.cat([up, s1], 1)))
    hw, hb = head
    return torch.einsum("bchw,c->bhw", d1, params[hw:hb]) + params[hb]


def masked_mse(out, target, wgt, inv_norm):
    return (wgt * (out - target) ** 2).sum() * inv_norm
