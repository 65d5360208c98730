"""Timing case of the learned preconditioner's U-Net on the 152 x 500 image
(padded to 160 x 512): forward (inference) and full training steps
(forward, loss, backward, Adam) at a batch of 8, timed with CUDA events on
the launching stream, and the convolutions' dense FLOP rate.

    python -m benchmarks.profile_net [--batch 8] [--steps 20] [--warmup 3]
"""
from __future__ import annotations

import argparse
import json

from stfwi_b200.learned.unet import LAYERS, UNet, padded_shape


def conv_flops(h, w, batch):
    """Multiply-adds x 2 of the 3x3 convolutions of one forward pass."""
    total = 0
    level = {"enc1": 0, "enc2": 1, "enc3": 2, "bot": 3, "dec3": 2, "dec2": 1, "dec1": 0}
    for name, cin, cout in LAYERS:
        lv = level[name[:-1]]
        total += 2 * 9 * cin * cout * (h >> lv) * (w >> lv) * batch
    return total


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)
    h, w = padded_shape(152, 500)
    net = UNet(h, w, seed=0)
    g = torch.Generator().manual_seed(0)
    x = net.pack(torch.randn((a.batch, 4, 152, 500), generator=g).cuda())
    tgt = torch.zeros((a.batch, h, w), device="cuda")
    tgt[:, :152, :500] = torch.randn((a.batch, 152, 500), generator=g).cuda()
    wgt = torch.zeros_like(tgt)
    wgt[:, :152, :500] = 1.0
    inv = 1.0 / float(wgt.sum())
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for _ in range(a.warmup):
        net.forward(x)
        net.train_step(x, tgt, wgt, 1e-4, inv_norm=inv)
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(a.steps):
        net.forward(x)
    ev[1].record()
    for _ in range(a.steps):
        net.train_step(x, tgt, wgt, 1e-4, inv_norm=inv)
    ev[2].record()
    torch.cuda.synchronize()
    net.check()
    fwd_ms = ev[0].elapsed_time(ev[1]) / a.steps
    step_ms = ev[1].elapsed_time(ev[2]) / a.steps
    f = conv_flops(h, w, a.batch)
    # a training step: forward, input gradients (all layers but the first) and weight gradients
    f_first = 2 * 9 * LAYERS[0][1] * LAYERS[0][2] * h * w * a.batch
    f_step = 3 * f - f_first
    print(json.dumps(dict(image=[h, w], batch=a.batch, steps=a.steps, forward_ms=fwd_ms, train_step_ms=step_ms,
                          conv_gflop_forward=f / 1e9, conv_gflop_train_step=f_step / 1e9,
                          forward_tflops=f / fwd_ms / 1e9, train_step_tflops=f_step / step_ms / 1e9)))


if __name__ == "__main__":
    main()
