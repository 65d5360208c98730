"""U-Net of the learned preconditioner on the library's tcgen05 kernels.

Four levels of 32, 64, 128 and 256 channels; each level has two 3x3
convolutions with bias and ReLU; 2x2 average pooling down, nearest 2x
upsampling up, the upsampled tensor concatenated with the level's skip
tensor (upsampled channels first); a 1x1 head gives one FP32 channel.
Input: 4 feature planes [gradient, illumination, Vp, Vs] (already
normalised) zero-padded to 16 channels and to a padded image whose width is
a multiple of 512 and height a multiple of 16.

Activations and weights are BF16 (NHWC), accumulation FP32 in tensor memory;
master weights, their gradients and the Adam moments are FP32 in one flat
device buffer.  Tensor memory for activations comes from torch (device
allocations only); every arithmetic step is a kernel of include/stfwi_nn.h.
"""
from __future__ import annotations

import ctypes as ct
import math

import numpy as np

from .. import _native as N

# (name, input channels, output channels) of the 3x3 convolutions, in forward order
LAYERS = (
    ("enc1a", 16, 32), ("enc1b", 32, 32),
    ("enc2a", 32, 64), ("enc2b", 64, 64),
    ("enc3a", 64, 128), ("enc3b", 128, 128),
    ("bota", 128, 256), ("botb", 256, 256),
    ("dec3a", 384, 128), ("dec3b", 128, 128),
    ("dec2a", 192, 64), ("dec2b", 64, 64),
    ("dec1a", 96, 32), ("dec1b", 32, 32),
)
HEAD_IN = 32
IN_CH = 16


def padded_shape(nz, nx):
    """Padded image (h, w): w a multiple of 512 (64-pixel rows at the lowest
    level), h a multiple of 16 (whole 128-pixel boxes at every level)."""
    return int(math.ceil(nz / 16) * 16), int(math.ceil(nx / 512) * 512)


def _check(status, what):
    if status != 0:
        msg = N.load().stfwi_nn_last_error().decode(errors="replace")
        raise N.StfwiError(status, f"{what}: {msg}")


def _p(t):
    return ct.c_void_p(t.data_ptr()) if t is not None else None


def _shape(name):
    return next((ci, co) for n, ci, co in LAYERS if n == name)


def param_layout():
    """Offsets (in floats) of every parameter block in the flat buffer:
    {name: (w_off, b_off)}, head (w_off, b_off), total."""
    off = 0
    lay = {}
    for name, cin, cout in LAYERS:
        lay[name] = (off, off + 9 * cout * cin)
        off += 9 * cout * cin + cout
    head = (off, off + HEAD_IN)
    off += HEAD_IN + 16            # head bias, padded to a 16-float boundary
    return lay, head, off


class UNet:
    """The network, its FP32 master parameters and Adam state on one device.

    ``h, w``: padded image size (``padded_shape``).  ``forward(x)`` takes
    the packed input [B, h, w, 16] BF16 (``pack``) and returns [B, h, w]
    FP32; ``train_step`` runs forward, the masked mean-square loss, the
    backward pass and one Adam step."""

    # storage type of activations and packed weights; the kernels read BF16,
    # a host-wiring test on the CPU swaps in FP64
    storage_dtype = None

    def __init__(self, h, w, seed=0, device="cuda"):
        import torch
        if w % 512 or h % 16:
            raise ValueError(f"padded image {h}x{w}: width must be a multiple of 512, height of 16")
        self.torch = torch
        self._act = self.storage_dtype or torch.bfloat16
        self.h, self.w = h, w
        self.device = torch.device(device)
        self.lay, self.head, self.nparam = param_layout()
        self.params = torch.zeros(self.nparam, dtype=torch.float32, device=self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self.init_params(seed)
        self.wf, self.wt = {}, {}
        for name, cin, cout in LAYERS:
            self.wf[name] = torch.empty((9, cout, cin), dtype=self._act, device=self.device)
            self.wt[name] = torch.empty((9, cin, cout), dtype=self._act, device=self.device)
        self._bufs = {}
        self.pack_weights()

    # ---------------------------------------------------------------- parameters

    def init_params(self, seed):
        """He-normal 3x3 weights over the real fan-in (4 input planes for the
        first layer, whose zero channels get zero weights), zero biases,
        a small head."""
        rng = np.random.default_rng(seed)
        p = np.zeros(self.nparam, dtype=np.float32)
        for name, cin, cout in LAYERS:
            wo, _ = self.lay[name]
            fan = 9 * (4 if name == "enc1a" else cin)
            wgt = rng.standard_normal((9, cout, cin)).astype(np.float32) * np.float32(math.sqrt(2.0 / fan))
            if name == "enc1a":
                wgt[:, :, 4:] = 0.0
            p[wo:wo + wgt.size] = wgt.ravel()
        hw, _ = self.head
        p[hw:hw + HEAD_IN] = rng.standard_normal(HEAD_IN).astype(np.float32) * np.float32(0.1 / math.sqrt(HEAD_IN))
        self.params.copy_(self.torch.from_numpy(p))

    def weight(self, name):
        wo, bo = self.lay[name]
        cin, cout = _shape(name)
        return self.params[wo:bo].view(9, cout, cin), self.params[bo:bo + cout]

    def grad(self, name):
        wo, bo = self.lay[name]
        cin, cout = _shape(name)
        return self.grads[wo:bo].view(9, cout, cin), self.grads[bo:bo + cout]

    def head_params(self):
        hw, hb = self.head
        return self.params[hw:hb], self.params[hb:hb + 1]

    def head_grads(self):
        hw, hb = self.head
        return self.grads[hw:hb], self.grads[hb:hb + 1]

    def pack_weights(self):
        L, st = N.load(), self._stream()
        for name, cin, cout in LAYERS:
            wo, bo = self.lay[name]
            _check(L.stfwi_nn_pack_weights(_p(self.params[wo:bo]), cout, cin, _p(self.wf[name]),
                                           _p(self.wt[name]), st), "pack_weights")

    def state_dict(self):
        return {"params": self.params.detach().cpu().numpy().copy(), "h": self.h, "w": self.w}

    def load_state_dict(self, sd):
        if int(sd["h"]) != self.h or int(sd["w"]) != self.w or np.asarray(sd["params"]).size != self.nparam:
            raise ValueError("state does not match this network")
        self.params.copy_(self.torch.from_numpy(np.asarray(sd["params"], dtype=np.float32)).to(self.device))
        self.pack_weights()

    def _stream(self):
        if self.device.type != "cuda":
            return None
        return ct.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    # ---------------------------------------------------------------- buffers

    def buffers(self, batch, train):
        """Activation (and, for training, gradient) buffers of a batch size."""
        key = (batch, bool(train))
        if key in self._bufs:
            return self._bufs[key]
        torch = self.torch
        h, w = self.h, self.w

        def t(hh, ww, c):
            return torch.empty((batch, hh, ww, c), dtype=self._act, device=self.device)

        s = [(h >> k, w >> k) for k in range(4)]
        b = {
            "a1": t(*s[0], 32), "cat1": t(*s[0], 96), "p1": t(*s[1], 32),
            "a2": t(*s[1], 64), "cat2": t(*s[1], 192), "p2": t(*s[2], 64),
            "a3": t(*s[2], 128), "cat3": t(*s[2], 384), "p3": t(*s[3], 128),
            "b1": t(*s[3], 256), "b2": t(*s[3], 256),
            "d3a": t(*s[2], 128), "d3b": t(*s[2], 128),
            "d2a": t(*s[1], 64), "d2b": t(*s[1], 64),
            "d1a": t(*s[0], 32), "d1b": t(*s[0], 32),
            "out": torch.empty((batch, h, w), dtype=torch.float32, device=self.device),
        }
        if train:
            for k in ("a1", "cat1", "p1", "a2", "cat2", "p2", "a3", "cat3", "p3", "b1", "b2",
                      "d3a", "d3b", "d2a", "d2b", "d1a", "d1b"):
                b["g_" + k] = torch.empty_like(b[k])
            b["g_s1"], b["g_s2"], b["g_s3"] = t(*s[0], 32), t(*s[1], 64), t(*s[2], 128)
            b["loss"] = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._bufs[key] = b
        return b

    def pack(self, feat, scale=(1.0, 1.0, 1.0, 1.0)):
        """features [B, 4, nz, nx] FP32 -> packed input [B, h, w, 16] BF16."""
        torch = self.torch
        feat = feat.to(device=self.device, dtype=torch.float32).contiguous()
        B, C, nz, nx = feat.shape
        if C != 4 or nz > self.h or nx > self.w:
            raise ValueError(f"features {tuple(feat.shape)} do not fit the {self.h}x{self.w} network")
        x = torch.empty((B, self.h, self.w, IN_CH), dtype=self._act, device=self.device)
        sc = (ct.c_float * 4)(*[float(v) for v in scale])
        _check(N.load().stfwi_nn_pack_input(_p(feat), B, nz, nx, self.h, self.w, sc, _p(x), self._stream()),
               "pack_input")
        return x

    # ---------------------------------------------------------------- forward

    def _conv(self, name, x, y, relu=True, y_coff=0):
        cin, cout = _shape(name)
        B, hh, ww, c = x.shape
        if c != cin:
            raise ValueError(f"{name}: input has {c} channels, expected {cin}")
        _, bias = self.weight(name)
        _check(N.load().stfwi_nn_conv3x3(_p(x), B, hh, ww, cin, _p(self.wf[name]), cout, _p(bias), int(relu),
                                         _p(y), y.shape[3], y_coff, self._stream()), name)

    def _pool(self, src, c, coff, dst):
        B, hh, ww, cs = src.shape
        _check(N.load().stfwi_nn_avgpool2(_p(src), B, hh, ww, c, cs, coff, _p(dst), self._stream()), "avgpool2")

    def _up(self, low, cat):
        B, hh, ww, c = low.shape
        _check(N.load().stfwi_nn_upsample2(_p(low), B, hh, ww, c, cat.shape[3], _p(cat), self._stream()),
               "upsample2")

    def forward(self, x, train=False):
        """Packed input [B, h, w, 16] -> output [B, h, w] FP32 (a view into
        the batch's buffers: copy it before the next call)."""
        B = x.shape[0]
        b = self.buffers(B, train)
        self._conv("enc1a", x, b["a1"])
        self._conv("enc1b", b["a1"], b["cat1"], y_coff=64)
        self._pool(b["cat1"], 32, 64, b["p1"])
        self._conv("enc2a", b["p1"], b["a2"])
        self._conv("enc2b", b["a2"], b["cat2"], y_coff=128)
        self._pool(b["cat2"], 64, 128, b["p2"])
        self._conv("enc3a", b["p2"], b["a3"])
        self._conv("enc3b", b["a3"], b["cat3"], y_coff=256)
        self._pool(b["cat3"], 128, 256, b["p3"])
        self._conv("bota", b["p3"], b["b1"])
        self._conv("botb", b["b1"], b["b2"])
        self._up(b["b2"], b["cat3"])
        self._conv("dec3a", b["cat3"], b["d3a"])
        self._conv("dec3b", b["d3a"], b["d3b"])
        self._up(b["d3b"], b["cat2"])
        self._conv("dec2a", b["cat2"], b["d2a"])
        self._conv("dec2b", b["d2a"], b["d2b"])
        self._up(b["d2b"], b["cat1"])
        self._conv("dec1a", b["cat1"], b["d1a"])
        self._conv("dec1b", b["d1a"], b["d1b"])
        hw, hb = self.head_params()
        npix = B * self.h * self.w
        _check(N.load().stfwi_nn_head(_p(b["d1b"]), npix, HEAD_IN, _p(hw), _p(hb), _p(b["out"]), self._stream()),
               "head")
        return b["out"]

    # ---------------------------------------------------------------- backward

    def _back(self, name, x, dz, dx=None, mask=None, m_coff=0):
        """Gradients of one convolution: bias and weights accumulate into the
        flat gradient buffer; dx (if given) receives the input gradient,
        masked by [mask > 0] when the input is a ReLU output."""
        L, st = N.load(), self._stream()
        cin, cout = _shape(name)
        B, hh, ww, _ = dz.shape
        gw, gb = self.grad(name)
        _check(L.stfwi_nn_bias_grad(_p(dz), B * hh * ww, cout, _p(gb), st), name + " bias_grad")
        _check(L.stfwi_nn_conv3x3_wgrad(_p(x), _p(dz), B, hh, ww, cin, cout, _p(gw), st), name + " wgrad")
        if dx is not None:
            mcs = mask.shape[3] if mask is not None else 0
            _check(L.stfwi_nn_conv3x3_dgrad(_p(dz), B, hh, ww, cout, _p(self.wt[name]), cin, _p(mask), mcs, m_coff,
                                            _p(dx), st), name + " dgrad")

    def _up_grad(self, dcat, low, dz):
        B, hh, ww, c = low.shape
        _check(N.load().stfwi_nn_upsample2_grad(_p(dcat), dcat.shape[3], _p(low), B, hh, ww, c, _p(dz),
                                                self._stream()), "upsample2_grad")

    def _skip_grad(self, dcat, cat, coff, dpool, dz):
        B, hh, ww, c = dz.shape
        _check(N.load().stfwi_nn_skip_grad(_p(dcat), _p(cat), cat.shape[3], coff, _p(dpool), B, hh, ww, c, _p(dz),
                                           self._stream()), "skip_grad")

    def backward(self, x, target, wgt, inv_norm):
        """After ``forward(x, train=True)``: the masked mean-square loss
        sum wgt (out - target)^2 * inv_norm (FP64, device) and the gradients of
        every parameter, accumulated into ``grads``."""
        B = x.shape[0]
        b = self.buffers(B, True)
        L, st = N.load(), self._stream()
        b["loss"].zero_()
        hw, _ = self.head_params()
        ghw, ghb = self.head_grads()
        _check(L.stfwi_nn_head_loss_grad(_p(b["d1b"]), B * self.h * self.w, HEAD_IN, _p(hw), _p(b["out"]),
                                         _p(target), _p(wgt), ct.c_float(inv_norm), _p(b["g_d1b"]), _p(ghw),
                                         _p(ghb), _p(b["loss"]), st), "head_loss_grad")
        self._back("dec1b", b["d1a"], b["g_d1b"], b["g_d1a"], mask=b["d1a"])
        self._back("dec1a", b["cat1"], b["g_d1a"], b["g_cat1"])
        self._up_grad(b["g_cat1"], b["d2b"], b["g_d2b"])
        self._back("dec2b", b["d2a"], b["g_d2b"], b["g_d2a"], mask=b["d2a"])
        self._back("dec2a", b["cat2"], b["g_d2a"], b["g_cat2"])
        self._up_grad(b["g_cat2"], b["d3b"], b["g_d3b"])
        self._back("dec3b", b["d3a"], b["g_d3b"], b["g_d3a"], mask=b["d3a"])
        self._back("dec3a", b["cat3"], b["g_d3a"], b["g_cat3"])
        self._up_grad(b["g_cat3"], b["b2"], b["g_b2"])
        self._back("botb", b["b1"], b["g_b2"], b["g_b1"], mask=b["b1"])
        self._back("bota", b["p3"], b["g_b1"], b["g_p3"])
        self._skip_grad(b["g_cat3"], b["cat3"], 256, b["g_p3"], b["g_s3"])
        self._back("enc3b", b["a3"], b["g_s3"], b["g_a3"], mask=b["a3"])
        self._back("enc3a", b["p2"], b["g_a3"], b["g_p2"])
        self._skip_grad(b["g_cat2"], b["cat2"], 128, b["g_p2"], b["g_s2"])
        self._back("enc2b", b["a2"], b["g_s2"], b["g_a2"], mask=b["a2"])
        self._back("enc2a", b["p1"], b["g_a2"], b["g_p1"])
        self._skip_grad(b["g_cat1"], b["cat1"], 64, b["g_p1"], b["g_s1"])
        self._back("enc1b", b["a1"], b["g_s1"], b["g_a1"], mask=b["a1"])
        self._back("enc1a", x, b["g_a1"])
        return b["loss"]

    def zero_grad(self):
        self.grads.zero_()

    def adam_step(self, lr, b1=0.9, b2=0.999, eps=1e-8, grad_scale=1.0):
        """One Adam update of the master weights (clears the gradients) and
        the BF16 repack."""
        self.step_count += 1
        t = self.step_count
        lr_t = lr * math.sqrt(1.0 - b2 ** t) / (1.0 - b1 ** t)
        _check(N.load().stfwi_nn_adam(_p(self.params), _p(self.grads), _p(self.m), _p(self.v), self.nparam,
                                      lr_t, b1, b2, eps, grad_scale, self._stream()), "adam")
        self.pack_weights()

    def train_step(self, x, target, wgt, lr, inv_norm=None):
        """Forward, loss, backward and one Adam step on a packed batch;
        returns the loss as a device FP64 tensor."""
        if inv_norm is None:
            inv_norm = 1.0 / max(float(wgt.sum()), 1.0)
        self.forward(x, train=True)
        loss = self.backward(x, target, wgt, inv_norm)
        self.adam_step(lr)
        return loss

    def check(self):
        """Synchronise and report a tensor-core pipeline wait that gave up."""
        _check(N.load().stfwi_nn_check(self._stream()), "network kernels")


def save_weights(path, params):
    """Store trained parameters compactly: the 3x3 convolution weights as the
    BF16 values the kernels read (their bits as uint16), the biases and the
    head in FP32.  Loading gives the network the kernels ran, unchanged."""
    import torch
    p = torch.as_tensor(np.asarray(params, dtype=np.float32))
    lay, head, total = param_layout()
    if p.numel() != total:
        raise ValueError("parameter count does not match the network")
    mask = np.zeros(total, dtype=bool)
    for wo, bo in lay.values():
        mask[wo:bo] = True
    w = p[torch.from_numpy(mask)].to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    np.savez_compressed(path, conv_bf16=w, rest_f32=p.numpy()[~mask], total=total)


def load_weights(path):
    """FP32 parameter vector from ``save_weights``."""
    import torch
    d = np.load(path)
    lay, _, total = param_layout()
    if int(d["total"]) != total:
        raise ValueError(f"{path}: parameter count does not match the network")
    mask = np.zeros(total, dtype=bool)
    for wo, bo in lay.values():
        mask[wo:bo] = True
    out = np.empty(total, dtype=np.float32)
    bits = torch.from_numpy(d["conv_bf16"].view(np.int16).copy())
    out[mask] = bits.view(torch.bfloat16).float().numpy()
    out[~mask] = d["rest_f32"]
    return out
