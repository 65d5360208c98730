"""A torch stand-in for the network entry points of include/stfwi_nn.h, for
testing the host wiring of stfwi_b200/learned/unet.py on the CPU: each
function restates the documented semantics of its C entry point in FP64
torch ops on the tensors the host code passes (the pointer helper is
replaced by the identity) and stores its result in the tensor's own dtype.
Test infrastructure only."""
import torch
import torch.nn.functional as F

from tests.unet_ref import conv


def _nchw(t, n, h, w, c):
    return t.reshape(n, h, w, c).permute(0, 3, 1, 2).double()


def _store(dst, n, h, w, cstride, coff, val_nchw):
    v = dst.view(n, h, w, cstride)
    v[..., coff:coff + val_nchw.shape[1]] = val_nchw.permute(0, 2, 3, 1).to(dst.dtype)


def _f(x):
    return float(x.value) if hasattr(x, "value") else float(x)


class FakeNN:
    def stfwi_nn_last_error(self):
        return b""

    def stfwi_nn_check(self, stream):
        return 0

    def stfwi_nn_conv3x3(self, x, n, h, w, cin, wt, cout, bias, relu, y, ycs, yoff, stream):
        out = conv(_nchw(x, n, h, w, cin), wt.reshape(9, cout, cin).double(), bias.double(), relu=bool(relu))
        _store(y, n, h, w, ycs, yoff, out)
        return 0

    def stfwi_nn_conv3x3_dgrad(self, dz, n, h, w, cout, wt_t, cin, mask, mcs, mcoff, dx, stream):
        out = conv(_nchw(dz, n, h, w, cout), wt_t.reshape(9, cin, cout).double())
        if mask is not None:
            out = out * (_nchw(mask, n, h, w, mcs)[:, mcoff:mcoff + cin] > 0)
        _store(dx, n, h, w, cin, 0, out)
        return 0

    def stfwi_nn_conv3x3_wgrad(self, x, dz, n, h, w, cin, cout, dw, stream):
        w9 = torch.zeros((9, cout, cin), dtype=torch.float64, requires_grad=True)
        conv(_nchw(x, n, h, w, cin), w9).backward(_nchw(dz, n, h, w, cout))
        dw.view(9, cout, cin).add_(w9.grad.to(dw.dtype))
        return 0

    def stfwi_nn_pack_input(self, feat, n, hd, wd, h, w, scale4, x, stream):
        xv = x.view(n, h, w, 16)
        xv.zero_()
        sc = torch.tensor([scale4[i] for i in range(4)], dtype=torch.float64)
        xv[:, :hd, :wd, :4] = (feat.double() * sc[None, :, None, None]).permute(0, 2, 3, 1).to(x.dtype)
        return 0

    def stfwi_nn_avgpool2(self, src, n, h, w, c, cs, coff, dst, stream):
        v = _nchw(src, n, h, w, cs)[:, coff:coff + c]
        _store(dst, n, h // 2, w // 2, c, 0, F.avg_pool2d(v, 2))
        return 0

    def stfwi_nn_skip_grad(self, dcat, ycat, cs, coff, dpool, n, h, w, c, dz, stream):
        g = F.interpolate(_nchw(dpool, n, h // 2, w // 2, c), scale_factor=2) / 4
        if dcat is not None:
            g = g + _nchw(dcat, n, h, w, cs)[:, coff:coff + c]
        _store(dz, n, h, w, c, 0, g * (_nchw(ycat, n, h, w, cs)[:, coff:coff + c] > 0))
        return 0

    def stfwi_nn_upsample2(self, low, n, h, w, c, ocs, out, stream):
        _store(out, n, 2 * h, 2 * w, ocs, 0, F.interpolate(_nchw(low, n, h, w, c), scale_factor=2))
        return 0

    def stfwi_nn_upsample2_grad(self, dcat, cs, low, n, h, w, c, dz, stream):
        g = F.avg_pool2d(_nchw(dcat, n, 2 * h, 2 * w, cs)[:, :c], 2) * 4
        _store(dz, n, h, w, c, 0, g * (_nchw(low, n, h, w, c) > 0))
        return 0

    def stfwi_nn_head(self, y, npix, c, wt, b, out, stream):
        out.view(-1)[:npix] = (y.reshape(npix, c).double() @ wt.double() + b.double()[0]).to(out.dtype)
        return 0

    def stfwi_nn_head_loss_grad(self, y, npix, c, wt, out, target, wgt, inv_norm, dz, dwt, db, loss, stream):
        inv = _f(inv_norm)
        yv = y.reshape(npix, c).double()
        r = out.reshape(-1).double() - target.reshape(-1).double()
        wv = wgt.reshape(-1).double()
        loss.add_((wv * r * r).sum() * inv)
        g = 2.0 * wv * r * inv
        db.add_(g.sum().to(db.dtype))
        dwt.add_((g @ yv).to(dwt.dtype))
        dz.view(npix, c)[:] = (g[:, None] * wt.double()[None, :] * (yv > 0)).to(dz.dtype)
        return 0

    def stfwi_nn_bias_grad(self, dz, npix, c, db, stream):
        db.add_(dz.reshape(npix, c).double().sum(0).to(db.dtype))
        return 0

    def stfwi_nn_pack_weights(self, w32, cout, cin, wf, wt, stream):
        w = w32.reshape(9, cout, cin)
        wf.view(9, cout, cin)[:] = w.to(wf.dtype)
        if wt is not None:
            wt.view(9, cin, cout)[:] = w.flip(0).transpose(1, 2).to(wt.dtype)
        return 0

    def stfwi_nn_adam(self, p, g, m, v, n, lr_t, b1, b2, eps, grad_scale, stream):
        lr_t, b1, b2, eps, gs = (_f(a) for a in (lr_t, b1, b2, eps, grad_scale))
        gi = g * gs
        m.mul_(b1).add_((1 - b1) * gi)
        v.mul_(b2).add_((1 - b2) * gi * gi)
        p.sub_(lr_t * m / (v.sqrt() + eps))
        g.zero_()
        return 0
