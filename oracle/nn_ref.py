"""TEST INFRASTRUCTURE ONLY (oracle).  FP64 CPU reference of the learned-start
network (clarity_b200/unet.py, csrc/nn.cu): the same layers written with
torch.nn.functional on float64 CPU tensors, so gradients come from autograd.
Only tests/ use it, to check the CUDA kernels (forward, backward data,
weight gradients) and the whole network's loss gradient.

Layouts follow the CUDA side: activations [D, H, W, C] (channels last),
weights [cout, 27, cin] with tap = (dz+1)*9 + (dy+1)*3 + (dx+1).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

T = torch.float64


def w_to_torch(w, cout, cin):
    """[cout, 27, cin] -> torch conv3d weight [cout, cin, 3, 3, 3] (tensors
    keep their autograd history)."""
    w = w if torch.is_tensor(w) else torch.as_tensor(np.asarray(w, np.float64))
    w = w.reshape(cout, 27, cin)
    return w.permute(0, 2, 1).reshape(cout, cin, 3, 3, 3)


def to_ncdhw(x):
    return x.permute(3, 0, 1, 2).unsqueeze(0)


def from_ncdhw(x):
    return x.squeeze(0).permute(1, 2, 3, 0)


def conv3(x1, w, cout, bias=None, relu=True, x2=None, mask=None):
    """x1 [D,H,W,c1] (+ x2 [D/2,H/2,W/2,c2] nearest-upsampled) -> [D,H,W,cout]."""
    xs = [x1]
    if x2 is not None:
        xs.append(x2.repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2))
    x = torch.cat(xs, dim=3)
    cin = x.shape[3]
    b = None
    if bias is not None:
        b = (bias if torch.is_tensor(bias) else torch.as_tensor(np.asarray(bias))).to(x.dtype)
    y = F.conv3d(to_ncdhw(x), w_to_torch(w, cout, cin).to(x.dtype), b, padding=1)
    y = from_ncdhw(y)
    if relu:
        y = F.relu(y)
    if mask is not None:
        y = y * (mask > 0).to(y.dtype)
    return y


def pool2(x):
    return from_ncdhw(F.avg_pool3d(to_ncdhw(x), 2))


def bf16_round(a):
    """Round an array to bfloat16 and back (the kernels' storage precision)."""
    return torch.as_tensor(np.asarray(a)).to(torch.bfloat16).to(T)


LAYERS = [("l0b", 16, 0, 16), ("l1a", 16, 0, 32), ("l1b", 32, 0, 32), ("l2a", 32, 0, 64),
          ("l2b", 64, 0, 64), ("l3a", 64, 0, 128), ("l3b", 128, 0, 128), ("l2c", 64, 128, 64),
          ("l2d", 64, 0, 64), ("l1c", 32, 64, 32), ("l1d", 32, 0, 32), ("l0c", 16, 32, 16),
          ("l0d", 16, 0, 16)]


def unet_loss(params: dict, inp, target):
    """The network's loss mean((r - target)^2) with `params` a dict of torch
    float64 tensors (requires_grad as wanted): name -> (w [cout,27,cin], b),
    'l0a' -> (w [16,27], b [16]), 'head' -> (w [16], b [1]).  Convolution
    weights are used as given (the caller rounds them to bf16 to match)."""
    x = torch.as_tensor(np.asarray(inp, np.float64)) if not torch.is_tensor(inp) else inp
    w0, b0 = params["l0a"]
    a0 = F.relu(from_ncdhw(F.conv3d(x[None, None], w0.reshape(16, 1, 3, 3, 3), b0, padding=1)))

    def cv(name, x1, x2=None):
        w, b = params[name]
        xs = [x1]
        if x2 is not None:
            xs.append(x2.repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2))
        xx = torch.cat(xs, dim=3)
        cout, cin = w.shape[0], xx.shape[3]
        wt = w.reshape(cout, 27, cin).permute(0, 2, 1).reshape(cout, cin, 3, 3, 3)
        return F.relu(from_ncdhw(F.conv3d(to_ncdhw(xx), wt, b, padding=1)))

    s0 = cv("l0b", a0)
    a1 = cv("l1a", pool2(s0))
    s1 = cv("l1b", a1)
    a2 = cv("l2a", pool2(s1))
    s2 = cv("l2b", a2)
    a3 = cv("l3a", pool2(s2))
    b3 = cv("l3b", a3)
    d2 = cv("l2d", cv("l2c", s2, b3))
    d1 = cv("l1d", cv("l1c", s1, d2))
    d0 = cv("l0d", cv("l0c", s0, d1))
    wh, bh = params["head"]
    r = (d0 * wh).sum(dim=3) + bh
    t = torch.as_tensor(np.asarray(target, np.float64))
    return ((r - t) ** 2).mean(), r
