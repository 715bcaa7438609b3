"""Learned start for Richardson-Lucy: a small 3-D U-Net that maps an early RL
iterate to an advanced one, from which RL resumes.

The network (4 levels, widths 16-32-64-128, 3x3x3 convolutions, ReLU, average
pooling down, nearest upsampling + skip concatenation up, a 1x1x1 head) runs
on this library's own kernels (csrc/nn.cu, through the C ABI): BF16 weights
and activations, FP32 accumulation on the tensor cores, FP32 master weights
and Adam.  PyTorch only provides device memory and streams.

Input and output are in the log domain of the mean-normalised estimate:
    a = x / mean(x),  in = log(a + EPS),  prediction = mean(x) ((a + EPS) e^r - EPS)
so the head's output r is a per-voxel log-ratio and the scale of the volume
does not matter.  Volumes must have dimensions divisible by 8 (three poolings).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import api

EPS = 0.01
WIDTHS = (16, 32, 64, 128)

# (name, cin of the full-resolution input, cin of the upsampled input, cout)
CONV_LAYERS = [
    ("l0b", 16, 0, 16),
    ("l1a", 16, 0, 32), ("l1b", 32, 0, 32),
    ("l2a", 32, 0, 64), ("l2b", 64, 0, 64),
    ("l3a", 64, 0, 128), ("l3b", 128, 0, 128),
    ("l2c", 64, 128, 64), ("l2d", 64, 0, 64),
    ("l1c", 32, 64, 32), ("l1d", 32, 0, 32),
    ("l0c", 16, 32, 16), ("l0d", 16, 0, 16),
]


def _lib():
    L = api.load()
    if not hasattr(L, "_nn_ready"):
        vp, i, f, ll = C.c_void_p, C.c_int, C.c_float, C.c_longlong
        L.clarityx_nn_conv3.argtypes = [vp, i, vp, i, i, i, i, vp, vp, i, i, vp, vp, vp]
        L.clarityx_nn_conv3_wgrad.argtypes = [vp, i, vp, i, i, i, i, vp, i, vp, vp, vp]
        L.clarityx_nn_conv_in.argtypes = [vp, i, i, i, vp, vp, vp, vp]
        L.clarityx_nn_conv_in_wgrad.argtypes = [vp, i, i, i, vp, vp, vp, vp]
        L.clarityx_nn_head.argtypes = [vp, ll, vp, vp, vp, vp]
        L.clarityx_nn_head_loss_grad.argtypes = [vp, ll, vp, vp, vp, vp, vp, vp, vp, vp]
        L.clarityx_nn_pool2.argtypes = [vp, i, i, i, i, vp, vp]
        L.clarityx_nn_merge_skip_grad.argtypes = [vp, i, vp, vp, i, i, i, i, vp, vp]
        L.clarityx_nn_up_grad.argtypes = [vp, i, i, i, vp, i, i, i, vp, vp]
        L.clarityx_nn_adam.argtypes = [vp, vp, vp, vp, ll, f, f, f, f, i, vp]
        L.clarityx_nn_pack_weights.argtypes = [vp, i, i, vp, vp, vp]
        for n in ("conv3", "conv3_wgrad", "conv_in", "conv_in_wgrad", "head", "head_loss_grad",
                  "pool2", "merge_skip_grad", "up_grad", "adam", "pack_weights"):
            getattr(L, f"clarityx_nn_{n}").restype = i
        L._nn_ready = True
    return L


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _s(stream):
    import torch
    return C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)


# ----------------------------------------------------------- primitives
def conv3(x1, w, cout, bias=None, relu=True, x2=None, mask=None, out=None, stream=None):
    """3x3x3 convolution of x1 [D,H,W,c1] (+ x2 [D/2,H/2,W/2,c2] upsampled)."""
    import torch
    D, H, W, c1 = x1.shape
    c2 = x2.shape[3] if x2 is not None else 0
    y = out if out is not None else torch.empty((D, H, W, cout), dtype=torch.bfloat16,
                                                 device=x1.device)
    api._check(_lib().clarityx_nn_conv3(_p(x1), c1, _p(x2), c2, D, H, W, _p(w), _p(bias), cout,
                                        1 if relu else 0, _p(mask), _p(y), _s(stream)))
    return y


def conv3_wgrad(x1, dy, dw, db=None, x2=None, stream=None):
    D, H, W, c1 = x1.shape
    c2 = x2.shape[3] if x2 is not None else 0
    api._check(_lib().clarityx_nn_conv3_wgrad(_p(x1), c1, _p(x2), c2, D, H, W, _p(dy),
                                              dy.shape[3], _p(dw), _p(db), _s(stream)))


def pool2(x, stream=None):
    import torch
    D, H, W, Cc = x.shape
    y = torch.empty((D // 2, H // 2, W // 2, Cc), dtype=torch.bfloat16, device=x.device)
    api._check(_lib().clarityx_nn_pool2(_p(x), Cc, D, H, W, _p(y), _s(stream)))
    return y


class UNet3D:
    """Parameters, forward, backward and Adam of the learned-start network."""

    def __init__(self, seed: int = 0, device: str = "cuda"):
        import torch
        self.device = device
        rng = np.random.default_rng(seed)
        specs = [("l0a", 1, 0, 16)] + CONV_LAYERS
        sizes, self.layout = [], {}
        off = 0
        for name, c1, c2, co in specs:
            nw = co * 27 * (c1 + c2)
            self.layout[name] = (off, nw, off + nw, co, c1, c2)
            off += nw + co
        self.layout["head"] = (off, 16, off + 16, 1, 16, 0)
        off += 17
        self.nparams = off
        p = np.zeros(off, np.float32)
        for name, c1, c2, co in specs:
            o, nw, ob, _, _, _ = self.layout[name]
            p[o:o + nw] = rng.standard_normal(nw) * math.sqrt(2.0 / (27 * (c1 + c2)))
        # zero head: the untrained network returns its input
        self.p = torch.from_numpy(p).to(device)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step_count = 0
        self.wf, self.wb = {}, {}
        for name, c1, c2, co in CONV_LAYERS:
            self.wf[name] = torch.empty(co * 27 * (c1 + c2), dtype=torch.bfloat16, device=device)
            self.wb[name] = torch.empty_like(self.wf[name])
        self.pack()

    # parameter views
    def w(self, name, t=None):
        o, nw, _, _, _, _ = self.layout[name]
        return (t if t is not None else self.p)[o:o + nw]

    def b(self, name, t=None):
        _, _, ob, co, _, _ = self.layout[name]
        return (t if t is not None else self.p)[ob:ob + co]

    def pack(self, stream=None):
        L = _lib()
        for name, c1, c2, co in CONV_LAYERS:
            api._check(L.clarityx_nn_pack_weights(_p(self.w(name)), co, c1 + c2,
                                                  _p(self.wf[name]), _p(self.wb[name]),
                                                  _s(stream)))

    def state(self) -> np.ndarray:
        return self.p.cpu().numpy()

    def load_state(self, arr) -> None:
        import torch
        arr = np.asarray(arr, np.float32)
        if arr.size != self.nparams:
            raise ValueError(f"expected {self.nparams} parameters, got {arr.size}")
        self.p.copy_(torch.from_numpy(arr).to(self.device))
        self.pack()

    # ------------------------------------------------------------ forward
    def forward(self, inp, stream=None, keep=False):
        """inp: float32 [D, H, W] (the log-domain input).  Returns r [D, H, W]
        (float32) and, with keep, the activations for backward."""
        import torch
        L = _lib()
        D, H, W = inp.shape
        if D % 8 or H % 8 or W % 8:
            raise ValueError("volume dimensions must be multiples of 8")
        st = _s(stream)
        A = {}
        a0 = torch.empty((D, H, W, 16), dtype=torch.bfloat16, device=inp.device)
        api._check(L.clarityx_nn_conv_in(_p(inp), D, H, W, _p(self.w("l0a")), _p(self.b("l0a")),
                                         _p(a0), st))
        A["a0"] = a0
        cv = lambda name, x1, x2=None: conv3(x1, self.wf[name], self.layout[name][3],
                                            bias=self.b(name), relu=True, x2=x2, stream=stream)
        A["s0"] = cv("l0b", a0)
        A["p0"] = pool2(A["s0"], stream)
        A["a1"] = cv("l1a", A["p0"])
        A["s1"] = cv("l1b", A["a1"])
        A["p1"] = pool2(A["s1"], stream)
        A["a2"] = cv("l2a", A["p1"])
        A["s2"] = cv("l2b", A["a2"])
        A["p2"] = pool2(A["s2"], stream)
        A["a3"] = cv("l3a", A["p2"])
        A["b3"] = cv("l3b", A["a3"])
        A["c2"] = cv("l2c", A["s2"], A["b3"])
        A["d2"] = cv("l2d", A["c2"])
        A["c1"] = cv("l1c", A["s1"], A["d2"])
        A["d1"] = cv("l1d", A["c1"])
        A["c0"] = cv("l0c", A["s0"], A["d1"])
        A["d0"] = cv("l0d", A["c0"])
        r = torch.empty((D, H, W), dtype=torch.float32, device=inp.device)
        api._check(L.clarityx_nn_head(_p(A["d0"]), D * H * W, _p(self.w("head")),
                                      _p(self.b("head")), _p(r), st))
        if keep:
            A["inp"] = inp
            A["r"] = r
            return r, A
        return r

    # ----------------------------------------------------------- backward
    def backward(self, A, target, loss_out, stream=None):
        """Accumulates parameter gradients of sum-of-squares loss mean((r -
        target)^2) into self.g; adds the loss to loss_out (float64 [1])."""
        import torch
        L = _lib()
        st = _s(stream)
        D, H, W = target.shape
        V = D * H * W
        g = self.g
        g_d0 = torch.empty_like(A["d0"])
        api._check(L.clarityx_nn_head_loss_grad(_p(A["d0"]), V, _p(self.w("head")), _p(A["r"]),
                                                _p(target), _p(g_d0), _p(self.w("head", g)),
                                                _p(self.b("head", g)), _p(loss_out), st))

        def lay(name, x1, dy, x2=None):
            conv3_wgrad(x1, dy, self.w(name, g), self.b(name, g), x2=x2, stream=stream)

        def bwd(name, dy, mask=None):
            c1, c2 = self.layout[name][4], self.layout[name][5]
            return conv3(dy, self.wb[name], c1 + c2, relu=False, mask=mask, stream=stream)

        def up_grad(dxcat, c1, c2, coarse):
            Dd, Hh, Ww, cc = dxcat.shape
            out = torch.empty_like(coarse)
            api._check(L.clarityx_nn_up_grad(_p(dxcat), cc, c1, c2, _p(coarse), Dd, Hh, Ww,
                                             _p(out), st))
            return out

        def skip_grad(dxcat, c1, dp, s):
            Dd, Hh, Ww, _ = s.shape
            out = torch.empty_like(s)
            api._check(L.clarityx_nn_merge_skip_grad(_p(dxcat), dxcat.shape[3], _p(dp), _p(s), c1,
                                                     Dd, Hh, Ww, _p(out), st))
            return out

        lay("l0d", A["c0"], g_d0)
        g_c0 = bwd("l0d", g_d0, mask=A["c0"])
        lay("l0c", A["s0"], g_c0, x2=A["d1"])
        dx0 = bwd("l0c", g_c0)
        g_d1 = up_grad(dx0, 16, 32, A["d1"])
        lay("l1d", A["c1"], g_d1)
        g_c1 = bwd("l1d", g_d1, mask=A["c1"])
        lay("l1c", A["s1"], g_c1, x2=A["d2"])
        dx1 = bwd("l1c", g_c1)
        g_d2 = up_grad(dx1, 32, 64, A["d2"])
        lay("l2d", A["c2"], g_d2)
        g_c2 = bwd("l2d", g_d2, mask=A["c2"])
        lay("l2c", A["s2"], g_c2, x2=A["b3"])
        dx2 = bwd("l2c", g_c2)
        g_b3 = up_grad(dx2, 64, 128, A["b3"])
        lay("l3b", A["a3"], g_b3)
        g_a3 = bwd("l3b", g_b3, mask=A["a3"])
        lay("l3a", A["p2"], g_a3)
        dp2 = bwd("l3a", g_a3)
        g_s2 = skip_grad(dx2, 64, dp2, A["s2"])
        lay("l2b", A["a2"], g_s2)
        g_a2 = bwd("l2b", g_s2, mask=A["a2"])
        lay("l2a", A["p1"], g_a2)
        dp1 = bwd("l2a", g_a2)
        g_s1 = skip_grad(dx1, 32, dp1, A["s1"])
        lay("l1b", A["a1"], g_s1)
        g_a1 = bwd("l1b", g_s1, mask=A["a1"])
        lay("l1a", A["p0"], g_a1)
        dp0 = bwd("l1a", g_a1)
        g_s0 = skip_grad(dx0, 16, dp0, A["s0"])
        lay("l0b", A["a0"], g_s0)
        g_a0 = bwd("l0b", g_s0, mask=A["a0"])
        api._check(L.clarityx_nn_conv_in_wgrad(_p(A["inp"]), D, H, W, _p(g_a0),
                                               _p(self.w("l0a", g)), _p(self.b("l0a", g)), st))

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, scale=1.0, stream=None):
        """One Adam step on the accumulated gradients (times `scale`), then
        zeroes them and repacks the BF16 weights."""
        if scale != 1.0:
            self.g.mul_(scale)
        self.step_count += 1
        api._check(_lib().clarityx_nn_adam(_p(self.p), _p(self.g), _p(self.m), _p(self.v),
                                           self.nparams, lr, b1, b2, eps, self.step_count,
                                           _s(stream)))
        self.g.zero_()
        self.pack(stream)


# ------------------------------------------------------------ data domain
def to_input(x):
    """(network input, mean) of an estimate x [D, H, W] (device float32)."""
    m = x.mean().clamp_min(1e-20)
    return (x / m + EPS).log(), m


def to_target(x_early, x_late):
    """Log-ratio target of the late iterate against the early one."""
    m = x_early.mean().clamp_min(1e-20)
    return ((x_late / m + EPS) / (x_early / m + EPS)).log()


def apply_prediction(x_early, r):
    m = x_early.mean().clamp_min(1e-20)
    return (m * ((x_early / m + EPS) * r.exp() - EPS)).clamp_min(0.0)


def predict(net: UNet3D, x_early, stream=None):
    """The network's advanced estimate from an early iterate, by the
    library's fused forward (clarityx_nn_predict: the domain transforms run
    inside the network's first and last kernels)."""
    import torch
    out = torch.empty_like(x_early)
    return api.nn_predict(net.p, x_early.contiguous(), out, stream=stream)


def predict_unfused(net: UNet3D, x_early, stream=None):
    """The same prediction through the training path's separate domain
    transforms (to_input, forward, apply_prediction): the check for the
    fused form."""
    inp, _ = to_input(x_early)
    r = net.forward(inp, stream=stream)
    return apply_prediction(x_early, r)
