"""GPU checks of the learned-start network's kernels (csrc/nn.cu) against an
FP64 CPU reference of the same layers (oracle/nn_ref.py, torch autograd).

Inputs and weights are BF16 on both sides (the reference computes on the
BF16-rounded values in FP64); the kernels accumulate in FP32 and store BF16,
so results agree to BF16 precision (relative error ~1e-2 of the largest
value), gradients of the whole network to a few per cent per layer and a
cosine similarity above 0.99.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

import nn_ref as R  # noqa: E402


def _close(got, want, rel=2e-2):
    got = got.detach().to(torch.float64).cpu()
    want = want.detach().to(torch.float64).cpu()
    err = (got - want).abs().max().item()
    scale = want.abs().max().item()
    assert err <= rel * max(scale, 1e-12), (err, scale)


def _rand(shape, g, scale=1.0):
    return (torch.randn(shape, generator=g, dtype=torch.float64) * scale).to(torch.bfloat16)


@pytest.mark.parametrize("c1,c2,cout,dims", [(16, 0, 16, (8, 12, 16)), (32, 0, 48, (6, 10, 8)),
                                             (16, 32, 64, (8, 8, 12)), (64, 128, 64, (4, 6, 8)),
                                             (128, 0, 128, (4, 4, 4)),
                                             # widths that are multiples of 32 take the
                                             # tcgen05 kernel: 128-, 64- and 32-wide MMA
                                             # tiles, 1, 2 or 4 rows per item, one or more
                                             # channel blocks, half-resolution chunks
                                             (16, 0, 16, (2, 4, 128)), (16, 32, 64, (2, 4, 128)),
                                             (32, 0, 48, (4, 2, 128)), (64, 0, 128, (2, 2, 256)),
                                             (16, 0, 80, (2, 4, 128)), (16, 32, 32, (4, 8, 64)),
                                             (32, 0, 48, (2, 6, 64)), (64, 64, 128, (2, 4, 32))])
def test_conv3_forward_backward_vs_reference(clarity_gpu, c1, c2, cout, dims):
    from clarity_b200 import unet
    g = torch.Generator().manual_seed(c1 * 7 + c2 + cout)
    D, H, W = dims
    x1 = _rand((D, H, W, c1), g)
    x2 = _rand((D // 2, H // 2, W // 2, c2), g) if c2 else None
    cin = c1 + c2
    wf32 = torch.randn((cout, 27, cin), generator=g, dtype=torch.float64) / np.sqrt(27 * cin)
    bias = torch.randn(cout, generator=g, dtype=torch.float64) * 0.1
    # BF16 weights in both layouts from the FP32 master copy
    wd = wf32.to(torch.float32).cuda().contiguous()
    wf = torch.empty(cout * 27 * cin, dtype=torch.bfloat16, device="cuda")
    wb = torch.empty_like(wf)
    clarity_gpu._check(unet._lib().clarityx_nn_pack_weights(
        unet._p(wd), cout, cin, unet._p(wf), unet._p(wb), unet._s(None)))
    wq = wd.to(torch.bfloat16).to(torch.float64).cpu()
    # forward with bias + ReLU
    y = unet.conv3(x1.cuda(), wf, cout, bias=bias.to(torch.float32).cuda(), relu=True,
                   x2=x2.cuda() if x2 is not None else None)
    torch.cuda.synchronize()
    xa = x1.to(torch.float64).requires_grad_(True)
    xb = x2.to(torch.float64).requires_grad_(True) if x2 is not None else None
    wt = wq.clone().requires_grad_(True)
    ref = R.conv3(xa, wt, cout, bias=bias.to(torch.float32).to(torch.float64), relu=False, x2=xb)
    _close(y, torch.relu(ref))
    # backward data: the same kernel with the mirrored, transposed weights
    dy = _rand((D, H, W, cout), g)
    dx = unet.conv3(dy.cuda(), wb, cin, relu=False)
    torch.cuda.synchronize()
    (ref * dy.to(torch.float64)).sum().backward()
    _close(dx[..., :c1], xa.grad)
    if xb is not None:
        # the upsampled part: summing 2x2x2 children gives the coarse gradient
        up = torch.empty((D // 2, H // 2, W // 2, c2), dtype=torch.bfloat16, device="cuda")
        ones = torch.ones((D // 2, H // 2, W // 2, c2), dtype=torch.bfloat16, device="cuda")
        clarity_gpu._check(unet._lib().clarityx_nn_up_grad(
            unet._p(dx), cin, c1, c2, unet._p(ones), D, H, W, unet._p(up), unet._s(None)))
        torch.cuda.synchronize()
        _close(up, xb.grad, rel=3e-2)
    # weight and bias gradients
    dw = torch.zeros(cout * 27 * cin, dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    unet.conv3_wgrad(x1.cuda(), dy.cuda(), dw, db, x2=x2.cuda() if x2 is not None else None)
    torch.cuda.synchronize()
    _close(dw.reshape(cout, 27, cin), wt.grad, rel=1e-2)
    _close(db, dy.to(torch.float64).sum(dim=(0, 1, 2)), rel=1e-2)


_CROSS = """
import sys, numpy as np, torch
from clarity_b200 import unet
x, w, m = (np.load(sys.argv[i]) for i in (1, 2, 3))
xd = torch.from_numpy(x).view(torch.bfloat16).cuda()
wd = torch.from_numpy(w).view(torch.bfloat16).cuda()
md = torch.from_numpy(m).view(torch.bfloat16).cuda()
cout = int(sys.argv[5])
b = torch.linspace(-0.5, 0.5, cout, device="cuda")
y = unet.conv3(xd, wd, cout, bias=b, relu=True)
ym = unet.conv3(xd, wd, cout, relu=False, mask=md)
torch.cuda.synchronize()
np.save(sys.argv[4], torch.stack([y, ym]).view(torch.int16).cpu().numpy())
"""


@pytest.mark.parametrize("dims,cin,cout", [((4, 4, 256), 32, 64), ((2, 8, 64), 48, 16),
                                           ((2, 8, 32), 64, 128)])
def test_conv3_tcgen05_matches_mma_sync_kernel(clarity_gpu, tmp_path, dims, cin, cout):
    # the same layers through both kernels, each in its own process:
    # CLARITY_NN_TCGEN05=require (a call the tcgen05 kernel cannot take is an
    # error, so this proves it ran) and CLARITY_NN_TCGEN05=0 (mma.sync)
    import os
    import subprocess
    import sys
    from conftest import ROOT
    g = torch.Generator().manual_seed(11 + cin + cout)
    x = _rand((*dims, cin), g)
    w = _rand((cout * 27 * cin,), g, 1.0 / np.sqrt(27 * cin))
    m = _rand((*dims, cout), g)
    for name, t in (("x", x), ("w", w), ("m", m)):
        np.save(tmp_path / f"{name}.npy", t.view(torch.int16).numpy())
    outs = {}
    for mode in ("require", "0"):
        env = dict(os.environ, CLARITY_NN_TCGEN05=mode, PYTHONPATH=ROOT)
        p = subprocess.run([sys.executable, "-c", _CROSS, *(str(tmp_path / f"{n}.npy")
                                                             for n in "xwm"),
                            str(tmp_path / f"y{mode}.npy"), str(cout)],
                           cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        outs[mode] = torch.from_numpy(np.load(tmp_path / f"y{mode}.npy")).view(torch.bfloat16)
    tc, ms = outs["require"], outs["0"]
    # FP32 sums in another order, then BF16 rounding: equal or one BF16 step apart
    _close(tc[0], ms[0], rel=1e-2)
    _close(tc[1], ms[1], rel=1e-2)
    assert torch.count_nonzero(tc[0]) > 0
    # and both against the FP64 reference of the layer
    wq = w.to(torch.float64).reshape(cout, 27, cin)
    ref = R.conv3(x.to(torch.float64), wq, cout,
                  bias=torch.linspace(-0.5, 0.5, cout, dtype=torch.float64), relu=False)
    _close(tc[0], torch.relu(ref))


@pytest.mark.parametrize("dims", [(8, 8, 8), (2, 4, 128), (2, 4, 32)])  # both kernels
def test_conv3_relu_mask_epilogue(clarity_gpu, dims):
    from clarity_b200 import unet
    g = torch.Generator().manual_seed(3)
    x = _rand((*dims, 16), g).cuda()
    m = _rand((*dims, 16), g).cuda()
    w = _rand((16 * 27 * 16,), g, 0.05).cuda()
    y = unet.conv3(x, w, 16, relu=False)
    ym = unet.conv3(x, w, 16, relu=False, mask=m)
    torch.cuda.synchronize()
    assert torch.equal(ym, torch.where(m > 0, y, torch.zeros_like(y)))


def test_pool_and_skip_merge(clarity_gpu):
    from clarity_b200 import unet
    g = torch.Generator().manual_seed(4)
    s = _rand((8, 6, 10, 16), g)
    p = unet.pool2(s.cuda())
    torch.cuda.synchronize()
    _close(p, R.pool2(s.to(torch.float64)), rel=1e-2)
    dxcat = _rand((8, 6, 10, 48), g)
    dp = _rand((4, 3, 5, 16), g)
    out = torch.empty((8, 6, 10, 16), dtype=torch.bfloat16, device="cuda")
    # device copies held in names: a temporary's memory could be reused by the
    # next one before the kernel runs
    dxd, dpd, sd = dxcat.cuda(), dp.cuda(), s.cuda()
    clarity_gpu._check(unet._lib().clarityx_nn_merge_skip_grad(
        unet._p(dxd), 48, unet._p(dpd), unet._p(sd), 16, 8, 6, 10, unet._p(out),
        unet._s(None)))
    torch.cuda.synchronize()
    up = dp.to(torch.float64).repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2)
    want = (dxcat.to(torch.float64)[..., :16] + up / 8) * (s.to(torch.float64) > 0)
    _close(out, want, rel=1e-2)


def _ref_params(net):
    p = torch.as_tensor(net.state(), dtype=torch.float64)
    out = {}
    for name, (o, nw, ob, co, c1, c2) in net.layout.items():
        w = p[o:o + nw]
        if name not in ("l0a", "head"):
            w = w.to(torch.float32).to(torch.bfloat16).to(torch.float64)  # the kernels' weights
        if name == "l0a":
            w = w.reshape(16, 27)
        elif name != "head":
            w = w.reshape(co, 27, c1 + c2)
        out[name] = (w.clone().requires_grad_(True), p[ob:ob + co].clone().requires_grad_(True))
    return out


def test_unet_loss_gradient_vs_reference(clarity_gpu):
    # the whole network: loss and every layer's gradient against FP64 autograd
    from clarity_b200 import unet
    net = unet.UNet3D(seed=5)
    g = torch.Generator().manual_seed(6)
    st = net.state()
    o, nw, ob, _, _, _ = net.layout["head"]
    st[o:o + nw] = np.random.default_rng(7).standard_normal(nw) * 0.3
    net.load_state(st)
    inp = torch.randn((16, 16, 16), generator=g, dtype=torch.float32)
    tgt = torch.randn((16, 16, 16), generator=g, dtype=torch.float32) * 0.1
    r, A = net.forward(inp.cuda(), keep=True)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    net.backward(A, tgt.cuda(), loss)
    torch.cuda.synchronize()
    params = _ref_params(net)
    ref_loss, ref_r = R.unet_loss(params, inp.to(torch.float64), tgt)
    ref_loss.backward()
    assert abs(loss.item() - ref_loss.item()) <= 0.05 * ref_loss.item()
    _close(r, ref_r, rel=5e-2)
    gpu_g = torch.as_tensor(net.g.cpu().numpy(), dtype=torch.float64)
    a, b = [], []
    for name, (o, nw, ob, co, c1, c2) in net.layout.items():
        wg, bg = params[name][0].grad.reshape(-1), params[name][1].grad.reshape(-1)
        mine_w, mine_b = gpu_g[o:o + nw], gpu_g[ob:ob + co]
        rel = (mine_w - wg).norm() / max(wg.norm().item(), 1e-30)
        assert rel <= 0.1, (name, rel.item())
        a += [mine_w, mine_b]
        b += [wg, bg]
    a, b = torch.cat(a), torch.cat(b)
    assert torch.dot(a, b) / (a.norm() * b.norm()) >= 0.99


def test_unet_training_reduces_loss(clarity_gpu):
    from clarity_b200 import unet
    net = unet.UNet3D(seed=8)
    g = torch.Generator().manual_seed(9)
    inp = torch.randn((16, 16, 16), generator=g).cuda()
    tgt = (0.3 * inp + 0.1 * torch.roll(inp, 1, 0)).contiguous()
    losses = []
    # the weight gradients are summed with atomics, so the trajectory differs
    # slightly from run to run: 60 steps, and the best of the last five
    for _ in range(60):
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        r, A = net.forward(inp, keep=True)
        net.backward(A, tgt, loss)
        net.adam_step(lr=3e-3)
        losses.append(loss.item())
    assert min(losses[-5:]) < 0.5 * losses[0], losses
