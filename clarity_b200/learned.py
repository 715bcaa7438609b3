"""Learned start: training data, training loop and the learned-start solve.

Training pairs are produced by the RL solver itself: synthetic patches
(spheres as the 256x256x64 workload at the same density, the halo PSF with
its sigmas scaled by U(0.7, 1.3), circular blur, Poisson noise) deconvolved to
iterate 5 (the network's input) and iterate 200 (its target) with batched RL
on the GPU.  The network (unet.UNet3D) learns the per-voxel log-ratio between
the two.  At solve time RL runs `pre` iterations, the network predicts an
advanced estimate, and RL resumes from it (clarityx_ml_ex_device with a start
estimate); plain RL remains the fallback, and the I-divergence traces of
both tell which is ahead.

    python -m clarity_b200.learned --patches 2000 --epochs 14 --early 5 --out weights.npy
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import time

import numpy as np

from . import api, synthetic as syn, unet

WEIGHTS = os.environ.get("CLARITY_LEARNED_WEIGHTS") or os.path.join(
    os.path.dirname(os.path.abspath(__file__)), "learned_start_weights.npy")
PATCH_ZYX = (48, 128, 128)
PRE = 5  # RL iterations before the network, unless the weights' metadata says otherwise


def meta_path(weights: str) -> str:
    """The JSON file beside a weights file: {"pre": ..., "epochs": ..., "patches": ...}."""
    return os.path.splitext(weights)[0] + ".json"


def make_patch(seed: int, shape_zyx=PATCH_ZYX):
    """(observed image, PSF) of one training patch (float32, z-y-x)."""
    r = syn.rng(seed)
    n = int(round(600 * np.prod(shape_zyx) / (64 * 256 * 256)))
    truth = syn.phantom(shape_zyx, n, r)
    psf = syn.halo_psf(shape_zyx, scale=float(r.uniform(0.7, 1.3)))
    return syn.observe(truth, psf, r), psf


def _make_patch_star(args):
    return make_patch(*args)


def generate_pairs(n: int, seed0: int = 10_000, early: int = 5, late: int = 200,
                   batch: int = 16, workers: int | None = None, log=print):
    """Device tensors (x_early, x_late), each [n, D, H, W] float32."""
    import torch
    workers = workers or min(16, os.cpu_count() or 4)
    ctx = mp.get_context("spawn")
    D, H, W = PATCH_ZYX
    xe = torch.empty((n, D, H, W), dtype=torch.float32, device="cuda")
    xl = torch.empty_like(xe)
    t0 = time.time()
    with ctx.Pool(workers) as pool:
        it = pool.imap(_make_patch_star, [(seed0 + i,) for i in range(n)], chunksize=4)
        for b0 in range(0, n, batch):
            imgs, psfs = [], []
            for _ in range(min(batch, n - b0)):
                img, psf = next(it)
                imgs.append(torch.from_numpy(img).cuda())
                psfs.append(torch.from_numpy(psf).cuda())
            k = len(imgs)
            api.ml_batch_device(imgs, psfs, [xe[b0 + i] for i in range(k)], early, graph=False)
            api.ml_batch_device(imgs, psfs, [xl[b0 + i] for i in range(k)], late, graph=False)
            if (b0 // batch) % 25 == 0:
                torch.cuda.synchronize()
                log(f"pairs {b0 + k}/{n}  {time.time() - t0:.1f}s")
    torch.cuda.synchronize()
    return xe, xl


def train(net: unet.UNet3D, xe, xl, epochs: int = 6, lr: float = 1e-3, batch: int = 4,
          seed: int = 0, log=print):
    """Adam on the log-ratio regression; returns the per-epoch mean losses."""
    import torch
    n = xe.shape[0]
    g = np.random.default_rng(seed)
    hist = []
    steps_total = epochs * ((n + batch - 1) // batch)
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        order = g.permutation(n)
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        for b0 in range(0, n, batch):
            idx = order[b0:b0 + batch]
            for i in idx:
                x, t = xe[int(i)], xl[int(i)]
                # random flips along x and y (the PSF is symmetric)
                flip = [d for d, f in ((1, g.random() < 0.5), (2, g.random() < 0.5)) if f]
                if flip:
                    x, t = x.flip(flip), t.flip(flip)
                inp, _ = unet.to_input(x.contiguous())
                tgt = unet.to_target(x, t).contiguous()
                _, A = net.forward(inp.contiguous(), keep=True)
                net.backward(A, tgt, loss)
            # cosine learning-rate decay
            lr_now = 0.5 * lr * (1 + np.cos(np.pi * step / max(steps_total, 1)))
            net.adam_step(lr=float(lr_now), scale=1.0 / len(idx))
            step += 1
        torch.cuda.synchronize()
        hist.append(loss.item() / n)
        log(f"epoch {ep + 1}/{epochs}: loss {hist[-1]:.5f}  {time.time() - t0:.1f}s")
    return hist


def learned_solve(net: unet.UNet3D, img_d, psf_d, out, post: int, pre: int | None = None,
                  idiv=None, stream=None, accel=False):
    """RL `pre` iterations (default: the iterate the network was trained on),
    the network's prediction, RL resumed for `post` iterations from it --
    plain, or accelerated (Biggs-Andrews) with accel (idiv: trace of the
    resumed part, post + 1 entries).  The plain form is one library call
    (clarityx_ml_learned_device)."""
    import torch
    if pre is None:
        pre = getattr(net, "pre", PRE)
    if not accel:
        return api.ml_learned_device(img_d, psf_d, net.p, out, pre, post, idiv=idiv,
                                     stream=stream)
    early = torch.empty_like(img_d)
    api.ml_device(img_d, psf_d, early, pre, stream)
    start = unet.predict(net, early, stream=stream).contiguous()
    if post <= 0:
        out.copy_(start)
        return out
    if accel:
        api.ml_accel_device(img_d, psf_d, out, post, idiv=idiv, stream=stream, start=start)
    else:
        api.ml_ex_device(img_d, psf_d, out, post, start=start, idiv=idiv, stream=stream)
    return out


def load_net(path: str = WEIGHTS) -> unet.UNet3D:
    net = unet.UNet3D()
    net.load_state(np.load(path))
    net.pre = PRE
    if os.path.exists(meta_path(path)):
        with open(meta_path(path)) as f:
            net.pre = int(json.load(f).get("pre", PRE))
    return net


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--patches", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--early", type=int, default=PRE,
                    help="the RL iterate the network starts from")
    ap.add_argument("--log", default=None)
    a = ap.parse_args()
    logf = open(a.log, "w") if a.log else None

    def log(msg):
        print(msg, flush=True)
        if logf:
            logf.write(msg + "\n")
            logf.flush()

    api.register()
    xe, xl = generate_pairs(a.patches, early=a.early, log=log)
    net = unet.UNet3D(seed=1)
    hist = train(net, xe, xl, epochs=a.epochs, lr=a.lr, batch=a.batch, log=log)
    np.save(a.out, net.state())
    with open(meta_path(a.out), "w") as f:
        json.dump({"pre": a.early, "epochs": a.epochs, "patches": a.patches}, f)
    log(json.dumps({"losses": hist, "out": a.out}))


if __name__ == "__main__":
    main()
