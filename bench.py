"""Benchmark: Richardson-Lucy (Clarity_MaximumLikelihoodDeconvolve) on a
256x256x64 fp32 volume with a same-size PSF (work box 512x512x128), 200
iterations per step -- the RL leg of the 256x256x64 plain-methods workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is whole-job throughput in image
voxel-iterations per second (G) with inputs resident in HBM, timed with CUDA
events on the launching stream, max over ranks; `e2e` is the same metric
through the public C API with host buffers (pinned), copies included.
Multi-GPU runs are independent replicas (one volume per GPU, no collective
on the data path); `value` sums the ranks' work over the slowest rank's time.

`--impl reference` times the reference's own CPU implementation (the
unmodified reference sources built into oracle/_ref with the project's
FFTW-API shim) on a bounded sample of the same workload, on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RL Gvoxel-iter/s @256²×64 fp32"
UNIT = "Gvoxel-iter/s"
IMAGE_ZYX = (64, 256, 256)
ITERS = 200
WORKLOAD = "Richardson-Lucy (MaximumLikelihoodDeconvolve) 256x256x64 fp32, same-size PSF " \
           "(0.9 G(2,5) + 0.1 G(6,12)), 200 iterations per step"


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for ln in f:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# --------------------------------------------------------------- CPU legs
def cpu_reference_rl(img, psf, iters):
    """Reference CPU code (oracle/_ref) or, where it was not built, the
    oracle restatement; returns (seconds, kind, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    if O.ReferenceCPU.available("ref"):
        ref = O.ReferenceCPU("ref")
        ref.set_threads(cores)
        t0 = time.perf_counter()
        ref.rl(img, psf, iters)
        return time.perf_counter() - t0, "reference", cores
    orc = O.Oracle()
    orc.set_threads(cores)
    t0 = time.perf_counter()
    orc.rl(img, psf, iters)
    return time.perf_counter() - t0, "port", cores


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    from clarity_b200 import synthetic as syn
    img, psf, _ = syn.cfg1(seed=1)
    # a bounded sample of the 200-iteration workload: four iterations per
    # step, so the per-call set-up (padding, the OTF's FFT, the energy sum)
    # is spread over several iterations as in the 200-iteration solve
    iters_per_step = 4
    for _ in range(args.warmup):
        cpu_reference_rl(img, psf, iters_per_step)
    times = []
    kind = cores = None
    for _ in range(args.steps):
        t, kind, cores = cpu_reference_rl(img, psf, iters_per_step)
        times.append(t)
    ms = 1e3 * sum(times) / len(times)
    vox = int(np.prod(IMAGE_ZYX))
    value = vox * iters_per_step / (ms / 1e3) / 1e9
    sample = f"RL on the 256x256x64 workload, {iters_per_step} iterations per step (work box " \
             f"512x512x128), all {cores} host threads"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD.replace("200 iterations", f"{iters_per_step} iterations"),
                       "image_xyz": [256, 256, 64], "psf_xyz": [256, 256, 64],
                       "iterations_per_step": iters_per_step, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU arm
def family_bytes(work, img_vox, ker_vox, iters):
    """Algorithmic HBM bytes of one RL solve, per kernel family.
    C = complex half spectrum 8*nz*ny*(nx/2+1); R = real work box 4*N; the
    image and kernel are read unpadded (Ri, Rk).  Schedule per solve: OTF
    (xy forward + z forward), one xy forward of the image, then per iteration
    z (h*cur), xy inverse+forward (ratio), z (h*r) and the product step, which
    also transforms u' for the next iteration except on the last one."""
    nz, ny, nx = work
    N = nx * ny * nz
    C = 8 * nz * ny * (nx // 2 + 1)
    R = 4 * N
    Ri, Rk = 4 * img_vox, 4 * ker_vox
    cur0 = Ri                       # first iteration reads the image
    prod_merged = [(C + (cur0 if k == 0 else R) + R + C) for k in range(iters - 1)]
    last = C + (cur0 if iters == 1 else R) + R
    return {
        "xy_forward": (Rk + C) + (Ri + C),
        "z": 2 * C + 2 * iters * 3 * C,
        "xy_inv_fwd": iters * (2 * C + Ri),
        "xy_product": sum(prod_merged),
        "xy_inverse": last,
        "per_iteration": 2 * R + Ri + 10 * C,
        "per_iteration_survey": 4 * R + 10 * C,
    }


# DRAM bytes (read + write) per launch of each steady-iteration kernel family,
# measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the
# steady launches of this workload's iteration 2 (z: the mean of its two
# launches, P2 and P4).
NCU_TRAFFIC = {"xy_product": 152.1e6 + 215.7e6, "xy_inv_fwd": 84.5e6 + 20.9e6,
               "z": (270.7e6 + 46.0e6 + 203.5e6 + 82.6e6) / 2}


def max_over_ranks(value, dist, device):
    """The slowest rank's figure (replicas: every rank solves its own volume;
    the job is done when the last one is).  `dist` None: one rank."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_to_target(api, torch, img_d, psf_d, stream, plain_iters=200, max_accel=60):
    """The second metric: device time until I-div(g, h*u) is within 1% of
    plain RL's value after `plain_iters` iterations, for plain RL and for the
    chosen form (the faster of Biggs-Andrews accelerated RL and, where its
    trained weights are present, the learned start), on the same GPU and
    inputs.
    The I-divergence of every plain iterate comes from the trace the ratio
    pass accumulates; the chosen form's iteration count is the smallest whose
    result meets the target (its own traced final I-divergence)."""
    out = torch.empty_like(img_d)
    tr = torch.zeros(plain_iters + 1, dtype=torch.float64, device="cuda")
    api.ml_ex_device(img_d, psf_d, out, plain_iters, idiv=tr, stream=stream)
    torch.cuda.synchronize()
    t = tr.cpu().numpy()
    target = 1.01 * float(t[plain_iters])
    k_plain = int(np.argmax(t <= target))
    k_acc, finals = None, {}
    for k in range(2, max_accel + 1):
        ta = torch.zeros(k + 1, dtype=torch.float64, device="cuda")
        api.ml_accel_device(img_d, psf_d, out, k, idiv=ta, stream=stream)
        torch.cuda.synchronize()
        finals[k] = float(ta[k].item())
        if finals[k] <= target:
            k_acc = k
            break

    def ev_ms(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    res = {"target": "I-divergence within 1% of plain RL after 200 iterations",
           "idiv_plain_200": float(t[plain_iters]), "idiv_target": target,
           "plain": {"iterations": k_plain,
                     "ms": ev_ms(lambda: api.ml_device(img_d, psf_d, out, k_plain, stream))},
           "chosen": {"form": "accelerated RL (Biggs-Andrews vector extrapolation)",
                      "iterations": k_acc}}
    if k_acc:
        res["chosen"]["ms"] = ev_ms(lambda: api.ml_accel_device(img_d, psf_d, out, k_acc,
                                                                stream=stream))
        res["chosen"]["idiv"] = finals[k_acc]
        res["speedup"] = res["plain"]["ms"] / res["chosen"]["ms"]
    # learned start (when trained weights are present): RL to the iterate the
    # network was trained on, the network's prediction, RL resumed from it
    # (plain or accelerated) until the target is met
    from clarity_b200 import learned
    if os.path.exists(learned.WEIGHTS):
        net = learned.load_net()
        for tag, accel in (("learned_start", False), ("learned_start_accel", True)):
            k_ls, ls_final = None, None
            # zero resumed iterations is the prediction itself (the plain form
            # traces it; the accelerated form starts at one iteration)
            for k in range(1 if accel else 0, max_accel + 1):
                tl = torch.zeros(k + 1, dtype=torch.float64, device="cuda")
                learned.learned_solve(net, img_d, psf_d, out, k, idiv=tl, stream=stream,
                                      accel=accel)
                torch.cuda.synchronize()
                if float(tl[k].item()) <= target:
                    k_ls, ls_final = k, float(tl[k].item())
                    break
            ls = {"form": f"learned start (3-D U-Net on RL iterate {net.pre}, BF16 tensor-core "
                          "kernels) " + ("+ accelerated RL" if accel else "+ resumed RL"),
                  "pre_iterations": net.pre, "resumed_iterations": k_ls}
            if k_ls is not None:
                ls["ms"] = ev_ms(lambda: learned.learned_solve(net, img_d, psf_d, out, k_ls,
                                                               stream=stream, accel=accel))
                ls["idiv"] = ls_final
                ls["speedup"] = res["plain"]["ms"] / ls["ms"]
            res[tag] = ls
        res["network"] = network_layers(torch, net)
    # the chosen form is the fastest one that meets the target: accelerated
    # RL needs no trained weights; the learned start (whose result the tests
    # hold to 1e-3 of the FP64 oracle) is faster where its weights are present
    res["accelerated"] = dict(res["chosen"])
    best = min((f for f in ("learned_start", "learned_start_accel") if "ms" in res.get(f, {})),
               key=lambda f: res[f]["ms"], default=None)
    if best and res[best]["ms"] < res["chosen"].get("ms", float("inf")):
        res["chosen"] = dict(res[best], iterations=res[best]["pre_iterations"] +
                             res[best]["resumed_iterations"])
        res["speedup"] = res[best]["speedup"]
    return res


def headline_parity(api, torch, img_d, psf_d, img, psf, stream, iters=10):
    """Error of the headline path's output after `iters` iterations (a
    bounded sample: the CPU references take about a second per iteration)
    against the reference's CPU build with a double flux sum (the parity
    target) and the FP64 oracle.  The full 200-iteration output is checked
    the same way by the GPU parity tests."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cores = os.cpu_count() or 1
    out = torch.empty_like(img_d)
    api.ml_device(img_d, psf_d, out, iters, stream)
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.float64)
    res = {"iterations": iters}
    if O.ReferenceCPU.available("ref_fp64sum"):
        ref = O.ReferenceCPU("ref_fp64sum")
        ref.set_threads(cores)
        r32 = ref.rl(img, psf, iters)
        res["rel_l2_vs_reference"] = O.rel_l2(got, r32)
        res["max_abs_vs_reference"] = float(np.abs(got - r32).max())
    orc = O.Oracle()
    orc.set_threads(cores)
    r64 = orc.rl(img, psf, iters, precision="f64")
    res["rel_l2_vs_fp64"] = O.rel_l2(got, r64)
    res["max_abs_vs_fp64"] = float(np.abs(got - r64).max())
    res["tolerance"] = "rel-L2 <= 1e-4 after several iterations (1e-5 after one)"
    return res


def network_layers(torch, net, shape_zyx=(64, 256, 256), reps=5):
    """Per-layer device time and TFLOP/s of the learned-start network's
    forward pass at the 256x256x64 volume (CUDA events around each layer's
    launch; 2 x voxels x cout x 27 x cin FLOPs per 3x3x3 convolution)."""
    from clarity_b200 import unet
    D, H, W = shape_zyx
    x = torch.rand((D, H, W), device="cuda") * 100 + 1
    inp, _ = unet.to_input(x)
    _, A = net.forward(inp.contiguous(), keep=True)  # the layers' inputs
    torch.cuda.synchronize()
    plan = [("l0b", A["a0"], None, 1), ("l1a", A["p0"], None, 2), ("l1b", A["a1"], None, 2),
            ("l2a", A["p1"], None, 4), ("l2b", A["a2"], None, 4), ("l3a", A["p2"], None, 8),
            ("l3b", A["a3"], None, 8), ("l2c", A["s2"], A["b3"], 4), ("l2d", A["c2"], None, 4),
            ("l1c", A["s1"], A["d2"], 2), ("l1d", A["c1"], None, 2), ("l0c", A["s0"], A["d1"], 1),
            ("l0d", A["c0"], None, 1)]
    rows, tot_ms, tot_fl = {}, 0.0, 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, x1, x2, f in plan:
        co = net.layout[name][3]
        cin = net.layout[name][4] + net.layout[name][5]
        vox = (D // f) * (H // f) * (W // f)
        fl = 2.0 * vox * co * 27 * cin
        call = lambda: unet.conv3(x1, net.wf[name], co, bias=net.b(name), relu=True, x2=x2)
        call()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            call()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        rows[name] = {"ms": ms, "tflops": fl / (ms / 1e3) / 1e12, "cin": cin, "cout": co,
                      "voxels": vox}
        tot_ms += ms
        tot_fl += fl
    e0.record()
    for _ in range(reps):
        out = torch.empty_like(x)
        from clarity_b200 import api
        api.nn_predict(net.p, x, out)
    e1.record()
    torch.cuda.synchronize()
    return {"layers": rows, "conv_ms": tot_ms, "conv_tflops": tot_fl / (tot_ms / 1e3) / 1e12,
            "predict_ms": e0.elapsed_time(e1) / reps,
            "note": "BF16 implicit-GEMM convolutions on tcgen05 (TMEM accumulators, TMA "
                    "operand loads), FP32 accumulation"}


def _cfg2_case(i):
    from clarity_b200 import synthetic as syn
    img, psf, _ = syn.cfg2_volume(i)
    return img, psf


def cached_reference(name, inputs):
    """A full-size CPU reference the GPU parity tests keep under
    tests/golden/_large (same key: the name and a digest of the inputs), or
    None when it has not been computed."""
    import hashlib
    h = hashlib.sha1()
    for a in inputs:
        h.update(np.ascontiguousarray(a).tobytes())
    path = os.path.join(ROOT, "tests", "golden", "_large", f"{name}-{h.hexdigest()[:16]}.npy")
    return np.load(path) if os.path.exists(path) else None


SUB = 16  # sample stride of the kept precision-form references


def precision_forms(api, torch, stream, iters=100):
    """The precision workload: RL for `iters` iterations on the 512x512x128
    volume (work box 1024x1024x256) with the FP32 register FFT and with the
    first radix-16 z stage as split hi+lo FP16 / BF16 tensor-core GEMMs; time
    (CUDA events) and the error against the FP64 oracle where its output has
    been computed (tests/golden/_large).  The full outputs (134 MB each) may
    be kept as every SUB-th voxel (name suffix "-sub"): the errors are then
    taken over that sample."""
    from clarity_b200 import synthetic as syn
    img, psf, _ = syn.cfg3()
    r64 = cached_reference(f"rl{iters}-f64", [img, psf])
    r32 = cached_reference(f"rl{iters}-ref32", [img, psf])
    pick = lambda a: a  # noqa: E731 (the whole volume)
    if r64 is None or r32 is None:
        r64 = cached_reference(f"rl{iters}-f64-sub", [img, psf])
        r32 = cached_reference(f"rl{iters}-ref32-sub", [img, psf])
        pick = lambda a: np.ascontiguousarray(a).ravel()[::SUB]  # noqa: E731
    if r64 is not None:
        r64 = r64.astype(np.float64)
    di, dk = torch.from_numpy(img).cuda(), torch.from_numpy(psf).cuda()
    out = torch.empty_like(di)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {"workload": f"RL 512x512x128 fp32 (work box 1024x1024x256), {iters} iterations",
           "fp64_reference": r64 is not None,
           "error_sample": None if r64 is None else (
               "every voxel" if r64.size == img.size else f"every {SUB}th voxel")}
    if r64 is not None and r32 is not None:
        res["reference_build_rel_l2_vs_fp64"] = float(np.linalg.norm(
            (r32.astype(np.float64) - r64).ravel()) / np.linalg.norm(r64.ravel()))
    for mode, name in ((0, "f32_simt"), (1, "f16_split_tc"), (2, "bf16_split_tc")):
        api.set_dft_precision(mode)
        try:
            api.ml_device(di, dk, out, 1, stream)  # warm-up
            torch.cuda.synchronize()
            e0.record(stream)
            api.ml_device(di, dk, out, iters, stream)
            e1.record(stream)
            torch.cuda.synchronize()
        finally:
            api.set_dft_precision(0)
        ms = e0.elapsed_time(e1)
        row = {"ms": ms, "value": img.size * iters / (ms / 1e3) / 1e9, "unit": "Gvoxel-iter/s"}
        if r64 is not None:
            got = pick(out.cpu().numpy()).astype(np.float64)
            row["rel_l2_vs_fp64"] = float(np.linalg.norm((got - r64).ravel()) /
                                          np.linalg.norm(r64.ravel()))
            row["max_abs_vs_fp64"] = float(np.abs(got - r64).max())
        res[name] = row
    return res


def other_configs(api, torch, stream, n_batch=64, batch_iters=30, cfg3_iters=10):
    """The batched and the large-volume workloads, measured beside the headline
    (G image-voxel-iterations/s; CUDA events on the launching stream)."""
    import multiprocessing as mp
    from clarity_b200 import synthetic as syn
    res = {}
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 4)) as pool:
        cases = pool.map(_cfg2_case, range(n_batch))
    imgs = [torch.from_numpy(a).cuda() for a, _ in cases]
    psfs = [torch.from_numpy(b).cuda() for _, b in cases]
    outs = [torch.empty_like(a) for a in imgs]
    vox = sum(a.numel() for a in imgs)
    # the schedule's bytes per RL iteration over the batch (2R + Ri + 10C per
    # volume, as the headline's schedule_bytes), for a bandwidth figure
    sched = 0
    for a in imgs:
        z, y, x = (2 * d for d in a.shape)
        sched += 2 * 4 * x * y * z + 4 * a.numel() + 10 * 8 * z * y * (x // 2 + 1)
    peak = peaks()[0]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    desc = (f"{n_batch} volumes of uneven sizes (x, y in 16*{{6..20}}, z in 8*{{2..12}}), "
            f"{batch_iters} RL iterations")

    def timed(persistent, tuned):
        if tuned:
            api.trim()
            api.autotune(True)
        try:
            # set-up (and tuning) and capture, outside the timed region
            api.ml_batch_device(imgs, psfs, outs, batch_iters, graph=True, stream=stream,
                                persistent=persistent)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(3):
                api.ml_batch_device(imgs, psfs, outs, batch_iters, graph=True, stream=stream,
                                    persistent=persistent)
            e1.record(stream)
            torch.cuda.synchronize()
        finally:
            if tuned:
                api.autotune(False)
        ms = e0.elapsed_time(e1) / 3
        gbps = sched * batch_iters / (ms / 1e3) / 1e9
        return {"workload": desc + (", iterations of all volumes in one persistent launch "
                                    "(work queue), in one captured CUDA graph" if persistent
                                    else ", per-volume launches on 8 streams, one captured "
                                         "CUDA graph"),
                "image_voxels": int(vox), "ms": ms,
                "value": vox * batch_iters / (ms / 1e3) / 1e9, "unit": "Gvoxel-iter/s",
                "schedule_GBps": gbps, "schedule_frac": gbps / peak,
                "plans": ("autotuned (fastest of the planner's best four tilings per work box)"
                          if tuned else "planner default")}

    res["batched_rl"] = timed(False, False)
    res["batched_rl_autotuned"] = timed(False, True)
    api.trim()
    res["batched_rl_persistent"] = timed(True, False)
    res["batched_rl_persistent_autotuned"] = timed(True, True)
    del imgs, psfs, outs
    img, psf, _ = syn.cfg3()
    di, dk = torch.from_numpy(img).cuda(), torch.from_numpy(psf).cuda()
    out = torch.empty_like(di)
    api.ml_device(di, dk, out, 1, stream)
    torch.cuda.synchronize()
    e0.record(stream)
    api.ml_device(di, dk, out, cfg3_iters, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    # the survey's per-iteration bytes (4R + 10C) of the work box, as the
    # headline's survey_frac
    fb = family_bytes(tuple(2 * d for d in img.shape), img.size, psf.size, cfg3_iters)
    large_gbps = fb["per_iteration_survey"] * cfg3_iters / (ms / 1e3) / 1e9
    res["large_rl"] = {"workload": f"RL 512x512x128 fp32 (work box 1024x1024x256), {cfg3_iters} "
                                   "iterations, FP32 SIMT FFT", "ms": ms,
                       "value": img.size * cfg3_iters / (ms / 1e3) / 1e9,
                       "unit": "Gvoxel-iter/s",
                       "survey_bytes_per_iteration": fb["per_iteration_survey"],
                       "survey_GBps": large_gbps, "survey_frac": large_gbps / peak}
    del di, dk, out
    res["precision_forms"] = precision_forms(api, torch, stream)
    return res


def run_gpu_arm(args, rank, world):
    import torch
    from clarity_b200 import api, synthetic as syn

    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    api.set_device(local)
    api.register()
    img, psf, _ = syn.cfg1(seed=1 + rank)
    img_d = torch.from_numpy(img).cuda()
    psf_d = torch.from_numpy(psf).cuda()
    out_d = torch.empty_like(img_d)
    stream = torch.cuda.current_stream()

    def step():
        api.ml_device(img_d, psf_d, out_d, ITERS, stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    if not args.quick:
        clocks.start()
    l0 = api.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = api.launch_count() - l0
    ms_total = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    # per-kernel-family durations: one more step, outside the timed region,
    # with CUDA events recorded around every fused-pass launch on its stream
    api.timing_enable(True)
    step()
    torch.cuda.synchronize()
    fam = api.timing_collect()
    api.timing_enable(False)
    if dist:
        dist.barrier()
    ms_step = ms_total / args.steps
    vox = int(np.prod(IMAGE_ZYX))
    value = world * vox * ITERS / (ms_step / 1e3) / 1e9

    if args.quick:
        api.unregister()
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"quick": True, "ms_per_step": ms_step, "value": value,
                              "families": {k: v for k, v in fam.items()}}), flush=True)
        return

    # end to end through the public C API with pinned host buffers
    img_h = torch.empty(IMAGE_ZYX, dtype=torch.float32, pin_memory=True).numpy()
    psf_h = torch.empty(IMAGE_ZYX, dtype=torch.float32, pin_memory=True).numpy()
    img_h[...] = img
    psf_h[...] = psf
    out_h = torch.empty(IMAGE_ZYX, dtype=torch.float32, pin_memory=True).numpy()
    lib = api.load()

    def e2e_step():
        rc = lib.Clarity_MaximumLikelihoodDeconvolve(img_h, api.dim3(img_h), psf_h,
                                                     api.dim3(psf_h), out_h, ITERS)
        api._check(rc)

    e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_ms = max_over_ranks(1e3 * (time.perf_counter() - t0) / args.steps, dist, "cuda")
    # the same call from pageable (malloc'ed) buffers, as every reference
    # caller passes them: the library's pinned bounce buffers stage the copies
    img_p, psf_p, out_p = img.copy(), psf.copy(), np.empty_like(img)

    def e2e_pageable_step():
        api._check(lib.Clarity_MaximumLikelihoodDeconvolve(img_p, api.dim3(img_p), psf_p,
                                                           api.dim3(psf_p), out_p, ITERS))

    e2e_pageable_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_pageable_step()
    e2e_pg_ms = max_over_ranks(1e3 * (time.perf_counter() - t0) / args.steps, dist, "cuda")
    clk = clocks.stop()
    e2e_value = world * vox * ITERS / (e2e_ms / 1e3) / 1e9

    # roofline of the dominant kernel family
    work = tuple(2 * s for s in IMAGE_ZYX)
    fb = family_bytes(work, vox, vox, ITERS)
    peak, peak_kind = peaks()
    fam_ms = {k: v for k, v in fam.items() if k != "other" and v[1] > 0}
    dom = max(fam_ms, key=lambda k: fam_ms[k][0]) if fam_ms else None
    roof = None
    if dom:
        tot_ms, cnt = fam_ms[dom]  # one step
        per_launch_ms = tot_ms / cnt
        bytes_per_launch = fb[dom] / cnt
        achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": NCU_TRAFFIC.get(dom), "traffic_unit": "bytes per launch",
                "bytes_per_launch": bytes_per_launch,
                "ms_per_launch": per_launch_ms,
                "share_of_step": tot_ms / sum(v[0] for v in fam_ms.values())}
    iter_bytes = fb["per_iteration_survey"]
    iter_ms = ms_step / ITERS
    own_bytes = fb["per_iteration"]
    families = {k: {"ms_per_launch": v[0] / v[1], "launches_per_step": v[1],
                    "GBps": (fb[k] / v[1]) / (v[0] / v[1] / 1e3) / 1e9}
                for k, v in fam_ms.items()}

    ttt = time_to_target(api, torch, img_d, psf_d, stream) if rank == 0 else None
    parity = headline_parity(api, torch, img_d, psf_d, img, psf, stream) if rank == 0 else None
    others = other_configs(api, torch, stream) if rank == 0 and world == 1 else None

    if rank == 0:
        sample_iters = max(1, args.cpu_iters)
        t_cpu, kind, cores = cpu_reference_rl(img, psf, sample_iters)
        cpu_value = vox * sample_iters / t_cpu / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded phantom, Poisson noise)",
            "config": {"workload": WORKLOAD, "image_xyz": [256, 256, 64],
                       "psf_xyz": [256, 256, 64], "work_box_xyz": [512, 512, 128],
                       "iterations_per_step": ITERS, "parallelism": f"replicas x{world}",
                       "l2": "inputs and working set (~0.7 GB) larger than L2"},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(img_h.nbytes + psf_h.nbytes),
                    "d2h_bytes_per_step": int(out_h.nbytes), "ms_per_step": e2e_ms},
            "e2e_pageable": {"value": world * vox * ITERS / (e2e_pg_ms / 1e3) / 1e9, "unit": UNIT,
                             "ms_per_step": e2e_pg_ms,
                             "note": "the public call from pageable host buffers (staged "
                                     "through the library's pinned bounce buffers)"},
            "gpu_launches": int(launches),
            "roofline": roof,
            "iteration": {"ms": iter_ms,
                          "survey_bytes": iter_bytes,
                          "survey_frac": iter_bytes / (iter_ms / 1e3) / 1e9 / peak,
                          "schedule_bytes": own_bytes,
                          "schedule_GBps": own_bytes / (iter_ms / 1e3) / 1e9,
                          "schedule_frac": own_bytes / (iter_ms / 1e3) / 1e9 / peak},
            "families": families,
            "cpu_baseline": {"value": cpu_value, "unit": UNIT, "cores": cores,
                             "kind": kind,
                             "sample": f"RL on the same 256x256x64 workload, {sample_iters} "
                                       f"iteration(s), {cores} host threads"},
            "clocks": clk,
            "time_to_target": ttt,
            "parity": parity,
            "other_configs": others,
        }
        print(json.dumps(line), flush=True)
    api.unregister()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def profile_case(which):
    """A small case of one kernel family for ncu captures (see --profile-case)."""
    import torch
    from clarity_b200 import api, unet, synthetic as syn
    api.load()
    api.register()
    if which == "conv":
        g = torch.Generator(device="cuda").manual_seed(0)
        for (D, H, W, c1, c2, co) in [(64, 256, 256, 16, 0, 16), (32, 128, 128, 32, 64, 32)]:
            def rnd(*shape, s=1.0):
                return ((torch.rand(shape, device="cuda", generator=g) - 0.5) * s).to(torch.bfloat16)
            x1 = rnd(D, H, W, c1)
            x2 = rnd(D // 2, H // 2, W // 2, c2) if c2 else None
            w = rnd(co, 27, c1 + c2, s=0.1)
            b = torch.zeros(co, device="cuda")
            for _ in range(2):
                unet.conv3(x1, w, co, bias=b, relu=True, x2=x2)
    else:
        cases = [syn.cfg2_volume(i)[:2] for i in (3, 5, 9, 12)]
        di = [torch.from_numpy(a).cuda() for a, _ in cases]
        dk = [torch.from_numpy(b).cuda() for _, b in cases]
        outs = [torch.empty_like(a) for a in di]
        api.ml_batch_device(di, dk, outs, 2, graph=False, persistent=True)
    torch.cuda.synchronize()
    api.synchronize()
    api.unregister()
    print(json.dumps({"profile_case": which, "ok": True}), flush=True)


def main():
    global ITERS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-iters", type=int, default=4)
    ap.add_argument("--iters", type=int, default=ITERS,
                    help="RL iterations per step (200 is the workload; fewer only "
                         "for profiling captures)")
    ap.add_argument("--quick", action="store_true",
                    help="device leg only (no e2e, no CPU baseline): for ncu captures")
    ap.add_argument("--profile-case", choices=["conv", "batch"], default=None,
                    help="run one small case for an ncu capture and exit: 'conv' two "
                         "launches each of the learned-start network's 16->16 layer at "
                         "64x256x256 and its 96->32 decoder layer at 32x128x128; 'batch' the "
                         "persistent batched RL launch over four batched-workload volumes, "
                         "two iterations")
    args = ap.parse_args()
    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    ITERS = args.iters
    if args.profile_case:
        profile_case(args.profile_case)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
    else:
        run_gpu_arm(args, rank, world)


if __name__ == "__main__":
    main()
