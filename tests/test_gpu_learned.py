"""The learned start as a method, on a held-out 256x256x64 volume.

The committed weights (clarity_b200/learned_start_weights.npy) were trained on
patches with seeds 10000..11999 (learned.generate_pairs); the volume here is
the 256x256x64 workload's recipe with seed 77, which no training patch used.

* The library's fused prediction (clarityx_nn_predict: the log-domain
  transforms inside the network's first and last kernels) equals the training
  path's separate transforms.
* Gain over the method without it: RL `pre` -> network -> RL resumed
  (clarityx_ml_learned_device, one call) reaches plain RL's 200-iteration
  I-divergence x 1.01 in fewer RL iterations and less device time than plain
  RL needs for the same target.
* Its result is within 1e-3 relative L2 of the FP64 oracle of the same
  procedure: the FP64 oracle's RL from the network's prediction (the network
  itself has no FP64 counterpart; its input, the GPU's RL iterate, is checked
  against the FP64 oracle's at 1e-4).
"""
import numpy as np
import pytest

from clarity_b200 import learned, synthetic as syn, unet
from conftest import rel_l2, report_error

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net():
    return learned.load_net()


@pytest.fixture(scope="module")
def held_out():
    import torch
    img, psf, _ = syn.cfg1(seed=77)
    return img, psf, torch.from_numpy(img).cuda(), torch.from_numpy(psf).cuda()


def _device_ms(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def test_fused_prediction_matches_training_transforms(clarity_gpu, net, held_out):
    import torch
    _, _, di, dk = held_out
    early = torch.empty_like(di)
    clarity_gpu.ml_device(di, dk, early, net.pre)
    fused = unet.predict(net, early)
    unfused = unet.predict_unfused(net, early)
    torch.cuda.synchronize()
    assert bool((fused >= 0).all())
    e = rel_l2(fused.cpu().numpy(), unfused.cpu().numpy())
    report_error("learned_prediction_fused_vs_unfused", rel_l2=e)
    # the activations are BF16: a last-bit difference in the log-domain input
    # (FP64 mean here, float mean there) moves some values across a BF16
    # rounding boundary (relative 2^-9), and that propagates through 15 layers
    assert e <= 2e-2


def test_learned_start_gains_over_plain_rl(clarity_gpu, oracle_lib, net, held_out):
    import torch
    img, psf, di, dk = held_out
    out = torch.empty_like(di)
    # plain RL: its 200-iteration I-divergence sets the target
    tr = torch.zeros(201, dtype=torch.float64, device="cuda")
    clarity_gpu.ml_ex_device(di, dk, out, 200, idiv=tr)
    torch.cuda.synchronize()
    t = tr.cpu().numpy()
    target = 1.01 * float(t[200])
    k_plain = int(np.argmax(t <= target))
    assert 0 < k_plain < 200
    # learned start: the fewest resumed iterations that meet the target
    pre, post = net.pre, None
    for k in range(0, 60):
        tl = torch.zeros(k + 1, dtype=torch.float64, device="cuda")
        learned.learned_solve(net, di, dk, out, k, idiv=tl)
        torch.cuda.synchronize()
        if float(tl[k].item()) <= target:
            post = k
            break
    assert post is not None, "the learned start never reached the target"
    ms_plain = _device_ms(lambda: clarity_gpu.ml_device(di, dk, out, k_plain))
    ms_learned = _device_ms(lambda: learned.learned_solve(net, di, dk, out, post))
    report_error("learned_start_time_to_target_256x256x64", plain_iterations=k_plain,
                 learned_pre=pre, learned_post=post, plain_ms=ms_plain, learned_ms=ms_learned,
                 speedup=ms_plain / ms_learned)
    assert pre + post < k_plain
    assert ms_learned < ms_plain
    # the procedure against its FP64 oracle (with at least three resumed
    # iterations, so the resumed RL is exercised even when the prediction
    # alone met the target)
    post_chk = max(post, 3)
    early = torch.empty_like(di)
    clarity_gpu.ml_device(di, dk, early, pre)
    pred = unet.predict(net, early)
    learned.learned_solve(net, di, dk, out, post_chk)
    torch.cuda.synchronize()
    e_pre = rel_l2(early.cpu().numpy(), oracle_lib.rl(img, psf, pre, precision="f64"))
    ref64, _ = oracle_lib.rl_ex(img, psf, post_chk, start=pred.cpu().numpy(), precision="f64")
    e_out = rel_l2(out.cpu().numpy(), ref64)
    report_error("learned_start_vs_fp64_256x256x64", pre_iterate_rel_l2=e_pre,
                 result_rel_l2=e_out, resumed_iterations=post_chk)
    assert e_pre <= 1e-4
    assert e_out <= 1e-3


def test_learned_solve_rejects_bad_arguments(clarity_gpu, net):
    import torch
    a = torch.ones((12, 16, 16), device="cuda")  # z = 12 is not a multiple of 8
    out = torch.empty_like(a)
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.ml_learned_device(a, a, net.p, out, 2, 2)
    assert e.value.code == clarity_gpu.CLARITY_INVALID_ARGUMENT
    b = torch.ones((16, 16, 16), device="cuda")
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.ml_learned_device(b, b, net.p[:-1].contiguous(), torch.empty_like(b), 2, 2)
    assert e.value.code == clarity_gpu.CLARITY_INVALID_ARGUMENT
