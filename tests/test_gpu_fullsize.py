"""GPU parity at the full workload sizes.

* 256x256x64 with the same-size halo PSF (0.9 G(2,5) + 0.1 G(6,12)): RL after
  1, 50 and 200 iterations, JVC after 50, Wiener at epsilon 1e-3
  (src/MaximumLikelihoodDeconvolve.cxx:255-332,
  src/JansenVanCittertDeconvolve.cxx:311-389, src/WienerDeconvolve.cxx:211-290);
* the 512x512x128 volume (work box 1024x1024x256, the largest specialised
  kernels) for two RL iterations;
* volumes of the batched workload whose work boxes need radices 7, 11, 13,
  17 and 19, in one batched call.

Every result is compared with the reference's own CPU build (oracle/_ref:
the unmodified sources with a double flux sum, the parity target) and with
the FP64 oracle.  Tolerances (relative L2 over the output image): 1e-5 after
one iteration or one pass, 1e-4 after several; against FP64 the result must
be within max(3 x the FP32 reference's own FP64 error, 1e-5).  The errors are
recorded (conftest.report_error) and written to $CLARITY_PARITY_REPORT.
The CPU references at these sizes take seconds to minutes; they are computed
once and kept in tests/golden/_large (conftest.cached).
"""
import numpy as np
import pytest

from clarity_b200 import synthetic as syn
from conftest import cached, rel_l2, report_error

pytestmark = pytest.mark.gpu

TOL_ONE = 1e-5
TOL_ITER = 1e-4


@pytest.fixture(scope="module")
def cfg1():
    img, psf, _ = syn.cfg1(seed=5)
    return img, psf


def _ref32(ref_cpu, oracle_lib, alg, img, psf, param):
    """The FP32 parity target: the reference build (or, where it was not
    built, the oracle's FP32 restatement, which is pinned bit-identical)."""
    def run():
        if ref_cpu is not None:
            return getattr(ref_cpu, alg)(img, psf, param)
        return getattr(oracle_lib, alg)(img, psf, param)
    return cached(f"{alg}{param}-ref32", [img, psf], run)


def _ref64(oracle_lib, alg, img, psf, param):
    return cached(f"{alg}{param}-f64", [img, psf],
                  lambda: getattr(oracle_lib, alg)(img, psf, param, precision="f64"))


def _check(name, out, r32, r64, tol):
    e32 = rel_l2(out, r32)
    e64 = rel_l2(out, r64)
    ref_e64 = rel_l2(r32, r64)
    report_error(name, rel_l2_vs_reference=e32, rel_l2_vs_fp64=e64,
                 reference_rel_l2_vs_fp64=ref_e64,
                 max_abs_vs_fp64=float(np.abs(out.astype(np.float64) - r64).max()),
                 max_abs_vs_reference=float(np.abs(out.astype(np.float64) - r32).max()))
    assert e32 <= tol, (name, e32)
    assert e64 <= max(3 * ref_e64, 1e-5), (name, e64, ref_e64)


@pytest.mark.parametrize("iters", [1, 50, 200])
def test_cfg1_rl(clarity_gpu, ref_cpu, oracle_lib, cfg1, iters):
    img, psf = cfg1
    out = clarity_gpu.maximum_likelihood_deconvolve(img, psf, iters)
    r32 = _ref32(ref_cpu, oracle_lib, "rl", img, psf, iters)
    r64 = _ref64(oracle_lib, "rl", img, psf, iters)
    _check(f"rl{iters}_256x256x64", out, r32, r64, TOL_ONE if iters == 1 else TOL_ITER)


def test_cfg1_jvc50(clarity_gpu, ref_cpu, oracle_lib, cfg1):
    # the JVC update fused into the TMA XY pass of the 512x512x128 work box
    img, psf = cfg1
    out = clarity_gpu.jansen_van_cittert_deconvolve(img, psf, 50)
    assert out.min() >= 0.0
    _check("jvc50_256x256x64", out, _ref32(ref_cpu, oracle_lib, "jvc", img, psf, 50),
           _ref64(oracle_lib, "jvc", img, psf, 50), TOL_ITER)


def test_cfg1_wiener(clarity_gpu, ref_cpu, oracle_lib, cfg1):
    # the Wiener filter fused into the specialised z pass of the same box
    img, psf = cfg1
    out = clarity_gpu.wiener_deconvolve(img, psf, 1e-3)
    _check("wiener_1e-3_256x256x64", out, _ref32(ref_cpu, oracle_lib, "wiener", img, psf, 1e-3),
           _ref64(oracle_lib, "wiener", img, psf, 1e-3), TOL_ONE)


def test_cfg1_device_entry_matches_host_entry(clarity_gpu, cfg1):
    # the benchmark's device call and the public host call agree bit for bit
    import torch
    img, psf = cfg1
    di, dk = torch.from_numpy(img).cuda(), torch.from_numpy(psf).cuda()
    out = torch.empty_like(di)
    clarity_gpu.ml_device(di, dk, out, 5)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(),
                          clarity_gpu.maximum_likelihood_deconvolve(img, psf, 5))


def test_cfg1_rl_correlate_opt_in(clarity_gpu, oracle_lib, cfg1):
    # the conjugate-for-correlation opt-in against the oracle's restatement of
    # it, and its distance from the reference form (reported)
    import torch
    img, psf = cfg1
    di, dk = torch.from_numpy(img).cuda(), torch.from_numpy(psf).cuda()
    out = torch.empty_like(di)
    clarity_gpu.ml_correlate_device(di, dk, out, 3)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    want = cached("rl_corr3-ref32", [img, psf], lambda: oracle_lib.rl_correlate(img, psf, 3))
    want64 = cached("rl_corr3-f64", [img, psf],
                    lambda: oracle_lib.rl_correlate(img, psf, 3, precision="f64"))
    plain = clarity_gpu.maximum_likelihood_deconvolve(img, psf, 3)
    report_error("rl_correlate3_256x256x64", rel_l2_vs_restatement=rel_l2(got, want),
                 rel_l2_vs_fp64=rel_l2(got, want64),
                 rel_l2_vs_reference_form=rel_l2(got, plain))
    assert rel_l2(got, want) <= TOL_ITER
    assert rel_l2(got, want64) <= max(3 * rel_l2(want, want64), 1e-5)


def test_large_box_rl(clarity_gpu, ref_cpu, oracle_lib):
    # the 512x512x128 volume: work box 1024x1024x256 (the ShapeW1024 kernels)
    img, psf, _ = syn.cfg3(seed=7)
    out = clarity_gpu.maximum_likelihood_deconvolve(img, psf, 2)
    _check("rl2_512x512x128", out, _ref32(ref_cpu, oracle_lib, "rl", img, psf, 2),
           _ref64(oracle_lib, "rl", img, psf, 2), TOL_ITER)


# batched-workload volumes whose work boxes need the odd radices:
# 7: (352, 544, 32) -> 11, 17; 23: (416, 224, 48) -> 7, 13;
# 33: (608, 224, 48) -> 7, 19; 49: (224, 352, 48) -> 7, 11; 14: (352, 608, 160) -> 11, 19
BATCH_IDS = [7, 23, 33, 49, 14]


def test_batched_workload_volumes(clarity_gpu, ref_cpu, oracle_lib):
    import torch
    iters = 5
    cases = [syn.cfg2_volume(i)[:2] for i in BATCH_IDS]
    di = [torch.from_numpy(a).cuda() for a, _ in cases]
    dk = [torch.from_numpy(b).cuda() for _, b in cases]
    outs = [torch.full_like(a, -1.0) for a in di]
    clarity_gpu.ml_batch_device(di, dk, outs, iters, graph=True)
    torch.cuda.synchronize()
    for i, (img, psf), o in zip(BATCH_IDS, cases, outs):
        got = o.cpu().numpy()
        _check(f"batched_vol{i}_rl{iters}_{img.shape[2]}x{img.shape[1]}x{img.shape[0]}", got,
               _ref32(ref_cpu, oracle_lib, "rl", img, psf, iters),
               _ref64(oracle_lib, "rl", img, psf, iters), TOL_ITER)
    # a batched volume equals its own single-volume solve, bit for bit
    one = torch.empty_like(di[0])
    clarity_gpu.ml_device(di[0], dk[0], one, iters)
    torch.cuda.synchronize()
    assert torch.equal(one, outs[0])
    # the persistent launch (all volumes' iterations through one work queue):
    # against the reference and FP64 like the per-volume batch, within 1e-6
    # of it (its z bodies use paired FP32 adds, the per-volume z kernels
    # scalar adds and FMAs), and a replay of its captured graph gives the
    # same bits
    pers = [torch.full_like(a, -1.0) for a in di]
    clarity_gpu.ml_batch_device(di, dk, pers, iters, graph=True, persistent=True)
    torch.cuda.synchronize()
    first = [p.clone() for p in pers]
    for i, (img, psf), a, b in zip(BATCH_IDS, cases, outs, pers):
        got = b.cpu().numpy()
        _check(f"batched_persistent_vol{i}_rl{iters}_{img.shape[2]}x{img.shape[1]}x"
               f"{img.shape[0]}", got, _ref32(ref_cpu, oracle_lib, "rl", img, psf, iters),
               _ref64(oracle_lib, "rl", img, psf, iters), TOL_ITER)
        assert rel_l2(got, a.cpu().numpy()) <= 1e-6, i
    clarity_gpu.ml_batch_device(di, dk, pers, iters, graph=True, persistent=True)
    torch.cuda.synchronize()
    for a, b in zip(first, pers):
        assert torch.equal(a, b)
    clarity_gpu.synchronize()
