"""The precision form of the 3-D FFT (clarityx_set_dft_precision): the first
radix-16 z stage of the 1024x1024x256 work box (a 512x512x128 volume with a
same-size PSF) as tensor-core GEMMs on split hi+lo FP16 or BF16 operands with
FP32 accumulation, beside the FP32 register passes.  Every form's result is
compared with the FP64 oracle (and the reference's CPU build); the errors
are recorded (conftest.report_error).  FP16 split must hold the FP32 parity
bar; BF16 split (8 + 8 significant bits) is reported and held to 1e-3.
"""
import numpy as np
import pytest

from clarity_b200 import synthetic as syn
from conftest import cached, rel_l2, report_error

pytestmark = pytest.mark.gpu

MODES = {0: "f32_simt", 1: "f16_split_tc", 2: "bf16_split_tc"}


@pytest.fixture(scope="module")
def large():
    img, psf, _ = syn.cfg3(seed=7)
    return img, psf


def _run_modes(api, fn):
    outs = {}
    try:
        for m in MODES:
            api.set_dft_precision(m)
            assert api.dft_precision() == m
            outs[m] = fn()
    finally:
        api.set_dft_precision(0)
    return outs


def test_precision_forms_rl_large_box(clarity_gpu, ref_cpu, oracle_lib, large):
    img, psf = large
    r32 = cached("rl2-ref32", [img, psf],
                 lambda: (ref_cpu or oracle_lib).rl(img, psf, 2))
    r64 = cached("rl2-f64", [img, psf], lambda: oracle_lib.rl(img, psf, 2, precision="f64"))
    ref_e64 = rel_l2(r32, r64)
    outs = _run_modes(clarity_gpu, lambda: clarity_gpu.maximum_likelihood_deconvolve(img, psf, 2))
    errs = {}
    for m, out in outs.items():
        errs[m] = rel_l2(out, r64)
        report_error(f"precision_{MODES[m]}_rl2_512x512x128", rel_l2_vs_fp64=errs[m],
                     max_abs_vs_fp64=float(np.abs(out.astype(np.float64) - r64).max()),
                     rel_l2_vs_reference=rel_l2(out, r32), reference_rel_l2_vs_fp64=ref_e64)
    # the tensor-core forms really ran (their results differ from FP32's)
    assert not np.array_equal(outs[1], outs[0])
    assert not np.array_equal(outs[2], outs[0])
    for m in (0, 1):
        assert errs[m] <= max(3 * ref_e64, 1e-5), (MODES[m], errs[m], ref_e64)
        assert rel_l2(outs[m], r32) <= 1e-4
    assert errs[2] <= 1e-3


def test_precision_forms_single_transform(clarity_gpu, oracle_lib, large):
    # one convolution: forward FFT, OTF product, inverse FFT
    img, psf = large
    r64 = cached("conv-f64", [img, psf], lambda: oracle_lib.convolve(img, psf, precision="f64"))
    outs = _run_modes(clarity_gpu, lambda: clarity_gpu.convolve(img, psf))
    for m, out in outs.items():
        report_error(f"precision_{MODES[m]}_convolve_512x512x128", rel_l2_vs_fp64=rel_l2(out, r64),
                     max_abs_vs_fp64=float(np.abs(out.astype(np.float64) - r64).max()))
    assert rel_l2(outs[0], r64) <= 1e-6
    assert rel_l2(outs[1], r64) <= 1e-6
    assert rel_l2(outs[2], r64) <= 1e-4


def test_precision_mode_argument_checked(clarity_gpu):
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.set_dft_precision(3)
    assert e.value.code == clarity_gpu.CLARITY_INVALID_ARGUMENT
    assert clarity_gpu.dft_precision() == 0
