"""CPU tests of the oracle itself: it must agree with the reference before it
may judge the CUDA library.

* the FFT restatement (the FFTW stand-in) against numpy's FFT;
* the restatement of every algorithm against the unmodified reference CPU
  build (bit-identical where the arithmetic order is the same);
* the reference's own test programs (tests/*/ compiled unchanged) as a
  known-answer check;
* the committed golden fixtures.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import load_golden, rel_l2


@pytest.mark.parametrize("shape", [(4, 6, 8), (5, 7, 9), (3, 10, 15), (8, 12, 19),
                                   (2, 2, 2), (1, 1, 6), (6, 11, 13)])
def test_fft_restatement_matches_numpy(oracle_lib, shape):
    x = np.random.default_rng(1).standard_normal(shape)
    ref = np.fft.rfftn(x)
    got64 = oracle_lib.r2c(x, "f64")
    assert np.abs(got64 - ref).max() <= 1e-12 * np.abs(ref).max()
    got32 = oracle_lib.r2c(x, "f32")
    assert np.abs(got32 - ref).max() <= 2e-6 * np.abs(ref).max()
    back = oracle_lib.c2r(ref, shape[2], "f64")
    assert np.abs(back - x * x.size).max() <= 1e-11 * x.size


def test_fft_c2r_ignores_self_conjugate_imaginary_parts(oracle_lib):
    # FFTW's c2r treats the input as Hermitian: the imaginary parts of the
    # x = 0 and x = nx/2 bins of the last axis do not contribute.
    x = np.random.default_rng(2).standard_normal((4, 6, 8))
    spec = np.fft.rfftn(x)
    spec2 = spec.copy()
    spec2[0, 0, 0] += 5j
    spec2[0, 0, 4] += 3j
    a = oracle_lib.c2r(spec, 8, "f64")
    b = oracle_lib.c2r(spec2, 8, "f64")
    assert np.abs(a - b).max() < 1e-9


ref_available = pytest.mark.skipif(not O.ReferenceCPU.available("ref"),
                                   reason="reference build (oracle/_ref) absent")


@ref_available
@pytest.mark.parametrize("case", ["small_even", "small_odd"])
def test_restatement_bit_identical_to_reference(oracle_lib, case):
    d = load_golden(case)
    img, psf = d["image"], d["psf"]
    ref = O.ReferenceCPU("ref")
    ref64 = O.ReferenceCPU("ref_fp64sum")
    assert np.array_equal(oracle_lib.convolve(img, psf), ref.convolve(img, psf))
    assert np.array_equal(oracle_lib.wiener(img, psf, 1e-3), ref.wiener(img, psf, 1e-3))
    assert np.array_equal(oracle_lib.jvc(img, psf, 4), ref.jvc(img, psf, 4))
    assert np.array_equal(oracle_lib.rl(img, psf, 4, sum_mode=O.SUM_SERIAL_FLOAT),
                          ref.rl(img, psf, 4))
    assert np.array_equal(oracle_lib.rl(img, psf, 4, sum_mode=O.SUM_DOUBLE),
                          ref64.rl(img, psf, 4))
    assert np.array_equal(oracle_lib.blind(img, psf, 3, sum_mode=O.SUM_SERIAL_FLOAT),
                          ref.blind(img, psf, 3))


@ref_available
def test_reference_pad_shift_matches_restatement(oracle_lib):
    import ctypes as C
    ref = O.ReferenceCPU("ref")
    L = ref.lib
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.Clarity_ImagePadSpatialShift.argtypes = [f32p, O._Dim3, f32p, O._Dim3,
                                               C.POINTER(C.c_int), C.c_float]
    src = np.random.default_rng(3).random((3, 5, 7)).astype(np.float32)
    for shift in [(0, 0, 0), (-3, -2, -1), (2, 1, 0), (-7, 5, -3)]:
        dst = np.empty((6, 9, 11), np.float32)
        sh = (C.c_int * 3)(*shift)
        L.Clarity_ImagePadSpatialShift(dst, O._Dim3(11, 9, 6), src, O._Dim3(7, 5, 3), sh, 0.5)
        ours = oracle_lib.pad_shift(src, (6, 9, 11), shift, 0.5)
        assert np.array_equal(dst, ours)


REF_BIN = os.path.join(os.path.dirname(O.HERE), "oracle", "_ref", "bin")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_BIN, "MaximumLikelihoodTest")),
                    reason="reference test programs not built")
def test_reference_test_program_known_answer(tmp_path):
    # tests/MaximumLikelihoodTest/MaximumLikelihoodTest.cxx at 16x16x8 with an
    # 8^3 kernel prints RMS 0.233955 when linked against a naive O(n^2) DFT in
    # place of FFTW; the project's FFT must reproduce it.
    env = dict(os.environ, CLARITY_IMAGE_SIZE_X="16", CLARITY_IMAGE_SIZE_Y="16",
               CLARITY_IMAGE_SIZE_Z="8", CLARITY_KERNEL_SIZE_X="8",
               CLARITY_KERNEL_SIZE_Y="8", CLARITY_KERNEL_SIZE_Z="8", CLARITY_NP="2")
    out = subprocess.run([os.path.join(REF_BIN, "MaximumLikelihoodTest")], env=env,
                         cwd=tmp_path, capture_output=True, text=True, timeout=120).stdout
    assert "RMS is: 0.233955" in out, out


@pytest.mark.parametrize("case", ["small_even", "small_odd", "testcommon_16x16x8"])
def test_restatement_matches_golden(oracle_lib, case):
    d = load_golden(case)
    img, psf = d["image"], d["psf"]
    n = int(d["rl_iters"])
    assert rel_l2(oracle_lib.rl(img, psf, n), d["rl_ref64"]) <= 1e-6
    assert rel_l2(oracle_lib.rl(img, psf, n, sum_mode=O.SUM_SERIAL_FLOAT), d["rl_ref"]) <= 1e-6
    assert rel_l2(oracle_lib.convolve(img, psf), d["convolve"]) <= 1e-6
    assert rel_l2(oracle_lib.wiener(img, psf, float(d["wiener_eps"])), d["wiener"]) <= 1e-6
    assert rel_l2(oracle_lib.jvc(img, psf, int(d["jvc_iters"])), d["jvc"]) <= 1e-6
    assert rel_l2(oracle_lib.blind(img, psf, int(d["blind_iters"])), d["blind_ref64"]) <= 1e-6


def test_restatement_matches_golden_cfg0(oracle_lib):
    d = load_golden("cfg0_rl10")
    got = oracle_lib.rl(d["image"], d["psf"], int(d["rl_iters"]))
    assert rel_l2(got, d["rl_ref64"]) <= 1e-6


def test_fp64_oracle_close_to_fp32(oracle_lib):
    d = load_golden("small_even")
    a = oracle_lib.rl(d["image"], d["psf"], 5, precision="f64")
    assert rel_l2(a, d["rl_ref64"]) < 1e-4
    c = oracle_lib.convolve(d["image"], d["psf"], precision="f64")
    assert rel_l2(c, d["convolve"]) < 1e-5


def test_rl_flux_conservation_on_work_box(oracle_lib):
    d = load_golden("small_even")
    out, work = oracle_lib.rl(d["image"], d["psf"], 3, precision="f64", work=True)
    assert abs(work.sum() - d["image"].astype(np.float64).sum()) < 1e-6 * d["image"].sum()


def test_idivergence_oracle(oracle_lib):
    g = np.array([1.0, 2.0, 0.0, 3.0], np.float32)
    gh = np.array([1.0, 1.0, 0.5, 3.0], np.float32)
    want = 2 * np.log(2.0) + 1.0 - 2.0 + 0.5
    assert abs(oracle_lib.idivergence(g, gh) - want) < 1e-12


def test_idiv_restoration_lowers_its_objective(oracle_lib):
    # the Markham-Conchello restatement: the work-box objective
    # sum g ln(g/gh) + gh - g + alpha sum s^2 (g zero-padded, gh = h * s, circular
    # on the padded box) falls with every conjugate-gradient step, and s >= 0
    d = load_golden("small_even")
    img, psf = d["image"].astype(np.float64), d["psf"].astype(np.float64)
    Z, Y, X = img.shape
    kz, ky, kx = psf.shape
    W = (Z + kz, Y + ky, X + kx)
    g = np.zeros(W)
    g[:Z, :Y, :X] = img
    h = np.zeros(W)
    h[:kz, :ky, :kx] = psf
    H = np.fft.rfftn(np.roll(h, (-(kz // 2), -(ky // 2), -(kx // 2)), (0, 1, 2)))

    def objective(est, alpha):
        s = np.zeros(W)
        s[:Z, :Y, :X] = est
        gh = np.fft.irfftn(np.fft.rfftn(s) * H, W, axes=(0, 1, 2))
        m = g > 0
        return float((g[m] * np.log(g[m] / gh[m])).sum() + gh.sum() - g.sum()
                     + alpha * (s ** 2).sum())

    for alpha in (0.0, 1e-4):
        ests = [oracle_lib.idiv_cg(d["image"], d["psf"], it, alpha, precision="f64")
                for it in (0, 1, 2, 4, 8)]
        js = [objective(e, alpha) for e in ests]
        assert all(b < a for a, b in zip(js, js[1:])), js
        assert all(e.min() >= 0 for e in ests)
