"""CPU emulation of the CUDA library: the library's own kernel and host
sources compiled as C++ (tests/emu, AddressSanitizer) and driven through the
public C API.  Every block runs on one host thread, so each kernel phase's
work items are all executed in order; this checks every shared- and
global-memory index the kernels compute (ASan aborts on any out-of-bounds
access) and the numerics against the oracle, without a GPU.

The shapes cover every plan form: split y (Ay > 1, several G/W choices),
whole-y-in-Z (Ay = 1), odd x (full complex rows), 1- and 2-pass axes and
prime radices.
"""
import os
import subprocess

import numpy as np
import pytest

from clarity_b200 import synthetic as syn
from conftest import ROOT, load_golden, rel_l2

EMU_DIR = os.path.join(ROOT, "_build", "emu")
EMU = os.path.join(EMU_DIR, "emu_main")


def _sources():
    out = []
    for d in ("clarity_b200/csrc", "tests/emu", "include"):
        for f in os.listdir(os.path.join(ROOT, d)):
            out.append(os.path.join(ROOT, d, f))
    return out


@pytest.fixture(scope="module")
def emu():
    newest = max(os.path.getmtime(f) for f in _sources())
    if not os.path.exists(EMU) or os.path.getmtime(EMU) < newest:
        subprocess.run([os.path.join(ROOT, "tests", "emu", "build_emu.sh"), ROOT],
                       check=True, capture_output=True)
    return EMU


def run_emu(emu, tmp_path, op, img, psf, param):
    img = np.ascontiguousarray(img, np.float32)
    psf = np.ascontiguousarray(psf, np.float32)
    a, b, o = (str(tmp_path / n) for n in ("img.raw", "psf.raw", "out.raw"))
    img.tofile(a)
    psf.tofile(b)
    z, y, x = img.shape
    kz, ky, kx = psf.shape
    p = subprocess.run([emu, op, str(x), str(y), str(z), str(kx), str(ky), str(kz),
                        repr(param), a, b, o], capture_output=True, text=True,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=0"))
    assert p.returncode == 0, p.stderr[-4000:]
    return np.fromfile(o, np.float32).reshape(img.shape)


@pytest.mark.parametrize("case", ["small_even", "small_odd", "testcommon_16x16x8"])
def test_emulated_library_matches_reference_golden(emu, tmp_path, case):
    d = load_golden(case)
    img, psf = d["image"], d["psf"]
    assert rel_l2(run_emu(emu, tmp_path, "convolve", img, psf, 0), d["convolve"]) <= 1e-6
    assert rel_l2(run_emu(emu, tmp_path, "convolve_noalloc", img, psf, 0),
                  d["convolve"]) <= 1e-6
    assert rel_l2(run_emu(emu, tmp_path, "wiener", img, psf, float(d["wiener_eps"])),
                  d["wiener"]) <= 2e-6
    assert rel_l2(run_emu(emu, tmp_path, "rl", img, psf, 1), d["rl1_ref64"]) <= 1e-6
    assert rel_l2(run_emu(emu, tmp_path, "rl", img, psf, int(d["rl_iters"])),
                  d["rl_ref64"]) <= 2e-6
    assert rel_l2(run_emu(emu, tmp_path, "jvc", img, psf, int(d["jvc_iters"])),
                  d["jvc"]) <= 2e-6
    assert rel_l2(run_emu(emu, tmp_path, "blind", img, psf, int(d["blind_iters"])),
                  d["blind_ref64"]) <= 2e-6


@pytest.mark.parametrize("img_zyx,psf_zyx", [
    ((16, 32, 32), (16, 32, 32)),   # work 64x64x32: compile-time specialised shape
    ((32, 64, 64), (32, 64, 64)),   # work 128x128x64: specialised shape of the small RL workload
    ((12, 24, 20), (12, 24, 20)),   # work 40x48x24: Ay 12, x radix 5*4
    ((10, 30, 18), (10, 30, 18)),   # work 36x60x20: Ay 4, By 15 (2 passes)
    ((15, 27, 25), (15, 27, 25)),   # work 50x54x30: Ay 3, By 18
    ((6, 9, 10), (3, 4, 5)),        # work 15x13x9: odd x, prime 13
    ((5, 8, 12), (3, 3, 5)),        # work 17x11x8: odd prime x 17, prime y 11
    ((1, 6, 8), (1, 2, 2)),         # work 10x8x2
])
def test_emulated_library_matches_oracle(emu, tmp_path, oracle_lib, img_zyx, psf_zyx):
    r = syn.rng(sum(img_zyx))
    img = (r.random(img_zyx) * 100 + 1).astype(np.float32)
    psf = syn.gaussian_psf(psf_zyx, 1.5, 1.2).astype(np.float32)
    assert rel_l2(run_emu(emu, tmp_path, "convolve", img, psf, 0),
                  oracle_lib.convolve(img, psf)) <= 1e-6
    assert rel_l2(run_emu(emu, tmp_path, "rl", img, psf, 2),
                  oracle_lib.rl(img, psf, 2)) <= 2e-6
    assert rel_l2(run_emu(emu, tmp_path, "jvc", img, psf, 2),
                  oracle_lib.jvc(img, psf, 2)) <= 2e-6
    assert rel_l2(run_emu(emu, tmp_path, "wiener", img, psf, 1e-2),
                  oracle_lib.wiener(img, psf, 1e-2)) <= 2e-6
    assert rel_l2(run_emu(emu, tmp_path, "sjvc", img, psf, 3),
                  oracle_lib.smoothed_jvc(img, psf, 3, 2, (1.0, 1.5, 0.7))) <= 2e-6
    # blind ML with PSF steps: one outer iteration agrees to FP32 level; the
    # alternating updates amplify roundoff after that (the FP32 oracle itself
    # drifts up to 7e-4 from FP64 at two iterations), so two iterations are
    # held to the FP64 oracle at max(1e-4, twice the FP32 oracle's drift)
    ob, _ = oracle_lib.blind_psf(img, psf, 1, 3)
    assert rel_l2(run_emu(emu, tmp_path, "blindpsf", img, psf, 1), ob) <= 2e-6
    ob32, _ = oracle_lib.blind_psf(img, psf, 2, 3)
    ob64, _ = oracle_lib.blind_psf(img, psf, 2, 3, precision="f64")
    assert rel_l2(run_emu(emu, tmp_path, "blindpsf", img, psf, 2), ob64) <= \
        max(1e-4, 2 * rel_l2(ob32, ob64))
    out, _ = oracle_lib.rl_accel(img, psf, 4)
    assert rel_l2(run_emu(emu, tmp_path, "accel", img, psf, 4), out) <= 2e-6
    # batched RL: three volumes, each identical to its own solve (checked in
    # emu_main), the first against the oracle
    assert rel_l2(run_emu(emu, tmp_path, "batch", img, psf, 2),
                  oracle_lib.rl(img, psf, 2)) <= 2e-6
    # the persistent batched launch: the same three volumes through one work
    # queue (checked against the single solves in emu_main), the first
    # against the oracle
    assert rel_l2(run_emu(emu, tmp_path, "batchp", img, psf, 3),
                  oracle_lib.rl(img, psf, 3)) <= 2e-6


@pytest.mark.parametrize("img_zyx,psf_zyx", [((16, 32, 32), (16, 32, 32)),
                                             ((12, 24, 20), (12, 24, 20)),
                                             ((6, 9, 10), (3, 4, 5))])
def test_emulated_persistent_batch_equals_single_solves(emu, tmp_path, img_zyx, psf_zyx):
    # with the runtime-planned kernels everywhere (CLARITY_STATIC=0) the
    # persistent launch's volumes equal their single solves bit for bit
    # (emu_main checks), whatever order the queue hands out work in
    r = syn.rng(3 + sum(img_zyx))
    img = (r.random(img_zyx) * 100 + 1).astype(np.float32)
    psf = syn.gaussian_psf(psf_zyx, 1.5, 1.2).astype(np.float32)
    os.environ["CLARITY_STATIC"] = "0"
    try:
        a = run_emu(emu, tmp_path, "batchp", img, psf, 2)
        os.environ["EMU_BLOCK_ORDER"] = "reverse"
        b = run_emu(emu, tmp_path, "batchp", img, psf, 2)
    finally:
        os.environ.pop("CLARITY_STATIC", None)
        os.environ.pop("EMU_BLOCK_ORDER", None)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("dims,chans", [((8, 6, 10), (16, 0, 16)), ((4, 6, 8), (16, 32, 48)),
                                        ((6, 4, 6), (32, 0, 64))])
def test_emulated_nn_conv3_matches_reference(emu, tmp_path, dims, chans):
    # the learned-start convolution kernels' tiles and index arithmetic (the
    # tensor-core fragments are replaced by scalar loops over the same shared
    # memory tiles) against the FP64 reference
    torch = pytest.importorskip("torch")
    import nn_ref as R
    D, H, W = dims
    c1, c2, co = chans
    pre = str(tmp_path / "nn")
    p = subprocess.run([emu, "nnconv", str(W), str(H), str(D), str(c1), str(c2), str(co), "1",
                        "-", "-", pre], capture_output=True, text=True,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=0"))
    assert p.returncode == 0, p.stderr[-2000:]
    rd = lambda s, shape: torch.from_numpy(np.fromfile(pre + "." + s, np.float32)
                                           .reshape(shape).astype(np.float64))
    cin = c1 + c2
    x1 = rd("x1", (D, H, W, c1)).requires_grad_(True)
    x2 = rd("x2", (D // 2, H // 2, W // 2, c2)) if c2 else None
    w = rd("w", (co, 27, cin)).requires_grad_(True)
    b = rd("b", (co,))
    dy = rd("dy", (D, H, W, co))
    ref = R.conv3(x1, w, co, bias=b, relu=False, x2=x2)
    y = rd("y", (D, H, W, co))
    assert (y - torch.relu(ref)).abs().max() <= 1e-2 * torch.relu(ref).abs().max()
    (ref * dy).sum().backward()
    dw = rd("dw", (co, 27, cin))
    assert (dw - w.grad).abs().max() <= 1e-4 * w.grad.abs().max()
    assert (rd("db", (co,)) - dy.sum(dim=(0, 1, 2))).abs().max() <= 1e-4 * dy.abs().sum()


@pytest.mark.parametrize("shape", [(12, 20, 24), (8, 30, 30)])
def test_emulated_results_do_not_depend_on_block_order(emu, tmp_path, shape):
    # every block of a pass owns its slice of the spectrum and of the output:
    # running the blocks last to first must give the same bits
    r = syn.rng(21)
    img = r.integers(0, 4000, size=shape).astype(np.float32)
    psf = syn.gaussian_psf(shape, 1.5, 2.0).astype(np.float32)
    for op, prm in (("convolve", 0), ("rl", 2), ("jvc", 2)):
        fwd = run_emu(emu, tmp_path, op, img, psf, prm)
        os.environ["EMU_BLOCK_ORDER"] = "reverse"
        try:
            rev = run_emu(emu, tmp_path, op, img, psf, prm)
        finally:
            del os.environ["EMU_BLOCK_ORDER"]
        assert np.array_equal(fwd, rev), op


@pytest.mark.parametrize("ishape,kshape", [((20, 30, 40), (12, 34, 24)),
                                           ((17, 29, 41), (15, 35, 23))])
def test_emulated_specialised_box_with_uneven_split(emu, tmp_path, ishape, kshape, oracle_lib):
    # a 64x64x32 work box (a specialised shape: TMA XY pass, per-line Z pass)
    # reached from image and PSF extents that are not multiples of the tile:
    # the ratio pass's live rows differ between lines and row groups
    r = syn.rng(5)
    img = (r.random(ishape) * 100).astype(np.float32)
    psf = syn.gaussian_psf(kshape, 1.5, 2.0).astype(np.float32)
    assert rel_l2(run_emu(emu, tmp_path, "rl", img, psf, 3), oracle_lib.rl(img, psf, 3)) <= 2e-6
    out, _ = oracle_lib.rl_accel(img, psf, 2)
    assert rel_l2(run_emu(emu, tmp_path, "accel", img, psf, 2), out) <= 2e-6


def test_emulated_u16_path_casts_like_x86(emu, tmp_path):
    # the raw-volume entry point (device casts in, RL, device cast out)
    # equals the float path's result cast as static_cast<unsigned short>
    # does on x86: truncation, low 16 bits (values above 65535 wrap)
    r = syn.rng(21)
    img = r.integers(0, 60000, size=(12, 20, 24)).astype(np.float32)
    psf = (syn.gaussian_psf((12, 20, 24), 1.5, 2.0) * 60000).astype(np.uint16).astype(np.float32)
    ref = run_emu(emu, tmp_path, "rl", img, psf, 3).astype(np.float64)
    v = np.trunc(ref).astype(np.int64) & 0xFFFF
    assert np.array_equal(run_emu(emu, tmp_path, "u16", img, psf, 3), v.astype(np.float32))


@pytest.mark.parametrize("case,op,alpha", [("small_even", "idiv", 0.0), ("small_odd", "idiva", 1e-4)])
def test_emulated_idiv_restoration_matches_oracle(emu, tmp_path, oracle_lib, case, op, alpha):
    # the Markham-Conchello I-divergence restoration: the library's passes and
    # reductions against the oracle's restatement of the same steps
    d = load_golden(case)
    img, psf = d["image"], d["psf"]
    for iters in (1, 4):
        got = run_emu(emu, tmp_path, op, img, psf, iters)
        ref64 = oracle_lib.idiv_cg(img, psf, iters, alpha, precision="f64")
        ref32 = oracle_lib.idiv_cg(img, psf, iters, alpha)
        assert rel_l2(got, ref64) <= max(2e-6, 4 * rel_l2(ref32, ref64))


@pytest.mark.parametrize("case", ["small_even", "small_odd"])
def test_emulated_correlation_opt_ins_match_oracle(emu, tmp_path, oracle_lib, case):
    # the conjugated OTF in the z pass: correlation, and RL whose second
    # convolution is the correlation
    d = load_golden(case)
    img, psf = d["image"], d["psf"]
    assert rel_l2(run_emu(emu, tmp_path, "correlate", img, psf, 0),
                  oracle_lib.correlate(img, psf)) <= 1e-6
    assert rel_l2(run_emu(emu, tmp_path, "rlcorr", img, psf, 3),
                  oracle_lib.rl_correlate(img, psf, 3)) <= 2e-6


def test_emulated_idiv_restoration_zero_iterations_returns_the_image(emu, tmp_path):
    # no step taken: s = (sqrt g)^2 on the image region, non-negative
    d = load_golden("small_even")
    img = d["image"]
    out = run_emu(emu, tmp_path, "idiv", img, d["psf"], 0)
    assert out.min() >= 0
    assert rel_l2(out, np.maximum(img, 0)) <= 1e-6
