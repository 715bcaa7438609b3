"""CPU tests of the C ABI library: it loads, exports every declared symbol,
keeps the reference's result codes, and its host-side logic (argument
checks, pad/clip utilities, planner) behaves without a GPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from clarity_b200 import api
from conftest import ROOT, gpu_available

HEADERS = [os.path.join(ROOT, "include", "clarity.h"),
           os.path.join(ROOT, "include", "clarity_ext.h")]


def declared_symbols():
    names = []
    for h in HEADERS:
        text = open(h).read()
        for m in re.finditer(r"^CLARITY_API\b[^;(]*?\b(\w+)\s*\(", text, re.S | re.M):
            names.append(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = api.load()
    names = declared_symbols()
    assert set(api.PUBLIC_SYMBOLS) <= set(names)
    assert set(api.EXTENSION_SYMBOLS) <= set(names)
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH],
                         capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for n in names:
        assert n in exported, n
        getattr(lib, n)


def test_result_codes_match_reference_enum_order():
    # Clarity.h.in:90-101: FFT_FAILED=0 ... SUCCESS=5
    text = open(HEADERS[0]).read()
    for name, val in [("CLARITY_FFT_FAILED", 0), ("CLARITY_OUT_OF_MEMORY", 1),
                      ("CLARITY_DEVICE_OUT_OF_MEMORY", 2), ("CLARITY_INVALID_OPERATION", 3),
                      ("CLARITY_INVALID_ARGUMENT", 4), ("CLARITY_SUCCESS", 5)]:
        assert re.search(rf"{name}\s*=\s*{val}\b", text)
        assert getattr(api, name) == val
        assert api.result_string(val) == name
    assert api.result_string(17) == "<unknown Clarity result>"


def test_dim3_from_array():
    arr = (C.c_int * 3)(7, 8, 9)
    d = api.load().Clarity_Dim3FromArray(arr)
    assert (d.x, d.y, d.z) == (7, 8, 9)


def test_pad_shift_and_clip_match_oracle(oracle_lib):
    src = np.random.default_rng(4).random((3, 5, 7)).astype(np.float32)
    for shift in [(0, 0, 0), (-3, -2, -1), (2, 1, 0), (-7, 5, -3)]:
        ours = api.image_pad_spatial_shift(src, (6, 9, 11), shift, 0.25)
        want = oracle_lib.pad_shift(src, (6, 9, 11), shift, 0.25)
        assert np.array_equal(ours, want)
    big = np.random.default_rng(5).random((6, 9, 11)).astype(np.float32)
    assert np.array_equal(api.image_clip(big, (3, 5, 7)), big[:3, :5, :7])


def test_argument_errors_without_device():
    img = np.ones((4, 4, 4), np.float32)
    L = api.load()
    # NULL buffers -> CLARITY_INVALID_ARGUMENT (src/ImageClip.cxx:34-36)
    f32p = L.Clarity_Convolve.argtypes
    L2 = C.CDLL(api.LIB_PATH)
    L2.Clarity_Convolve.argtypes = [C.c_void_p, api.Dim3, C.c_void_p, api.Dim3, C.c_void_p]
    L2.Clarity_Convolve.restype = C.c_int
    assert L2.Clarity_Convolve(None, api.Dim3(4, 4, 4), None, api.Dim3(4, 4, 4), None) == 4
    # non-positive dimensions
    with pytest.raises(api.ClarityError) as e:
        api._check(L.Clarity_Convolve(img, api.Dim3(0, 4, 4), img, api.Dim3(4, 4, 4), img))
    assert e.value.code == api.CLARITY_INVALID_ARGUMENT
    assert "dimension" in str(e.value)
    assert f32p is not None


def test_idiv_restoration_argument_errors_without_device():
    # iterations < 0 and a negative or NaN penalty are rejected before any
    # device work, with the reason in clarityx_last_error
    L = api.load()
    d3 = api.Dim3(4, 4, 4)
    for iters, alpha, word in ((-1, 0.0, "iterations"), (2, -1.0, "alpha"),
                               (2, float("nan"), "alpha")):
        rc = L.clarityx_idiv_deconvolve_device(C.c_void_p(16), d3, C.c_void_p(16), d3,
                                               C.c_void_p(16), iters, C.c_float(alpha), None)
        assert rc == api.CLARITY_INVALID_ARGUMENT
        assert word in L.clarityx_last_error().decode()


@pytest.mark.skipif(gpu_available(), reason="a GPU is present")
def test_register_without_gpu_is_invalid_operation():
    code = api.load().Clarity_Register()
    assert code == api.CLARITY_INVALID_OPERATION
    img = np.ones((4, 4, 4), np.float32)
    with pytest.raises(api.ClarityError) as e:
        api.convolve(img, img)
    assert e.value.code == api.CLARITY_INVALID_OPERATION
    assert "Register" in str(e.value)


@pytest.mark.parametrize("work", [(16, 32, 32), (64, 128, 128), (128, 512, 512),
                                  (256, 1024, 1024), (11, 15, 19), (1, 1, 2), (2, 3, 5),
                                  (176, 608, 544), (32, 192, 640), (96, 448, 224)])
def test_planner_invariants(work):
    z, y, x = work
    p = api.plan_info(work)
    assert p["Ay"] * p["By"] == y
    assert p["By"] % p["G"] == 0
    assert p["KG"] * p["W"] >= p["XS"]
    assert p["xmode"] == (x % 2)
    assert p["M"] == (x // 2 if x % 2 == 0 else x)
    assert p["xy_smem"] <= 200 * 1024 and p["z_smem"] <= 200 * 1024
    assert p["z_blocks"] == p["Ay"] * p["KG"]
    assert p["xy_blocks"] == z * (p["By"] // p["G"])


def test_benchmark_box_gets_the_specialised_tiling():
    # the 512x512x128 box (256x256x64 image + same-size PSF) must plan exactly
    # the compile-time shape its TMA XY pass and per-line Z pass are built for
    # (x radices 16.16, Ay 16, y0 radices 8.4, z radices 16.8, G 2, W 2)
    p = api.plan_info((128, 512, 512))
    assert (p["M"], p["Ay"], p["By"], p["G"], p["W"]) == (256, 16, 32, 2, 2)
    assert (p["x_passes"], p["y0_passes"], p["z_passes"]) == (2, 2, 2)


def test_planner_rejects_unsupported_prime():
    with pytest.raises(api.ClarityError) as e:
        api.plan_info((8, 8, 2 * 23))
    assert e.value.code == api.CLARITY_INVALID_ARGUMENT


def test_raw_image_app_usage_without_gpu():
    # the drop-in app mirrors the reference's command line (usage text, exit 1)
    app = os.path.join(os.path.dirname(api.LIB_PATH), "bin", "deconvolve_raw_images")
    p = subprocess.run([app], capture_output=True, text=True)
    assert p.returncode == 1
    assert "<image filename> <x> <y> <z> <psf filename> <x> <y> <z> <output file name>" in p.stdout


def test_network_parameter_count_matches_the_python_layout():
    # the C forward reads the FP32 parameter vector in unet.UNet3D's order:
    # per layer weights [co][27][c1 + c2] then bias [co], then the head
    from clarity_b200 import learned, unet
    specs = [("l0a", 1, 0, 16)] + unet.CONV_LAYERS
    n = sum(co * 27 * (c1 + c2) + co for _, c1, c2, co in specs) + 16 + 1
    assert api.nn_param_count() == n
    assert np.load(learned.WEIGHTS).size == n


def test_learned_start_argument_errors_without_device():
    L = api.load()
    d3 = api.Dim3(16, 16, 16)
    n = api.nn_param_count()
    rc = L.clarityx_ml_learned_device(C.c_void_p(16), d3, C.c_void_p(16), d3, None, n, 5,
                                      C.c_void_p(16), 2, None, None)
    assert rc == api.CLARITY_INVALID_ARGUMENT
    rc = L.clarityx_ml_learned_device(C.c_void_p(16), d3, C.c_void_p(16), d3, C.c_void_p(16),
                                      n - 1, 5, C.c_void_p(16), 2, None, None)
    assert rc == api.CLARITY_INVALID_ARGUMENT
    assert "parameters" in L.clarityx_last_error().decode()


def test_compat_header_compiles_a_reference_style_caller(tmp_path):
    # `#include <Clarity.h>` with include/compat on the path declares the
    # reference's API from this library's header
    src = tmp_path / "caller.c"
    src.write_text('#include <Clarity.h>\n'
                   'int main(void) { Clarity_Dim3 d = {1, 2, 3};\n'
                   '  return Clarity_ResultString(CLARITY_SUCCESS) != 0 && d.z == 3 ? 0 : 1; }\n')
    exe = tmp_path / "caller"
    p = subprocess.run(["gcc", "-I", os.path.join(ROOT, "include", "compat"), str(src), "-o",
                        str(exe), "-L", os.path.dirname(api.LIB_PATH), "-lclarity",
                        f"-Wl,-rpath,{os.path.dirname(api.LIB_PATH)}"],
                       capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    assert subprocess.run([str(exe)]).returncode == 0
