"""The drop-in claim, checked at the boundary: the reference's own five test
programs (tests/*Test/*Test.cxx) and its raw-image app
(apps/DeconvolveRawImages/DeconvolveRawImages.cxx), compiled UNCHANGED
against libclarity.so (oracle/_ref/dropin, built by `make -C oracle dropin`
from the reference sources through include/compat/Clarity.h), run here and
compared with the same programs linked to the reference's CPU build
(oracle/_ref/bin).  The programs read their sizes from the environment
(tests/common/Test_Common.h:51-89) and write their volumes as raw float32
files into the working directory; the RMS lines they print and the volumes
they write must agree within the float tolerances of the parity tests.

Both sets of programs are prebuilt (the reference sources are read only at
build time); the test is skipped where they were not built.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "bin")
DROPIN_BIN = os.path.join(ROOT, "oracle", "_ref", "dropin")
IMAGE_XYZ = (64, 48, 24)
KERNEL_XYZ = (16, 16, 8)
ENV = {"CLARITY_IMAGE_SIZE_X": str(IMAGE_XYZ[0]), "CLARITY_IMAGE_SIZE_Y": str(IMAGE_XYZ[1]),
       "CLARITY_IMAGE_SIZE_Z": str(IMAGE_XYZ[2]), "CLARITY_KERNEL_SIZE_X": str(KERNEL_XYZ[0]),
       "CLARITY_KERNEL_SIZE_Y": str(KERNEL_XYZ[1]), "CLARITY_KERNEL_SIZE_Z": str(KERNEL_XYZ[2])}

# program -> (file holding its result, tolerance)
PROGRAMS = {
    "ConvolutionTest": ("convolved_f32.raw", 1e-5),
    "WienerFilterTest": ("deconvolved_f32.raw", 1e-5),
    "MaximumLikelihoodTest": ("deconvolved_f32.raw", 1e-4),
    "JansenVanCittertTest": ("deconvolved_f32.raw", 1e-4),
    "BlindMaximumLikelihoodTest": ("deconvolved_f32.raw", 1e-4),
}


def _run(exe, cwd, args=()):
    env = dict(os.environ, **ENV)
    p = subprocess.run([exe, *args], cwd=cwd, env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout


def _numbers(text, label):
    return [float(m) for m in re.findall(label + r"\s*(-?[0-9.]+(?:e[-+]?\d+)?)", text)]


def _need(*paths):
    for p in paths:
        if not os.path.exists(p):
            pytest.skip(f"{p} was not built (make -C oracle ref dropin REF=<reference tree>)")


@pytest.mark.parametrize("program", sorted(PROGRAMS))
def test_reference_program_relinked_against_libclarity(program, tmp_path):
    ref_exe = os.path.join(REF_BIN, program)
    new_exe = os.path.join(DROPIN_BIN, program)
    _need(ref_exe, new_exe)
    (tmp_path / "ref").mkdir()
    (tmp_path / "new").mkdir()
    out_ref = _run(ref_exe, tmp_path / "ref")
    out_new = _run(new_exe, tmp_path / "new")
    n = int(np.prod(IMAGE_XYZ))
    result, tol = PROGRAMS[program]
    # the inputs the programs generate are the same bytes
    for f in ("image_f32.raw", "psf_f32.raw"):
        assert (tmp_path / "ref" / f).read_bytes() == (tmp_path / "new" / f).read_bytes()
    for f in sorted({"convolved_f32.raw", result}):
        a = np.fromfile(tmp_path / "new" / f, np.float32)
        b = np.fromfile(tmp_path / "ref" / f, np.float32)
        assert a.size == b.size == n
        assert np.isfinite(a).all()
        assert rel_l2(a, b) <= (1e-5 if f == "convolved_f32.raw" else tol), f
    # the printed report: the same lines, numbers within the float tolerance
    rms_ref, rms_new = _numbers(out_ref, "RMS is:"), _numbers(out_new, "RMS is:")
    assert len(rms_ref) == len(rms_new)
    for a, b in zip(rms_new, rms_ref):
        assert abs(a - b) <= 1e-4 * max(1.0, abs(b)) + 2e-6
    # difference of total intensities: float sums over the image, each voxel
    # within the parity tolerance
    tot_ref = _numbers(out_ref, "between images:")
    tot_new = _numbers(out_new, "between images:")
    assert len(tot_ref) == len(tot_new)
    for a, b in zip(tot_new, tot_ref):
        assert abs(a - b) <= tol * n
    strip = lambda t: [ln for ln in t.splitlines() if not re.search(r"\d\.\d", ln)
                       and "initialized" not in ln]
    assert strip(out_new) == strip(out_ref)


def test_raw_image_app_relinked_against_libclarity(tmp_path):
    ref_exe = os.path.join(REF_BIN, "DeconvolveRawImages")
    new_exe = os.path.join(DROPIN_BIN, "DeconvolveRawImages")
    _need(ref_exe, new_exe)
    r = np.random.Generator(np.random.PCG64(41))
    x, y, z = 40, 36, 12
    img = r.integers(0, 4000, size=(z, y, x)).astype(np.uint16)
    t = [np.exp(-0.5 * ((np.arange(n) - n // 2) / s) ** 2) for n, s in ((z, 2.0), (y, 1.5), (x, 1.5))]
    psf = (t[0][:, None, None] * t[1][None, :, None] * t[2][None, None, :])
    psf = (psf / psf.max() * 60000).astype(np.uint16)
    img.tofile(tmp_path / "img.raw")
    psf.tofile(tmp_path / "psf.raw")
    outs = {}
    for tag, exe in (("ref", ref_exe), ("new", new_exe)):
        args = [str(tmp_path / "img.raw"), str(x), str(y), str(z), str(tmp_path / "psf.raw"),
                str(x), str(y), str(z), str(tmp_path / f"out_{tag}.raw")]
        text = _run(exe, tmp_path, args)
        outs[tag] = (text, np.fromfile(tmp_path / f"out_{tag}.raw", np.uint16))
    keep = lambda t: [ln for ln in t.splitlines()
                      if "initialized" not in ln and not ln.startswith("Output file name")]
    assert keep(outs["new"][0]) == keep(outs["ref"][0])
    a, b = outs["new"][1].astype(np.int64), outs["ref"][1].astype(np.int64)
    assert a.size == b.size == img.size
    # float results within the parity tolerance truncate to the same count
    # except where they lie next to an integer: at most one count apart, rarely
    assert np.abs(a - b).max() <= 1
    assert np.count_nonzero(a != b) <= 0.01 * a.size
