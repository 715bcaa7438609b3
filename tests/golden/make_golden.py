"""Generate the golden fixtures from the REFERENCE itself.

Runs only where the reference sources were built into oracle/_ref (this needs
the read-only reference checkout; the GPU machine only reads the committed
.npz files).  Inputs are seeded synthetic volumes; outputs come from the
unmodified reference CPU code (src/*.cxx) linked with the project's FFTW-API
shim, called through the reference's own C API:

  ref        verbatim reference (serial float flux sum)
  ref64      the same with Clarity_ReduceSum accumulating in double

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from clarity_b200 import synthetic as syn  # noqa: E402


def case(name, img, psf, rl_iters, jvc_iters, blind_iters, eps=1e-3, full=True):
    ref = O.ReferenceCPU("ref")
    ref64 = O.ReferenceCPU("ref_fp64sum")
    out = {"image": img, "psf": psf,
           "rl_iters": np.int32(rl_iters), "jvc_iters": np.int32(jvc_iters),
           "blind_iters": np.int32(blind_iters), "wiener_eps": np.float32(eps)}
    out["rl_ref"] = ref.rl(img, psf, rl_iters)
    out["rl_ref64"] = ref64.rl(img, psf, rl_iters)
    out["rl1_ref64"] = ref64.rl(img, psf, 1)
    if full:
        out["convolve"] = ref.convolve(img, psf)
        out["wiener"] = ref.wiener(img, psf, eps)
        out["jvc"] = ref.jvc(img, psf, jvc_iters)
        out["blind_ref64"] = ref64.blind(img, psf, blind_iters)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, img.shape, psf.shape, {k: v.shape for k, v in out.items() if hasattr(v, 'shape') and v.ndim})


def main():
    # even work box 32x26x16 (x,y,z)
    img, psf, _ = syn.make_case((12, 20, 24), 8, 1.5, 2.0, seed=11)
    psf = syn.gaussian_psf((4, 6, 8), 1.2, 1.5).astype(np.float32)
    case("small_even", img, psf, 5, 4, 3)
    # odd work box 19x15x11 (x odd -> full complex x; radices 19, 5, 3, 11)
    img, psf, _ = syn.make_case((7, 10, 13), 5, 1.2, 1.5, seed=12)
    psf = syn.gaussian_psf((4, 5, 6), 1.0, 1.3).astype(np.float32)
    case("small_odd", img, psf, 5, 4, 3)
    # the reference test fixture (tests/common/Test_Common.h:99-161) at a
    # reduced size: box of ones over the central half, sigma-2 Gaussian kernel
    dims = (8, 16, 16)
    t = np.zeros(dims, np.float32)
    t[2:6, 4:12, 4:12] = 1.0
    k = syn.gaussian_psf((8, 8, 8), 2.0, 2.0).astype(np.float32)
    conv = O.ReferenceCPU("ref").convolve(t, k)
    case("testcommon_16x16x8", conv, k, 10, 10, 10)
    # the small RL workload: 64x64x32, 40 spheres, sigma 1.5/3.0, RL 10 iterations
    img, psf, _ = syn.cfg0(seed=0)
    case("cfg0_rl10", img, psf, 10, 10, 10, full=False)


if __name__ == "__main__":
    main()
