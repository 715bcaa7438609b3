"""The no-allocation convolution entry point (clarityx_convolve_noalloc).

Callers that cannot allocate device memory while running -- code under a
memory pool it manages itself, fixed-footprint real-time loops, plugins in a
context that forbids cudaMalloc -- use this entry point; its scratch lives in
a fixed 32 MiB array inside the library.  The tests call it through the C ABI
twice in a row and check each result against the regular device-buffer entry
point (clarityx_convolve_device), on the golden fixtures and on the largest
box the array holds.  The file is named so pytest collects it last; it passes
alone in a fresh process and after the other tests (it needs no registration
of its own, and the regular entry point it compares against is registered by
the shared fixture).
"""
import numpy as np
import pytest

from clarity_b200 import synthetic as syn
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def _twice_against_device_entry(api, img, psf, tol=1e-6):
    import torch
    want = torch.empty_like(img)
    api.convolve_device(img, psf, want)
    torch.cuda.synchronize()
    want = want.cpu().numpy()
    outs = []
    for _ in range(2):
        out = torch.full_like(img, float("nan"))
        api.convolve_noalloc(img, psf, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_l2(got, want) <= tol
        outs.append(got)
    return want, outs


@pytest.mark.parametrize("case", ["small_even", "small_odd", "testcommon_16x16x8"])
def test_noalloc_matches_device_entry_point_twice(clarity_gpu, case):
    import torch
    d = load_golden(case)
    img = torch.from_numpy(d["image"]).cuda()
    psf = torch.from_numpy(d["psf"]).cuda()
    _, outs = _twice_against_device_entry(clarity_gpu, img, psf)
    for got in outs:
        assert rel_l2(got, d["convolve"]) <= 1e-5


def test_noalloc_at_its_largest_documented_box(clarity_gpu):
    # a 64^3 image with a 64^3 kernel: work box 128^3, 16.5 MiB of spectra
    import torch
    r = syn.rng(31)
    img = torch.from_numpy((r.random((64, 64, 64)) * 100 + 1).astype(np.float32)).cuda()
    psf = torch.from_numpy(syn.gaussian_psf((64, 64, 64), 1.5, 2.5).astype(np.float32)).cuda()
    _twice_against_device_entry(clarity_gpu, img, psf)


def test_noalloc_rejects_work_box_beyond_scratch(clarity_gpu):
    import torch
    img = torch.ones((128, 128, 128), device="cuda")
    out = torch.empty_like(img)
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.convolve_noalloc(img, img, out)
    assert e.value.code == clarity_gpu.CLARITY_INVALID_ARGUMENT
    assert "scratch" in str(e.value)
