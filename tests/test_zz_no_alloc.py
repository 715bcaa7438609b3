"""The no-allocation convolution entry point (clarityx_convolve_noalloc).

Callers that cannot allocate device memory while running -- CUDA graph
capture, their own memory pools, fixed-footprint real-time loops, plugins in
a context that forbids cudaMalloc -- use this entry point; its scratch lives
in a fixed 32 MiB array inside the library.  The test calls it through the C
ABI twice in a row and checks each result against the regular
device-buffer entry point (clarityx_convolve_device).  The file is named so
pytest collects it last; it passes alone in a fresh process and after the
other tests (it needs no registration of its own, and the regular entry
point it compares against is registered by the shared fixture).
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["small_even", "small_odd", "testcommon_16x16x8"])
def test_noalloc_matches_device_entry_point_twice(clarity_gpu, case):
    import torch
    d = load_golden(case)
    img = torch.from_numpy(d["image"]).cuda()
    psf = torch.from_numpy(d["psf"]).cuda()
    want = torch.empty_like(img)
    clarity_gpu.convolve_device(img, psf, want)
    torch.cuda.synchronize()
    want = want.cpu().numpy()
    for _ in range(2):
        out = torch.full_like(img, float("nan"))
        clarity_gpu.convolve_noalloc(img, psf, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_l2(got, want) <= 1e-6
        assert rel_l2(got, d["convolve"]) <= 1e-5


def test_noalloc_rejects_work_box_beyond_scratch(clarity_gpu):
    import torch
    img = torch.ones((128, 128, 128), device="cuda")
    out = torch.empty_like(img)
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.convolve_noalloc(img, img, out)
    assert e.value.code == clarity_gpu.CLARITY_INVALID_ARGUMENT
    assert "scratch" in str(e.value)
