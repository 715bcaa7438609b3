"""Failure detection on the GPU without a GPU fault.

The fused passes wait for their tile copies with bounded waits; a wait that
gives up records a timeout in the library's error word and its kernel
returns.  clarityx_inject_wait_timeout runs exactly such a wait with nothing
to wait for (a barrier armed for bytes no copy delivers, no copy issued, a
bound of a few thousand polls), so the wait runs out, the kernel returns and
the context stays usable.  These tests check that the failure reaches the
caller through the public calls, once, and that the library works afterwards.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def test_timed_out_wait_is_reported_by_synchronize(clarity_gpu):
    import torch
    s = torch.cuda.current_stream()
    clarity_gpu.synchronize(s)  # nothing pending
    clarity_gpu.inject_wait_timeout(s)
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.synchronize(s)
    assert e.value.code == clarity_gpu.CLARITY_INVALID_OPERATION
    assert "timed out" in str(e.value)
    clarity_gpu.synchronize(s)  # reported once, then cleared
    clarity_gpu.inject_wait_timeout(s)
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.synchronize(None)  # the whole device
    assert e.value.code == clarity_gpu.CLARITY_INVALID_OPERATION


def test_device_call_reports_an_earlier_timeout_and_enqueues_nothing(clarity_gpu, oracle_lib):
    import torch
    d = load_golden("small_even")
    img = torch.from_numpy(d["image"]).cuda()
    psf = torch.from_numpy(d["psf"]).cuda()
    clarity_gpu.inject_wait_timeout()
    torch.cuda.synchronize()  # the probe has finished; the word is set
    out = torch.full_like(img, -1.0)
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.ml_device(img, psf, out, 3)
    assert e.value.code == clarity_gpu.CLARITY_INVALID_OPERATION
    torch.cuda.synchronize()
    assert bool((out == -1.0).all())  # nothing ran
    # the next call runs and is right
    clarity_gpu.ml_device(img, psf, out, 3)
    clarity_gpu.synchronize(torch.cuda.current_stream())
    assert rel_l2(out.cpu().numpy(), oracle_lib.rl(d["image"], d["psf"], 3)) <= 1e-4


def test_host_call_reports_an_earlier_timeout(clarity_gpu):
    import torch
    d = load_golden("small_odd")
    clarity_gpu.inject_wait_timeout()
    torch.cuda.synchronize()
    with pytest.raises(clarity_gpu.ClarityError) as e:
        clarity_gpu.convolve(d["image"], d["psf"])
    assert e.value.code == clarity_gpu.CLARITY_INVALID_OPERATION
    out = clarity_gpu.convolve(d["image"], d["psf"])
    assert rel_l2(out, d["convolve"]) <= 1e-5
    assert np.isfinite(out).all()
