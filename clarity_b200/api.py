"""Python mirror of the Clarity C API over the in-tree libclarity.so.

The function names, argument meaning and result codes follow the reference
header (Clarity.h.in:88-383): ``Clarity_MaximumLikelihoodDeconvolve(inImage,
imageDim, kernelImage, kernelDim, outImage, iterations)`` becomes
``maximum_likelihood_deconvolve(image, kernel, iterations)`` on numpy arrays in
(z, y, x) order (x fastest, the reference's memory layout), returning a new
array.  Every call goes through the C ABI; a non-success code raises
:class:`ClarityError` carrying the code and the library's message.

The ``*_device`` variants take torch CUDA tensors and run on the given (or
current) torch stream without host copies.

There is no CPU fallback: loading fails loudly if libclarity.so is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# CLARITY_LIB selects another build of the library (e.g. a variant built
# with `python -m clarity_b200.build -D... --lib PATH`).
LIB_PATH = os.environ.get("CLARITY_LIB", os.path.join(_HERE, "libclarity.so"))

# ClarityResult_t (Clarity.h.in:90-101); the numeric order is ABI.
CLARITY_FFT_FAILED = 0
CLARITY_OUT_OF_MEMORY = 1
CLARITY_DEVICE_OUT_OF_MEMORY = 2
CLARITY_INVALID_OPERATION = 3
CLARITY_INVALID_ARGUMENT = 4
CLARITY_SUCCESS = 5

RESULT_NAMES = {
    0: "CLARITY_FFT_FAILED", 1: "CLARITY_OUT_OF_MEMORY",
    2: "CLARITY_DEVICE_OUT_OF_MEMORY", 3: "CLARITY_INVALID_OPERATION",
    4: "CLARITY_INVALID_ARGUMENT", 5: "CLARITY_SUCCESS",
}

# Every symbol include/clarity.h and include/clarity_ext.h declare.
PUBLIC_SYMBOLS = [
    "Clarity_Dim3FromArray", "Clarity_Register", "Clarity_UnRegister",
    "Clarity_SetNumberOfThreads", "Clarity_ImagePadSpatialShift", "Clarity_ImageClip",
    "Clarity_ResultString", "Clarity_WienerDeconvolve",
    "Clarity_JansenVanCittertDeconvolve", "Clarity_SmoothedJansenVanCittertDeconvolve",
    "Clarity_IDivergenceDeconvolve", "Clarity_MaximumLikelihoodDeconvolve",
    "Clarity_BlindMaximumLikelihoodDeconvolve", "Clarity_Convolve",
]
EXTENSION_SYMBOLS = [
    "clarityx_last_error", "clarityx_set_device", "clarityx_inject_device_alloc_failure",
    "clarityx_trim", "clarityx_synchronize", "clarityx_inject_wait_timeout",
    "clarityx_convolve_device",
    "clarityx_wiener_device", "clarityx_ml_device", "clarityx_correlate_device",
    "clarityx_ml_correlate_device", "clarityx_blind_ml_device",
    "clarityx_jvc_device", "clarityx_idivergence", "clarityx_plan_info",
    "clarityx_launch_count", "clarityx_timing_enable", "clarityx_timing_collect",
    "clarityx_convolve_noalloc", "clarityx_ml_batch_device", "clarityx_autotune",
    "clarityx_ml_ex_device", "clarityx_ml_accel_device", "clarityx_ml_u16",
    "clarityx_blind_ml_psf_device",
    "clarityx_idiv_deconvolve_device",
    "clarityx_nn_conv3", "clarityx_nn_conv3_wgrad", "clarityx_nn_conv_in",
    "clarityx_nn_conv_in_wgrad", "clarityx_nn_head", "clarityx_nn_head_loss_grad",
    "clarityx_nn_pool2", "clarityx_nn_merge_skip_grad", "clarityx_nn_up_grad",
    "clarityx_nn_adam", "clarityx_nn_pack_weights",
    "clarityx_ml_learned_device", "clarityx_nn_predict", "clarityx_nn_param_count",
    "clarityx_set_dft_precision", "clarityx_dft_precision",
]
DFT_F32, DFT_F16_SPLIT, DFT_BF16_SPLIT = 0, 1, 2
BATCH_GRAPH = 1  # CLARITYX_BATCH_GRAPH
BATCH_PERSISTENT = 2  # CLARITYX_BATCH_PERSISTENT


class ClarityError(RuntimeError):
    def __init__(self, code: int, message: str):
        self.code = code
        super().__init__(f"{RESULT_NAMES.get(code, code)}: {message}")


class Dim3(C.Structure):
    """Clarity_Dim3 (Clarity.h.in:110-114)."""
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]

    def __repr__(self) -> str:
        return f"Dim3({self.x}, {self.y}, {self.z})"


_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_lib = None
_lib_lock = threading.Lock()


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libclarity.so (raises if it has not been built)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} is missing: build it with `python -m clarity_b200.build`")
        L = C.CDLL(path)
        i, u, f, vp = C.c_int, C.c_uint, C.c_float, C.c_void_p
        L.Clarity_Dim3FromArray.argtypes = [C.POINTER(C.c_int)]
        L.Clarity_Dim3FromArray.restype = Dim3
        L.Clarity_Register.restype = i
        L.Clarity_UnRegister.restype = i
        L.Clarity_SetNumberOfThreads.argtypes = [u]
        L.Clarity_SetNumberOfThreads.restype = i
        L.Clarity_ImagePadSpatialShift.argtypes = [_f32p, Dim3, _f32p, Dim3,
                                                   C.POINTER(C.c_int), f]
        L.Clarity_ImagePadSpatialShift.restype = i
        L.Clarity_ImageClip.argtypes = [_f32p, Dim3, _f32p, Dim3]
        L.Clarity_ImageClip.restype = i
        L.Clarity_ResultString.argtypes = [i]
        L.Clarity_ResultString.restype = C.c_char_p
        for name, extra in [("Clarity_WienerDeconvolve", [f]),
                            ("Clarity_JansenVanCittertDeconvolve", [i]),
                            ("Clarity_MaximumLikelihoodDeconvolve", [i]),
                            ("Clarity_BlindMaximumLikelihoodDeconvolve", [i]),
                            ("Clarity_Convolve", []),
                            ("Clarity_IDivergenceDeconvolve", [])]:
            fn = getattr(L, name)
            fn.argtypes = [_f32p, Dim3, _f32p, Dim3, _f32p] + extra
            fn.restype = i
        L.Clarity_SmoothedJansenVanCittertDeconvolve.argtypes = [
            _f32p, Dim3, _f32p, Dim3, _f32p, u, u, C.POINTER(C.POINTER(C.c_float))]
        L.Clarity_SmoothedJansenVanCittertDeconvolve.restype = i
        L.clarityx_last_error.restype = C.c_char_p
        L.clarityx_set_device.argtypes = [i]
        L.clarityx_set_device.restype = i
        L.clarityx_inject_device_alloc_failure.argtypes = [i]
        L.clarityx_inject_device_alloc_failure.restype = None
        L.clarityx_trim.restype = i
        L.clarityx_synchronize.argtypes = [vp]
        L.clarityx_synchronize.restype = i
        L.clarityx_inject_wait_timeout.argtypes = [vp]
        L.clarityx_inject_wait_timeout.restype = i
        for name, extra in [("clarityx_convolve_device", []),
                            ("clarityx_correlate_device", []),
                            ("clarityx_ml_correlate_device", [i]),
                            ("clarityx_wiener_device", [f]),
                            ("clarityx_ml_device", [i]),
                            ("clarityx_blind_ml_device", [i]),
                            ("clarityx_jvc_device", [i])]:
            fn = getattr(L, name)
            fn.argtypes = [vp, Dim3, vp, Dim3, vp] + extra + [vp]
            fn.restype = i
        L.clarityx_idivergence.argtypes = [_f32p, _f32p, C.c_longlong,
                                           C.POINTER(C.c_double)]
        L.clarityx_idivergence.restype = i
        L.clarityx_plan_info.argtypes = [Dim3, C.POINTER(C.c_int), i]
        L.clarityx_plan_info.restype = i
        L.clarityx_convolve_noalloc.argtypes = [vp, Dim3, vp, Dim3, vp, vp]
        L.clarityx_convolve_noalloc.restype = i
        L.clarityx_ml_batch_device.argtypes = [i, C.POINTER(vp), C.POINTER(Dim3),
                                               C.POINTER(vp), C.POINTER(Dim3),
                                               C.POINTER(vp), i, i, vp]
        L.clarityx_ml_batch_device.restype = i
        L.clarityx_ml_ex_device.argtypes = [vp, Dim3, vp, Dim3, vp, vp, i, vp, vp]
        L.clarityx_ml_ex_device.restype = i
        L.clarityx_ml_accel_device.argtypes = [vp, Dim3, vp, Dim3, vp, vp, i, vp, vp]
        L.clarityx_ml_accel_device.restype = i
        _u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
        L.clarityx_ml_u16.argtypes = [_u16p, Dim3, _u16p, Dim3, _u16p, i]
        L.clarityx_ml_u16.restype = i
        L.clarityx_blind_ml_psf_device.argtypes = [vp, Dim3, vp, Dim3, vp, vp, i, i, vp]
        L.clarityx_blind_ml_psf_device.restype = i
        L.clarityx_idiv_deconvolve_device.argtypes = [vp, Dim3, vp, Dim3, vp, i, C.c_float, vp]
        L.clarityx_idiv_deconvolve_device.restype = i
        L.clarityx_ml_learned_device.argtypes = [vp, Dim3, vp, Dim3, vp, C.c_longlong, i, vp, i,
                                                 vp, vp]
        L.clarityx_ml_learned_device.restype = i
        L.clarityx_nn_predict.argtypes = [vp, C.c_longlong, vp, Dim3, vp, vp]
        L.clarityx_nn_predict.restype = i
        L.clarityx_nn_param_count.restype = C.c_longlong
        L.clarityx_set_dft_precision.argtypes = [i]
        L.clarityx_set_dft_precision.restype = i
        L.clarityx_dft_precision.restype = i
        L.clarityx_autotune.argtypes = [i]
        L.clarityx_autotune.restype = None
        L.clarityx_launch_count.restype = C.c_longlong
        L.clarityx_timing_enable.argtypes = [i]
        L.clarityx_timing_enable.restype = None
        L.clarityx_timing_collect.argtypes = [C.POINTER(C.c_double),
                                              C.POINTER(C.c_longlong), i]
        L.clarityx_timing_collect.restype = None
        _lib = L
        return L


def _check(code: int) -> None:
    if code != CLARITY_SUCCESS:
        msg = load().clarityx_last_error().decode(errors="replace")
        raise ClarityError(code, msg)


def dim3(a) -> Dim3:
    """numpy (z, y, x) shape (or array) -> Clarity_Dim3(x, y, z)."""
    shape = a.shape if hasattr(a, "shape") else tuple(a)
    z, y, x = shape
    return Dim3(int(x), int(y), int(z))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------ lifecycle
def register() -> None:
    """Clarity_Register (src/Clarity.cxx:46-79)."""
    _check(load().Clarity_Register())


def unregister() -> None:
    """Clarity_UnRegister (src/Clarity.cxx:82-91)."""
    _check(load().Clarity_UnRegister())


def set_number_of_threads(n: int) -> None:
    _check(load().Clarity_SetNumberOfThreads(int(n)))


def result_string(code: int) -> str:
    return load().Clarity_ResultString(int(code)).decode()


def set_device(device: int) -> None:
    _check(load().clarityx_set_device(int(device)))


def inject_device_alloc_failure(countdown: int) -> None:
    load().clarityx_inject_device_alloc_failure(int(countdown))


def trim() -> None:
    _check(load().clarityx_trim())


def synchronize(stream=None) -> None:
    """clarityx_synchronize: wait for `stream` (None: every stream of the
    library's device) and raise the first asynchronous failure, such as a
    device-side bounded wait that gave up."""
    ptr = None if stream is None else C.c_void_p(stream.cuda_stream)
    _check(load().clarityx_synchronize(ptr))


def inject_wait_timeout(stream=None) -> None:
    """clarityx_inject_wait_timeout: enqueue a kernel whose bounded wait runs
    out (no copy in flight), recording a timeout as a fused pass would."""
    _check(load().clarityx_inject_wait_timeout(_stream_ptr(stream)))


# ------------------------------------------------------------- utilities
def image_pad_spatial_shift(src, dst_shape_zyx, shift_xyz, fill=0.0) -> np.ndarray:
    """Clarity_ImagePadSpatialShift (src/ImagePadSpatialShift.cxx:32-69)."""
    src = _f32(src)
    dst = np.empty(tuple(dst_shape_zyx), dtype=np.float32)
    sh = (C.c_int * 3)(*[int(v) for v in shift_xyz])
    _check(load().Clarity_ImagePadSpatialShift(dst, dim3(dst), src, dim3(src), sh,
                                               float(fill)))
    return dst


def image_clip(src, dst_shape_zyx) -> np.ndarray:
    """Clarity_ImageClip (src/ImageClip.cxx:30-50)."""
    src = _f32(src)
    dst = np.empty(tuple(dst_shape_zyx), dtype=np.float32)
    _check(load().Clarity_ImageClip(dst, dim3(dst), src, dim3(src)))
    return dst


# ------------------------------------------------------------ algorithms
def _host(name, image, kernel, *extra) -> np.ndarray:
    image, kernel = _f32(image), _f32(kernel)
    out = np.empty_like(image)
    _check(getattr(load(), name)(image, dim3(image), kernel, dim3(kernel), out, *extra))
    return out


def convolve(image, kernel) -> np.ndarray:
    """Clarity_Convolve (src/Convolve.cxx:41-115)."""
    return _host("Clarity_Convolve", image, kernel)


def wiener_deconvolve(image, kernel, epsilon: float) -> np.ndarray:
    """Clarity_WienerDeconvolve (src/WienerDeconvolve.cxx:211-290)."""
    return _host("Clarity_WienerDeconvolve", image, kernel, float(epsilon))


def maximum_likelihood_deconvolve(image, kernel, iterations: int) -> np.ndarray:
    """Clarity_MaximumLikelihoodDeconvolve (src/MaximumLikelihoodDeconvolve.cxx:255-332)."""
    return _host("Clarity_MaximumLikelihoodDeconvolve", image, kernel, int(iterations))


def blind_maximum_likelihood_deconvolve(image, kernel, iterations: int) -> np.ndarray:
    """Clarity_BlindMaximumLikelihoodDeconvolve (src/BlindMaximumLikelihoodDeconvolve.cxx:249-317)."""
    return _host("Clarity_BlindMaximumLikelihoodDeconvolve", image, kernel,
                 int(iterations))


def jansen_van_cittert_deconvolve(image, kernel, iterations: int) -> np.ndarray:
    """Clarity_JansenVanCittertDeconvolve (src/JansenVanCittertDeconvolve.cxx:311-389)."""
    return _host("Clarity_JansenVanCittertDeconvolve", image, kernel, int(iterations))


def smoothed_jansen_van_cittert_deconvolve(image, kernel, iterations: int,
                                           smooth_interval: int,
                                           smooth_sigma_xyz=None) -> np.ndarray:
    """Clarity_SmoothedJansenVanCittertDeconvolve (Clarity.h.in:285-291)."""
    image, kernel = _f32(image), _f32(kernel)
    out = np.empty_like(image)
    if smooth_sigma_xyz is None:
        arr = None
    else:
        vals = [C.c_float(float(s)) for s in smooth_sigma_xyz]
        arr = (C.POINTER(C.c_float) * 3)(*[C.pointer(v) for v in vals])
    _check(load().Clarity_SmoothedJansenVanCittertDeconvolve(
        image, dim3(image), kernel, dim3(kernel), out, int(iterations),
        int(smooth_interval), arr))
    return out


def idivergence_deconvolve(image, kernel) -> np.ndarray:
    """Clarity_IDivergenceDeconvolve: the reference stub writes zeros."""
    return _host("Clarity_IDivergenceDeconvolve", image, kernel)


def idivergence(g, ghat) -> float:
    """FP64 I-divergence sum g ln(g/ghat) + ghat - g (clarityx_idivergence)."""
    g, ghat = _f32(g).ravel(), _f32(ghat).ravel()
    if g.size != ghat.size:
        raise ValueError("size mismatch")
    r = C.c_double(0.0)
    _check(load().clarityx_idivergence(g, ghat, g.size, C.byref(r)))
    return float(r.value)


def plan_info(work_shape_zyx) -> dict:
    keys = ["M", "XS", "Ay", "By", "G", "W", "KG", "xy_blocks", "z_blocks", "xy_smem",
            "z_smem", "x_passes", "y0_passes", "z_passes", "xmode", "spec_kelems"]
    f = (C.c_int * 16)()
    _check(load().clarityx_plan_info(dim3(work_shape_zyx), f, 16))
    return dict(zip(keys, list(f)))


# ------------------------------------------------------------ probes
KERNEL_FAMILIES = ["xy_forward", "z", "xy_inv_fwd", "xy_inverse", "other", "xy_product"]


def launch_count() -> int:
    return int(load().clarityx_launch_count())


def timing_enable(on: bool = True) -> None:
    load().clarityx_timing_enable(1 if on else 0)


def timing_collect() -> dict:
    n = len(KERNEL_FAMILIES)
    ms = (C.c_double * n)()
    cnt = (C.c_longlong * n)()
    load().clarityx_timing_collect(ms, cnt, n)
    return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_FAMILIES)}


# ------------------------------------------------------ device variants
def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _dev(name, image, kernel, out, extra, stream):
    for t in (image, kernel, out):
        if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
            raise ValueError("device variants need contiguous float32 CUDA tensors")
    _check(getattr(load(), name)(C.c_void_p(image.data_ptr()), dim3(image),
                                 C.c_void_p(kernel.data_ptr()), dim3(kernel),
                                 C.c_void_p(out.data_ptr()), *extra, _stream_ptr(stream)))
    return out


def convolve_device(image, kernel, out, stream=None):
    return _dev("clarityx_convolve_device", image, kernel, out, [], stream)


def correlate_device(image, kernel, out, stream=None):
    """clarityx_correlate_device: circular correlation with the kernel (its
    spectrum conjugated in the z pass; an opt-in with no reference
    counterpart)."""
    return _dev("clarityx_correlate_device", image, kernel, out, [], stream)


def ml_correlate_device(image, kernel, out, iterations, stream=None):
    """clarityx_ml_correlate_device: RL whose second convolution per
    iteration is a correlation with the kernel (conjugated OTF)."""
    return _dev("clarityx_ml_correlate_device", image, kernel, out, [int(iterations)], stream)


def convolve_noalloc(image, kernel, out, stream=None):
    """clarityx_convolve_noalloc: convolution of device tensors with all
    scratch in the library's fixed 32 MiB device array (no allocation)."""
    return _dev("clarityx_convolve_noalloc", image, kernel, out, [], stream)


def wiener_device(image, kernel, out, epsilon, stream=None):
    return _dev("clarityx_wiener_device", image, kernel, out, [C.c_float(epsilon)], stream)


def ml_device(image, kernel, out, iterations, stream=None):
    return _dev("clarityx_ml_device", image, kernel, out, [int(iterations)], stream)


def blind_ml_device(image, kernel, out, iterations, stream=None):
    return _dev("clarityx_blind_ml_device", image, kernel, out, [int(iterations)], stream)


def jvc_device(image, kernel, out, iterations, stream=None):
    return _dev("clarityx_jvc_device", image, kernel, out, [int(iterations)], stream)


def ml_batch_device(images, kernels, outs, iterations, graph=True, stream=None,
                    persistent=False):
    """clarityx_ml_batch_device: Richardson-Lucy on lists of device tensors
    (volumes of any sizes, one kernel each), run concurrently; with graph the
    batch is captured into a CUDA graph and replayed on later identical
    calls; with persistent the iterations of all volumes run in one
    persistent launch over a shared work queue.  Asynchronous on
    `stream`."""
    n = len(images)
    if len(kernels) != n or len(outs) != n:
        raise ValueError("images, kernels and outs must have the same length")
    for t in list(images) + list(kernels) + list(outs):
        if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
            raise ValueError("batch volumes must be contiguous float32 CUDA tensors")
    vp = C.c_void_p
    imgs = (vp * n)(*[t.data_ptr() for t in images])
    kers = (vp * n)(*[t.data_ptr() for t in kernels])
    outp = (vp * n)(*[t.data_ptr() for t in outs])
    ids = (Dim3 * n)(*[dim3(t) for t in images])
    kds = (Dim3 * n)(*[dim3(t) for t in kernels])
    _check(load().clarityx_ml_batch_device(n, imgs, ids, kers, kds, outp, int(iterations),
                                           (BATCH_GRAPH if graph else 0) |
                                           (BATCH_PERSISTENT if persistent else 0),
                                           _stream_ptr(stream)))
    return outs


def set_dft_precision(mode: int) -> None:
    """clarityx_set_dft_precision: 0 FP32 register passes (default), 1 the
    split hi+lo FP16 tensor-core first z stage, 2 the same in BF16."""
    _check(load().clarityx_set_dft_precision(int(mode)))


def dft_precision() -> int:
    return int(load().clarityx_dft_precision())


def autotune(on: bool = True) -> None:
    """clarityx_autotune: time candidate plans on first use of a work box."""
    load().clarityx_autotune(1 if on else 0)


def ml_ex_device(image, kernel, out, iterations, start=None, idiv=None, stream=None):
    """clarityx_ml_ex_device: RL from `start` (an image-shaped device tensor;
    None: the image) with an optional I-divergence trace into `idiv` (a float64
    device tensor of `iterations` + 1 entries: the estimate at the start of each
    iteration, then the result)."""
    for t in (image, kernel, out) + ((start,) if start is not None else ()):
        if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
            raise ValueError("device variants need contiguous float32 CUDA tensors")
    if start is not None and tuple(start.shape) != tuple(image.shape):
        raise ValueError("start must have the image's shape")
    if idiv is not None and not (idiv.is_cuda and str(idiv.dtype) == "torch.float64"
                                 and idiv.numel() >= max(int(iterations), 0) + 1):
        raise ValueError("idiv must be a float64 CUDA tensor of `iterations` + 1 entries")
    vp = C.c_void_p
    _check(load().clarityx_ml_ex_device(
        vp(image.data_ptr()), dim3(image), vp(kernel.data_ptr()), dim3(kernel),
        vp(start.data_ptr()) if start is not None else None, vp(out.data_ptr()),
        int(iterations), vp(idiv.data_ptr()) if idiv is not None else None,
        _stream_ptr(stream)))
    return out


def ml_accel_device(image, kernel, out, iterations, idiv=None, stream=None, start=None):
    """clarityx_ml_accel_device: accelerated RL (Biggs-Andrews extrapolation)
    from `start` (None: the image) with an optional I-divergence trace
    (`iterations` + 1 float64 entries)."""
    if start is not None and tuple(start.shape) != tuple(image.shape):
        raise ValueError("start must have the image's shape")
    for t in (image, kernel, out) + ((start,) if start is not None else ()):
        if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
            raise ValueError("device variants need contiguous float32 CUDA tensors")
    if idiv is not None and not (idiv.is_cuda and str(idiv.dtype) == "torch.float64"
                                 and idiv.numel() >= max(int(iterations), 0) + 1):
        raise ValueError("idiv must be a float64 CUDA tensor of `iterations` + 1 entries")
    vp = C.c_void_p
    _check(load().clarityx_ml_accel_device(
        vp(image.data_ptr()), dim3(image), vp(kernel.data_ptr()), dim3(kernel),
        vp(start.data_ptr()) if start is not None else None,
        vp(out.data_ptr()), int(iterations), vp(idiv.data_ptr()) if idiv is not None else None,
        _stream_ptr(stream)))
    return out


def ml_learned_device(image, kernel, params, out, pre, post, idiv=None, stream=None):
    """clarityx_ml_learned_device: RL `pre` iterations, the learned-start
    network's prediction (FP32 parameter tensor `params` on the device), RL
    resumed for `post` iterations (optional float64 trace of post + 1
    entries)."""
    for t in (image, kernel, out, params):
        if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
            raise ValueError("device variants need contiguous float32 CUDA tensors")
    if idiv is not None and not (idiv.is_cuda and str(idiv.dtype) == "torch.float64"
                                 and idiv.numel() >= max(int(post), 0) + 1):
        raise ValueError("idiv must be a float64 CUDA tensor of `post` + 1 entries")
    vp = C.c_void_p
    _check(load().clarityx_ml_learned_device(
        vp(image.data_ptr()), dim3(image), vp(kernel.data_ptr()), dim3(kernel),
        vp(params.data_ptr()), params.numel(), int(pre), vp(out.data_ptr()), int(post),
        vp(idiv.data_ptr()) if idiv is not None else None, _stream_ptr(stream)))
    return out


def nn_predict(params, x, out, stream=None):
    """clarityx_nn_predict: the learned-start network's advanced estimate
    from the volume x (domain transforms fused into its first and last
    kernels)."""
    for t in (params, x, out):
        if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
            raise ValueError("nn_predict needs contiguous float32 CUDA tensors")
    vp = C.c_void_p
    _check(load().clarityx_nn_predict(vp(params.data_ptr()), params.numel(), vp(x.data_ptr()),
                                      dim3(x), vp(out.data_ptr()), _stream_ptr(stream)))
    return out


def nn_param_count() -> int:
    return int(load().clarityx_nn_param_count())


def maximum_likelihood_deconvolve_u16(image, kernel, iterations: int) -> np.ndarray:
    """clarityx_ml_u16: RL on uint16 volumes (casts on the device), as the
    reference's DeconvolveRawImages app around Clarity_MaximumLikelihoodDeconvolve."""
    image = np.ascontiguousarray(image, np.uint16)
    kernel = np.ascontiguousarray(kernel, np.uint16)
    out = np.empty_like(image)
    _check(load().clarityx_ml_u16(image, dim3(image), kernel, dim3(kernel), out, int(iterations)))
    return out


def idiv_deconvolve_device(image, kernel, out, iterations, alpha=0.0, stream=None):
    """clarityx_idiv_deconvolve_device: I-divergence restoration
    (Markham-Conchello conjugate gradients on s = a^2)."""
    return _dev("clarityx_idiv_deconvolve_device", image, kernel, out,
                [int(iterations), C.c_float(float(alpha))], stream)


def blind_ml_psf_device(image, kernel, out, iterations, psf_subiterations=5, psf_out=None,
                        stream=None):
    """clarityx_blind_ml_psf_device: blind ML alternating one object step and
    `psf_subiterations` PSF steps per iteration; psf_out (kernel-shaped) gets
    the PSF estimate."""
    for t in (image, kernel, out) + ((psf_out,) if psf_out is not None else ()):
        if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
            raise ValueError("device variants need contiguous float32 CUDA tensors")
    vp = C.c_void_p
    _check(load().clarityx_blind_ml_psf_device(
        vp(image.data_ptr()), dim3(image), vp(kernel.data_ptr()), dim3(kernel), vp(out.data_ptr()),
        vp(psf_out.data_ptr()) if psf_out is not None else None, int(iterations),
        int(psf_subiterations), _stream_ptr(stream)))
    return out
