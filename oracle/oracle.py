"""TEST INFRASTRUCTURE ONLY (oracle).

ctypes access to the two CPU checkers built by ``oracle/Makefile``:

* ``_build/liboracle.so`` -- this project's restatement of the reference path
  (``clarity_oracle.cpp``), in float (parity target) and double (the FP64
  oracle every error is stated against).
* ``_ref/liboracle_ref.so`` and ``_ref/liboracle_ref_fp64sum.so`` -- the
  unmodified reference CPU sources linked with the project's FFTW-API shim,
  called through the reference's own public C API (``Clarity_*``).  These
  exist only where the reference sources were present at build time.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (CPU baseline and
the reference arm) import this module.  The product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = {
    "ref": os.path.join(HERE, "_ref", "liboracle_ref.so"),
    "ref_fp64sum": os.path.join(HERE, "_ref", "liboracle_ref_fp64sum.so"),
}
# The reference source tree the checker builds from: CLARITY_REFERENCE_DIR,
# or the `reference_dir` argument of build().  Nothing at run time reads it.
REFERENCE_DIR = os.environ.get("CLARITY_REFERENCE_DIR", "")

SUM_SERIAL_FLOAT = 0
SUM_DOUBLE = 1

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(with_reference: bool | None = None, reference_dir: str | None = None) -> None:
    """Compile the oracle and, when the reference sources are given and
    present, _ref (the reference build, its test programs and app) and the
    drop-in builds of those programs against libclarity.so (build the library
    first)."""
    ref = reference_dir if reference_dir is not None else REFERENCE_DIR
    if with_reference is None:
        with_reference = bool(ref) and os.path.isdir(os.path.join(ref, "src"))
    targets = ["oracle"] + (["ref", "dropin"] if with_reference else [])
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref}", *targets], check=True)


class _Dim3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


def _dims(a: np.ndarray) -> tuple[int, int, int]:
    """numpy (z, y, x) shape -> Clarity (x, y, z)."""
    z, y, x = a.shape
    return x, y, z


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class Oracle:
    """The project's CPU restatement (float and double)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(with_reference=False)
        self.lib = C.CDLL(path)
        L = self.lib
        i = C.c_int
        for name, extra in [("convolve", []), ("rl", [i, i]),
                            ("wiener", [C.c_float]), ("jvc", [i]),
                            ("sjvc", [i, i, C.c_double, C.c_double, C.c_double]),
                            ("blind", [i, i])]:
            fn = getattr(L, f"oracle_{name}_f32")
            fn.argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p] + extra + [C.c_void_p]
            fn.restype = None
            fn64 = getattr(L, f"oracle_{name}_f64")
            extra64 = [C.c_double if e is C.c_float else e for e in extra]
            if name in ("rl", "blind"):
                extra64 = [i]  # no sum mode: always double
            fn64.argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p] + extra64 + [C.c_void_p]
            fn64.restype = None
        for p in ("f32", "f64"):
            getattr(L, f"oracle_correlate_{p}").argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p]
            getattr(L, f"oracle_rl_corr_{p}").argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p,
                                                         i]
        L.oracle_rl_ex_f32.argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p, i, i,
                                       C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_rl_ex_f32.restype = None
        L.oracle_rl_ex_f64.argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p, i,
                                       C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_rl_ex_f64.restype = None
        L.oracle_rl_accel_f32.argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p, i, i,
                                          C.c_void_p]
        L.oracle_rl_accel_f32.restype = None
        L.oracle_rl_accel_f64.argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p, i,
                                          C.c_void_p]
        L.oracle_rl_accel_f64.restype = None
        for pr in ("f32", "f64"):
            fn = getattr(L, f"oracle_blind_psf_{pr}")
            fn.argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p, _f32p, i, i]
            fn.restype = None
        for p in ("f32", "f64"):
            getattr(L, f"oracle_idiv_cg_{p}").argtypes = [_f32p, i, i, i, _f32p, i, i, i, _f32p,
                                                         i, C.c_double]
        L.oracle_idivergence.argtypes = [_f32p, _f32p, C.c_long, C.POINTER(C.c_long)]
        L.oracle_idivergence.restype = C.c_double
        L.oracle_pad_shift.argtypes = [_f32p, i, i, i, _f32p, i, i, i,
                                       C.POINTER(C.c_int), C.c_float]
        for p, T in (("f32", _f32p), ("f64", _f64p)):
            getattr(L, f"oracle_r2c_3d_{p}").argtypes = [i, i, i, T, T]
            getattr(L, f"oracle_c2r_3d_{p}").argtypes = [i, i, i, T, T]
        L.oracle_set_threads.argtypes = [i]

    def set_threads(self, n: int) -> None:
        self.lib.oracle_set_threads(int(n))

    def _run(self, name, img, psf, extra, precision="f32", work=False):
        img, psf = _f32(img), _f32(psf)
        out = np.empty_like(img)
        ix, iy, iz = _dims(img)
        kx, ky, kz = _dims(psf)
        wshape = (iz + kz, iy + ky, ix + kx)
        wdt = np.float32 if precision == "f32" else np.float64
        w = np.empty(wshape, dtype=wdt) if work else None
        fn = getattr(self.lib, f"oracle_{name}_{precision}")
        fn(img, ix, iy, iz, psf, kx, ky, kz, out, *extra,
           w.ctypes.data if work else None)
        return (out, w) if work else out

    def convolve(self, img, psf, precision="f32", work=False):
        return self._run("convolve", img, psf, [], precision, work)

    def correlate(self, img, psf, precision="f32"):
        """Circular correlation: Clarity_Convolve with the kernel's spectrum
        conjugated (the library's opt-in; no reference counterpart)."""
        img, psf = _f32(img), _f32(psf)
        out = np.empty_like(img)
        getattr(self.lib, f"oracle_correlate_{precision}")(img, *_dims(img), psf, *_dims(psf),
                                                           out)
        return out

    def rl_correlate(self, img, psf, iters, precision="f32"):
        """RL whose second convolution per iteration is a correlation with
        the kernel (conjugated OTF), double flux sums."""
        img, psf = _f32(img), _f32(psf)
        out = np.empty_like(img)
        getattr(self.lib, f"oracle_rl_corr_{precision}")(img, *_dims(img), psf, *_dims(psf), out,
                                                         int(iters))
        return out

    def rl(self, img, psf, iters, precision="f32", sum_mode=SUM_DOUBLE, work=False):
        extra = [iters, sum_mode] if precision == "f32" else [iters]
        return self._run("rl", img, psf, extra, precision, work)

    def rl_ex(self, img, psf, iters, start=None, precision="f32", sum_mode=SUM_DOUBLE):
        """RL from `start` (image-shaped; None: the image); returns (out, idiv
        trace of `iters` + 1 entries: per iteration start, then the result)."""
        img, psf = _f32(img), _f32(psf)
        out = np.empty_like(img)
        st = _f32(start) if start is not None else None
        tr = np.zeros(max(int(iters), 0) + 1, np.float64)
        ix, iy, iz = _dims(img)
        kx, ky, kz = _dims(psf)
        sp = st.ctypes.data if st is not None else None
        if precision == "f32":
            self.lib.oracle_rl_ex_f32(img, ix, iy, iz, psf, kx, ky, kz, out, int(iters),
                                      int(sum_mode), sp, tr.ctypes.data, None)
        else:
            self.lib.oracle_rl_ex_f64(img, ix, iy, iz, psf, kx, ky, kz, out, int(iters),
                                      sp, tr.ctypes.data, None)
        return out, tr

    def rl_accel(self, img, psf, iters, precision="f32", sum_mode=SUM_DOUBLE):
        """Accelerated RL (Biggs-Andrews); returns (out, idiv trace of
        `iters` + 1 entries: at each extrapolated point, then the result)."""
        img, psf = _f32(img), _f32(psf)
        out = np.empty_like(img)
        tr = np.zeros(max(int(iters), 0) + 1, np.float64)
        ix, iy, iz = _dims(img)
        kx, ky, kz = _dims(psf)
        if precision == "f32":
            self.lib.oracle_rl_accel_f32(img, ix, iy, iz, psf, kx, ky, kz, out, int(iters),
                                         int(sum_mode), tr.ctypes.data)
        else:
            self.lib.oracle_rl_accel_f64(img, ix, iy, iz, psf, kx, ky, kz, out, int(iters),
                                         tr.ctypes.data)
        return out, tr

    def blind_psf(self, img, psf, iters, sub, precision="f32"):
        """Blind ML with the PSF update: (object estimate, PSF estimate)."""
        img, psf = _f32(img), _f32(psf)
        out = np.empty_like(img)
        pout = np.empty_like(psf)
        ix, iy, iz = _dims(img)
        kx, ky, kz = _dims(psf)
        getattr(self.lib, f"oracle_blind_psf_{precision}")(img, ix, iy, iz, psf, kx, ky, kz, out,
                                                           pout, int(iters), int(sub))
        return out, pout

    def idiv_cg(self, img, psf, iters, alpha=0.0, precision="f32"):
        """I-divergence restoration (Markham-Conchello conjugate gradients on
        s = a^2); returns the estimate on the image region."""
        img, psf = _f32(img), _f32(psf)
        out = np.empty_like(img)
        ix, iy, iz = _dims(img)
        kx, ky, kz = _dims(psf)
        getattr(self.lib, f"oracle_idiv_cg_{precision}")(img, ix, iy, iz, psf, kx, ky, kz, out,
                                                         int(iters), float(alpha))
        return out

    def wiener(self, img, psf, eps, precision="f32", work=False):
        return self._run("wiener", img, psf, [eps], precision, work)

    def jvc(self, img, psf, iters, precision="f32", work=False):
        return self._run("jvc", img, psf, [iters], precision, work)

    def smoothed_jvc(self, img, psf, iters, interval, sigma_xyz, precision="f32", work=False):
        sx, sy, sz = (float(v) for v in sigma_xyz)
        return self._run("sjvc", img, psf, [iters, interval, sx, sy, sz], precision, work)

    def blind(self, img, psf, iters, precision="f32", sum_mode=SUM_DOUBLE, work=False):
        extra = [iters, sum_mode] if precision == "f32" else [iters]
        return self._run("blind", img, psf, extra, precision, work)

    def idivergence(self, g, ghat) -> float:
        g, ghat = _f32(g).ravel(), _f32(ghat).ravel()
        sk = C.c_long(0)
        v = self.lib.oracle_idivergence(g, ghat, g.size, C.byref(sk))
        return float(v)

    def pad_shift(self, src, dst_shape_zyx, shift_xyz, fill=0.0):
        src = _f32(src)
        dst = np.empty(dst_shape_zyx, dtype=np.float32)
        sh = (C.c_int * 3)(*shift_xyz)
        dz, dy, dx = dst_shape_zyx
        sx, sy, sz = _dims(src)
        self.lib.oracle_pad_shift(dst, dx, dy, dz, src, sx, sy, sz, sh, fill)
        return dst

    def r2c(self, a, precision="f32"):
        dt = np.float32 if precision == "f32" else np.float64
        a = np.ascontiguousarray(a, dtype=dt)
        nz, ny, nx = a.shape
        out = np.empty((nz, ny, nx // 2 + 1, 2), dtype=dt)
        getattr(self.lib, f"oracle_r2c_3d_{precision}")(nz, ny, nx, a, out)
        return out[..., 0] + 1j * out[..., 1]

    def c2r(self, spec, nx, precision="f32"):
        dt = np.float32 if precision == "f32" else np.float64
        s = np.ascontiguousarray(np.stack([spec.real, spec.imag], -1), dtype=dt)
        nz, ny, _ = spec.shape
        out = np.empty((nz, ny, nx), dtype=dt)
        getattr(self.lib, f"oracle_c2r_3d_{precision}")(nz, ny, nx, s, out)
        return out


class ReferenceCPU:
    """The unmodified reference CPU library, called through its C API."""

    def __init__(self, variant: str = "ref_fp64sum"):
        path = REF_SO[variant]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        d3 = _Dim3
        L.Clarity_Register.restype = C.c_int
        L.Clarity_UnRegister.restype = C.c_int
        L.Clarity_SetNumberOfThreads.argtypes = [C.c_uint]
        for name, extra in [("Clarity_Convolve", []),
                            ("Clarity_MaximumLikelihoodDeconvolve", [C.c_int]),
                            ("Clarity_BlindMaximumLikelihoodDeconvolve", [C.c_int]),
                            ("Clarity_JansenVanCittertDeconvolve", [C.c_int]),
                            ("Clarity_WienerDeconvolve", [C.c_float])]:
            fn = getattr(L, name)
            fn.argtypes = [_f32p, d3, _f32p, d3, _f32p] + extra
            fn.restype = C.c_int
        rc = L.Clarity_Register()
        assert rc == 5, rc

    @staticmethod
    def available(variant: str = "ref_fp64sum") -> bool:
        return os.path.exists(REF_SO[variant])

    def set_threads(self, n: int) -> None:
        self.lib.Clarity_SetNumberOfThreads(int(n))

    def _call(self, name, img, psf, *extra):
        img, psf = _f32(img), _f32(psf)
        out = np.zeros_like(img)
        rc = getattr(self.lib, name)(img, _Dim3(*_dims(img)), psf,
                                     _Dim3(*_dims(psf)), out, *extra)
        if rc != 5:
            raise RuntimeError(f"{name} returned {rc}")
        return out

    def convolve(self, img, psf):
        return self._call("Clarity_Convolve", img, psf)

    def rl(self, img, psf, iters):
        return self._call("Clarity_MaximumLikelihoodDeconvolve", img, psf, iters)

    def blind(self, img, psf, iters):
        return self._call("Clarity_BlindMaximumLikelihoodDeconvolve", img, psf, iters)

    def jvc(self, img, psf, iters):
        return self._call("Clarity_JansenVanCittertDeconvolve", img, psf, iters)

    def wiener(self, img, psf, eps):
        return self._call("Clarity_WienerDeconvolve", img, psf, float(eps))


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
