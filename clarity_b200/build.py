"""Build libclarity.so in-tree with nvcc for sm_100a.

    python -m clarity_b200.build [--force] [--jobs N]

Every .cu/.cpp file in csrc/ is compiled to an object under _build/obj
(in parallel), then linked into clarity_b200/libclarity.so with the CUDA
runtime linked statically, so the library needs nothing from PyTorch.
A file is rebuilt when it or any header in csrc/ or include/ is newer than
its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "libclarity.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++20", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-fvisibility=hidden", "-diag-suppress", "177,550"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[str]:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return hs


def _stale(src: str, obj: str, newest_header: float) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or newest_header > t


def _compile(src: str, obj: str, extra: list[str]) -> tuple[str, int, str]:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    return src, p.returncode, p.stdout + p.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False,
          ptxas_info: bool = False, defines: list[str] | None = None,
          lib: str = LIB, obj_dir: str = OBJ) -> str:
    """Compile and link.  `defines` adds -D flags (build variants); a variant
    should use its own `lib` and `obj_dir`."""
    os.makedirs(obj_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    newest = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(obj_dir, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(s, o, newest):
            todo.append((s, o))
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    extra += [f"-D{d}" for d in (defines or [])]
    if todo:
        jobs = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(_compile, s, o, extra) for s, o in todo]
            failed = []
            for f in cf.as_completed(futs):
                src, rc, out = f.result()
                if verbose or rc != 0 or ptxas_info:
                    sys.stderr.write(f"== {os.path.basename(src)} (rc={rc})\n{out}\n")
                if rc != 0:
                    failed.append(src)
            if failed:
                raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    if todo or not os.path.exists(lib):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart", "static",
               "-o", lib, *objs]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stdout + p.stderr)
    if lib == LIB:
        build_apps(lib)
    return lib


def build_apps(lib: str = LIB) -> list[str]:
    """The example applications (apps/*.cpp), linked against libclarity.so."""
    out_dir = os.path.join(PKG, "bin")
    os.makedirs(out_dir, exist_ok=True)
    built = []
    for src in sorted(glob.glob(os.path.join(PKG, "apps", "*.cpp"))):
        exe = os.path.join(out_dir, os.path.splitext(os.path.basename(src))[0])
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(src),
                                                                 os.path.getmtime(lib)):
            built.append(exe)
            continue
        cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
               src, "-o", exe, "-L", PKG, "-lclarity", "-Wl,-rpath,$ORIGIN/.."]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("app build failed:\n" + p.stdout + p.stderr)
        built.append(exe)
    return built


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("-D", dest="defines", action="append", default=[],
                    help="extra preprocessor definition (build variant)")
    ap.add_argument("--lib", default=LIB, help="output library path")
    ap.add_argument("--obj-dir", default=OBJ, help="object directory")
    a = ap.parse_args()
    print(build(a.force, a.jobs, a.verbose, a.ptxas_info, a.defines, a.lib, a.obj_dir))


if __name__ == "__main__":
    main()
