"""Build the opgpu shared library (CUDA kernels for sm_100a + C ABI) in-tree.

    python -m openphase_b200.build_ext            # builds openphase_b200/lib/libopgpu.so

Every .cu translation unit is compiled by nvcc for sm_100a only; step_f64.cu, step_f32.cu and
adjoint.cu additionally with --fmad=false (the FP64 form reproduces the reference's unfused double
arithmetic; the adjoint repeats the forward's per-voxel arithmetic of either form exactly).  The host-side
initialisers are compiled by the system g++ with OpenMP.  Objects go to openphase_b200/_build/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libopgpu.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "-I", str(INCLUDE),
               "-I", str(CSRC), "--expt-relaxed-constexpr"]
CU_UNITS = {
    "opgpu.cu": [],
    "step_f64.cu": ["--fmad=false"],
    "step_f32.cu": ["--fmad=false"],
    "adjoint.cu": ["--fmad=false"],
    "average.cu": ["--fmad=false"],
}
CPP_UNITS = ["host_init.cpp"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _env():
    env = dict(os.environ)
    # some images point CC/CXX at a compiler without OpenMP support files; use the system ones
    env.pop("CC", None)
    env.pop("CXX", None)
    return env


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, env=_env())


def source_hash() -> str:
    """SHA-256 (first 16 hex digits) over the library's sources, headers and compile flags: the
    build stamp the library reports through opgpu_build_info()."""
    import hashlib
    h = hashlib.sha256()
    files = sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp"), *CSRC.glob("*.h"), *CSRC.glob("*.cuh"),
                    *INCLUDE.glob("*.h")], key=lambda f: f.name)
    for f in files:
        h.update(f.name.encode())
        h.update(f.read_bytes())
    h.update(repr((ARCH, [x for x in NVCC_COMMON if not x.startswith("/")], CU_UNITS)).encode())
    return h.hexdigest()[:16]


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    stamp = source_hash()
    # the stamp is compiled into opgpu.cu; rebuild it when the stamp changes
    stamp_file = BUILD / "source_hash.txt"
    if not stamp_file.exists() or stamp_file.read_text() != stamp:
        stamp_file.write_text(stamp)
        hdrs = hdrs + [stamp_file]
    objs = []
    jobs = []
    for unit, extra in CU_UNITS.items():
        src = CSRC / unit
        obj = BUILD / (unit + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *hdrs]):
            jobs.append([nvcc, *ARCH, *NVCC_COMMON, *extra, f"-DOPGPU_SOURCE_HASH=\"{stamp}\"", "-c", str(src),
                         "-o", str(obj)])
    for unit in CPP_UNITS:
        src = CSRC / unit
        obj = BUILD / (unit + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *hdrs]):
            jobs.append(["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I", str(INCLUDE), "-I", str(CSRC),
                         "-c", str(src), "-o", str(obj)])
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, env=_env())))
    for cmd, p in procs:
        if p.wait() != 0:
            raise RuntimeError("build failed: " + " ".join(cmd))
    if force or jobs or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static",
              "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
