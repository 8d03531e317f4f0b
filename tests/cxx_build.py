"""Compile tests/cxx/normal_gg.cpp against include/opgpu.hpp and the in-tree libopgpu.so."""
from __future__ import annotations

import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cxx" / "normal_gg.cpp"
LIBDIR = ROOT / "openphase_b200" / "lib"


def build_normal_gg(out_dir: Path) -> Path:
    exe = Path(out_dir) / "normal_gg"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
           "-L", str(LIBDIR), "-lopgpu", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe
