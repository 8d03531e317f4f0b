"""CPU tests of the C ABI library: it loads without a GPU, exports every declared entry point,
rejects bad arguments, and its host-side initialisers are exact."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from openphase_b200 import _lib, initializations as init
from openphase_b200._lib import Grid, lib

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "opgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(opgpu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = lib()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing
    # the Python binding knows every one of them
    assert set(names) <= set(_lib._SIGS)


def test_abi_version_and_device_query():
    assert lib().opgpu_abi_version() == 2
    assert lib().opgpu_device_count() >= 0


def test_create_rejects_bad_grids_and_missing_device():
    L = lib()
    h = C.c_void_p()
    bad = Grid(nx=2, ny=8, nz=8, dx=1.0, iwidth=5.0, laplacian_stencil=2, gradient_stencil=1, precision=0,
               k_slots=8, device=0)
    assert L.opgpu_create(C.byref(bad), C.byref(h)) == _lib.E_INVALID
    bad_k = Grid(nx=8, ny=8, nz=8, dx=1.0, iwidth=5.0, laplacian_stencil=2, gradient_stencil=1, precision=0,
                 k_slots=7, device=0)
    assert L.opgpu_create(C.byref(bad_k), C.byref(h)) == _lib.E_INVALID
    if L.opgpu_device_count() == 0:
        good = Grid(nx=8, ny=8, nz=8, dx=1.0, iwidth=5.0, laplacian_stencil=2, gradient_stencil=1, precision=0,
                    k_slots=8, device=0)
        assert L.opgpu_create(C.byref(good), C.byref(h)) == _lib.E_NODEVICE
    assert L.opgpu_destroy(None) == 0


def _splitmix64(x):
    M = (1 << 64) - 1
    z = (x + 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def test_uniform_is_splitmix64_keyed():
    M = (1 << 64) - 1
    for seed, stream, a, b in [(1, 1, 0, 0), (2, 2, 17, 1999), (123456789, 3, 5, 0), (5, 1, 19999, 2)]:
        h = _splitmix64(seed ^ ((stream * 0xD1B54A32D192ED03) & M))
        h = _splitmix64(h ^ a)
        h = _splitmix64(h ^ ((b * 0x8CB92BA72F3D8DD7) & M))
        assert init.uniform(seed, stream, a, b) == (h >> 11) * 2.0 ** -53


def test_voronoi_owner_is_brute_force_argmin():
    nx, ny, nz, G, seed = 20, 17, 13, 25, 3
    own = init.voronoi_owner(nx, ny, nz, G, seed)
    pos = np.array([[min(int(init.uniform(seed, 1, g, a) * n), n - 1) for a, n in enumerate((nx, ny, nz))]
                    for g in range(G)])
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    best = np.full(X.shape, 1 << 60)
    arg = np.zeros(X.shape, int)
    for g in range(G):
        d = [np.minimum(np.abs(A - p), n - np.abs(A - p)) for A, p, n in zip((X, Y, Z), pos[g], (nx, ny, nz))]
        dd = d[0] ** 2 + d[1] ** 2 + d[2] ** 2
        m = dd < best
        best[m] = dd[m]
        arg[m] = g
    assert np.array_equal(arg.ravel(), own)


def test_spread_boundaries_lists():
    nx, ny, nz = 6, 5, 4
    rng = np.random.default_rng(0)
    owner = rng.integers(0, 4, size=nx * ny * nz).astype(np.int32)
    counts, idx, val = init.spread_boundaries(nx, ny, nz, owner)
    own3 = owner.reshape(nx, ny, nz)
    off = 0
    for v in range(nx * ny * nz):
        i, j, k = np.unravel_index(v, (nx, ny, nz))
        expect = [int(own3[i, j, k])]
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for dk in (-1, 0, 1):
                    g = int(own3[(i + di) % nx, (j + dj) % ny, (k + dk) % nz])
                    if g not in expect:
                        expect.append(g)
        assert list(idx[off:off + counts[v]]) == expect
        off += counts[v]
    assert np.all(val == 1.0)


def test_pair_table_and_driving_forces():
    t = init.sigma_table(50, 7, 0.8, 0.4)
    assert np.array_equal(t, t.T)
    assert t.min() >= 0.8 and t.max() < 1.2
    assert t[3, 41] == 0.8 + 0.4 * init.uniform(7, init.STREAM_SIGMA, 3, 41)
    d = init.driving_forces(30, 7, 0.05)
    assert d[11] == 0.05 * init.uniform(7, init.STREAM_DRIVING_FORCE, 11, 0)


def test_raw_format_round_trip(tmp_path):
    counts = np.array([1, 2, 0, 3], dtype=np.int32)
    idx = np.array([4, 1, 2, 7, 8, 9], dtype=np.int32)
    val = np.array([1.0, 0.25, 0.75, 0.1, 0.2, 0.7])
    data = init.raw_bytes(1, 2, 2, counts, idx, val)
    # layout of PhaseField::Write: 3 x int32, then per voxel u64 count and (u64 index, f64 value)
    assert len(data) == 12 + 8 * (4 + 2 * 6)
    dims, c2, i2, v2 = init.parse_raw(data)
    assert dims == (1, 2, 2)
    assert np.array_equal(c2, counts) and np.array_equal(i2, idx) and np.array_equal(v2, val)


def test_cxx_mirror_compiles_and_links(tmp_path):
    """The C++ mirror of the reference classes (include/opgpu.hpp) builds into a NormalGG-shaped
    caller linked against the in-tree library."""
    from tests.cxx_build import build_normal_gg
    exe = build_normal_gg(tmp_path)
    assert exe.exists()
