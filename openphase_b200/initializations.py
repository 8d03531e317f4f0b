"""Seeded initial states and parameter tables (the counterpart of the reference's Initializations
module, src/Initializations.cpp).

All values come from the counter-based generator of the C library (opgpu_uniform: SplitMix64 over
(seed, stream, a, b)), so the states are reproducible bit for bit anywhere.

* voronoi(...)       periodic Voronoi grains with spread grain boundaries (ragged lists)
* sigma_table(...)   symmetric per-grain-pair interface energies lo + span*u
* driving_forces(...) per-grain stored-energy driving forces scale*u
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import OpgpuError, lib, ptr

STREAM_POSITION = 1
STREAM_SIGMA = 2
STREAM_DRIVING_FORCE = 3


def uniform(seed: int, stream: int, a: int, b: int) -> float:
    return float(lib().opgpu_uniform(seed, stream, a, b))


def voronoi_owner(nx: int, ny: int, nz: int, ngrains: int, seed: int, threads: int = 0) -> np.ndarray:
    owner = np.empty(nx * ny * nz, dtype=np.int32)
    rc = lib().opgpu_voronoi_owner_host(nx, ny, nz, ngrains, seed, threads, ptr(owner))
    if rc:
        raise OpgpuError(rc, "voronoi_owner")
    return owner


def spread_boundaries(nx: int, ny: int, nz: int, owner: np.ndarray, threads: int = 0):
    """Ragged lists (counts, idx, val) of an owner map with spread grain boundaries."""
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    counts = np.empty(nx * ny * nz, dtype=np.int32)
    total = C.c_int64(0)
    L = lib()
    rc = L.opgpu_spread_boundaries_host(nx, ny, nz, ptr(owner), threads, ptr(counts), None, C.byref(total))
    if rc:
        raise OpgpuError(rc, "spread_boundaries")
    idx = np.empty(total.value, dtype=np.int32)
    rc = L.opgpu_spread_boundaries_host(nx, ny, nz, ptr(owner), threads, ptr(counts), ptr(idx), C.byref(total))
    if rc:
        raise OpgpuError(rc, "spread_boundaries")
    val = np.ones(total.value, dtype=np.float64)
    return counts, idx, val


def voronoi(nx: int, ny: int, nz: int, ngrains: int, seed: int, threads: int = 0):
    """Seeded periodic Voronoi state as ragged lists (counts, idx, val)."""
    return spread_boundaries(nx, ny, nz, voronoi_owner(nx, ny, nz, ngrains, seed, threads), threads)


def sigma_table(ngrains: int, seed: int, lo: float = 0.8, span: float = 0.4) -> np.ndarray:
    """Symmetric G x G table sigma(a,b) = lo + span*u(seed, SIGMA, min, max); diagonal = lo."""
    t = np.empty((ngrains, ngrains), dtype=np.float64)
    rc = lib().opgpu_pair_table_host(ngrains, seed, STREAM_SIGMA, lo, span, ptr(t))
    if rc:
        raise OpgpuError(rc, "pair_table_host")
    return t


def driving_forces(ngrains: int, seed: int, scale: float) -> np.ndarray:
    """Per-grain stored-energy driving forces scale*u(seed, DRIVING_FORCE, g, 0)."""
    d = np.empty(ngrains, dtype=np.float64)
    rc = lib().opgpu_grain_values_host(ngrains, seed, STREAM_DRIVING_FORCE, scale, ptr(d))
    if rc:
        raise OpgpuError(rc, "grain_values_host")
    return d


def raw_bytes(nx: int, ny: int, nz: int, counts, idx, val) -> bytes:
    """Serialise ragged lists in the reference's raw PhaseField format (PhaseField::Write)."""
    counts = np.asarray(counts, dtype=np.int64)
    n = counts.size
    total = int(counts.sum())
    # per voxel: u64 count, then count x (u64 index, f64 value)
    words = np.empty(n + 2 * total, dtype=np.uint64)
    starts = np.zeros(n, dtype=np.int64)
    starts[1:] = np.cumsum(1 + 2 * counts[:-1])
    words[starts] = counts.astype(np.uint64)
    entry_pos = np.repeat(starts + 1, counts) + 2 * (np.arange(total) - np.repeat(np.cumsum(counts) - counts, counts))
    words[entry_pos] = np.asarray(idx, dtype=np.int64).astype(np.uint64)
    words[entry_pos + 1] = np.asarray(val, dtype=np.float64).view(np.uint64)
    return np.array([nx, ny, nz], dtype=np.int32).tobytes() + words.tobytes()


def parse_raw(data: bytes):
    """Parse a raw PhaseField file into (dims, counts, idx, val)."""
    nx, ny, nz = np.frombuffer(data[:12], dtype=np.int32)
    words = np.frombuffer(data[12:], dtype=np.uint64)
    n = int(nx) * int(ny) * int(nz)
    counts = np.empty(n, dtype=np.int32)
    pos = 0
    # counts are needed sequentially; walk with a vectorised jump table in chunks
    for v in range(n):
        c = int(words[pos])
        counts[v] = c
        pos += 1 + 2 * c
    if pos != words.size:
        raise ValueError("raw file size does not match its counts")
    starts = np.zeros(n, dtype=np.int64)
    starts[1:] = np.cumsum(1 + 2 * counts[:-1].astype(np.int64))
    total = int(counts.sum())
    entry_pos = np.repeat(starts + 1, counts) + 2 * (np.arange(total) - np.repeat(np.cumsum(counts) - counts, counts))
    idx = words[entry_pos].astype(np.int32)
    val = words[entry_pos + 1].view(np.float64).copy()
    return (int(nx), int(ny), int(nz)), counts, idx, val


STREAM_ORIENTATION = 5


def nucleus_centres(ngrains: int, nx: int, ny: int, nz: int, seed: int) -> np.ndarray:
    """Centres of nuclei 1..ngrains-1 (grain 0 is the matrix): u(seed, POSITION, g, axis)*n."""
    c = np.empty((ngrains, 3))
    for g in range(ngrains):
        for ax, n in enumerate((nx, ny, nz)):
            c[g, ax] = uniform(seed, STREAM_POSITION, g, ax) * n
    return c


def nuclei(nx: int, ny: int, nz: int, ngrains: int, seed: int, radius: float, iwidth: float):
    """Grain 0 fills the box; grains 1..ngrains-1 are spheres of the given radius at seeded centres
    with the diffuse profile of Initializations::Sphere (src/Initializations.cpp:341-389): inside
    R - iWidth/2 the voxel holds only the sphere; out to R + iWidth/2 the sphere gets
    p = 0.5 - 0.5*sin(pi*(r - R)/iWidth) and the values already present are scaled by 1 - p.
    Distances are periodic minimum-image distances to the centre; nuclei are placed in index order.
    Returns ragged lists (counts, idx, val) (not normalised; finalize normalises)."""
    N = nx * ny * nz
    lists = [dict() for _ in range(N)]
    for v in range(N):
        lists[v][0] = 1.0
    centres = nucleus_centres(ngrains, nx, ny, nz, seed)
    reach = int(np.ceil(radius + 0.5 * iwidth)) + 1
    for g in range(1, ngrains):
        cx, cy, cz = centres[g]
        ix = np.arange(int(np.floor(cx)) - reach, int(np.floor(cx)) + reach + 2)
        iy = np.arange(int(np.floor(cy)) - reach, int(np.floor(cy)) + reach + 2)
        iz = np.arange(int(np.floor(cz)) - reach, int(np.floor(cz)) + reach + 2)
        seen = set()
        for i in ix:
            for j in iy:
                for k in iz:
                    v = ((i % nx) * ny + (j % ny)) * nz + (k % nz)
                    if v in seen:
                        continue
                    seen.add(v)
                    dx = min(abs(i % nx - cx), nx - abs(i % nx - cx))
                    dy = min(abs(j % ny - cy), ny - abs(j % ny - cy))
                    dz = min(abs(k % nz - cz), nz - abs(k % nz - cz))
                    rad = float(np.sqrt(dx * dx + dy * dy + dz * dz))
                    if rad < radius - 0.5 * iwidth:
                        lists[v] = {g: 1.0}
                    elif rad <= radius + 0.5 * iwidth:
                        prof = 0.5 - 0.5 * np.sin(np.pi * (rad - radius) / iwidth)
                        for key in lists[v]:
                            lists[v][key] *= 1.0 - prof
                        lists[v][g] = prof
    counts = np.array([len(d) for d in lists], dtype=np.int32)
    idx = np.fromiter((k for d in lists for k in d), dtype=np.int32, count=int(counts.sum()))
    val = np.fromiter((x for d in lists for x in d.values()), dtype=np.float64, count=int(counts.sum()))
    return counts, idx, val


def small_rotations(ngrains: int, seed: int, spread: float) -> np.ndarray:
    """Unit quaternions (s, x, y, z) of rotations by an angle uniform in [0, spread) about axes
    uniform on the sphere: orientations whose pairwise disorientations are mostly small."""
    q = np.empty((ngrains, 4))
    for g in range(ngrains):
        u1, u2, u3 = (uniform(seed, STREAM_ORIENTATION, g, k) for k in range(3))
        cz = 2.0 * u1 - 1.0
        r = np.sqrt(max(0.0, 1.0 - cz * cz))
        axis = (r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2), cz)
        half = 0.5 * spread * u3
        q[g] = (np.cos(half), axis[0] * np.sin(half), axis[1] * np.sin(half), axis[2] * np.sin(half))
    return q


def quaternions(ngrains: int, seed: int) -> np.ndarray:
    """Uniform random unit quaternions (s, x, y, z) per grain by Shoemake's method (Graphics Gems
    III, 1992): u1, u2, u3 uniform; q = (sqrt(1-u1) sin 2pi u2, sqrt(1-u1) cos 2pi u2,
    sqrt(u1) sin 2pi u3, sqrt(u1) cos 2pi u3)."""
    q = np.empty((ngrains, 4))
    for g in range(ngrains):
        u1, u2, u3 = (uniform(seed, STREAM_ORIENTATION, g, k) for k in range(3))
        a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
        x, y = a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2)
        z, w = b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)
        q[g] = (w, x, y, z)
    return q


def write_vtk(path, nx: int, ny: int, nz: int, counts, idx, val, grain_phase=None, nphases: int = 1,
              stencil: str = "LB", gradient_stencil: str = "ISOTROPIC"):
    """PhaseField::WriteVTK of ragged host lists (no device needed; opgpu_write_vtk_host)."""
    from ._lib import STENCIL
    c = np.ascontiguousarray(counts, dtype=np.int32)
    i = np.ascontiguousarray(idx, dtype=np.int32)
    v = np.ascontiguousarray(val, dtype=np.float64)
    ngrains = int(i.max()) + 1 if i.size else 1
    gp = None
    if grain_phase is not None:
        gp = np.ascontiguousarray(grain_phase, dtype=np.int32)
        ngrains = gp.size
    rc = lib().opgpu_write_vtk_host(nx, ny, nz, ptr(c), ptr(i), ptr(v), ngrains, ptr(gp), nphases,
                                    STENCIL[stencil], STENCIL[gradient_stencil], str(path).encode())
    if rc:
        raise OpgpuError(rc, "write_vtk_host")
