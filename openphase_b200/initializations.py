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
