"""Output files against the reference's own (no device needed).

The fixtures under tests/golden/ (made by tests/golden/make_golden.py from the compiled reference)
hold a reference state and the files the reference wrote for it: PhaseField::WriteVTK's .vts and the
GrainsProperties restart file.  opgpu_write_vtk_host, given the same state (its stored, positive
entries), must write the same bytes; the grain-record layout read here must reproduce the
reference's volumes.
"""
import struct
from pathlib import Path

import numpy as np
import pytest

from openphase_b200.initializations import write_vtk
from oracle.bridge import positive_entries
from tests.golden.make_golden import OUTPUT_CASES

GOLDEN = Path(__file__).resolve().parent / "golden"

# Grain::Write (include/GrainsProperties.h:197-231): Exist, Mobile (bool), Stage (int), Parent, Phase,
# Variant (size_t), State (int), Density, RefVolume, Volume, MAXVolume, 30 motion doubles, quaternion
GRAIN_RECORD = struct.Struct("<??iQQQi4d30d4d")


def parse_grains_file(data: bytes):
    (size,) = struct.unpack_from("<Q", data, 0)
    assert len(data) == 8 + size * GRAIN_RECORD.size
    out = []
    for g in range(size):
        f = GRAIN_RECORD.unpack_from(data, 8 + g * GRAIN_RECORD.size)
        out.append({"exist": f[0], "mobile": f[1], "stage": f[2], "parent": f[3], "phase": f[4], "variant": f[5],
                    "state": f[6], "density": f[7], "ref_volume": f[8], "volume": f[9], "max_volume": f[10],
                    "quat": f[41:45]})
    return out


@pytest.mark.parametrize("name", list(OUTPUT_CASES))
def test_vtk_writer_matches_reference_bytes(name, tmp_path):
    case, step = OUTPUT_CASES[name]
    z = np.load(GOLDEN / f"{name}.npz")
    counts, idx, val = positive_entries(z["counts"].astype(np.int32), z["idx"].astype(np.int32), z["val"])
    out = tmp_path / "pf.vts"
    write_vtk(out, case.nx, case.ny, case.nz, counts, idx, val, grain_phase=case.grain_phase(),
              nphases=case.nphases, stencil=case.stencil, gradient_stencil=case.gradient_stencil)
    ours = out.read_bytes()
    ref = z["vtk"].tobytes()
    if ours != ref:
        a, b = ours.decode().splitlines(), ref.decode().splitlines()
        first = next((i for i, (x, y) in enumerate(zip(a, b)) if x != y), min(len(a), len(b)))
        pytest.fail(f"{name}: first differing line {first}: ours {a[first:first + 2]} reference {b[first:first + 2]}")


@pytest.mark.parametrize("name", list(OUTPUT_CASES))
def test_grain_file_layout_matches_reference(name):
    """The record layout the library writes and reads (opgpu_write_grains / opgpu_read_grains)
    parses the reference's file into its own volumes and volume ratios."""
    case, step = OUTPUT_CASES[name]
    z = np.load(GOLDEN / f"{name}.npz")
    grains = parse_grains_file(z["grains_file"].tobytes())
    assert len(grains) == case.ngrains
    vol = np.array([g["volume"] for g in grains])
    ratio = np.array([min(1.0, g["max_volume"] / g["ref_volume"]) if g["exist"] else 1.0 for g in grains])
    assert np.array_equal(vol, z["volume"])
    assert np.allclose(ratio, z["volume_ratio"], rtol=0, atol=1e-15)
    assert all(g["phase"] == p for g, p in zip(grains, case.grain_phase()))
    # the defaults the library writes for what it does not model
    assert all(g["mobile"] and g["parent"] == 0 and g["variant"] == 0 for g in grains)
