"""Restart files and VTK output of the CUDA path, against itself and against the reference.

* A restart (raw state + grain records, then finalize) continues like the run that wrote it: the
  same lists and max|dphi| <= 1e-9, grains below the reference volume included (their volumes,
  sums over the grid in an order the atomics decide, feed back at the last bit).
* The files interchange with the reference: the reference restarts from files this library wrote
  and continues like the GPU (the parity bar), and this library restarts from files the reference
  wrote.
* opgpu_write_vtk writes the reference's PhaseField::WriteVTK file byte for byte.
"""
import numpy as np
import pytest

from openphase_b200.cases import Case
from openphase_b200.context import Context
from oracle.bridge import parse_raw, positive_entries, reference_available, run_reference
from tests.parity import compare_states

pytestmark = pytest.mark.gpu
TOL = 1e-9
needs_ref = pytest.mark.skipif(not reference_available(), reason="reference build (oracle/_ref) not present")

SMALL = Case(24, 24, 24, 30, seed=7, iwidth=6.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4), dg_scale=0.05,
             name="restart_small_grains")
DRIVEN = Case(32, 28, 24, 12, seed=8, iwidth=5.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4), dg_scale=0.05,
              name="restart_driven")


def _grains_close(a, b, rel=1e-12):
    """Grain records of two contexts: exist and stage identical, volumes, MAXVolume and VolumeRatio
    within `rel` (the volumes are sums over the grid whose order the atomics decide)."""
    ga, gb = a.grains(), b.grains()
    diff = {k: float(np.max(np.abs(ga[k] - gb[k]) / np.maximum(np.abs(gb[k]), 1.0)))
            for k in ("volume", "max_volume", "volume_ratio")}
    same = np.array_equal(ga["exist"], gb["exist"]) and np.array_equal(ga["stage"], gb["stage"])
    return same and all(d <= rel for d in diff.values()), diff


def test_restart_continues_bit_for_bit(tmp_path):
    case = SMALL
    a = Context.from_case(case, precision="fp64", k_slots=16)
    a.step(case.dt, 20)
    raw, grains = tmp_path / "PhaseField_20.dat", tmp_path / "GrainsProperties_20.dat"
    a.write_restart(raw, grains)
    b = Context.from_case(case, precision="fp64", k_slots=16, restart=(raw, grains))
    ok, diff = _grains_close(a, b)
    assert ok, diff
    assert any(v < 1.0 for v in b.grains()["volume_ratio"])   # grains below the reference volume
    a.step(case.dt, 30)
    b.step(case.dt, 30)
    r = compare_states(a.download(), b.download(), case.ngrains)
    assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= TOL, r
    ok, diff = _grains_close(a, b)
    assert ok, diff


@needs_ref
def test_reference_restarts_from_our_files(tmp_path):
    """GPU: 10 steps, restart files; the reference restarts from them (PhaseField::Read + Finalize)
    and runs 20 steps; the GPU runs the same 20 steps: identical states."""
    case = DRIVEN
    ctx = Context.from_case(case, precision="fp64", k_slots=16)
    ctx.step(case.dt, 10)
    raw, grains = tmp_path / "PhaseField_10.dat", tmp_path / "GrainsProperties_10.dat"
    ctx.write_restart(raw, grains)
    _, c, i, v = parse_raw(raw.read_bytes())
    ref, _ = run_reference(case, c, i, v, [20], threads=4, restart_grains=str(grains))
    ctx.step(case.dt, 20)
    rc, ri, rv, rvol, rvr = ref[20]
    r = compare_states(ctx.download(), positive_entries(rc, ri, rv), case.ngrains)
    assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= TOL, r
    g = ctx.grains()
    assert np.max(np.abs(g["volume"] - rvol) / np.maximum(rvol, 1.0)) <= 1e-12
    assert np.max(np.abs(g["volume_ratio"] - rvr)) <= 1e-12


@needs_ref
def test_we_restart_from_reference_files(tmp_path):
    """The reference: 15 steps, its own restart files (PhaseField::Write, GrainsProperties::Write);
    a GPU context restarts from them and runs 15 more; the GPU run of 30 steps from the start ends
    in the same state."""
    case = DRIVEN
    state = case.initial_state()
    wd = tmp_path / "ref"
    ref, _ = run_reference(case, *state, [15], threads=4, workdir=wd)
    b = Context.from_case(case, precision="fp64", k_slots=16,
                          restart=(wd / "out" / "PF_15.dat", wd / "out" / "FP_15.dat"))
    a = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    a.step(case.dt, 15)
    ok, diff = _grains_close(a, b)
    assert ok, diff
    a.step(case.dt, 15)
    b.step(case.dt, 15)
    r = compare_states(a.download(), b.download(), case.ngrains)
    assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= TOL, r


@needs_ref
@pytest.mark.parametrize("case", [
    # every grain far above the reference volume (VolumeRatio = 1): the GPU state equals the
    # reference's bit for bit, so the ASCII files must be byte-identical
    Case(40, 36, 32, 10, seed=8, iwidth=4.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4), dg_scale=0.05,
         name="vtk_driven"),
    Case(32, 30, 28, 3, seed=6, iwidth=3.0, dt=0.05, sigma=1.2, stencil="SIMPLE",
         phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)), phase_solid=(0, 1),
         phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=7.0, name="vtk_nuclei_simple"),
], ids=lambda c: c.name)
def test_vtk_matches_reference_file(case, tmp_path):
    state = case.initial_state()
    _, stats = run_reference(case, *state, [12], threads=4, vtk_steps=(12,))
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    ctx.step(case.dt, 12)
    out = tmp_path / "PhaseField_12.vts"
    ctx.write_vtk(out)
    assert out.read_bytes() == stats["vtk"][12]
