"""Liquid + solid nuclei with CUBIC solid-liquid interface energy and per-grain orientations (the
two-phase solidification set-up): the per-voxel anisotropic energies need the gradients of every
list entry (InterfaceProperties::SetSR, src/InterfaceProperties.cpp:617-673).  The nuclei have
VolumeRatio < 1, so the triple-junction term and the volume-ratio scaling are active.

FP64 form against the oracle (pinned to the reference by tests/golden/cubic_nuclei_24.npz): the
energies use pow(n, 4) (CUDA vs libm) and the volume sums feed back through VolumeRatio, so the bar
is max|dphi| <= 1e-9 with identical index sets (borderline decisions counted).  FP32 form: the
error against the FP64 oracle is stated.
"""
import numpy as np
import pytest

from openphase_b200._lib import OpgpuError
from openphase_b200.cases import Case
from openphase_b200.context import Context
from oracle.bridge import Oracle
from tests.parity import compare_states

pytestmark = pytest.mark.gpu


def _case(n, grains, seed=3):
    return Case(n, n, n, grains, seed=seed, iwidth=5.0, dt=0.05, sigma=1.2,
                phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)), phase_solid=(0, 1),
                phase_cubic_eps=((0.0, 0.02), (0.02, 0.0)), phase_dg=(0.1, 0.0), init="nuclei",
                nucleus_radius=4.0, orientations=True, name=f"solidification_{n}")


@pytest.mark.parametrize("n,grains,checkpoints", [(24, 7, (1, 10, 40, 100)), (40, 17, (1, 20, 80))])
def test_fp64_cubic_nuclei_match_oracle(n, grains, checkpoints):
    case = _case(n, grains)
    state = case.initial_state()
    ora = Oracle(case, *state)
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    prev = 0
    for s in checkpoints:
        st = ctx.step(case.dt, s - prev)
        ora.step(s - prev)
        prev = s
        assert st & 0b11 == 0
        r = compare_states(ctx.download(), ora.state(positive_only=True), case.ngrains)
        g, go = ctx.grains(), ora.grains()
        vol = float(np.max(np.abs(g["volume"] - go["volume"]) / np.maximum(go["volume"], 1.0)))
        print(n, s, r, vol)
        assert r["non_borderline_mismatch_voxels"] == 0, (s, r)
        assert r["max_dphi"] <= 1e-9, (s, r)
        assert vol <= 1e-10


@pytest.mark.parametrize("name", ["cubic_nuclei_24", "hexboettger_nuclei_24", "hexsun_nuclei_24",
                                  "hexyang_nuclei_24", "faceted_nuclei_24", "facetedexp_nuclei_24",
                                  "mobility_cubic_24", "mobility_hexboettger_24", "mobility_hexsun_24",
                                  "mobility_hexyang_24", "mobility_faceted_24"])
def test_fp64_energy_models_match_oracle_and_reference(name):
    """CUBIC, the hexagonal models (HEXBOETTGER, HEXSUN, HEXYANG), FACETED and FACETEDEXP with {100}
    and {111} facet families (InterfaceEnergyModel.h:325-438), and the anisotropic mobilities
    including FACETED (InterfaceMobilityModel.h:210-288), on the solid-liquid pairs: the FP64 form against the oracle over 100 steps and against the
    reference's own states (tests/golden/<name>.npz) at its checkpoints."""
    from tests.golden.make_golden import GOLDEN_CASES
    from pathlib import Path
    case, golden_steps = GOLDEN_CASES[name]
    z = np.load(Path(__file__).resolve().parent / "golden" / f"{name}.npz")
    state = case.initial_state()
    ora = Oracle(case, *state)
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    prev = 0
    for s in sorted(set(golden_steps) | {100}):
        assert ctx.step(case.dt, s - prev) & 0b11 == 0
        ora.step(s - prev)
        prev = s
        mine = ctx.download()
        r = compare_states(mine, ora.state(positive_only=True), case.ngrains)
        assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= 1e-9, (s, r)
        if f"s{s}_val" in z:
            c, i, v = z[f"s{s}_counts"].astype(np.int64), z[f"s{s}_idx"].astype(np.int32), z[f"s{s}_val"]
            keep = v > 0.0
            ref = (np.bincount(np.repeat(np.arange(c.size), c)[keep], minlength=c.size).astype(np.int32),
                   i[keep], v[keep])
            r = compare_states(mine, ref, case.ngrains)
            assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= 1e-9, (s, r)


def test_fp32_cubic_nuclei_error_against_fp64_oracle():
    case = _case(40, 17)
    state = case.initial_state()
    ora = Oracle(case, *state)
    ctx = Context.from_case(case, precision="fp32", k_slots=16, state=state)
    prev = 0
    report = []
    for s in (1, 10, 80):
        ctx.step(case.dt, s - prev)
        ora.step(s - prev)
        prev = s
        r = compare_states(ctx.download(), ora.state(positive_only=True), case.ngrains)
        g, go = ctx.grains()["volume"], ora.grains()["volume"]
        live = go > 50.0
        vol = float(np.max(np.abs(g[live] - go[live]) / go[live]))
        report.append((s, r["max_dphi"], r["frac_over_1e4"], vol))
    print(report)
    assert report[0][1] <= 1e-6
    assert all(v <= 1e-2 for _, _, _, v in report)


def test_adjoint_refuses_anisotropic_energies():
    case = _case(24, 7)
    ctx = Context.from_case(case, precision="fp64", k_slots=16)
    with pytest.raises(OpgpuError):
        ctx.adjoint_begin(np.zeros(case.ngrains))
    with pytest.raises(OpgpuError):
        ctx.tlm_begin()


@pytest.mark.parametrize("aniso", [True, False])
def test_step_timing_on_every_path(aniso):
    """opgpu_set_timing on the per-voxel path of anisotropic energies (no classify phase) and on the
    tiled path: every timed step is counted and the classify share lies within the step."""
    case = _case(24, 7) if aniso else Case(24, 24, 24, 10, seed=3, iwidth=5.0, dt=0.1, name="iso_24")
    ctx = Context.from_case(case, precision="fp64", k_slots=16)
    ctx.step(case.dt, 2)
    ctx.set_timing(True)
    ctx.step(case.dt, 3)
    s = ctx.stats()
    assert s["timed_launches"] == 3
    assert s["timed_kernel_ms"] > 0.0
    assert 0.0 <= s["timed_classify_ms"] <= s["timed_kernel_ms"]
    if aniso:
        assert s["timed_classify_ms"] < 0.1 * s["timed_kernel_ms"]
