"""DISORIENTATION interface-energy model (InterfaceEnergyModel::CalculateDisorientation,
include/InterfaceProperties/InterfaceEnergyModel.h:308-323, with Tools::getDisorientationCubic,
src/Tools.cpp:626-678): the energy of a grain pair is a Read-Shockley-type function of the cubic
disorientation of the two grains' orientations, capped above 0.349066 rad.  The library tabulates
it per grain pair on the host (the host's log and acos, as in the reference) and the step reads the
table; the oracle evaluates it per voxel and pair the way InterfaceProperties::SetSR does.

The oracle is pinned to the reference by tests/golden/disorientation_20.npz (bit-identical), so the
FP64 form must reproduce the oracle bit for bit: identical index sets and max|dphi| = 0.
"""
from pathlib import Path

import numpy as np
import pytest

from openphase_b200._lib import OpgpuError
from openphase_b200.cases import Case
from openphase_b200.context import Context
from oracle.bridge import Oracle
from tests.golden.make_golden import GOLDEN_CASES
from tests.parity import compare_states

pytestmark = pytest.mark.gpu


def _case(n, grains, seed, spread=0.6):
    return Case(n, n, n, grains, seed=seed, iwidth=4.0, dt=0.1, orientations=True, orientation_spread=spread,
                disorientation=True, name=f"disorientation_{n}")


def _positive(z, s):
    """The reference's stored lists at step s without their zero-valued entries."""
    c, i, v = z[f"s{s}_counts"].astype(np.int64), z[f"s{s}_idx"].astype(np.int32), z[f"s{s}_val"]
    keep = v > 0.0
    owner = np.repeat(np.arange(c.size), c)
    return np.bincount(owner[keep], minlength=c.size).astype(np.int32), i[keep], v[keep]


@pytest.mark.parametrize("variant", ["tiled", "generic"])
def test_fp64_matches_reference_golden(variant):
    case, steps = GOLDEN_CASES["disorientation_20"]
    z = np.load(Path(__file__).resolve().parent / "golden" / "disorientation_20.npz")
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=case.initial_state())
    ctx.set_kernel_variant(variant)
    prev = 0
    for s in steps:
        assert ctx.step(case.dt, s - prev) & 0b11 == 0
        prev = s
        r = compare_states(ctx.download(), _positive(z, s), case.ngrains)
        assert r["same_sets"] and r["max_dphi"] == 0.0, (s, r)


@pytest.mark.parametrize("n,grains,seed,spread,steps", [(40, 30, 21, 0.6, 100), (32, 40, 22, 1.5, 60)])
def test_fp64_matches_oracle(n, grains, seed, spread, steps):
    case = _case(n, grains, seed, spread)
    state = case.initial_state()
    ora = Oracle(case, *state)
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    prev = 0
    for s in (1, steps // 2, steps):
        assert ctx.step(case.dt, s - prev) & 0b11 == 0
        ora.step(s - prev)
        prev = s
        r = compare_states(ctx.download(), ora.state(positive_only=True), case.ngrains)
        assert r["same_sets"] and r["max_dphi"] == 0.0, (s, r)
        assert np.max(np.abs(ctx.grains()["volume"] - ora.grains()["volume"])) <= 1e-9


def test_orientation_change_rebuilds_the_table():
    """New orientations take effect at the next step, like GrainsProperties::Orientation does at the
    next InterfaceProperties::Set."""
    case = _case(24, 16, 23)
    state = case.initial_state()
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    ctx.step(case.dt, 5)
    case2 = _case(24, 16, 23, spread=1.2)
    ctx.set_orientations(case2.quaternions())
    ctx.step(case.dt, 5)
    ora = Oracle(case, *state)
    ora.step(5)
    ora2 = Oracle(case2, *ora.state(positive_only=True))
    ora2.step(5)
    r = compare_states(ctx.download(), ora2.state(positive_only=True), case.ngrains)
    assert r["same_sets"] and r["max_dphi"] <= 1e-12, r


def test_hash_energies_are_refused():
    case = _case(16, 8, 24)
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=case.initial_state())
    ctx.set_pair_hash(5, 0.8, 0.4)
    with pytest.raises(OpgpuError):
        ctx.step(case.dt, 1)
