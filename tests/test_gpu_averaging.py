"""Driving-force averaging ($Average Yes, the reference default) on the GPU.

The oracle's restatement of DrivingForce::Average is pinned to the reference by the fixtures
tests/golden/average_*.npz (tests/test_oracle.py); here the CUDA path (opgpu_set_averaging) is held
to the oracle and to those fixtures.  The averaged force of each voxel pair goes through CUDA's tanh
in the limiter (the value differs per voxel, so no per-pair table applies), which can differ from
the C library's in the last bit: the bar is the parity bar (identical lists, borderline voxels
counted, max|dphi| <= 1e-9) over the tested windows.
"""
from pathlib import Path

import numpy as np
import pytest

from openphase_b200.cases import Case
from openphase_b200.context import Context
from oracle.bridge import Oracle, positive_entries
from tests.golden.make_golden import GOLDEN_CASES
from tests.parity import compare_states

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-9


@pytest.mark.parametrize("name", ["average_20", "average_eta6_24"])
def test_averaging_matches_reference_fixture_and_oracle(name):
    case, steps = GOLDEN_CASES[name]
    z = np.load(GOLDEN / f"{name}.npz")
    state = case.initial_state()
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    ora = Oracle(case, *state)
    prev = 0
    for s in steps:
        st = ctx.step(case.dt, s - prev)
        ora.step(s - prev)
        prev = s
        assert st & 0b11 == 0 and not st & (1 << 7), st
        gpu = ctx.download()
        ref = positive_entries(z[f"s{s}_counts"].astype(np.int32), z[f"s{s}_idx"].astype(np.int32), z[f"s{s}_val"])
        for other in (ref, ora.state(positive_only=True)):
            r = compare_states(gpu, other, case.ngrains)
            assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= TOL, (s, r)


def test_averaging_larger_grid():
    case = Case(48, 40, 32, 14, seed=31, iwidth=5.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4), dg_scale=0.15,
                average=True, name="average_48")
    state = case.initial_state()
    tiled = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    ora = Oracle(case, *state)
    plain = Context.from_case(case.with_(average=False), precision="fp64", k_slots=16, state=state)
    prev = 0
    for s in (1, 10, 30):
        tiled.step(case.dt, s - prev)
        plain.step(case.dt, s - prev)
        ora.step(s - prev)
        prev = s
        r = compare_states(tiled.download(), ora.state(positive_only=True), case.ngrains)
        assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= TOL, (s, r)
    # averaging is not a rounding-level change: pairs far from their interface core lose their force
    r = compare_states(tiled.download(), plain.download(), case.ngrains)
    assert r["max_dphi"] > 1e-3, r


def test_averaging_refused_where_unsupported():
    from openphase_b200._lib import E_INVALID, OpgpuError
    from openphase_b200.adjoint import Rollout
    case, _ = GOLDEN_CASES["average_20"]
    ctx = Context.from_case(case, precision="fp64", k_slots=16)
    R = Rollout(ctx, case.dt, 4)
    R.forward()
    with pytest.raises(OpgpuError) as e:
        R.backward(np.ones(case.ngrains))
    assert e.value.code & E_INVALID
