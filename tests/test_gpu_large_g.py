"""Large grain counts: grain indices up to 17000 and device-generated pair energies.

The 512^3 scale set-up has 20000 grains, where a G*G energy table is impractical on the host side
of a user program: opgpu_set_pair_hash generates sigma(a,b) = lo + span*u(seed, min, max) on the
device with the counter-based generator.  These tests run a grid whose grains carry indices spread
over [0, 17000) (a Voronoi state of 80 grains, renumbered) so that int16 indices, the G-sized grain
records and the G*G limited-driving-force table are exercised at large G, and compare with the
oracle given the same energies as a host table (opgpu_pair_table_host, same keys): identical lists,
max|dphi| <= 1e-9 (every grain stays above the reference volume, so the result is bit-identical in
practice).
"""
import numpy as np
import pytest

from openphase_b200.cases import Case
from openphase_b200.context import Context
from openphase_b200.initializations import voronoi
from oracle.bridge import Oracle
from tests.parity import compare_states

pytestmark = pytest.mark.gpu

G_LARGE = 17000
STRIDE = 212          # grain g of the 80-grain Voronoi state becomes grain g * STRIDE


def _case_and_state():
    # 80 grains of about 2400 voxels each, far above the reference volume at eta = 4 (268 voxels)
    case = Case(64, 64, 48, G_LARGE, seed=12, iwidth=4.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4),
                dg_scale=0.05, name="large_g")
    counts, idx, val = voronoi(case.nx, case.ny, case.nz, 80, case.seed)
    return case, (counts, idx * STRIDE, val)


@pytest.mark.parametrize("mode", ["table", "hash"])
def test_large_grain_count_matches_oracle(mode):
    case, state = _case_and_state()
    ora = Oracle(case, *state)
    ctx = Context.from_case(case, precision="fp64", k_slots=16, state=state)
    if mode == "hash":
        lo, span = case.sigma_pairs
        ctx.set_pair_hash(case.seed, lo, span)
    prev = 0
    for s in (1, 10, 60):
        st = ctx.step(case.dt, s - prev)
        ora.step(s - prev)
        prev = s
        g, go = ctx.grains(), ora.grains()
        assert st & 0b11 == 0
        r = compare_states(ctx.download(), ora.state(positive_only=True), case.ngrains)
        assert r["non_borderline_mismatch_voxels"] == 0 and r["max_dphi"] <= 1e-9, (mode, s, r)
        assert (go["volume_ratio"][go["volume"] > 0] == 1.0).all()
        live = go["volume"] > 0
        assert np.max(np.abs(g["volume"][live] - go["volume"][live]) / go["volume"][live]) <= 1e-12
        assert np.array_equal(g["exist"], go["exist"])
