"""The C++ mirror of the reference classes (include/opgpu.hpp), driven in the reference's call
order by a NormalGG-shaped program (tests/cxx/normal_gg.cpp), against the oracle."""
import subprocess

import numpy as np
import pytest

from openphase_b200.cases import Case
from openphase_b200.initializations import parse_raw, raw_bytes
from oracle.bridge import Oracle
from tests.cxx_build import build_normal_gg
from tests.parity import compare_states

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("with_dg", [False, True])
def test_cxx_normal_gg_matches_oracle(tmp_path, with_dg):
    case = Case(32, 32, 32, 8, seed=3, iwidth=5.0, dt=0.1, dg_scale=0.05 if with_dg else 0.0,
                name="cxx_normal_gg")
    nsteps = 30
    counts, idx, val = case.initial_state()
    (tmp_path / "in.raw").write_bytes(raw_bytes(case.nx, case.ny, case.nz, counts, idx, val))
    args = [str(build_normal_gg(tmp_path)), str(tmp_path / "in.raw"), str(tmp_path / "out.raw"),
            str(case.nx), str(case.ny), str(case.nz), str(case.ngrains), str(case.iwidth), str(case.dt),
            str(nsteps)]
    if with_dg:
        np.savetxt(tmp_path / "dg.txt", case.driving_force(), fmt="%.17g")
        args.append(str(tmp_path / "dg.txt"))
    run = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    vol = np.array([float(x) for x in run.stdout.split()])
    _, c, i, v = parse_raw((tmp_path / "out.raw").read_bytes())

    ora = Oracle(case, counts, idx, val)
    ora.step(nsteps)
    r = compare_states((c, i, v), ora.state(positive_only=True), case.ngrains)
    assert r["non_borderline_mismatch_voxels"] == 0, r
    assert r["max_dphi"] <= 1e-9, r
    g = ora.grains()["volume"]
    assert np.max(np.abs(vol - g) / np.maximum(g, 1.0)) <= 1e-12
