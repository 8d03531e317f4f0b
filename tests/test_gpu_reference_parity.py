"""The FP64 CUDA step against the reference itself, at the sizes of the benchmark set-ups.

The other parity tests hold the CUDA path to the oracle (the C restatement); these run the
unmodified reference (oracle/_ref/ref_driver: OpenPhase compiled from its own sources and driven
through its public C++ API, on all host cores) on the same seeded input and compare its dumped
states with the GPU's:

* grain_growth_dg_256: 256^3 periodic, 2000 Voronoi grains, eta = 6 dx, sigma ~ U[0.8, 1.2] per grain
  pair, mu = 1, dG_g ~ U[0, 0.05], LB stencil, dt = 0.08.  A 50-step prefix (the reference takes
  seconds per step at this size), compared at steps 1, 10 and 50.
* normal_grain_growth_64: 64^3 periodic, 32 Voronoi grains, eta = 5 dx, sigma = mu = 1, no driving
  force, dt = 0.1; all 1000 steps, compared at steps 1, 100 and 1000.
* solidification_128: 128^3, a liquid with 64 solid nuclei of radius 4 (CUBIC solid-liquid energy,
  eps = 0.02, per-nucleus orientations), liquid -> solid driving force 0.1, dt = 0.05; a 200-step
  prefix compared at steps 1, 50 and 200, and the FP32 form's error against the FP64 form there.

Bar: per-voxel index lists identical (extra entries within 1e-12 of the finalize erase threshold
count as borderline and are reported), max|dphi| <= 1e-9, grain volumes within 1e-12 relative.
Each comparison is printed as one `PARITY {...}` JSON line.
"""
import json
import os

import numpy as np
import pytest

from openphase_b200.cases import grain_growth_dg_256, normal_grain_growth_64, solidification_128
from openphase_b200.context import Context
from oracle.bridge import positive_entries, reference_available, run_reference
from tests.parity import compare_states

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference_available(), reason="reference build (oracle/_ref) not present")]

TOL = 1e-9


def _last(x):
    return int(x[-1] if isinstance(x, list) else x)


def _against_reference(case, checkpoints, k_slots):
    state = case.initial_state(threads=os.cpu_count() or 0)
    ref, stats = run_reference(case, *state, dump_steps=list(checkpoints), threads=os.cpu_count() or 0)
    ctx = Context.from_case(case, precision="fp64", k_slots=k_slots, state=state)
    out, prev = [], 0
    for s in checkpoints:
        st = ctx.step(case.dt, s - prev)
        prev = s
        c, i, v, vol, vr = ref[s]
        r = compare_states(ctx.download(), positive_entries(c, i, v), case.ngrains)
        g = ctx.grains()
        r["step"] = s
        r["status_gpu"] = st
        r["vol_rel"] = float(np.max(np.abs(g["volume"] - vol) / np.maximum(vol, 1.0)))
        r["vr_max"] = float(np.max(np.abs(g["volume_ratio"] - vr)))
        r["grains_below_ref_volume"] = int(np.count_nonzero(vr < 1.0))
        out.append(r)
        print("PARITY " + json.dumps({"case": case.name, **r}))
    steps = stats["step_seconds"] if isinstance(stats["step_seconds"], list) else [stats["step_seconds"]]
    print("PARITY " + json.dumps({"case": case.name, "reference_threads": stats["threads"],
                                  "reference_s_per_step_median": float(np.median(steps)),
                                  "reference_wide_last": _last(stats["wide"]),
                                  "gpu_wide_last": int(np.count_nonzero(ctx.flags()))}))
    return out, stats, ctx


def test_fp64_matches_reference_grain_growth_dg_256_prefix():
    """The headline workload, first 50 steps, against the reference."""
    case = grain_growth_dg_256()
    res, stats, ctx = _against_reference(case, (1, 10, 50), k_slots=16)
    for r in res:
        assert r["status_gpu"] & 0b11 == 0, r          # no K / list overflow
        assert r["non_borderline_mismatch_voxels"] == 0, r
        assert r["max_dphi"] <= TOL, r
        assert r["vol_rel"] <= 1e-12, r
    # wide-interface voxels (flag != 0) of the final state
    assert int(np.count_nonzero(ctx.flags())) == _last(stats["wide"])


def test_fp64_matches_reference_normal_grain_growth_64_1000_steps():
    """Normal grain growth over all 1000 steps, against the reference."""
    case = normal_grain_growth_64()
    res, stats, ctx = _against_reference(case, (1, 100, 1000), k_slots=8)
    for r in res:
        assert r["status_gpu"] & 0b11 == 0, r
        assert r["non_borderline_mismatch_voxels"] == 0, r
        assert r["max_dphi"] <= TOL, r
        assert r["vol_rel"] <= 1e-12, r


def test_fp64_matches_reference_solidification_128_prefix():
    """Two-phase solidification with cubic anisotropy at its full size, against the reference.  The
    nuclei start below the reference volume (VolumeRatio < 1), so the grain volumes -- sums over the
    grid whose order differs between the two engines in the last bit -- feed back into the
    kinetics: the lists must agree (borderline voxels counted) within the 1e-9 bar."""
    from openphase_b200.compare import precision_error
    case = solidification_128()
    res, stats, ctx = _against_reference(case, (1, 50, 200), k_slots=16)
    for r in res:
        assert r["status_gpu"] & 0b11 == 0, r
        assert r["non_borderline_mismatch_voxels"] == 0, r
        assert r["max_dphi"] <= TOL, r
        assert r["vol_rel"] <= 1e-9, r
    f32 = Context.from_case(case, precision="fp32", k_slots=16)
    f32.step(case.dt, 200)
    err = precision_error(f32.download(), f32.grains()["volume"], ctx.download(), ctx.grains()["volume"],
                          case.ngrains)
    print("PARITY " + json.dumps({"case": case.name, "fp32_error_after_200_steps": err}))
