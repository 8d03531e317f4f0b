"""Comparison of two ragged phase-field states, and the error figures of the FP32 form.

A state is (counts[N], idx[total], val[total]): per voxel (x slowest, z fastest) the number of
stored fields, then the (grain, value) entries of all voxels concatenated in that order.
"""
from __future__ import annotations

import numpy as np


def dense_keys(counts, idx, ngrains):
    vox = np.repeat(np.arange(counts.size, dtype=np.int64), counts)
    return vox * ngrains + np.asarray(idx, dtype=np.int64)


def compare_states(a, b, ngrains, borderline=1e-12, eps_snap=np.finfo(np.float64).eps):
    """Compare two ragged states (counts, idx, val).

    Returns a dict with
      same_sets          per-voxel index lists identical (same order)
      set_mismatch_voxels number of voxels whose index *sets* differ
      borderline_voxels  mismatching voxels whose extra entries sit within `borderline` of the
                          finalize erase threshold in the engine that kept them
      max_dphi           max |phi_a - phi_b| over the union of entries (missing entries count as 0)
      frac_over_1e4      fraction of the union entries with |phi_a - phi_b| > 1e-4
    """
    ca, ia, va = a
    cb, ib, vb = b
    out = {}
    out["same_sets"] = bool(np.array_equal(ca, cb) and np.array_equal(ia, ib))
    if out["same_sets"]:
        d = np.abs(np.asarray(va) - np.asarray(vb))
        out["max_dphi"] = float(d.max()) if d.size else 0.0
        out["frac_over_1e4"] = float(np.count_nonzero(d > 1e-4)) / max(1, d.size)
        out["set_mismatch_voxels"] = 0
        out["borderline_voxels"] = 0
        out["non_borderline_mismatch_voxels"] = 0
        return out
    ka = dense_keys(ca, ia, ngrains)
    kb = dense_keys(cb, ib, ngrains)
    oa, ob = np.argsort(ka, kind="stable"), np.argsort(kb, kind="stable")
    ka, va_s = ka[oa], np.asarray(va)[oa]
    kb, vb_s = kb[ob], np.asarray(vb)[ob]
    keys = np.union1d(ka, kb)
    pa = np.zeros(keys.size)
    pb = np.zeros(keys.size)
    ina = np.isin(keys, ka)
    inb = np.isin(keys, kb)
    pa[ina] = va_s
    pb[inb] = vb_s
    out["max_dphi"] = float(np.max(np.abs(pa - pb))) if keys.size else 0.0
    out["frac_over_1e4"] = float(np.count_nonzero(np.abs(pa - pb) > 1e-4)) / max(1, keys.size)
    only = ina ^ inb
    vox = keys[only] // ngrains
    out["set_mismatch_voxels"] = int(np.unique(vox).size)
    extra_val = np.where(ina[only], pa[only], pb[only])
    near = np.abs(extra_val - eps_snap) <= borderline
    bad_vox = np.unique(vox[~near])
    out["borderline_voxels"] = int(out["set_mismatch_voxels"] - bad_vox.size)
    out["non_borderline_mismatch_voxels"] = int(bad_vox.size)
    return out


def mean_radius(volume):
    """Mean equivalent-sphere radius (3V/4pi)^(1/3) over the grains with positive volume."""
    v = np.asarray(volume, dtype=np.float64)
    v = v[v > 0.0]
    return float(np.mean(np.cbrt(3.0 * v / (4.0 * np.pi)))) if v.size else 0.0


def precision_error(state, volume, state_ref, volume_ref, ngrains, min_volume=1.0):
    """Error of a state (the FP32 form's) against a reference state (the FP64 form's) of the same
    run: max|dphi| and the fraction of entries off by more than 1e-4, voxels whose field sets differ,
    the worst per-grain volume error relative to the reference volume (grains of at least
    `min_volume` voxels), and the relative error of the mean grain radius."""
    r = compare_states(state, state_ref, ngrains)
    v, vr = np.asarray(volume), np.asarray(volume_ref)
    big = vr >= min_volume
    rel = np.abs(v[big] - vr[big]) / vr[big]
    r0 = mean_radius(vr)
    return {"max_dphi": r["max_dphi"], "frac_over_1e4": r["frac_over_1e4"],
            "set_mismatch_voxels": r["set_mismatch_voxels"],
            "volume_rel_max": float(rel.max()) if rel.size else 0.0,
            "volume_rel_mean": float(rel.mean()) if rel.size else 0.0,
            "mean_radius_rel": abs(mean_radius(v) - r0) / r0 if r0 else 0.0}
