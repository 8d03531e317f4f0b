"""State comparison used by the parity tests."""
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
