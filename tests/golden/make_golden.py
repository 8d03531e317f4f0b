"""Generate the golden fixtures of the phase-field step from the unmodified reference.

Runs the reference (compiled from its own sources by `make -C oracle ref`, driven through its public
API by oracle/ref_driver.cpp) on small seeded cases and stores, per case, the states and grain
records at a few checkpoints.  The fixtures pin the oracle (tests/test_oracle.py) without needing the
reference at test time.  OUTPUT_CASES also store the reference's VTK file and grain-record restart
file of one state (tests/test_output_files.py).

    python tests/golden/make_golden.py [name ...]  # writes tests/golden/<name>.npz (all by default)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from openphase_b200.cases import Case  # noqa: E402
from oracle.bridge import run_reference  # noqa: E402

GOLDEN_CASES = {
    "lb_16": (Case(16, 16, 16, 6, seed=3, iwidth=4.0, dt=0.1, name="lb_16"), [1, 10, 50]),
    "isotropic_24x20x16": (Case(24, 20, 16, 10, seed=5, iwidth=5.0, dt=0.1, stencil="ISOTROPIC",
                                name="isotropic_24x20x16"), [1, 40]),
    "simple_24x20x16": (Case(24, 20, 16, 10, seed=5, iwidth=5.0, dt=0.1, stencil="SIMPLE",
                             name="simple_24x20x16"), [1, 40]),
    "pairs_dg_24": (Case(24, 24, 24, 30, seed=7, iwidth=6.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4),
                         dg_scale=0.05, name="pairs_dg_24"), [1, 60]),
    "dg_strong_20": (Case(20, 20, 20, 40, seed=9, iwidth=4.0, dt=0.1, sigma=1.2, sigma_pairs=(0.8, 0.4),
                          dg_scale=0.3, name="dg_strong_20"), [1, 60]),
    # liquid + solid nuclei (VolumeRatio < 1, triple-junction term), CUBIC solid-liquid energy with
    # per-grain orientations (gradients of the candidate lists), liquid -> solid driving force
    "cubic_nuclei_24": (Case(24, 24, 24, 7, seed=3, iwidth=5.0, dt=0.05, sigma=1.2,
                             phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                             phase_solid=(0, 1), phase_cubic_eps=((0.0, 0.02), (0.02, 0.0)), phase_dg=(0.1, 0.0),
                             init="nuclei", nucleus_radius=4.0, orientations=True, name="cubic_nuclei_24"),
                        [1, 10, 40]),
    # the hexagonal energy models on the solid-liquid pairs of the nuclei set-up
    "hexboettger_nuclei_24": (Case(24, 24, 24, 7, seed=4, iwidth=5.0, dt=0.05, sigma=1.2,
                                   phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                                   phase_solid=(0, 1), phase_cubic_eps=((0.0, 0.05), (0.05, 0.0)),
                                   phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                                   hex_model="HEXBOETTGER", name="hexboettger_nuclei_24"), [1, 30]),
    "hexsun_nuclei_24": (Case(24, 24, 24, 7, seed=5, iwidth=5.0, dt=0.05, sigma=1.2,
                              phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                              phase_solid=(0, 1), phase_cubic_eps=((0.0, -0.03), (-0.03, 0.0)),
                              phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                              hex_model="HEXSUN", hex_eps=(0.01, 0.002, 0.004), name="hexsun_nuclei_24"), [1, 30]),
    "hexyang_nuclei_24": (Case(24, 24, 24, 7, seed=6, iwidth=5.0, dt=0.05, sigma=1.2,
                               phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                               phase_solid=(0, 1), phase_cubic_eps=((0.0, -0.03), (-0.03, 0.0)),
                               phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                               hex_model="HEXYANG", hex_eps=(0.1, 0.2, 0.0), name="hexyang_nuclei_24"), [1, 30]),
    # anisotropic interface mobility (CUBIC, HEX*) on the solid-liquid pairs, each with the
    # matching energy model
    "mobility_cubic_24": (Case(24, 24, 24, 7, seed=8, iwidth=5.0, dt=0.05, sigma=1.2,
                               phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                               phase_solid=(0, 1), phase_cubic_eps=((0.0, 0.02), (0.02, 0.0)),
                               phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                               mobility_model="CUBIC", mobility_eps=(0.2, 0.0, 0.0, 0.0),
                               name="mobility_cubic_24"), [1, 30]),
    "mobility_hexboettger_24": (Case(24, 24, 24, 7, seed=9, iwidth=5.0, dt=0.05, sigma=1.2,
                                     phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                                     phase_solid=(0, 1), phase_cubic_eps=((0.0, 0.05), (0.05, 0.0)),
                                     phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                                     hex_model="HEXBOETTGER", mobility_model="HEXBOETTGER",
                                     mobility_eps=(0.15, 0.0, 0.0, 0.0), name="mobility_hexboettger_24"), [1, 30]),
    "mobility_hexsun_24": (Case(24, 24, 24, 7, seed=10, iwidth=5.0, dt=0.05, sigma=1.2,
                                phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                                phase_solid=(0, 1), phase_cubic_eps=((0.0, -0.03), (-0.03, 0.0)),
                                phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                                hex_model="HEXSUN", hex_eps=(0.01, 0.002, 0.004), mobility_model="HEXSUN",
                                mobility_eps=(-0.05, 0.02, 0.01, 0.005), name="mobility_hexsun_24"), [1, 30]),
    "mobility_hexyang_24": (Case(24, 24, 24, 7, seed=11, iwidth=5.0, dt=0.05, sigma=1.2,
                                 phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                                 phase_solid=(0, 1), phase_cubic_eps=((0.0, -0.03), (-0.03, 0.0)),
                                 phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                                 hex_model="HEXYANG", hex_eps=(0.1, 0.2, 0.0), mobility_model="HEXYANG",
                                 mobility_eps=(-0.04, 0.1, 0.2, 0.0), name="mobility_hexyang_24"), [1, 30]),
    # FACETED energy model ({100} and {111} facet families) on the solid-liquid pairs
    "faceted_nuclei_24": (Case(24, 24, 24, 7, seed=7, iwidth=5.0, dt=0.05, sigma=1.2,
                               phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                               phase_solid=(0, 1), phase_cubic_eps=((0.0, 1.0), (1.0, 0.0)),
                               phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                               facets=((1, 0, 0, 1.0, 0.7), (1, 1, 1, 1.1, 0.8)), name="faceted_nuclei_24"),
                          [1, 10, 30]),
    # FACETEDEXP energy model ({100} and {111} families, cusp powers 4 and 6) on the solid-liquid pairs
    "facetedexp_nuclei_24": (Case(24, 24, 24, 7, seed=12, iwidth=5.0, dt=0.05, sigma=1.2,
                                  phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                                  phase_solid=(0, 1), phase_cubic_eps=((0.0, 1.0), (1.0, 0.0)),
                                  phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                                  facets=((1, 0, 0, 0.05, 4.0), (1, 1, 1, 0.03, 6.0)), facet_exp=True,
                                  name="facetedexp_nuclei_24"), [1, 10, 30]),
    # FACETED mobility ({100} and {111} families) with the CUBIC energy on the solid-liquid pairs
    "mobility_faceted_24": (Case(24, 24, 24, 7, seed=13, iwidth=5.0, dt=0.05, sigma=1.2,
                                 phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                                 phase_solid=(0, 1), phase_cubic_eps=((0.0, 0.02), (0.02, 0.0)),
                                 phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=4.0, orientations=True,
                                 mobility_model="FACETED", mobility_facets=((1, 0, 0, 2.0, 0.3), (1, 1, 1, 1.5, 0.5)),
                                 name="mobility_faceted_24"), [1, 30]),
    # DISORIENTATION energy model: per-grain-pair energies from the cubic disorientation of
    # orientations spread over up to 0.6 rad (pairs below and above the 0.349 rad cap)
    "disorientation_20": (Case(20, 20, 20, 12, seed=11, iwidth=4.0, dt=0.1, orientations=True,
                               orientation_spread=0.6, disorientation=True, name="disorientation_20"),
                          [1, 40]),
    # driving-force averaging ($Average Yes, the reference default): Range = iWidth, threshold
    # iWidth/15 below 5 cells (first case) and 1/3 from 5 cells on (second case)
    "average_20": (Case(20, 18, 16, 12, seed=21, iwidth=4.0, dt=0.1, sigma=1.2, sigma_pairs=(0.8, 0.4),
                        dg_scale=0.1, average=True, name="average_20"), [1, 10, 20]),
    "average_eta6_24": (Case(24, 24, 20, 10, seed=23, iwidth=6.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4),
                             dg_scale=0.2, average=True, name="average_eta6_24"), [1, 10]),
}


# output files of the reference (PhaseField::WriteVTK and the grain-record restart file) for a state
# of each case at one step: they pin opgpu_write_vtk_host and the grain-record format
OUTPUT_CASES = {
    "vtk_pairs_12": (Case(12, 10, 8, 8, seed=5, iwidth=3.0, dt=0.1, sigma=1.2, sigma_pairs=(0.8, 0.4),
                          dg_scale=0.05, name="vtk_pairs_12"), 5),
    "vtk_simple_nuclei_12": (Case(12, 12, 10, 4, seed=6, iwidth=3.0, dt=0.05, sigma=1.2, stencil="SIMPLE",
                                  phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)),
                                  phase_solid=(0, 1), phase_dg=(0.1, 0.0), init="nuclei", nucleus_radius=3.0,
                                  name="vtk_simple_nuclei_12"), 4),
}


def output_fixture(name):
    case, step = OUTPUT_CASES[name]
    counts, idx, val = case.initial_state()
    res, stats = run_reference(case, counts, idx, val, [step], threads=2, vtk_steps=(step,))
    c, i, v, vol, vr = res[step]
    arrays = {"counts": c.astype(np.uint8), "idx": i.astype(np.int16), "val": v, "volume": vol,
              "volume_ratio": vr, "vtk": np.frombuffer(stats["vtk"][step], dtype=np.uint8),
              "grains_file": np.frombuffer(stats["grains_file"][step], dtype=np.uint8)}
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    print(name, arrays["vtk"].size, arrays["grains_file"].size)


def main(names=None):
    for name in OUTPUT_CASES:
        if not names or name in names:
            output_fixture(name)
    for name, (case, steps) in GOLDEN_CASES.items():
        if names and name not in names:
            continue
        counts, idx, val = case.initial_state()
        res, stats = run_reference(case, counts, idx, val, [0] + steps, threads=4)
        arrays = {"init_counts": counts.astype(np.uint8), "init_idx": idx.astype(np.int16)}
        for s in [0] + steps:
            c, i, v, vol, vr = res[s]
            arrays[f"s{s}_counts"] = c.astype(np.uint8)
            arrays[f"s{s}_idx"] = i.astype(np.int16)
            arrays[f"s{s}_val"] = v
            arrays[f"s{s}_volume"] = vol
            arrays[f"s{s}_volume_ratio"] = vr
        arrays["wide"] = np.asarray(stats["wide"] if isinstance(stats["wide"], list) else [stats["wide"]],
                                    dtype=np.int64)
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print(name, {k: v.shape for k, v in arrays.items() if k.endswith("_val")})


if __name__ == "__main__":
    main(sys.argv[1:])
