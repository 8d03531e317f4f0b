"""Simulation set-ups: grid, phases, grains, interface and driving-force parameters of one run.

A `Case` carries everything both engines need (the CUDA path and the CPU checkers) to run the same
seeded problem.  The named workloads mirror the benchmark set-ups of the multiphase-field step:

  normal_grain_growth_64      64^3 periodic, 32 Voronoi grains, eta = 5 dx, sigma = mu = 1,
                              no driving force, dt = 0.1, 1000 steps
  grain_growth_dg_256         256^3 periodic, 2000 Voronoi grains, eta = 6 dx, sigma ~ U[0.8, 1.2]
                              per grain pair, mu = 1, dG_g ~ U[0, 0.05], dt = 0.08, 2000 steps
  adjoint_calibration_128     128^3 periodic, 256 grains, eta = 5 dx, sigma ~ U[0.8, 1.2],
                              dG_g ~ U[0, 0.03], dt = 0.08, 200 steps
  scale_512                   512^3 periodic, 20000 grains, eta = 6 dx, sigma ~ U[0.8,1.2], mu = 1,
                              dG_g ~ U[0, 0.05], dt = 0.08, 1000 steps
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Optional

import numpy as np

from . import initializations as init


@dataclass
class Case:
    nx: int
    ny: int
    nz: int
    ngrains: int
    seed: int = 1
    dx: float = 1.0
    iwidth: float = 5.0
    stencil: str = "LB"               # Laplacian: SIMPLE | ISOTROPIC | LB (the D3Q27 stencil)
    gradient_stencil: str = "ISOTROPIC"
    dt: float = 0.1
    nsteps: int = 100
    sigma: float = 1.0                # phase-pair ISO energy (also MaxEnergy of the limiter)
    mu: float = 1.0
    sigma_pairs: Optional[tuple] = None   # (lo, span): per-grain-pair sigma table
    dg_scale: float = 0.0             # per-grain driving force scale (0 = none)
    limiting: bool = True
    average: bool = False             # DrivingForce $Average (reference default Yes; the benchmarks use No)
    limit: float = 0.95
    regularization: float = 1.0
    tj_factor: float = 0.0
    name: str = ""
    # multi-phase set-ups (default: one solid phase holding every grain, ISO energy sigma, mu)
    phase_sigma: Optional[tuple] = None        # P x P interface energy per phase pair
    phase_mu: Optional[tuple] = None           # P x P mobility per phase pair
    phase_solid: Optional[tuple] = None        # per phase: 1 solid, 0 liquid
    phase_cubic_eps: Optional[tuple] = None    # P x P: CUBIC energy model with this epsilon (0 = ISO)
    phase_dg: Optional[tuple] = None           # per-phase driving force: dG(g) = phase_dg[phase(g)]
    init: str = "voronoi"                      # "voronoi" or "nuclei" (grain 0 = matrix)
    nucleus_radius: float = 4.0
    orientations: bool = False                 # random unit quaternion per grain
    orientation_spread: float = 0.0            # > 0: rotations by at most this angle (rad) instead
    disorientation: bool = False               # DISORIENTATION energy model for every phase pair
    hex_model: str = ""                        # HEXBOETTGER / HEXSUN / HEXYANG in place of CUBIC
    hex_eps: tuple = (0.0, 0.0, 0.0)           # Epsilon2..4 of the HEX model (Epsilon1: phase_cubic_eps)
    facets: tuple = ()                         # FACETED in place of CUBIC: (h, k, l, SigmaF, EpsilonEF) each
    facet_families: bool = True                # every facet stands for its family of permutations
    facet_exp: bool = False                    # FACETEDEXP in place of FACETED: facets are (h, k, l, EpsilonEF, PowerEF)
    mobility_model: str = ""                   # CUBIC / HEXBOETTGER / HEXSUN / HEXYANG / FACETED mobility on the pairs
    mobility_eps: tuple = (0.0, 0.0, 0.0, 0.0)  # with anisotropic energy (phase_cubic_eps != 0): Epsilon1..4
    mobility_facets: tuple = ()                # FACETED mobility: (h, k, l, MuF, EpsilonMF) each
    mobility_facet_families: bool = True

    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def nphases(self) -> int:
        return len(self.phase_sigma) if self.phase_sigma else 1

    def sigma_phase(self) -> np.ndarray:
        return np.array(self.phase_sigma, dtype=np.float64) if self.phase_sigma else np.array([[self.sigma]])

    def mu_phase(self) -> np.ndarray:
        return np.array(self.phase_mu, dtype=np.float64) if self.phase_mu else np.array([[self.mu]])

    def limit_phase(self) -> np.ndarray:
        return np.full((self.nphases, self.nphases), self.limit)

    def solid_phase(self) -> np.ndarray:
        return np.array(self.phase_solid if self.phase_solid else (1,) * self.nphases, dtype=np.int32)

    def cubic_eps(self) -> Optional[np.ndarray]:
        return np.array(self.phase_cubic_eps, dtype=np.float64) if self.phase_cubic_eps else None

    def energy_models(self) -> Optional[np.ndarray]:
        """P x P model codes: 0 ISO, 1 CUBIC, 2 DISORIENTATION."""
        if self.disorientation:
            return np.full((self.nphases, self.nphases), 2, dtype=np.int32)
        e = self.cubic_eps()
        if e is None:
            return None
        if self.facets:
            code = 7 if self.facet_exp else 6
        else:
            code = {"": 1, "HEXBOETTGER": 3, "HEXSUN": 4, "HEXYANG": 5}[self.hex_model]
        return np.where(e != 0.0, code, 0).astype(np.int32)

    def mobility_models(self) -> Optional[np.ndarray]:
        """P x P mobility model codes (0 ISO, 1 CUBIC, 3..5 HEX*, 6 FACETED)."""
        if not self.mobility_model or self.phase_cubic_eps is None:
            return None
        code = {"CUBIC": 1, "HEXBOETTGER": 3, "HEXSUN": 4, "HEXYANG": 5, "FACETED": 6}[self.mobility_model]
        return np.where(np.array(self.phase_cubic_eps) != 0.0, code, 0).astype(np.int32)

    def mobility_eps_table(self) -> Optional[np.ndarray]:
        if self.mobility_models() is None:
            return None
        return np.broadcast_to(np.asarray(self.mobility_eps, dtype=np.float64), (self.nphases, self.nphases, 4)).copy()

    def facet_tables(self):
        """(facet_start[P*P+1], facet_data[F, 5], facet_family[P*P]) for the FACETED pairs, or None."""
        em = self.energy_models()
        if not self.facets or em is None:
            return None
        return self._facet_rows(em, (6, 7), self.facets, self.facet_families)

    def mobility_facet_tables(self):
        """(start[P*P+1], data[F, 5], family[P*P]) for the FACETED mobility pairs, or None."""
        mm = self.mobility_models()
        if not self.mobility_facets or mm is None:
            return None
        return self._facet_rows(mm, (6,), self.mobility_facets, self.mobility_facet_families)

    def _facet_rows(self, codes, which, facets, families):
        P = self.nphases
        start, rows = [0], []
        for q in range(P * P):
            if codes.flat[q] in which:
                rows += [list(f) for f in facets]
            start.append(len(rows))
        fam = np.full(P * P, int(families), dtype=np.int32)
        return np.array(start, dtype=np.int32), np.array(rows, dtype=np.float64).reshape(-1, 5), fam

    def model_eps(self) -> Optional[np.ndarray]:
        """P x P x 3: Epsilon2..4 of the HEX models."""
        if not self.hex_model or self.phase_cubic_eps is None:
            return None
        return np.broadcast_to(np.asarray(self.hex_eps, dtype=np.float64), (self.nphases, self.nphases, 3)).copy()

    def grain_phase(self) -> np.ndarray:
        g = np.zeros(self.ngrains, dtype=np.int32)
        if self.init == "nuclei":
            g[1:] = 1
        return g

    def quaternions(self) -> Optional[np.ndarray]:
        if not self.orientations:
            return None
        if self.orientation_spread > 0.0:
            return init.small_rotations(self.ngrains, self.seed, self.orientation_spread)
        return init.quaternions(self.ngrains, self.seed)

    def initial_state(self, threads: int = 0):
        if self.init == "nuclei":
            return init.nuclei(self.nx, self.ny, self.nz, self.ngrains, self.seed, self.nucleus_radius,
                               self.iwidth)
        return init.voronoi(self.nx, self.ny, self.nz, self.ngrains, self.seed, threads)

    def pair_sigma(self) -> Optional[np.ndarray]:
        if self.sigma_pairs is None:
            return None
        lo, span = self.sigma_pairs
        return init.sigma_table(self.ngrains, self.seed, lo, span)

    def driving_force(self) -> Optional[np.ndarray]:
        if self.phase_dg:
            return np.array(self.phase_dg, dtype=np.float64)[self.grain_phase()]
        if not self.dg_scale:
            return None
        return init.driving_forces(self.ngrains, self.seed, self.dg_scale)

    def with_(self, **kw) -> "Case":
        return replace(self, **kw)


def normal_grain_growth_64() -> Case:
    return Case(64, 64, 64, 32, seed=1, iwidth=5.0, dt=0.1, nsteps=1000, sigma=1.0, mu=1.0,
                name="normal_grain_growth_64")


def grain_growth_dg_256() -> Case:
    # sigma ~ U[0.8, 1.2]: the limiter's MaxEnergy is the largest pair energy, 1.2
    return Case(256, 256, 256, 2000, seed=2, iwidth=6.0, dt=0.08, nsteps=2000, sigma=1.2, mu=1.0,
                sigma_pairs=(0.8, 0.4), dg_scale=0.05, name="grain_growth_dg_256")


def grain_growth_dg_128() -> Case:
    """The 256^3 workload scaled to 128^3 at the same mean grain size (250 grains): the case the
    kernel profiles are captured on."""
    return Case(128, 128, 128, 250, seed=2, iwidth=6.0, dt=0.08, nsteps=2000, sigma=1.2, mu=1.0,
                sigma_pairs=(0.8, 0.4), dg_scale=0.05, name="grain_growth_dg_128")


def solidification_128() -> Case:
    """Liquid (grain 0, phase 0) with 64 solid nuclei of radius 4 (phase 1), liquid -> solid driving
    force 0.1, solid-liquid sigma = 1.0 with cubic anisotropy eps = 0.02 and per-nucleus random
    orientations, solid-solid sigma = 1.2, mu_sl = 2.0, mu_ss = 0.5, eta = 5 dx, dt = 0.05."""
    return Case(128, 128, 128, 65, seed=3, iwidth=5.0, dt=0.05, nsteps=1500, sigma=1.2,
                phase_sigma=((1.0, 1.0), (1.0, 1.2)), phase_mu=((2.0, 2.0), (2.0, 0.5)), phase_solid=(0, 1),
                phase_cubic_eps=((0.0, 0.02), (0.02, 0.0)), phase_dg=(0.1, 0.0), init="nuclei",
                nucleus_radius=4.0, orientations=True, name="solidification_128")


def adjoint_calibration_128() -> Case:
    return Case(128, 128, 128, 256, seed=4, iwidth=5.0, dt=0.08, nsteps=200, sigma=1.2, mu=1.0,
                sigma_pairs=(0.8, 0.4), dg_scale=0.03, name="adjoint_calibration_128")


def scale_512() -> Case:
    return Case(512, 512, 512, 20000, seed=5, iwidth=6.0, dt=0.08, nsteps=1000, sigma=1.2, mu=1.0,
                sigma_pairs=(0.8, 0.4), dg_scale=0.05, name="scale_512")
