"""Gradients of grain-volume losses through a rollout of the phase-field step.

`Rollout` runs T steps from a fixed initial state with checkpoints every C = ceil(sqrt(T)) steps
and, given dL/dV of the final grain volumes, sweeps backwards: each segment of C steps is
recomputed from its checkpoint (its states kept in C more slots), then reversed step by step by
the adjoint kernels (opgpu_adjoint_step).  Memory: ceil(T/C) + C state copies; cost: one extra
forward pass plus the reverse steps.

`GrainVolumes` wraps it as a torch.autograd.Function of the parameters
(sigma[G, G], mu[G, G], dG[G]) -> V[G] (final grain volumes).

The gradients are those of the forward run's discrete decisions held fixed (list members, zeroed
and limited increments, snapped and erased fields), with VolumeRatio held fixed; see
csrc/adjoint.cu.  No reference counterpart: OpenPhase has no adjoint.
"""
from __future__ import annotations

import math

import numpy as np

from .context import Context


class Rollout:
    def __init__(self, ctx: Context, dt: float, nsteps: int, interval: int | None = None):
        self.ctx = ctx
        self.dt = float(dt)
        self.T = int(nsteps)
        self.C = int(interval) if interval else max(1, math.ceil(math.sqrt(self.T)))
        self.nseg = max(1, math.ceil(self.T / self.C))
        # slot 0: initial state; 1..nseg: segment starts; then C slots for a recomputed segment
        self.seg0 = 1
        self.buf0 = 1 + self.nseg
        ctx.checkpoint_reserve(self.buf0 + self.C)
        ctx.checkpoint_save(0)

    def set_parameters(self, sigma=None, mu=None, dg=None):
        self.ctx.set_pair_table(sigma, mu)
        if dg is not None:
            self.ctx.set_driving_force(dg)

    def forward(self, fingerprint: bool = False) -> np.ndarray:
        """Run T steps from the initial state; returns the final grain volumes.  With fingerprint,
        self.fingerprint records the stored-entry count after every step (a change of the active
        sets between two runs shows up there)."""
        ctx = self.ctx
        ctx.checkpoint_load(0)
        status = 0
        self.fingerprint = []
        start = ctx.stats()["entries_out_total"] if fingerprint else 0
        for t in range(self.T):
            if t % self.C == 0:
                ctx.checkpoint_save(self.seg0 + t // self.C)
            status |= ctx.step(self.dt, 1)
            if fingerprint:
                self.fingerprint.append(ctx.stats()["entries_out_total"])
        if fingerprint:
            self.fingerprint = list(np.diff([start] + self.fingerprint))
        self.status = status
        return ctx.grains()["volume"].copy()

    def backward(self, dL_dV):
        """Reverse sweep from the state the last forward() left; returns (dsigma, dmu, ddG)."""
        ctx = self.ctx
        ctx.adjoint_begin(dL_dV)
        status = 0
        for seg in reversed(range(self.nseg)):
            t0 = seg * self.C
            t1 = min(self.T, t0 + self.C)
            ctx.checkpoint_load(self.seg0 + seg)
            for t in range(t0, t1):
                ctx.step_save_input(self.dt, self.buf0 + (t - t0))
            for t in range(t1 - 1, t0 - 1, -1):
                status |= ctx.adjoint_step(self.buf0 + (t - t0), self.dt)
        self.adjoint_status = status
        return ctx.adjoint_gradients()

    def tangent(self, dsigma=None, dmu=None, ddg=None) -> np.ndarray:
        """Tangent-linear model: dV(T) for the given parameter tangents (FP64 form)."""
        ctx = self.ctx
        ctx.checkpoint_load(0)
        ctx.tlm_begin(dsigma, dmu, ddg)
        ctx.tlm_step(self.dt, self.T)
        return ctx.tlm_volumes()


def grain_volumes_function():
    """torch.autograd.Function: (sigma[G,G], mu[G,G], dG[G], rollout) -> V[G] (float64, CPU)."""
    import torch

    class GrainVolumes(torch.autograd.Function):
        @staticmethod
        def forward(fctx, sigma, mu, dg, rollout):
            rollout.set_parameters(sigma.detach().cpu().numpy().astype(np.float64),
                                   mu.detach().cpu().numpy().astype(np.float64),
                                   dg.detach().cpu().numpy().astype(np.float64))
            fctx.rollout = rollout
            return torch.from_numpy(rollout.forward())

        @staticmethod
        def backward(fctx, gV):
            ds, dm, dd = fctx.rollout.backward(gV.detach().cpu().numpy().astype(np.float64))
            return torch.from_numpy(ds), torch.from_numpy(dm), torch.from_numpy(dd), None

    return GrainVolumes
