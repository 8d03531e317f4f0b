"""Slab decomposition of the step over ranks, one GPU each.

The global grid is cut into x-slabs.  A rank's context holds its slab plus one halo plane on each
side (local nx = slab + 2).  Every step:
  1. the first and last interior planes are packed and exchanged with the neighbouring ranks
     (periodic in x), and unpacked into the halo planes;
  2. the step runs on the local grid (its y/z wrap is the global one; the halo planes' own updates
     are discarded); the grain volumes are summed over the interior planes only;
  3. the partial volume sums are all-reduced and the grain update (VolumeRatio, MAXVolume, ...)
     completes the step on every rank.
The reference does the same with MPI: halo cells (include/BoundaryConditions.h:2747-2854) and an
all-reduce of the grain volumes (src/PhaseField.cpp:854-892).

Communication goes through a `comm` object with exchange(send_lo, send_hi) -> (recv_lo, recv_hi)
and allreduce(tensor): `DistComm` uses torch.distributed (NCCL on the device buffers; with gloo the
buffers are staged through host memory).  The context runs stream-ordered (its slab calls only
enqueue work on its own stream): the stepper makes torch's stream wait for the context's stream
before a buffer is sent or reduced, and the context's stream wait for torch's before a received
buffer is used, so no step synchronises the host except for the staging of a gloo exchange and the
status read at the end of `step`.
"""
from __future__ import annotations

import numpy as np

from .context import Context


def slab_bounds(nx: int, world: int, rank: int):
    """Global planes [x0, x1) of rank's slab (sizes differ by at most one plane)."""
    if world < 1 or not 0 <= rank < world or nx < world:
        raise ValueError("need 1 <= world <= nx and 0 <= rank < world")
    base, rem = divmod(nx, world)
    x0 = rank * base + min(rank, rem)
    return x0, x0 + base + (1 if rank < rem else 0)


def local_lists(counts, idx, val, dims, x0: int, x1: int):
    """Ragged lists of global planes x0-1 .. x1 (periodic in x): the slab with its two halo planes."""
    nx, ny, nz = dims
    P = ny * nz
    counts = np.asarray(counts)
    off = np.zeros(counts.size + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    planes = [(x0 - 1) % nx] + list(range(x0, x1)) + [x1 % nx]
    c_parts, i_parts, v_parts = [], [], []
    for x in planes:
        a, b = x * P, (x + 1) * P
        c_parts.append(counts[a:b])
        i_parts.append(np.asarray(idx)[off[a]:off[b]])
        v_parts.append(np.asarray(val)[off[a]:off[b]])
    return (np.concatenate(c_parts).astype(np.int32), np.concatenate(i_parts).astype(np.int32),
            np.concatenate(v_parts).astype(np.float64))


class DistComm:
    """Periodic neighbour exchange and all-reduce over torch.distributed."""

    def __init__(self, dist, group=None):
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    @property
    def staged(self) -> bool:
        """gloo moves host tensors only: device buffers go through host memory."""
        return self.dist.get_backend(self.group) == "gloo"

    def exchange(self, send_lo, send_hi):
        """send_lo (first interior plane) goes to rank-1 as its upper halo, send_hi (last interior
        plane) to rank+1 as its lower halo.  Two phases, each with one send and one receive per
        neighbour, so that the messages cannot pair up wrongly when both neighbours are one rank.
        The operations run on torch's current stream (which the caller has ordered after the
        packing); the received buffers are ready on that stream when this returns."""
        import torch
        if self.world == 1:
            return send_hi.clone(), send_lo.clone()
        d = self.dist
        dev = send_lo.device
        if self.staged and send_lo.is_cuda:
            send_lo, send_hi = send_lo.cpu(), send_hi.cpu()
        lo, hi = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        recv_lo, recv_hi = torch.empty_like(send_lo), torch.empty_like(send_hi)
        for op in d.batch_isend_irecv([d.P2POp(d.isend, send_hi, hi, self.group),
                                       d.P2POp(d.irecv, recv_lo, lo, self.group)]):
            op.wait()
        for op in d.batch_isend_irecv([d.P2POp(d.isend, send_lo, lo, self.group),
                                       d.P2POp(d.irecv, recv_hi, hi, self.group)]):
            op.wait()
        if recv_lo.device != dev:
            recv_lo, recv_hi = recv_lo.to(dev), recv_hi.to(dev)
        return recv_lo, recv_hi

    def allreduce(self, t):
        """In place on torch's current stream (through host memory with gloo)."""
        if self.world > 1:
            if self.staged and t.is_cuda:
                h = t.cpu()
                self.dist.all_reduce(h, group=self.group)
                t.copy_(h)
            else:
                self.dist.all_reduce(t, group=self.group)
        return t


class SlabStepper:
    """One rank's slab of a case: a context over the slab plus halos, stepped in the three phases."""

    def __init__(self, case, rank: int, world: int, *, precision="fp64", k_slots=16, device=0, state=None,
                 sigma=None, mu=None, dg=None):
        import torch
        self.case = case
        self.rank, self.world = rank, world
        self.x0, self.x1 = slab_bounds(case.nx, world, rank)
        self.nxl = self.x1 - self.x0 + 2
        self.device = device
        ctx = Context(self.nxl, case.ny, case.nz, dx=case.dx, iwidth=case.iwidth, stencil=case.stencil,
                      gradient_stencil=case.gradient_stencil, precision=precision, k_slots=k_slots, device=device)
        ctx.set_model(case.sigma_phase(), case.mu_phase(), limit=case.limit_phase(), limiting=case.limiting,
                      regularization=case.regularization, tj_factor=case.tj_factor,
                      energy_model=case.energy_models(), cubic_eps=case.cubic_eps(), phase_solid=case.solid_phase())
        ctx.set_grains(case.ngrains, phase=case.grain_phase())
        if case.orientations:
            ctx.set_orientations(case.quaternions())
        ps = case.pair_sigma() if sigma is None else sigma
        if ps is not None or mu is not None:
            ctx.set_pair_table(ps, mu)
        ctx.set_driving_force(case.driving_force() if dg is None else dg)
        ctx.set_volume_window(1, self.nxl - 1)
        counts, idx, val = state if state is not None else case.initial_state()
        ctx.upload(*local_lists(counts, idx, val, (case.nx, case.ny, case.nz), self.x0, self.x1))
        ctx.finalize_initialization()
        ctx.set_stream_ordered(True)
        self.ctx = ctx
        self.torch_device = torch.device("cuda", device)
        self.ctx_stream = torch.cuda.ExternalStream(ctx.stream, device=self.torch_device)
        nb = ctx.plane_bytes()
        self.send_lo = torch.empty(nb, dtype=torch.uint8, device=self.torch_device)
        self.send_hi = torch.empty(nb, dtype=torch.uint8, device=self.torch_device)
        self.acc = torch.empty(case.ngrains, dtype=torch.float64, device=self.torch_device)

    # ---- stream order between the context's stream and torch's current stream
    def to_torch(self):
        """Work enqueued on the context's stream so far comes before torch's next operations."""
        import torch
        torch.cuda.current_stream(self.torch_device).wait_stream(self.ctx_stream)

    def from_torch(self):
        """torch's operations so far come before the context's next work."""
        import torch
        self.ctx_stream.wait_stream(torch.cuda.current_stream(self.torch_device))

    # ---- the three phases of a step (each returns with its buffers ready on torch's stream)
    def pack(self):
        self.from_torch()   # the previous exchange has read the send buffers
        self.ctx.pack_plane(1, self.send_lo.data_ptr())
        self.ctx.pack_plane(self.nxl - 2, self.send_hi.data_ptr())
        self.to_torch()
        return self.send_lo, self.send_hi

    def unpack(self, recv_lo, recv_hi):
        self.from_torch()
        self.ctx.unpack_plane(0, recv_lo.data_ptr())
        self.ctx.unpack_plane(self.nxl - 1, recv_hi.data_ptr())
        self._keep = (recv_lo, recv_hi)   # alive until the context's stream has read them

    def step_partial(self, dt) -> int:
        st = self.ctx.step_partial(dt)
        self.ctx.volume_accumulator(self.acc.data_ptr())
        self.to_torch()
        return st

    def recount(self):
        self.ctx.volume_recount()
        self.ctx.volume_accumulator(self.acc.data_ptr())
        self.to_torch()

    def complete(self, total, initial=False) -> int:
        self.from_torch()
        return self.ctx.step_complete(total.data_ptr(), initial)

    def sync(self) -> int:
        """Wait for the context's stream; the soft status its steps raised."""
        return self.ctx.sync()

    def interior(self):
        """Ragged lists of the interior planes (global planes x0 .. x1-1)."""
        counts, idx, val = self.ctx.download()
        P = self.case.ny * self.case.nz
        off = np.zeros(counts.size + 1, dtype=np.int64)
        np.cumsum(counts, out=off[1:])
        a, b = P, (self.nxl - 1) * P
        return counts[a:b], idx[off[a]:off[b]], val[off[a]:off[b]]


def initialize(stepper: SlabStepper, comm):
    """Global grain volumes of the initial state (FinalizeInitialization's update)."""
    stepper.recount()
    comm.allreduce(stepper.acc)
    stepper.complete(stepper.acc, initial=True)
    return stepper.sync()


def step(stepper: SlabStepper, comm, dt: float, nsteps: int = 1) -> int:
    """nsteps slab steps; returns the soft status they raised (one host synchronisation at the end,
    besides the staging of a gloo exchange)."""
    for _ in range(nsteps):
        lo, hi = stepper.pack()
        rlo, rhi = comm.exchange(lo, hi)
        stepper.unpack(rlo, rhi)
        stepper.step_partial(dt)
        comm.allreduce(stepper.acc)
        stepper.complete(stepper.acc)
    return stepper.sync()
