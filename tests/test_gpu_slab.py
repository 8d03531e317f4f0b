"""Slab decomposition on one GPU.

1. W ranks emulated in one process, each with its own context over its slab plus halo planes,
   stepped phase by phase (pack, exchange, step, volume all-reduce, complete) with the exchange
   and the all-reduce done by torch operations between the contexts' streams.
2. Two real ranks: two processes on the same GPU, joined by torch.distributed over gloo (the
   buffers staged through host memory), running the library's slab driver (`slab.initialize`,
   `slab.step`).  No kernel waits on another: every exchange goes through the host.
The assembled interior states must equal the single-domain run."""
import datetime
import os

import numpy as np
import pytest
import torch

from openphase_b200.cases import Case
from openphase_b200.context import Context
from openphase_b200.slab import SlabStepper
from tests.parity import compare_states

pytestmark = pytest.mark.gpu


def _emulated(steppers, dt, nsteps):
    W = len(steppers)
    for _ in range(nsteps):
        packs = [s.pack() for s in steppers]
        for r, s in enumerate(steppers):
            s.unpack(packs[(r - 1) % W][1], packs[(r + 1) % W][0])
        for s in steppers:
            s.step_partial(dt)
        total = sum(s.acc for s in steppers)
        for s in steppers:
            s.complete(total)
    for s in steppers:
        assert s.sync() & 0b11 == 0


def _assemble(steppers):
    parts = [s.interior() for s in steppers]
    return (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
            np.concatenate([p[2] for p in parts]))


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_slab_decomposition_equals_single_domain(world, precision):
    case = Case(48, 40, 32, 12, seed=8, iwidth=5.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4), dg_scale=0.05,
                name="slab_48")
    state = case.initial_state()
    ref = Context.from_case(case, precision=precision, k_slots=16, state=state)
    steppers = [SlabStepper(case, r, world, precision=precision, k_slots=16, state=state) for r in range(world)]
    for s in steppers:
        s.recount()
    total = sum(s.acc for s in steppers)
    for s in steppers:
        s.complete(total, initial=True)
    for n in (1, 10, 30):
        _emulated(steppers, case.dt, n)
        ref.step(case.dt, n)
        r = compare_states(_assemble(steppers), ref.download(), case.ngrains)
        vol = steppers[0].ctx.grains()["volume"]
        vref = ref.grains()["volume"]
        if precision == "fp64":
            assert r["same_sets"] and r["max_dphi"] <= 1e-12, r
            assert np.max(np.abs(vol - vref) / np.maximum(vref, 1.0)) <= 1e-12
        else:
            # FP32: the single-domain and slab runs contract multiply-adds alike; differences come
            # only from the volume-sum order
            assert r["max_dphi"] <= 1e-5, r
        for s in steppers[1:]:
            assert np.array_equal(s.ctx.grains()["volume"], vol)


def _slab_case():
    return Case(48, 40, 32, 12, seed=8, iwidth=5.0, dt=0.08, sigma=1.2, sigma_pairs=(0.8, 0.4), dg_scale=0.05,
                name="slab_48")


def _rank_worker(rank, world, port, nsteps, out):
    import torch.distributed as dist
    from openphase_b200 import slab
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        case = _slab_case()
        comm = slab.DistComm(dist)
        st = SlabStepper(case, comm.rank, comm.world, precision="fp64", k_slots=16, device=0)
        status = slab.initialize(st, comm)
        status |= slab.step(st, comm, case.dt, nsteps)
        out.put((rank, status, st.interior(), st.ctx.grains()["volume"]))
    finally:
        dist.destroy_process_group()


def test_two_processes_over_gloo_equal_single_domain():
    import torch.multiprocessing as mp
    case = _slab_case()
    world, nsteps = 2, 30
    mpc = mp.get_context("spawn")
    out = mpc.Queue()
    port = 29700 + os.getpid() % 200
    procs = [mpc.Process(target=_rank_worker, args=(r, world, port, nsteps, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(world):
            r, status, interior, vol = out.get(timeout=300)
            res[r] = (status, interior, vol)
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.terminate()
    assert all(p.exitcode == 0 for p in procs)
    ref = Context.from_case(case, precision="fp64", k_slots=16, state=case.initial_state())
    ref.step(case.dt, nsteps)
    parts = [res[r][1] for r in range(world)]
    got = (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
           np.concatenate([p[2] for p in parts]))
    r = compare_states(got, ref.download(), case.ngrains)
    assert all(res[k][0] & 0b11 == 0 for k in res)
    assert r["same_sets"] and r["max_dphi"] <= 1e-12, r
    vref = ref.grains()["volume"]
    for k in res:
        assert np.max(np.abs(res[k][2] - vref) / np.maximum(vref, 1.0)) <= 1e-12
