"""Host logic of the slab decomposition on CPU (no GPU): the slab split, the local lists with their
periodic halo planes, and the neighbour exchange / all-reduce pattern over torch.distributed with
world size 2 and 3 on gloo."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from openphase_b200.slab import DistComm, local_lists, slab_bounds


def test_slab_bounds_cover_the_grid():
    for nx in (5, 16, 257):
        for world in range(1, 6):
            spans = [slab_bounds(nx, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nx
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def test_local_lists_hold_slab_and_periodic_halos():
    nx, ny, nz = 6, 2, 3
    P = ny * nz
    # voxel v holds (v % 3) + 1 entries whose indices encode the plane
    counts = np.array([(v % 3) + 1 for v in range(nx * P)], dtype=np.int32)
    idx = np.concatenate([np.full(c, v // P) for v, c in enumerate(counts)]).astype(np.int32)
    val = np.concatenate([np.full(c, float(v)) for v, c in enumerate(counts)])
    for x0, x1 in ((0, 3), (3, 6), (2, 4)):
        c, i, v = local_lists(counts, idx, val, (nx, ny, nz), x0, x1)
        planes = [(x0 - 1) % nx] + list(range(x0, x1)) + [x1 % nx]
        assert c.size == len(planes) * P
        off = np.concatenate([[0], np.cumsum(c)])
        for lp, gp in enumerate(planes):
            for k in range(P):
                gv = gp * P + k
                lv = lp * P + k
                assert c[lv] == counts[gv]
                assert np.all(i[off[lv]:off[lv + 1]] == gp)
                assert np.all(v[off[lv]:off[lv + 1]] == float(gv))


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        comm = DistComm(dist)
        # each rank's first / last interior planes carry (rank, 0) / (rank, 1)
        lo = torch.tensor([rank, 0], dtype=torch.uint8)
        hi = torch.tensor([rank, 1], dtype=torch.uint8)
        rlo, rhi = comm.exchange(lo, hi)
        acc = torch.full((3,), float(rank + 1), dtype=torch.float64)
        comm.allreduce(acc)
        out.put((rank, rlo.tolist(), rhi.tolist(), acc.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_and_volume_allreduce_over_gloo(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + world * 7 + os.getpid() % 200
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, rlo, rhi, acc = out.get(timeout=120)
        res[r] = (rlo, rhi, acc)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    total = sum(range(1, world + 1))
    for r in range(world):
        rlo, rhi, acc = res[r]
        # lower halo = last interior plane of rank-1, upper halo = first interior plane of rank+1
        assert rlo == [(r - 1) % world, 1]
        assert rhi == [(r + 1) % world, 0]
        assert acc == [float(total)] * 3


def test_single_rank_exchange_is_periodic_wrap():
    class One:
        @staticmethod
        def get_rank(group=None):
            return 0

        @staticmethod
        def get_world_size(group=None):
            return 1
    comm = DistComm(One)
    lo, hi = torch.tensor([1]), torch.tensor([2])
    rlo, rhi = comm.exchange(lo, hi)
    assert rlo.tolist() == [2] and rhi.tolist() == [1]
