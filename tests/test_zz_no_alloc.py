"""opgpu_download_flags_noalloc: the allocation-free flag download gives the same flags as
opgpu_download_flags, call after call, and rejects grids beyond its fixed scratch.

Collected last on purpose (file name), so that it also runs after every other GPU test in the
same process.
"""
import numpy as np
import pytest

from openphase_b200._lib import E_INVALID, OpgpuError
from openphase_b200.cases import Case
from openphase_b200.context import Context

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_flags_noalloc_matches_flags(precision):
    case = Case(40, 36, 32, 12, seed=21, iwidth=5.0, dt=0.1, dg_scale=0.05, name="noalloc")
    ctx = Context.from_case(case, precision=precision, k_slots=16)
    for _ in range(2):
        ref = ctx.flags()
        first = ctx.flags_noalloc()
        second = ctx.flags_noalloc()          # two calls in a row
        assert np.array_equal(first, ref)
        assert np.array_equal(second, ref)
        assert (ref == 2).any() and (ref == 1).any() and (ref == 0).any()
        ctx.step(case.dt, 3)


def test_flags_noalloc_allocates_no_device_memory():
    """The property the entry point exists for: after its one-time set-up, calls leave the device's
    free memory unchanged (no allocation, not even a transient one that a free would hide from a
    before/after count in the caller's memory pool)."""
    import torch
    case = Case(40, 36, 32, 12, seed=22, iwidth=5.0, dt=0.1, name="noalloc_mem")
    ctx = Context.from_case(case, precision="fp64", k_slots=16)
    ref = ctx.flags()
    ctx.flags_noalloc()                       # one-time set-up of this context
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert np.array_equal(ctx.flags_noalloc(), ref)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_flags_noalloc_rejects_grid_beyond_scratch():
    ctx = Context(257, 256, 256, iwidth=5.0, precision="fp32", k_slots=8)
    with pytest.raises(OpgpuError) as e:
        ctx.flags_noalloc()
    assert e.value.code & E_INVALID
    assert "16777216" in str(e.value)
