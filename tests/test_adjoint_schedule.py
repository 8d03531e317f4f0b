"""Checkpoint schedule of the adjoint rollout (host logic only, no GPU): a recording stand-in for
the context checks that every reverse step gets the state its forward step started from."""
import math

import numpy as np
import pytest

from openphase_b200.adjoint import Rollout


class Recorder:
    """Stand-in context whose 'state' is the step counter t."""

    def __init__(self):
        self.t = None
        self.slots = {}
        self.nslots = 0
        self.reverse = []
        self.ngrains = 3

    def checkpoint_reserve(self, n):
        self.nslots = max(self.nslots, n)

    def checkpoint_save(self, k):
        assert 0 <= k < self.nslots
        self.slots[k] = self.t

    def checkpoint_load(self, k):
        self.t = self.slots[k]

    def step(self, dt, n):
        self.t += n
        return 0

    def step_save_input(self, dt, k):
        self.checkpoint_save(k)
        return self.step(dt, 1)

    def stats(self):
        return {"entries_out_total": 0}

    def grains(self):
        return {"volume": np.zeros(3)}

    def adjoint_begin(self, w):
        self.lam_at = self.t

    def adjoint_step(self, k, dt):
        # the adjoint is aligned with the current state, which must be one step after the slot's
        assert self.lam_at == self.t and self.slots[k] == self.t - 1
        self.reverse.append(self.slots[k])
        # the slot and the current state exchange their buffers
        self.t, self.slots[k] = self.slots[k], self.t
        self.lam_at = self.t
        return 0

    def adjoint_gradients(self):
        return None, None, None


@pytest.mark.parametrize("T,interval", [(1, None), (7, None), (16, None), (30, None), (30, 1), (30, 30), (200, 16)])
def test_reverse_visits_every_step_once_from_its_own_state(T, interval):
    ctx = Recorder()
    ctx.t = 0
    R = Rollout(ctx, 0.1, T, interval)
    assert R.C == (interval or max(1, math.ceil(math.sqrt(T))))
    R.forward()
    assert ctx.t == T
    R.backward(np.zeros(3))
    assert ctx.reverse == list(range(T - 1, -1, -1))
    # memory: segment starts + one segment of states + the initial state
    assert ctx.nslots == 1 + math.ceil(T / R.C) + R.C
