"""Host logic of the device MC runner that needs no GPU: the launch shapes
MCRunner picks for a batch and for the last chains of a run."""
import types

import numpy as np
import pytest

from protein_physics_b200 import _lib
from protein_physics_b200.mc import TAIL_MAX_TEAMS, MCRunner, auto_shape


@pytest.mark.parametrize("sms", [148, 132])
def test_auto_shape_fills_the_sms(sms):
    for n in range(1, 3 * sms):
        cl, k = auto_shape(n, sms)
        assert cl in (1, 2, 4, 8, 16) and 1 <= k <= TAIL_MAX_TEAMS
        if n * 2 <= sms:
            assert n * cl * k <= sms  # every team of every system resident
            assert cl == 16 or n * 2 * cl > sms  # the largest cluster that fits
        else:
            assert (cl, k) == (1, 1)
    assert auto_shape(1, 148) == (16, 4) and auto_shape(74, 148) == (2, 1) and auto_shape(75, 148) == (1, 1)


def _runner(sizes, sms=148, tail_shape=True):
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    return types.SimpleNamespace(tail_shape=tail_shape, _sms=sms, b=types.SimpleNamespace(atom_off_h=off))


def _states(steps):
    st = np.zeros(len(steps), dtype=_lib.STATE_DTYPE)
    st["step"] = steps
    return st


def test_tail_plan_launches_the_chains_left_largest_first():
    rng = np.random.default_rng(1)
    sizes = rng.integers(800, 10000, size=256)
    R = _runner(sizes)
    steps = np.full(256, 100)
    left = rng.choice(256, size=40, replace=False)
    steps[left] = rng.integers(0, 100, size=40)
    order, n, cl, k = MCRunner._tail_plan(R, _states(steps), 100)
    assert n == 40 and (cl, k) == auto_shape(40, 148)
    assert sorted(order.tolist()) == sorted(left.tolist())
    assert order.dtype == np.int32
    assert np.all(np.diff(sizes[order]) <= 0)  # largest first


def test_tail_plan_keeps_the_batch_shape_while_the_sms_are_busy():
    sizes = np.full(256, 5000)
    R = _runner(sizes)
    assert MCRunner._tail_plan(R, _states(np.zeros(256)), 100) is None  # every chain left
    steps = np.full(256, 100)
    steps[:75] = 3  # 75 chains: more than half the SMs
    assert MCRunner._tail_plan(R, _states(steps), 100) is None
    steps[74] = 100
    assert MCRunner._tail_plan(R, _states(steps), 100)[1:] == (74, 2, 1)
    assert MCRunner._tail_plan(R, _states(np.full(256, 100)), 100) is None  # none left
    assert MCRunner._tail_plan(_runner(sizes, tail_shape=False), _states(steps), 100) is None


def test_tail_plan_leaves_a_small_batch_its_own_shape_until_a_chain_is_done():
    sizes = np.full(16, 65000)
    R = _runner(sizes)
    assert MCRunner._tail_plan(R, _states(np.full(16, 40)), 100) is None  # the caller's / the tuner's shape
    steps = np.full(16, 40)
    steps[3] = 100
    assert MCRunner._tail_plan(R, _states(steps), 100)[1:] == (15,) + auto_shape(15, 148)

