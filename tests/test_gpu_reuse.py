"""A solver handle reused across solves.

The first traversal of a handle counts every step before writing it and sizes the list
and frontier buffers; later traversals run without count passes on those buffers and fall
back to the counted form when a buffer turns out too small.  Both forms must give the same
lists (they are sorted by target and source) and therefore bitwise the same results.
"""
import importlib

import numpy as np
import pytest

from oracle import rel_l2

pytestmark = pytest.mark.gpu
fmm = importlib.import_module("exafmm-dev_b200")


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_second_traversal_gives_the_same_lists(prec, datasets):
    x, q = datasets.make("plummer", 40000, seed=5, precision=prec)
    s = fmm.Solver(P=6, theta=0.4, ncrit=32, precision=prec)
    s.set_bodies(x, q)
    s.build_tree()
    s.upward_pass()
    s.traverse()                      # counted form (first traversal of the handle)
    m2l1, p2p1 = s.lists()
    s.traverse()                      # device-counted form on the sized buffers
    m2l2, p2p2 = s.lists()
    assert len(m2l1) > 0 and len(p2p1) > 0
    assert np.array_equal(m2l1, m2l2)
    assert np.array_equal(p2p1, p2p2)


def test_growing_inputs_on_one_handle_match_fresh_handles(datasets):
    # each input needs larger buffers than the one before: the device-counted traversal
    # overflows, is detected, and the counted form redoes it
    s = fmm.Solver(P=6, theta=0.4, ncrit=32)
    for k, n in enumerate((2000, 30000, 120000, 5000)):
        x, q = datasets.make(("cube", "plummer", "sphere", "plummer")[k], n, seed=20 + k,
                             precision="f32")
        got = s.solve(x, q)
        fresh = fmm.Solver(P=6, theta=0.4, ncrit=32)
        ref = fresh.solve(x, q)
        ok = ~np.isnan(ref)
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        assert np.array_equal(got[ok], ref[ok]), n
        assert s.list_counts() == fresh.list_counts()


def test_autotune_ncrit_picks_the_fastest_candidate(datasets):
    x, q = datasets.make("plummer", 60000, seed=8, precision="f32")
    s = fmm.Solver(P=8, theta=0.4, ncrit=64)
    best, times = s.autotune_ncrit(x, q, candidates=(8, 64, 256), repeats=2)
    assert best in (8, 64, 256) and all(t > 0 for t in times.values())
    assert times[best] == min(times.values())
    # the handle now solves with the tuned ncrit: bitwise a fresh handle at that ncrit
    got = s.solve(x, q)
    assert np.array_equal(got, fmm.Solver(P=8, theta=0.4, ncrit=best).solve(x, q))


def test_autotune_p2p_lanes(datasets):
    """fmm_b200_autotune_p2p: the thresholds picked are a candidate, and the solves after it
    agree with the default mapping to rounding (only the split of a target's sources over its
    lanes changes)."""
    x, q = datasets.make("plummer", 60000, seed=5, precision="f32")
    s = fmm.Solver(P=8, theta=0.4, ncrit=64, use_ropt=0)
    ref = s.solve(x, q)
    cands = ((8, 16), (0, 16), (0, 0))
    best, ms = s.autotune_p2p(candidates=cands, repeats=2)
    assert best in cands and all(v > 0 for v in ms.values())
    got = s.solve(x, q)
    pot, acc = rel_l2(got, ref)
    assert pot < 1e-6 and acc < 1e-6, (pot, acc)
    with pytest.raises(fmm.FmmError):
        s.autotune_p2p(candidates=((9, 16),))


def test_growth_keeps_grown_out_buffers_until_trim(datasets):
    """A handle that grows (a larger solve after a smaller one) allocates without freeing
    during the solve; fmm_b200_trim then frees the buffers it grew out of, and later solves
    give bitwise the same results."""
    xs, qs = datasets.make("plummer", 20000, seed=31, precision="f32")
    xl, ql = datasets.make("plummer", 200000, seed=32, precision="f32")
    s = fmm.Solver(P=8, theta=0.4, ncrit=64, use_ropt=0)
    s.solve(xs, qs)
    a0 = fmm.device_allocations()
    big = s.solve(xl, ql)
    assert fmm.device_allocations() > a0  # the arrays grew
    s.trim()
    assert np.array_equal(s.solve(xl, ql), big)
    a1 = fmm.device_allocations()
    small = s.solve(xs, qs)
    assert fmm.device_allocations() == a1  # no growth for a smaller solve
    assert np.array_equal(small, fmm.Solver(P=8, theta=0.4, ncrit=64, use_ropt=0).solve(xs, qs))
