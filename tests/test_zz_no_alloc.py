"""fmm_b200_direct_noalloc: the FP64 direct sum for callers that cannot allocate device memory.

Its device staging lives in a static array shared by every call, so the checks are: the
result is bitwise fmm_b200_direct's (same kernel, same inputs) on two calls in a row, the
second smaller than the first, so that anything the first call left in the array and the
second wrongly read would show; a call at exactly the size limits covers the largest
layout; sizes beyond the limits are rejected before the device is touched (that check runs
without a GPU too).  This file is collected last, after every other test.
"""
import importlib

import numpy as np
import pytest

from oracle import Oracle, rel_l2

fmm = importlib.import_module("exafmm-dev_b200")


@pytest.mark.gpu
def test_two_calls_in_a_row_match_direct(datasets):
    rng = np.random.default_rng(7)
    # call 1: targets are sources (their r^2 == 0 self pairs are skipped), no softening
    xs1, qs1 = datasets.make("plummer", 60000, seed=1, precision="f64")
    xt1 = xs1[rng.choice(len(xs1), 3000, replace=False)]
    # call 2: fewer targets and sources than call 1, softened
    xs2, qs2 = datasets.make("cube", 513, seed=2, precision="f64")
    xt2 = rng.uniform(-1, 1, (700, 3))
    got1 = fmm.direct_noalloc(xt1, xs1, qs1, eps2=0.0)
    got2 = fmm.direct_noalloc(xt2, xs2, qs2, eps2=1e-4)
    ref1 = fmm.direct(xt1, xs1, qs1, eps2=0.0)
    ref2 = fmm.direct(xt2, xs2, qs2, eps2=1e-4)
    assert np.isfinite(got1).all() and np.isfinite(got2).all()
    # same kernel on the same inputs: tolerance zero
    assert np.array_equal(got1, ref1)
    assert np.array_equal(got2, ref2)


@pytest.mark.gpu
def test_at_the_size_limits_matches_direct(datasets):
    nt, ns = fmm.DIRECT_NOALLOC_MAX_TARGETS, fmm.DIRECT_NOALLOC_MAX_SOURCES
    xs, qs = datasets.make("sphere", ns, seed=3, precision="f64")
    xt = np.random.default_rng(8).uniform(-2, 2, (nt, 3))
    got = fmm.direct_noalloc(xt, xs, qs)
    assert np.array_equal(got, fmm.direct(xt, xs, qs))
    # no sources gives zeros; no targets gives nothing
    assert np.array_equal(fmm.direct_noalloc(xt[:5], xs[:0], qs[:0]), np.zeros((5, 4)))
    assert fmm.direct_noalloc(xt[:0], xs, qs).shape == (0, 4)


def test_sizes_beyond_the_limits_are_rejected():
    nt, ns = fmm.DIRECT_NOALLOC_MAX_TARGETS, fmm.DIRECT_NOALLOC_MAX_SOURCES
    for mt, ms in ((nt + 1, 10), (10, ns + 1)):
        with pytest.raises(fmm.FmmError) as e:
            fmm.direct_noalloc(np.zeros((mt, 3)), np.zeros((ms, 3)), np.ones(ms))
        assert e.value.code == fmm.FMM_ERR_INVALID
        assert "limits of %d targets / %d sources" % (nt, ns) in str(e.value)


@pytest.mark.gpu
def test_matches_the_oracle_direct_sum(datasets):
    """Both GPU direct sums against the oracle's FP64 sum: softened, unsoftened, and targets
    that coincide with sources (skipped pairs); rounding differences only (FMA contraction)."""
    xs, qs = datasets.make("plummer", 20000, seed=9, precision="f64")
    rng = np.random.default_rng(10)
    xt = np.concatenate([xs[:1000], rng.uniform(-1, 1, (1000, 3))])
    o64 = Oracle("f64")
    for eps2 in (0.0, 1e-3):
        want = o64.direct(xt, xs, qs, eps2=eps2)
        for got in (fmm.direct_noalloc(xt, xs, qs, eps2=eps2), fmm.direct(xt, xs, qs, eps2=eps2)):
            pot, acc = rel_l2(got, want)
            assert pot < 1e-13 and acc < 1e-13, (eps2, pot, acc)


@pytest.mark.gpu
def test_a_success_clears_the_last_error(datasets):
    lib = fmm.load_library()
    nt = fmm.DIRECT_NOALLOC_MAX_TARGETS
    with pytest.raises(fmm.FmmError):
        fmm.direct_noalloc(np.zeros((nt + 1, 3)), np.zeros((4, 3)), np.ones(4))
    assert b"limits" in lib.fmm_b200_last_error(None)
    xs, qs = datasets.make("cube", 100, seed=4, precision="f64")
    fmm.direct_noalloc(xs[:10], xs, qs)
    assert lib.fmm_b200_last_error(None) == b""


def test_limits_come_from_the_header():
    hdr = open(__file__.replace("tests/test_zz_no_alloc.py", "include/exafmm_b200.h")).read()
    assert "#define FMM_DIRECT_NOALLOC_MAX_TARGETS %d" % fmm.DIRECT_NOALLOC_MAX_TARGETS in hdr
    assert "#define FMM_DIRECT_NOALLOC_MAX_SOURCES %d" % fmm.DIRECT_NOALLOC_MAX_SOURCES in hdr
