"""The FP64 direct sum on the GPU (fmm_b200_direct: Traversal::direct + normalize,
include/traversal.h:304-337) against the oracle's FP64 direct sum (oracle/fmm_oracle.c).

This kernel is the accuracy reference of the bench and of the full-size tests, so it is
pinned on its own: plain and softened sums, targets that coincide with sources (their
r^2 == 0 pairs are skipped, as the reference's P2P does at LaplaceP2PCPU.cxx:149), and
duplicated source positions.  Both sums run in double with the same pair order; the only
differences are fused multiply-adds, so the bar is 1e-13 relative (rel-L2 per quantity).
"""
import importlib

import numpy as np
import pytest

from oracle import Oracle, rel_l2

fmm = importlib.import_module("exafmm-dev_b200")


def cases(datasets):
    rng = np.random.default_rng(21)
    xs, qs = datasets.make("plummer", 20000, seed=5, precision="f64")
    # 2,000 targets: half of them source positions (coincident pairs), half free points
    xt = np.concatenate([xs[rng.choice(len(xs), 1000, replace=False)],
                         rng.uniform(-1.5, 1.5, (1000, 3))])
    # duplicated sources: the first 500 positions again, with other charges
    xd = np.concatenate([xs, xs[:500]])
    qd = np.concatenate([qs, rng.uniform(-1, 1, 500)])
    return [("plain", xt, xs, qs, 0.0), ("softened", xt, xs, qs, 1e-3),
            ("duplicates", xt, xd, qd, 0.0), ("integer_eps2", xt[:300], xd, qd, 1.0)]


@pytest.mark.gpu
def test_direct_matches_oracle(datasets):
    o64 = Oracle("f64")
    for name, xt, xs, qs, eps2 in cases(datasets):
        want = o64.direct(xt, xs, qs, eps2=eps2)
        got = fmm.direct(xt, xs, qs, eps2=eps2)
        assert np.isfinite(got).all(), name
        pot, acc = rel_l2(got, want)
        assert pot < 1e-13 and acc < 1e-13, (name, pot, acc)


def test_direct_rejects_bad_arguments():
    lib = fmm.load_library()
    rc = lib.fmm_b200_direct(0, -1, None, 0, None, None, 0.0, None)
    assert rc == fmm.FMM_ERR_INVALID
    assert b"invalid argument" in lib.fmm_b200_last_error(None)
