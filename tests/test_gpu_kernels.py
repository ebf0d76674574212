"""The single-operator C ABI (fmm_b200_kernel_*: namespace kernel, include/kernel.h:6-14).

* examples/kernel.cxx:23-92 run through it: P2M -> M2M -> M2L -> L2L -> L2P against P2P on
  the example's geometry and drand48 inputs, reproducing the reference's chain errors
  (tests/golden/kernel_chain.json, made from the reference) for spherical P = 4..10 and
  Cartesian P = 4..6;
* each operator on hand-made cells against the oracle's single operators (FP64: 1e-12);
* a whole FMM driven operator by operator over a solver's own tree and lists, equal to the
  solver's result (FP64: 1e-13);
* the argument checks (out-of-range indices, concurrent entries that would race).
"""
import importlib
import json
import os

import numpy as np
import pytest

from oracle import CARTESIAN, SPHERICAL, Oracle, rel_l2

pytestmark = pytest.mark.gpu
fmm = importlib.import_module("exafmm-dev_b200")


class Drand48:
    """POSIX drand48 from glibc's unseeded state (X = 0): X <- (a X + c) mod 2^48."""

    def __init__(self):
        self.x = 0

    def __call__(self):
        self.x = (0x5DEECE66D * self.x + 0xB) & ((1 << 48) - 1)
        return self.x / float(1 << 48)


def chain_error(basis, P, precision):
    """examples/kernel.cxx: cells Cj (centre 1, 16 sources), CJ (centre 0, child Cj),
    CI (centre R + 4), Ci (centre R + 3, parent CI, 16 targets), theta = 0.5, R = 2 / theta."""
    d = Drand48()
    R = 2 / 0.5
    xs = np.zeros((16, 3)); qs = np.zeros(16)
    for b in range(16):
        xs[b] = [2 * d(), 2 * d(), 2 * d()]
        qs[b] = d()
    xt = np.zeros((16, 3)); qt = np.zeros(16)
    for b in range(16):
        xt[b] = [R + 2 + 2 * d(), R + 2 + 2 * d(), R + 2 + 2 * d()]
        qt[b] = d()
    s = fmm.Solver(basis=basis, P=P, precision=precision)
    s.set_bodies(np.concatenate([xs, xt]), np.concatenate([qs, qt]))
    X = np.array([[1, 1, 1], [0, 0, 0], [R + 4] * 3, [R + 3] * 3], float)
    s.kernel_set_cells(X, np.ones(4), ibody=[0, 0, 0, 16], nbody=[16, 0, 0, 16],
                       ichild=[0, 0, 0, 0], nchild=[0, 1, 0, 0], iparent=[0, 0, 0, 2])
    s.kernel_p2m([0])
    s.kernel_m2m([1])
    s.kernel_m2l([2], [1])
    s.kernel_l2l([3])
    s.kernel_l2p([3])
    fmm_pot = s.kernel_trg()[16:, 0]
    s.kernel_set_trg(None)
    s.kernel_p2p([3], [0])
    direct = s.kernel_trg()[16:, 0]
    return float(np.sqrt(((fmm_pot - direct) ** 2).sum() / (direct ** 2).sum()))


def test_kernel_chain_reproduces_the_reference(golden_dir):
    with open(os.path.join(golden_dir, "kernel_chain.json")) as f:
        gold = json.load(f)
    for key, val in sorted(gold.items()):
        basis, P = key.split("_p")
        got = chain_error(basis, int(P), "f64")
        assert abs(got - val) <= 2e-3 * val, (key, got, val)
        got32 = chain_error(basis, int(P), "f32")
        assert abs(got32 - val) <= 0.1 * val, (key, got32, val)


def flat(e, spherical):
    e = np.asarray(e)
    return np.stack([e.real, e.imag], axis=-1).ravel() if spherical else e.ravel()


@pytest.mark.parametrize("basis,P", [("spherical", 4), ("spherical", 10), ("cartesian", 5)])
def test_single_operators_match_oracle(basis, P):
    rng = np.random.default_rng(P)
    sph = basis == "spherical"
    b = SPHERICAL if sph else CARTESIAN
    o = Oracle("f64")
    # cells: 0 a leaf of 24 bodies, 1 its parent, 2 a far cell, 3 a child of 2
    Xc = np.array([[0.2, -0.1, 0.3], [0.0, 0.0, 0.0], [4.0, 3.5, -3.0], [4.2, 3.3, -2.8]])
    xb = Xc[0] + rng.uniform(-0.25, 0.25, (24, 3))
    qb = rng.uniform(-1, 1, 24)
    s = fmm.Solver(basis=basis, P=P, precision="f64")
    s.set_bodies(xb, qb)
    s.kernel_set_cells(Xc, np.ones(4), ibody=[0, 0, 0, 0], nbody=[24, 0, 0, 0],
                       ichild=[0, 0, 0, 0], nchild=[0, 1, 0, 0], iparent=[0, 0, 0, 2])
    s.kernel_p2m([0])
    Mg = s.expansion(0)
    M0 = o.op_p2m(b, P, Xc[0], np.concatenate([xb, qb[:, None]], axis=1), np.zeros(Mg[0].size * (2 if sph else 1)))
    assert np.allclose(flat(Mg[0], sph), M0, rtol=1e-12, atol=1e-14 * np.abs(M0).max())
    s.kernel_m2m([1])
    M1 = o.op_m2m(b, P, Xc[1], Xc[0], M0, np.zeros_like(M0))
    Mg = s.expansion(0)
    assert np.allclose(flat(Mg[1], sph), M1, rtol=1e-12, atol=1e-14 * np.abs(M1).max())
    s.kernel_m2l([2], [1])
    L2 = o.op_m2l(b, P, Xc[2], Xc[1], M1, np.zeros_like(M1))
    Lg = s.expansion(1)
    assert np.allclose(flat(Lg[2], sph), L2, rtol=1e-12, atol=1e-14 * np.abs(L2).max())
    # accumulate: a second M2L from the same source doubles the local expansion
    s.kernel_m2l([2], [1])
    assert np.allclose(flat(s.expansion(1)[2], sph), 2 * L2, rtol=1e-12,
                       atol=1e-14 * np.abs(L2).max())
    s.kernel_set_expansion(1, 0.5 * s.expansion(1))
    s.kernel_l2l([3])
    L3 = o.op_l2l(b, P, Xc[3], Xc[2], L2, np.zeros_like(L2))
    assert np.allclose(flat(s.expansion(1)[3], sph), L3, rtol=1e-12,
                       atol=1e-14 * np.abs(L3).max())


def test_whole_fmm_through_the_operators(datasets):
    """The reference's pipeline as its passes call the kernel plugin: P2M on the leaves,
    M2M level by level upward, M2L and P2P over the traversal's lists, L2L downward, L2P on
    the leaves -- over a solver's own tree, equal to that solver's result."""
    x, q = datasets.make("cube", 4000, seed=3, precision="f64")
    kw = dict(P=6, theta=0.4, ncrit=32, use_ropt=0, precision="f64")
    ref = fmm.Solver(**kw)
    want = ref.solve(x, q)
    m2l, p2p = ref.lists()
    s = fmm.Solver(**kw)
    s.set_bodies(x, q)
    s.build_tree()
    c = s.cells()
    nc, maxlevel = s.num_cells()
    lev, nch = c["level"], c["nchild"]
    leaves = np.flatnonzero(nch == 0)
    s.kernel_p2m(leaves)
    for l in range(maxlevel - 1, -1, -1):
        s.kernel_m2m(np.flatnonzero((lev == l) & (nch > 0)))
    s.kernel_m2l(m2l >> 32, m2l & ((1 << 27) - 1), (m2l >> 27) & 31)
    s.kernel_p2p(p2p >> 32, p2p & ((1 << 27) - 1), (p2p >> 27) & 31)
    for l in range(1, maxlevel + 1):
        s.kernel_l2l(np.flatnonzero(lev == l))
    s.kernel_l2p(leaves)
    got = np.zeros_like(want)
    got[s.order()] = s.kernel_trg()
    pot, acc = rel_l2(got, want)
    assert pot < 1e-13 and acc < 1e-13, (pot, acc)


def test_operator_arguments_are_checked(datasets):
    x, q = datasets.make("cube", 64, seed=1, precision="f64")
    s = fmm.Solver(P=4, precision="f64")
    s.set_bodies(x, q)
    X = np.array([[0.0, 0.0, 0.0], [0.3, 0.2, 0.1], [-0.3, -0.2, -0.1]])
    s.kernel_set_cells(X, np.ones(3), ibody=[0, 0, 32], nbody=[64, 32, 32], ichild=[1, 0, 0],
                       nchild=[2, 0, 0], iparent=[0, 0, 0])
    bad = [lambda: s.kernel_p2m([3]),                      # out of range
           lambda: s.kernel_p2m([1, 1]),                   # listed twice
           lambda: s.kernel_m2m([0, 1]),                   # a cell with its child
           lambda: s.kernel_l2l([0]),                      # its own parent
           lambda: s.kernel_l2l([1, 0]),                   # a cell with its parent
           lambda: s.kernel_l2p([0, 1]),                   # overlapping bodies
           lambda: s.kernel_p2p([0, 1], [2, 2]),           # overlapping target bodies
           lambda: s.kernel_m2l([1], [2], image=[27]),     # image code out of range
           lambda: s.kernel_m2l([1], [-1])]
    for f in bad:
        with pytest.raises(fmm.FmmError) as e:
            f()
        assert e.value.code == fmm.FMM_ERR_INVALID
    with pytest.raises(fmm.FmmError) as e:
        s.kernel_set_cells(X, np.ones(3), ibody=[0, 0, 40], nbody=[64, 32, 32],
                           ichild=[1, 0, 0], nchild=[2, 0, 0], iparent=[0, 0, 0])
    assert e.value.code == fmm.FMM_ERR_INVALID
    # the handle still works after the rejections
    s.kernel_p2m([1, 2])
    s.kernel_m2m([0])
    assert np.isfinite(s.expansion(0)).all()
