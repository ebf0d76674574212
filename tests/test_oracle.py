"""The oracle (CPU restatement, oracle/fmm_oracle.c) pinned against the reference.

Two pins: the committed golden fixtures made by tests/golden/make_golden.py from the
reference compiled from its own sources, and (where oracle/_ref was built) the reference
itself run on fresh inputs.  Trees, body order and interaction lists must match bit for
bit; potentials and gradients within rounding of the working precision.
"""
import json
import os

import numpy as np
import pytest

from oracle import (CARTESIAN, SPHERICAL, TREE_ADAPTIVE, TREE_UNIFORM, Oracle, Reference,
                    have_reference, rel_l2)

CELL_KEYS = ("iparent", "ichild", "nchild", "ibody", "nbody", "level", "X", "R_built", "R")


def _params(p):
    basis = SPHERICAL if p["config"].startswith("sph") else CARTESIAN
    P = int(p["config"].split("_")[1][1:])
    mass = int(p["config"].endswith("_mass"))
    kahan = int("f32k" in p["config"])
    return basis, P, mass, kahan


@pytest.mark.parametrize("case", ["sph_p6_f64_cube", "sph_p10_f32k_plummer",
                                  "cart_p5_f32_sphere", "sph_p6_f64_periodic"])
def test_oracle_matches_golden(case, golden_dir):
    g = np.load(os.path.join(golden_dir, case + ".npz"))
    p = json.loads(str(g["params"]))
    basis, P, mass, kahan = _params(p)
    o = Oracle(p["precision"]).run(g["x"], g["q"], basis=basis, P=P, theta=p["theta"],
                                   ncrit=p["ncrit"], use_ropt=p["use_ropt"], mass=mass,
                                   kahan=kahan, images=p.get("images", 0),
                                   cycle=p.get("cycle", 2 * np.pi))
    cells = o.cells()
    for k in CELL_KEYS:
        assert np.array_equal(cells[k], g["cell_" + k]), k
    shallow = cells["level"] <= 10  # the reference's 32-bit key arithmetic holds to level 10
    assert np.array_equal(cells["icell"][shallow], g["cell_icell"][shallow])
    assert np.array_equal(o.order(), g["order"])
    assert np.array_equal(np.sort(o.m2l()), g["m2l"])
    assert np.array_equal(np.sort(o.p2p()), g["p2p"])
    tol = 2e-6 if p["precision"] == "f32" else 5e-7  # reference P2P: AVX rsqrt + one Newton step
    pot, acc = rel_l2(o.trg(), g["trg"])
    assert pot < tol and acc < tol, (pot, acc)


def test_kernel_chain_matches_golden(golden_dir):
    with open(os.path.join(golden_dir, "kernel_chain.json")) as f:
        gold = json.load(f)
    o = Oracle("f64")
    for key, val in gold.items():
        basis, P = key.split("_p")
        got = o.kernel_chain(SPHERICAL if basis == "spherical" else CARTESIAN, int(P))
        assert abs(got - val) <= 2e-3 * val, (key, got, val)


def test_kernel_chain_converges():
    """Cartesian and spherical truncations agree, and the error falls with P."""
    o = Oracle("f64")
    errs = [o.kernel_chain(SPHERICAL, P) for P in (4, 6, 8, 10, 12)]
    assert all(a > 5 * b for a, b in zip(errs, errs[1:])), errs


def test_direct_and_rel_l2(datasets):
    x, q = datasets.make("cube", 300, precision="f64")
    o = Oracle("f64")
    d = o.direct(x, x, q)
    # brute force in numpy
    dx = x[:, None, :] - x[None, :, :]
    r2 = (dx ** 2).sum(-1)
    np.fill_diagonal(r2, np.inf)
    inv = 1 / np.sqrt(r2)
    pot = (q[None, :] * inv).sum(1)
    g = -(q[None, :, None] * dx * inv[..., None] ** 3).sum(1)
    assert np.allclose(d[:, 0], pot, rtol=1e-12)
    assert np.allclose(d[:, 1:], g, rtol=1e-10)
    assert rel_l2(d, d) == (0.0, 0.0)


def test_empty_and_single_body():
    o = Oracle("f64")
    r = o.run(np.zeros((0, 3)), np.zeros(0))
    assert r.num_cells == 0
    # One body sits at its leaf centre: the spherical L2P divides by r and sin(theta) there
    # (kernels/LaplaceSphericalCPU.cxx:17-26,45), so the reference returns a NaN gradient.
    r = o.run(np.array([[0.5, 0.25, -0.5]]), np.array([1.0]))
    assert r.num_cells == 1
    t = r.trg()
    assert t[0, 0] == 0 and np.all(np.isnan(t[0, 1:]))
    x = np.array([[0.5, 0.25, -0.5], [0.1, 0.2, 0.3]])
    t = o.run(x, np.array([1.0, 2.0])).trg()
    d = o.direct(x, x, np.array([1.0, 2.0]))
    assert np.allclose(t, d, rtol=1e-12)


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("cfg,prec,dist,n,kw", [
    ("sph_p6_f64", "f64", "cube", 16384, dict(ncrit=64, theta=0.4, use_ropt=0)),
    ("sph_p6_f32k", "f32", "cube", 20000, dict(ncrit=32, theta=0.4, use_ropt=0, nspawn=500)),
    ("sph_p8_f32k_mass", "f32", "plummer", 30000, dict(ncrit=64, theta=0.4, use_ropt=1)),
    ("cart_p5_f32", "f32", "sphere", 30000, dict(ncrit=32, theta=0.5, use_ropt=0)),
    ("cart_p4_f64", "f64", "cube", 10000, dict(ncrit=16, theta=0.6, use_ropt=0)),
    # the uniform Morton tree (include/build_tree_omp.h): depths 3, 4, 4, 1 and 0
    ("uni_sph_p6_f64", "f64", "cube", 16384, dict(ncrit=64, theta=0.4, use_ropt=0)),
    ("uni_sph_p8_f32k", "f32", "plummer", 20000, dict(ncrit=32, theta=0.4, use_ropt=0)),
    ("uni_cart_p4_f64", "f64", "sphere", 12000, dict(ncrit=16, theta=0.5, use_ropt=0)),
    ("uni_sph_p6_f64", "f64", "cube", 100, dict(ncrit=64, theta=0.4, use_ropt=0)),
    ("uni_sph_p6_f64", "f64", "plummer", 30, dict(ncrit=64, theta=0.4, use_ropt=0)),
])
def test_oracle_matches_reference(cfg, prec, dist, n, kw, datasets):
    R = Reference(cfg)
    x, q = datasets.make(dist, n, seed=7, precision=prec)
    r = R.run(x, q, **kw)
    o = Oracle(prec).run(x, q, basis=SPHERICAL if R.spherical else CARTESIAN, P=R.P,
                         mass=int(R.mass), kahan=int(R.kahan),
                         tree=TREE_UNIFORM if R.uniform else TREE_ADAPTIVE, **kw)
    rc, oc = r.cells(), o.cells()
    for k in CELL_KEYS:
        assert np.array_equal(rc[k], oc[k]), k
    assert np.array_equal(r.order(), o.order())
    assert np.array_equal(r.m2l(), o.m2l())  # same pairs in the same visiting order
    assert np.array_equal(r.p2p(), o.p2p())
    pot, acc = rel_l2(o.trg(), r.trg())
    tol = 2e-6 if prec == "f32" else 5e-7  # the reference P2P uses AVX rsqrt + one Newton step
    assert pot < tol and acc < tol, (pot, acc)


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("cfg,prec,images", [("sph_p6_f64", "f64", 1), ("sph_p6_f64", "f64", 2),
                                             ("sph_p6_f64", "f64", 4), ("sph_p6_f32k", "f32", 3)])
def test_oracle_matches_reference_periodic(cfg, prec, images, datasets):
    """Traversal with the 27 shifted source trees and traversePeriodic's super-cells
    (include/traversal.h:127-185, 250-260): the same pairs, with their image codes, in the
    same visiting order, and the same potentials."""
    R = Reference(cfg)
    x, q = datasets.make("cube", 3000, seed=11, precision=prec)
    kw = dict(ncrit=32, theta=0.4, use_ropt=0, images=images, cycle=2.0)
    r = R.run(x, q, **kw)
    o = Oracle(prec).run(x, q, P=R.P, kahan=int(R.kahan), **kw)
    assert np.array_equal(r.m2l(), o.m2l())
    assert np.array_equal(r.p2p(), o.p2p())
    assert len(np.unique(o.m2l() >> 27 & 31)) == 27  # every image contributes
    pot, acc = rel_l2(o.trg(), r.trg())
    tol = 2e-6 if prec == "f32" else 5e-7
    assert pot < tol and acc < tol, (pot, acc)


def test_uniform_level_rule():
    """include/build_tree_omp.h:218: 1 + int(log(N / ncrit) / ln 2 / 3) with integer N / ncrit,
    0 below ncrit; exact powers of 8 of N / ncrit start a new level."""
    o = Oracle("f64")
    assert o.uniform_level(30, 64) == 0 and o.uniform_level(64, 64) == 1
    assert o.uniform_level(64 * 8 - 1, 64) == 1 and o.uniform_level(64 * 8, 64) == 2
    assert o.uniform_level(16384, 64) == 3 and o.uniform_level(1 << 20, 64) == 5
    assert o.uniform_level(64 * 4096, 64) == 5 and o.uniform_level(64 * 4095, 64) == 4


def test_periodic_direct_sum():
    """oracle_direct_periodic: the shifts |i| <= sum_{l < images} 3^l; one image level is
    the 27 nearest copies."""
    rng = np.random.default_rng(3)
    xs = rng.uniform(-1, 1, (40, 3))
    qs = rng.uniform(-1, 1, 40)
    xt = xs[:5]
    o = Oracle("f64")
    got = o.direct_periodic(xt, xs, qs, 1, 2.0)
    ref = np.zeros((5, 4))
    for ix in (-1, 0, 1):
        for iy in (-1, 0, 1):
            for iz in (-1, 0, 1):
                ref += o.direct(xt - 2.0 * np.array([ix, iy, iz]), xs, qs)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)
    assert np.allclose(o.direct_periodic(xt, xs, qs, 0, 2.0), o.direct(xt, xs, qs), rtol=1e-14)


def _ij_run(prec, g, kw, P, mass, kahan, basis=SPHERICAL):
    return Oracle(prec).run_ij(g["xt"], g["qt"], g["xs"], g["qs"], basis=basis, P=P, mass=mass,
                               kahan=kahan, **kw)


def test_oracle_ij_matches_golden(golden_dir):
    """Separate target and source trees (examples/serial.cxx IneJ) against the reference's
    recorded lists and potentials."""
    g = np.load(os.path.join(golden_dir, "sph_p8_f32k_ij.npz"))
    p = json.loads(str(g["params"]))
    basis, P, mass, kahan = _params(p)
    kw = dict(ncrit=p["ncrit"], theta=p["theta"], use_ropt=p["use_ropt"])
    o = _ij_run(p["precision"], g, kw, P, mass, kahan, basis)
    assert np.array_equal(np.sort(o.m2l()), g["m2l"])
    assert np.array_equal(np.sort(o.p2p()), g["p2p"])
    pot, acc = rel_l2(o.trg(), g["trg"])
    assert pot < 2e-6 and acc < 2e-6, (pot, acc)


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("cfg,prec,common", [("sph_p6_f64", "f64", 1), ("cart_p5_f32", "f32", 1),
                                             ("sph_p10_f32k_mass", "f32", 1),
                                             ("sph_p8_f32k_mass", "f32", 0)])
def test_oracle_ij_matches_reference(cfg, prec, common, datasets):
    R = Reference(cfg)
    xt, qt = datasets.make("cube", 2500, seed=3, precision=prec)
    xs, qs = datasets.make("sphere", 3500, seed=4, precision=prec)
    xt = xt * 0.5 + 0.25
    kw = dict(ncrit=32, theta=0.4, use_ropt=0)
    r = R.run_ij(xt, qt, xs, qs, common_box=common, **kw)
    o = Oracle(prec).run_ij(xt, qt, xs, qs, basis=SPHERICAL if R.spherical else CARTESIAN,
                            P=R.P, mass=int(R.mass), kahan=int(R.kahan), common_box=common, **kw)
    assert np.array_equal(r.m2l(), o.m2l())  # visiting order too
    assert np.array_equal(r.p2p(), o.p2p())
    pot, acc = rel_l2(o.trg(), r.trg())
    tol = 2e-6 if prec == "f32" else 5e-7
    assert pot < tol and acc < tol, (pot, acc)


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("cfg,prec", [("sph_p6_f64", "f64"), ("cart_p5_f32", "f32"),
                                      ("sph_p8_f32k_mass", "f32")])
def test_oracle_mutual_matches_reference(cfg, prec, datasets):
    """dualTreeTraversal with mutual = true: each unordered pair once (TraverseRange drops
    the (latter, former) quarter of a range against itself), both cells updated."""
    R = Reference(cfg)
    x, q = datasets.make("plummer", 9000, seed=17, precision=prec)
    kw = dict(ncrit=32, theta=0.4, use_ropt=1, nspawn=500)
    r = R.run(x, q, mutual=1, **kw)
    o = Oracle(prec).run(x, q, basis=SPHERICAL if R.spherical else CARTESIAN, P=R.P,
                         kahan=int(R.kahan), mass=int(R.mass), mutual=1, **kw)
    assert np.array_equal(r.m2l(), o.m2l())
    assert np.array_equal(r.p2p(), o.p2p())
    pot, acc = rel_l2(o.trg(), r.trg())
    tol = 2e-6 if prec == "f32" else 5e-7
    assert pot < tol and acc < tol, (pot, acc)
