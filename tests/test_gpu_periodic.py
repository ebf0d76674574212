"""Periodic boundaries (images > 0) on the CUDA path, against the oracle and the reference.

The traversal runs from (root, root shifted by (ix, iy, iz) cycle) for |i| <= 1 and the
root's local expansion takes the super-cells of traversePeriodic (include/traversal.h:
127-185, 250-260).  Bar as for open boundaries: interaction lists (with their image codes)
bit-exact for use_ropt = 0; potentials and gradients within 1e-10 (FP64) or 2e-5 (FP32)
of the oracle on the same tree.
"""
import importlib
import json
import os

import numpy as np
import pytest

from oracle import CARTESIAN, SPHERICAL, Oracle, rel_l2

pytestmark = pytest.mark.gpu
fmm = importlib.import_module("exafmm-dev_b200")


@pytest.mark.parametrize("prec,images,P,basis", [
    ("f64", 1, 6, "spherical"), ("f64", 3, 6, "spherical"), ("f32", 2, 8, "spherical"),
    ("f32", 4, 10, "spherical"), ("f64", 1, 5, "cartesian"), ("f64", 3, 5, "cartesian"),
    ("f32", 2, 6, "cartesian")])
def test_periodic_matches_oracle(prec, images, P, basis, datasets):
    x, q = datasets.make("cube", 6000, seed=21, precision=prec)
    kw = dict(ncrit=32, theta=0.4, use_ropt=0)
    o = Oracle(prec).run(x, q, P=P, kahan=int(prec == "f32"), images=images, cycle=2.0,
                         basis=SPHERICAL if basis == "spherical" else CARTESIAN, **kw)
    s = fmm.Solver(basis=basis, P=P, precision=prec, images=images, cycle=2.0, **kw)
    s.set_bodies(x, q)
    s.build_tree()
    s.upward_pass()
    s.traverse()
    s.downward_pass()
    m2l, p2p = s.lists()
    assert np.array_equal(m2l, np.sort(o.m2l()))
    assert np.array_equal(p2p, np.sort(o.p2p()))
    pot, acc = rel_l2(s.trg(), o.trg())
    tol = 2e-5 if prec == "f32" else 1e-10
    assert pot < tol and acc < tol, (pot, acc)


def test_periodic_golden_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "sph_p6_f64_periodic.npz"))
    p = json.loads(str(g["params"]))
    s = fmm.Solver(P=6, theta=p["theta"], ncrit=p["ncrit"], use_ropt=p["use_ropt"],
                   precision="f64", images=p["images"], cycle=p["cycle"])
    trg = s.solve(g["x"], g["q"])
    m2l, p2p = s.lists()
    assert np.array_equal(m2l, g["m2l"]) and np.array_equal(p2p, g["p2p"])
    pot, acc = rel_l2(trg, g["trg"])
    assert pot < 5e-7 and acc < 5e-7, (pot, acc)


def test_periodic_converges_to_the_image_sum(datasets):
    """With one image level the FMM sums exactly the 27 nearest copies; against the direct
    sum over them the error is the truncation error of the expansions."""
    x, q = datasets.make("cube", 4000, seed=5, precision="f64")
    kw = dict(P=12, theta=0.35, ncrit=32, use_ropt=0, images=1, cycle=2.0)
    trg = fmm.Solver(precision="f64", **kw).solve(x, q)
    o = Oracle("f64")
    idx = datasets.sample_targets(len(q), 64)
    d = o.direct_periodic(x[idx], x, q, 1, 2.0)
    pot, acc = rel_l2(trg[idx], d)
    opot, oacc = rel_l2(o.run(x, q, **kw).trg()[idx], d)  # 2.5e-6, 8.4e-6
    assert opot < 5e-6 and oacc < 2e-5, (opot, oacc)
    assert pot < 1.05 * opot + 1e-9 and acc < 1.05 * oacc + 1e-9, (pot, acc, opot, oacc)


def test_periodic_batch_equals_alone(datasets):
    sizes = [3000, 800, 5000]
    xs, qs = [], []
    for i, n in enumerate(sizes):
        x, q = datasets.make(("cube", "plummer", "cube")[i], n, seed=40 + i, precision="f32")
        xs.append(np.clip(x, -0.999, 0.999))
        qs.append(q)
    s = fmm.Solver(P=8, theta=0.4, ncrit=32, images=2, cycle=2.0)
    batch = s.solve_batch(xs, qs)
    alone = fmm.Solver(P=8, theta=0.4, ncrit=32, images=2, cycle=2.0)
    for x, q, got in zip(xs, qs, batch):
        assert np.array_equal(got, alone.solve(x, q))


def test_gromacs_wrapper_periodic(datasets):
    """FMM_Init(images) + FMM_Coulomb(cycle): the periodic solve minus the dipole
    correction (up_down_pass.h:160-168), as the reference wrapper computes it."""
    lib = fmm.load_library()
    x, q = datasets.make("cube", 5000, seed=3, precision="f64")
    x = np.ascontiguousarray(x * 0.999)
    n = len(q)
    cycle = 2.0
    lib.FMM_Init(2)
    p = np.zeros(n)
    f = np.zeros(3 * n)
    xf = np.ascontiguousarray(x.reshape(-1))
    lib.FMM_Coulomb(n, fmm._p(xf), fmm._p(q), fmm._p(p), fmm._p(f), cycle)
    lib.FMM_Finalize()
    ref = fmm.Solver(P=10, theta=0.4, ncrit=32, use_ropt=1, images=2, cycle=cycle).solve(x, q)
    dip = (x * q[:, None]).sum(0)
    coef = 4 * np.pi / (3 * cycle ** 3)
    ep = ref[:, 0] - coef * (dip ** 2).sum() / n / q
    ef = ref[:, 1:] - coef * dip
    assert np.allclose(p, ep, rtol=1e-12, atol=1e-12)
    assert np.allclose(f.reshape(-1, 3), ef, rtol=1e-12, atol=1e-12)
