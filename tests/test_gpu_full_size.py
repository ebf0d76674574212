"""The benchmark configurations at their full sizes, through size-independent properties.

At these sizes the oracle would take minutes, so each solve is held to properties that do
not depend on N: the rel-L2 error of potential and gradient against an FP64 direct sum
(on the GPU) over stride-sampled targets stays within the bound of the method at that P
and theta; the solve is deterministic (bitwise the same twice); the batched form returns
every solve bitwise as alone.
"""
import importlib

import numpy as np
import pytest

from oracle import rel_l2

pytestmark = pytest.mark.gpu
fmm = importlib.import_module("exafmm-dev_b200")


def direct_error(datasets, x, q, trg, ntarget=512):
    idx = datasets.sample_targets(len(q), ntarget)
    d = fmm.direct(x[idx], x, q)
    return rel_l2(trg[idx], d)


def test_precision_form_plummer_1m(datasets):
    """Plummer N = 1,048,576, spherical P = 10, theta = 0.35, ncrit = 64, FP32 +
    compensation, q = 1/N: rel-L2 <= 1e-4 against FP64 direct (measured 3.3e-7 / 1.9e-5)."""
    x, q = datasets.make("plummer", 1 << 20, seed=43, precision="f32")
    s = fmm.Solver(P=10, theta=0.35, ncrit=64, nspawn=1000, use_rmax=1, use_ropt=1)
    a = s.solve(x, q)
    pot, acc = direct_error(datasets, x, q, a)
    assert pot < 1e-4 and acc < 1e-4, (pot, acc)
    assert np.array_equal(a, s.solve(x, q))


def test_cartesian_sphere_4m(datasets):
    """Sphere surface N = 4,194,304, Cartesian P = 5, theta = 0.5, ncrit = 32, FP32: the
    deep, unbalanced tree and long P2P lists of that configuration."""
    x, q = datasets.make("sphere", 1 << 22, seed=44, precision="f32")
    s = fmm.Solver(basis="cartesian", P=5, theta=0.5, ncrit=32, use_ropt=0)
    a = s.solve(x, q)
    pot, acc = direct_error(datasets, x, q, a)
    # the reference CPU build at this configuration: pot 2.28e-3, acc 5.33e-5
    assert pot < 5e-3 and acc < 1e-3, (pot, acc)
    nm2l, np2p, pairs = s.list_counts()
    assert nm2l > 0 and np2p > 0 and pairs > len(q)


def test_plain_fmm_cube_16k_fp64(datasets):
    """Cube N = 16,384, spherical P = 6, theta = 0.4, ncrit = 64, FP64, with and without the
    error-optimised radius (with it, zero net charge turns the solve into a direct sum, as in
    the reference)."""
    x, q = datasets.make("cube", 16384, seed=42, precision="f64")
    # the reference CPU build: pot 5.21e-4, acc 6.51e-4 (use_ropt 0); 2.2e-8 (use_ropt 1)
    for use_ropt, bound in ((0, 2e-3), (1, 1e-6)):
        s = fmm.Solver(P=6, theta=0.4, ncrit=64, use_ropt=use_ropt, precision="f64")
        a = s.solve(x, q)
        idx = datasets.sample_targets(len(q), 128)
        pot, acc = rel_l2(a[idx], fmm.direct(x[idx], x, q))
        assert pot < bound and acc < bound, (use_ropt, pot, acc)


def test_batched_256_solves(datasets):
    """256 solves, N log-uniform in [1e3, 2e5], cube / Plummer / sphere by i mod 3,
    spherical P = 8: every solve of the batch bitwise as alone (checked on a sample of them)
    and every solve within the method's error of FP64 direct.  At the configuration's
    theta = 0.4 the zero-net-charge cubes reach ~2.3e-4 (the reference's FP64 build measures
    the same on them), so the bound there is 5e-4; at theta = 0.3 every solve meets 1e-4."""
    rng = np.random.default_rng(44)
    sizes = np.rint(np.exp(rng.uniform(np.log(1e3), np.log(2e5), 256))).astype(int)
    dists = ("cube", "plummer", "sphere")
    xs, qs = [], []
    for i, n in enumerate(sizes):
        x, q = datasets.make(dists[i % 3], int(n), seed=1000 + i, precision="f32")
        xs.append(x)
        qs.append(q)
    idx = [datasets.sample_targets(len(q), 128) for q in qs]
    ref = [fmm.direct(x[k], x, q) for x, q, k in zip(xs, qs, idx)]
    for theta, bound in ((0.4, 5e-4), (0.3, 1e-4)):
        kw = dict(P=8, theta=theta, ncrit=64, use_ropt=0)
        batch = fmm.Solver(**kw).solve_batch(xs, qs)
        if theta == 0.4:
            alone = fmm.Solver(**kw)
            for i in (0, 1, 2, 100, 255):
                assert np.array_equal(batch[i], alone.solve(xs[i], qs[i])), i
        for i in range(len(xs)):
            pot, acc = rel_l2(batch[i][idx[i]], ref[i])
            assert pot < bound and acc < bound, (theta, i, dists[i % 3], len(qs[i]), pot, acc)


def test_serving_mixed_orders_meet_1e4(datasets):
    """Serving: requests of 2e4, 2e5 and 1e6 bodies at P = 6, 8 and 10,
    cube and Plummer, through the continuous-batching server with the opening angle per
    order (P = 6: 0.22, P = 8: 0.30, P = 10: 0.35): every request within rel-L2 1e-4 of
    potential and gradient against FP64 direct."""
    thetas = {6: 0.22, 8: 0.30, 10: 0.35}
    srv = fmm.Server(theta=0.4, ncrit=64, use_ropt=0, hbm_budget_gb=40.0, workers=2,
                     max_batch=8)
    for P, t in thetas.items():
        srv.set_theta(P, t)
    reqs, k = [], 0
    for n in (20000, 200000, 1000000):
        for P in (6, 8, 10):
            x, q = datasets.make(("cube", "plummer")[k % 2], n, seed=300 + k, precision="f32")
            reqs.append((x, q, P, srv.submit(x, q, P)))
            k += 1
    for x, q, P, rid in reqs:
        out, _, _ = srv.wait(rid)
        pot, acc = direct_error(datasets, x, q, out, 256)
        assert pot < 1e-4 and acc < 1e-4, (P, len(q), pot, acc)
    srv.close()