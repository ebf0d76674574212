"""Batched solves (forest of independent trees) and the continuous-batching server.

The property tested throughout: a solve's result does not depend on what it is batched
with — it is bitwise the result it gets alone — and matches the oracle.
"""
import importlib
import threading
import time

import numpy as np
import pytest

from oracle import SPHERICAL, Oracle, rel_l2

pytestmark = pytest.mark.gpu
fmm = importlib.import_module("exafmm-dev_b200")


def mixed_solves(datasets, sizes, seed=0, precision="f32"):
    dists = ("cube", "plummer", "sphere")
    out = []
    for i, n in enumerate(sizes):
        if n == 0:  # an empty solve in the batch
            out.append((np.zeros((0, 3)), np.zeros(0)))
            continue
        x, q = datasets.make(dists[i % 3], n, seed=seed + i, precision=precision)
        out.append((x, q))
    return out


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_batch_bitwise_equals_alone(prec, datasets):
    sizes = [1500, 20000, 7, 64, 65, 3000, 50000, 1, 999]
    solves = mixed_solves(datasets, sizes, precision=prec)
    s = fmm.Solver(P=8, theta=0.4, ncrit=64, precision=prec)
    batch = s.solve_batch([x for x, _ in solves], [q for _, q in solves])
    alone = fmm.Solver(P=8, theta=0.4, ncrit=64, precision=prec)
    for (x, q), got in zip(solves, batch):
        ref = alone.solve(x, q)
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        ok = ~np.isnan(ref)
        assert np.array_equal(got[ok], ref[ok])


def test_batch_cells_are_the_alone_trees(datasets):
    sizes = [5000, 0, 12000, 300]
    solves = mixed_solves(datasets, sizes, seed=3)
    s = fmm.Solver(P=6, theta=0.4, ncrit=32, use_ropt=0)
    counts = np.array(sizes, np.int32)
    x = np.concatenate([a for a, _ in solves])
    q = np.concatenate([b for _, b in solves])
    s.set_bodies(x, q)
    # batch through the C ABI stages: set the segments with a batch solve, then inspect
    s.solve_batch([a for a, _ in solves], [b for _, b in solves])
    roots, rsolve = s.roots()
    assert list(rsolve) == [0, 2, 3]  # the empty solve has no root
    cells = s.cells()
    alone = fmm.Solver(P=6, theta=0.4, ncrit=32, use_ropt=0)
    bounds = list(roots) + [len(cells["nbody"])]
    body0 = np.concatenate([[0], np.cumsum(counts)])
    for r, sv in enumerate(rsolve):
        xa, qa = solves[sv]
        alone.set_bodies(xa, qa)
        alone.build_tree()
        ca = alone.cells()
        lo, hi = bounds[r], bounds[r + 1]
        assert hi - lo == len(ca["nbody"])
        assert np.array_equal(cells["nbody"][lo:hi], ca["nbody"])
        assert np.array_equal(cells["nchild"][lo:hi], ca["nchild"])
        assert np.array_equal(cells["X"][lo:hi], ca["X"])
        assert np.array_equal(cells["ibody"][lo:hi] - body0[sv], ca["ibody"])
        internal = ca["nchild"] > 0
        assert np.array_equal(cells["ichild"][lo:hi][internal] - lo, ca["ichild"][internal])
        assert np.array_equal(cells["iparent"][lo:hi] - lo, ca["iparent"])


def test_batch_matches_oracle(datasets):
    sizes = [4000, 9000, 2500]
    solves = mixed_solves(datasets, sizes, seed=9, precision="f64")
    s = fmm.Solver(P=8, theta=0.4, ncrit=48, precision="f64")
    batch = s.solve_batch([x for x, _ in solves], [q for _, q in solves])
    o = Oracle("f64")
    for (x, q), got in zip(solves, batch):
        ref = o.run(x, q, basis=SPHERICAL, P=8, theta=0.4, ncrit=48, use_ropt=1).trg()
        pot, acc = rel_l2(got, ref)
        assert pot < 1e-10 and acc < 1e-10, (pot, acc)


def test_server_mixed_orders_bitwise_and_latency(datasets):
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(40):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(60000))))
        P = int(rng.choice([6, 8, 10]))
        x, q = datasets.make(("cube", "plummer")[i % 2], n, seed=100 + i, precision="f32")
        reqs.append((x, q, P))
    srv = fmm.Server(theta=0.4, ncrit=64, hbm_budget_gb=8.0, workers=3, max_batch=16)
    ids = []
    # submit from two threads while batches are running
    lock = threading.Lock()

    def submit(part):
        for k in part:
            x, q, P = reqs[k]
            rid = srv.submit(x, q, P)
            with lock:
                ids.append((k, rid))
            time.sleep(0.001)

    t1 = threading.Thread(target=submit, args=(range(0, 40, 2),))
    t2 = threading.Thread(target=submit, args=(range(1, 40, 2),))
    t1.start(); t2.start(); t1.join(); t2.join()
    results = {}
    for k, rid in ids:
        out, lat, que = srv.wait(rid)
        assert lat > 0 and 0 <= que <= lat
        results[k] = out
    st = srv.stats()
    assert st["completed"] == 40 and st["pending"] == 0 and 1 <= st["batches"] <= 40
    srv.close()
    solvers = {}
    for k, (x, q, P) in enumerate(reqs):
        s = solvers.setdefault(P, fmm.Solver(P=P, theta=0.4, ncrit=64))
        ref = s.solve(x, q)
        got = results[k]
        ok = ~np.isnan(ref)
        assert np.array_equal(got[ok], ref[ok]), k


def test_server_rejects_requests_beyond_budget(datasets):
    srv = fmm.Server(hbm_budget_gb=0.001, workers=1)
    x, q = datasets.make("cube", 200000, precision="f32")
    with pytest.raises(fmm.FmmError) as e:
        srv.submit(x, q, 8)
    assert e.value.code == fmm.FMM_ERR_NO_MEMORY
    with pytest.raises(fmm.FmmError):
        srv.submit(x[:10], q[:10], 3)  # order not compiled
    srv.close()


@pytest.mark.parametrize("basis,prec,orders", [("cartesian", "f32", (4, 5)),
                                                ("spherical", "f64", (6, 8))])
def test_server_other_bases_and_precisions(basis, prec, orders, datasets):
    """The serving loop on the Cartesian basis (whose compiled orders do not include the
    configuration's default P = 10) and in FP64: every result bitwise the same request
    solved alone."""
    rng = np.random.default_rng(9)
    reqs = []
    for i in range(12):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(30000))))
        P = int(orders[i % len(orders)])
        x, q = datasets.make(("cube", "plummer")[i % 2], n, seed=700 + i, precision=prec)
        reqs.append((x, q, P))
    srv = fmm.Server(basis=basis, theta=0.45, ncrit=32, use_ropt=0, precision=prec,
                     hbm_budget_gb=8.0, workers=2, max_batch=8)
    ids = [(k, srv.submit(x, q, P)) for k, (x, q, P) in enumerate(reqs)]
    results = {k: srv.wait(rid)[0] for k, rid in ids}
    srv.trim()  # frees the grown-out buffers; the handles stay usable
    x, q, P = reqs[-1]
    again = srv.wait(srv.submit(x, q, P))[0]
    ok = ~np.isnan(again)
    assert np.array_equal(again[ok], results[len(reqs) - 1][ok])
    srv.close()
    solvers = {}
    for k, (x, q, P) in enumerate(reqs):
        s = solvers.setdefault(P, fmm.Solver(basis=basis, P=P, theta=0.45, ncrit=32,
                                             use_ropt=0, precision=prec))
        ref = s.solve(x, q)
        ok = ~np.isnan(ref)
        assert np.array_equal(results[k][ok], ref[ok]), k
