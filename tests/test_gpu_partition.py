"""A solve split over GPUs by target parts (fmm_b200_set_partition), its parts run in turn on
one GPU: the parts' body ranges tile the tree's bodies at leaf starts, each part's result is
0 outside its bodies, and the sum of the parts' results equals the whole solve bit for bit
(each body's result comes from one part; the reduction that joins the GPUs adds zeros).
The tree, the upward pass and the traversal's pairs of each target are those of the whole
solve, so nothing may differ.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
fmm = importlib.import_module("exafmm-dev_b200")


def parts_of(s, x, q, nparts):
    outs, ranges = [], []
    for r in range(nparts):
        s.set_partition(r, nparts)
        outs.append(s.solve(x, q))
        part, np_, b, e = s.partition()
        assert (part, np_) == (r, nparts)
        ranges.append((b, e))
    s.set_partition(0, 1)
    return outs, ranges


def check_parts(s, x, q, nparts):
    n = len(q)
    whole = s.solve(x, q)
    outs, ranges = parts_of(s, x, q, nparts)
    # ranges tile [0, n) in order, each cut at the start of a leaf
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (b0, e0), (b1, e1) in zip(ranges, ranges[1:]):
        assert e0 == b1 and b0 <= e0
    cells = s.cells()
    leaf = cells["nchild"] == 0
    starts = set(cells["ibody"][leaf].tolist()) | {n}
    assert all(b in starts for b, _ in ranges)
    # each part: zero outside its bodies (tree order -> caller order through get_order)
    order = s.order()
    total = np.zeros_like(whole)
    for (b, e), o in zip(ranges, outs):
        mine = np.zeros(n, bool)
        mine[order[b:e]] = True
        assert not np.any(o[~mine]), "results outside the part"
        total += o
    assert np.array_equal(total, whole)
    return ranges


@pytest.mark.parametrize("basis,P,prec,tree", [
    ("spherical", 10, "f32", "adaptive"), ("spherical", 8, "f64", "adaptive"),
    ("cartesian", 5, "f32", "adaptive"), ("spherical", 6, "f32", "uniform"),
    ("cartesian", 4, "f64", "uniform")])
@pytest.mark.parametrize("nparts", [2, 3, 8])
def test_parts_sum_to_the_whole_solve(basis, P, prec, tree, nparts, datasets):
    x, q = datasets.make("plummer", 20000, seed=11, precision=prec)
    s = fmm.Solver(basis=basis, P=P, theta=0.4, ncrit=32, precision=prec, tree=tree)
    ranges = check_parts(s, x, q, nparts)
    c = s.cells()
    maxleaf = int(c["nbody"][c["nchild"] == 0].max())
    sizes = [e - b for b, e in ranges]
    assert max(sizes) <= -(-len(q) // nparts) + maxleaf  # each cut within a leaf of k n / nparts


def test_parts_periodic(datasets):
    x, q = datasets.make("cube", 8000, seed=3, precision="f64")
    s = fmm.Solver(P=6, theta=0.4, ncrit=32, precision="f64", images=2, cycle=2.0)
    check_parts(s, x, q, 4)


def test_parts_lists_are_the_whole_lists_of_their_targets(datasets):
    """Every part's M2L and P2P pairs are the whole traversal's pairs of the part's target
    cells, and the parts' lists together are the whole lists."""
    x, q = datasets.make("plummer", 12000, seed=4, precision="f32")
    s = fmm.Solver(P=8, theta=0.35, ncrit=32, precision="f32")
    s.solve(x, q)
    m2l, p2p = s.lists()
    got_m, got_p = [], []
    for r in range(3):
        s.set_partition(r, 3)
        s.solve(x, q)
        m, p = s.lists()
        got_m.append(m)
        got_p.append(p)
    s.set_partition(0, 1)
    # a cell that straddles a cut is a target of both parts: compare as sets
    assert np.array_equal(np.unique(np.concatenate(got_m)), np.unique(m2l))
    assert np.array_equal(np.unique(np.concatenate(got_p)), np.unique(p2p))
    assert sum(len(m) for m in got_m) >= len(m2l)
    assert sum(len(p) for p in got_p) == len(p2p)  # leaves belong to one part


def test_more_parts_than_leaves(datasets):
    x, q = datasets.make("cube", 40, seed=2, precision="f64")
    s = fmm.Solver(P=6, ncrit=64, precision="f64")  # one leaf: every part but one is empty
    whole = s.solve(x, q)
    outs, ranges = parts_of(s, x, q, 5)
    assert np.array_equal(sum(outs), whole)
    assert sorted(e - b for b, e in ranges)[-1] == 40


def test_partition_rejects(datasets):
    x, q = datasets.make("cube", 2000, seed=1, precision="f64")
    s = fmm.Solver(P=6, precision="f64")
    with pytest.raises(fmm.FmmError):
        s.set_partition(2, 2)
    with pytest.raises(fmm.FmmError):
        s.set_partition(0, 0)
    s.set_partition(1, 2)
    with pytest.raises(fmm.FmmError) as e:
        s.solve_batch([x[:1000], x[1000:]], [q[:1000], q[1000:]])
    assert e.value.code == fmm.FMM_ERR_NOT_SUPPORTED
    sm = fmm.Solver(P=6, precision="f64", mutual=1)
    sm.set_partition(0, 2)
    with pytest.raises(fmm.FmmError) as e:
        sm.solve(x, q)
    assert e.value.code == fmm.FMM_ERR_NOT_SUPPORTED


def test_distributed_solver_one_rank(datasets):
    """DistributedSolver on its GPU path with NCCL, one rank: the all_gather, the partitioned
    solve and the reduce_scatter give the plain solve's result bit for bit."""
    import socket

    import torch
    import torch.distributed as dist

    dmod = importlib.import_module("exafmm-dev_b200.distributed")
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1, device_id=torch.device("cuda", 0))
    try:
        x, q = datasets.make("plummer", 30000, seed=8, precision="f32")
        b = torch.tensor(np.concatenate([x, q[:, None]], 1), dtype=torch.float32, device="cuda")
        ds = dmod.DistributedSolver(P=8, theta=0.35, ncrit=32, precision="f32")
        got = ds.solve(b)
        s = fmm.Solver(P=8, theta=0.35, ncrit=32, precision="f32")
        want = torch.empty_like(b)
        s.solve_device(len(q), b.data_ptr(), want.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(got, want)
    finally:
        dist.destroy_process_group()
