"""The host side of a solve spread over ranks (exafmm-dev_b200.distributed), on CPU ranks
with the gloo backend: the bodies' all_gather with ranks of unequal (and zero) body counts,
the part each rank computes, and the reduce_scatter that returns every body's result to
its owner.  The GPU solve is replaced by a direct sum over the gathered bodies that
computes one contiguous part of the targets and zeros for the rest, as a partitioned
handle does; each rank must end with the direct sum at its own bodies."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def direct(xt, xs, qs):
    d = xt[:, None, :] - xs[None, :, :]
    r2 = (d * d).sum(-1)
    inv = np.where(r2 > 0, 1.0 / np.sqrt(np.where(r2 > 0, r2, 1.0)), 0.0)
    pot = (qs[None, :] * inv).sum(1)
    grad = -(qs[None, :, None] * d * (inv ** 3)[:, :, None]).sum(1)
    return np.concatenate([pot[:, None], grad], 1)


def fake_part(all_bodies, part, nparts):
    b = all_bodies.numpy()
    n = len(b)
    lo, hi = part * n // nparts, (part + 1) * n // nparts
    out = np.zeros_like(b)
    out[lo:hi] = direct(b[lo:hi, :3], b[:, :3], b[:, 3])
    return torch.from_numpy(out)


def bodies_of(rank, counts, seed=7):
    rng = np.random.default_rng(seed + rank)
    n = counts[rank]
    return np.concatenate([rng.uniform(-1, 1, (n, 3)), rng.uniform(0.1, 1, (n, 1))], 1)


def worker(rank, world, port, counts, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mod = importlib.import_module("exafmm-dev_b200.distributed")
        ds = mod.DistributedSolver(compute=fake_part)
        mine = bodies_of(rank, counts)
        got = ds.solve(torch.from_numpy(mine)).numpy()
        everything = np.concatenate([bodies_of(r, counts) for r in range(world)])
        want = direct(mine[:, :3], everything[:, :3], everything[:, 3])
        ok = got.shape == want.shape and np.allclose(got, want, rtol=1e-12, atol=0)
        q.put((rank, bool(ok), float(np.abs(got - want).max()) if len(want) else 0.0))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("counts", [[300, 300], [250, 0, 411], [1, 2, 3, 500]])
def test_distributed_solve_host_logic(counts):
    world = len(counts)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, counts, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, err in sorted(res):
        assert ok, (rank, err)
