"""One FMM solve over the GPUs of one node: torch.distributed ranks (NCCL), one GPU each.

The reference spreads a solve over MPI ranks by an ORB partition of the bodies
(include/partition.h:69-195), the exchange of every rank's local essential tree
(include/tree_mpi.h:225-369) and traversals of the local tree against the remote ones.  On
one node of B200s, each with room for all the bodies, the exchange is replaced by two
collectives around one partitioned solve per GPU:

  1. all_gather of the ranks' bodies (x, y, z, q: 16 bytes a body in FP32), so that every
     rank holds all of them, in rank order;
  2. every rank builds the same tree and upward pass from the same bodies and computes the
     targets of its own part of them (Solver.set_partition(rank, world): the traversal keeps
     the pairs of that part's target cells, L2L and L2P run on that part's cells and bodies,
     every other body's result is 0);
  3. reduce_scatter (sum) of the results back to the ranks that own the bodies.  Each
     body's result comes from exactly one rank and the others add zeros, so every rank ends
     with the one-GPU solve's results for its own bodies, bit for bit.

The tree build and the upward pass are not divided; the traversal, M2L, P2P, L2L and L2P
are.
"""
import torch
import torch.distributed as dist

from . import Solver

__all__ = ["DistributedSolver"]


class DistributedSolver:
    """The FMM over the ranks of a process group, each rank on its own GPU.

    solve(bodies) takes this rank's bodies, a (n_local, 4) tensor of (x, y, z, q) on this
    rank's device in the working precision, and returns their (n_local, 4) results
    (phi, grad phi per unit charge) as the one-GPU solve of all ranks' bodies gives them.
    Every rank calls it with its own bodies at the same time (it runs collectives).

    compute(all_bodies, part, nparts) may replace the GPU solve (the host logic's tests run
    it on CPU ranks): it returns the (n, 4) results of the given part of the bodies and zeros
    for the others."""

    def __init__(self, group=None, compute=None, **solver_kwargs):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.solver = None
        if compute is None:
            self.solver = Solver(**solver_kwargs)
            self.solver.set_partition(self.rank, self.world)
            compute = self._gpu_compute
        self.compute = compute

    def _gpu_compute(self, all_bodies, part, nparts):
        trg = torch.empty_like(all_bodies)
        if all_bodies.shape[0]:
            self.solver.set_stream(torch.cuda.current_stream(all_bodies.device).cuda_stream)
            self.solver.solve_device(all_bodies.shape[0], all_bodies.data_ptr(),
                                     trg.data_ptr())
        return trg

    def gather_counts(self, n_local, device):
        """Bodies per rank (one small all_gather, read on the host)."""
        c = torch.tensor([n_local], dtype=torch.int64, device=device)
        out = torch.empty(self.world, dtype=torch.int64, device=device)
        dist.all_gather_into_tensor(out, c, group=self.group)
        return out.tolist()

    def solve(self, bodies):
        if bodies.dim() != 2 or bodies.shape[1] != 4:
            raise ValueError("bodies: (n, 4) tensor of x, y, z, q")
        bodies = bodies.contiguous()
        dev = bodies.device
        n_local = bodies.shape[0]
        counts = self.gather_counts(n_local, dev)
        nmax = max(counts)
        if nmax == 0:
            return torch.zeros_like(bodies)
        # every rank's bodies in one block of nmax rows (all_gather takes equal sizes)
        if n_local == nmax:
            pad = bodies
        else:
            pad = torch.zeros((nmax, 4), dtype=bodies.dtype, device=dev)
            pad[:n_local] = bodies
        gathered = torch.empty((self.world * nmax, 4), dtype=bodies.dtype, device=dev)
        dist.all_gather_into_tensor(gathered, pad, group=self.group)
        mine = torch.empty_like(pad)
        if all(c == nmax for c in counts):  # no padding: the gathered block is the bodies
            trg = self.compute(gathered, self.rank, self.world)
            dist.reduce_scatter_tensor(mine, trg, op=dist.ReduceOp.SUM, group=self.group)
            return mine
        rows = torch.cat([torch.arange(r * nmax, r * nmax + counts[r], device=dev)
                          for r in range(self.world)])
        all_bodies = gathered[rows].contiguous()  # rank order, the padding left out
        trg = self.compute(all_bodies, self.rank, self.world)
        out = torch.zeros_like(gathered)
        out[rows] = trg
        dist.reduce_scatter_tensor(mine, out, op=dist.ReduceOp.SUM, group=self.group)
        return mine[:n_local]
