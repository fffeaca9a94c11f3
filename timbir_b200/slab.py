"""z-slab sharding of one reconstruction over ranks (the reference's MPI
decomposition, TIMBIR src/MBIR_4D/XT_MPI.c:47-122 and XT_Engine.c:93-104).

Each rank holds a contiguous slab of detector rows and the matching slab of
slices (the sinogram is row-disjoint between slabs, so the data term
separates); the prior couples the slabs through one boundary slice per frame
on each side.  Per rank: a :class:`timbir_b200.Stage` built from its rows,
made slab `rank` of `ranks` (its cost, variance and convergence sums go
through the communicator's all-reduce, as the reference's MPI_Reduce /
MPI_Allreduce calls do), and after the prologue and after every ICD
iteration its boundary slices go to its neighbours' halos (the reference's
MPI_Send_Recv_Z_Slices / MPI_Wait_Z_Slices, which it runs between half-sweeps
of an iteration; here between iterations, one sweep of the super-voxel
schedule covering every voxel once).

Communicators:

* :class:`TorchComm` -- torch.distributed (NCCL between GPUs, gloo on CPU):
  the all-reduce of a few doubles, and the halo exchange as point-to-point
  sends and receives of the boundary slices.
* :class:`ThreadComm` -- ranks run as threads of one process (several slabs on
  one GPU, e.g. to check that a sharded solve reaches the whole volume's MAP
  estimate): the same two operations through shared memory and a barrier.
  No kernel of one rank waits on another rank's kernels; ranks meet only on
  the host, between launches.
"""
from __future__ import annotations

import threading

import numpy as np

from . import synth


def check_slab_split(proj_rows: int, ranks: int) -> int:
    """Rows per slab; the reference's preconditions (XT_Engine.c:101-104):
    proj_rows divisible by the ranks, an even number of rows per slab, at
    least 2."""
    if ranks < 1:
        raise ValueError("ranks must be at least 1")
    if proj_rows % ranks:
        raise ValueError(f"proj_rows = {proj_rows} is not divisible by {ranks} ranks")
    r = proj_rows // ranks
    if r < 2 or r % 2:
        raise ValueError(f"{r} detector rows per slab: must be even and at least 2")
    return r


def split_scan(scan: synth.Scan, rank: int, ranks: int) -> synth.Scan:
    """Slab `rank` of a scan: detector rows [rank r, (rank + 1) r) of the
    projections and weights (layout [views][rows][cols], as each MPI rank of
    the reference reads its slab, bin_data/XT_Main.c:126-134), the phantom's
    matching slices."""
    r = check_slab_split(scan.proj_rows, ranks)
    sl = slice(rank * r, (rank + 1) * r)
    ph = None if scan.phantom is None else np.ascontiguousarray(scan.phantom[:, sl])
    return synth.Scan(np.ascontiguousarray(scan.projections[:, sl]), np.ascontiguousarray(scan.weights[:, sl]),
                      scan.proj_angles, scan.proj_times, scan.recon_times, r, scan.proj_cols, scan.proj_num,
                      scan.recon_num, scan.vox_wid, scan.rot_center, ph)


def split_volume(x: np.ndarray, rank: int, ranks: int) -> np.ndarray:
    """Slices of slab `rank` of an object [N_time][N_z][N_y][N_x]."""
    n = x.shape[1] // ranks
    return np.ascontiguousarray(x[:, rank * n:(rank + 1) * n])


class TorchComm:
    """torch.distributed communicator of the slab ranks (the default group,
    or `group`).  Tensors live on `device` (a CUDA device for NCCL, "cpu" for
    gloo)."""

    def __init__(self, device=None, group=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.ranks = dist.get_world_size(group)
        if device is None:
            device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        self.device = torch.device(device)

    def allreduce(self, v: np.ndarray) -> None:
        t = self.torch.from_numpy(np.array(v, np.float64)).to(self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        v[:] = t.cpu().numpy()

    def exchange(self, lo, hi):
        """Send this rank's bottom face `lo` to rank - 1 and its top face `hi`
        to rank + 1; returns (halo_lo, halo_hi): rank - 1's top face and
        rank + 1's bottom face (None at the ends)."""
        torch, dist = self.torch, self.dist
        lo = lo.to(self.device).contiguous()
        hi = hi.to(self.device).contiguous()
        halo_lo = torch.empty_like(lo) if self.rank > 0 else None
        halo_hi = torch.empty_like(hi) if self.rank < self.ranks - 1 else None
        peer = lambda r: r if self.group is None else dist.get_global_rank(self.group, r)  # noqa: E731
        ops = []
        if self.rank > 0:
            ops.append(dist.P2POp(dist.isend, lo, peer(self.rank - 1), self.group))
            ops.append(dist.P2POp(dist.irecv, halo_lo, peer(self.rank - 1), self.group))
        if self.rank < self.ranks - 1:
            ops.append(dist.P2POp(dist.isend, hi, peer(self.rank + 1), self.group))
            ops.append(dist.P2POp(dist.irecv, halo_hi, peer(self.rank + 1), self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return halo_lo, halo_hi


class ThreadComm:
    """Communicator of `ranks` slab ranks run as threads of one process.
    Every rank makes the same calls in the same order; each call meets the
    other ranks at a barrier (timeout: seconds a rank waits for the others
    before the call fails)."""

    def __init__(self, ranks: int, timeout: float = 120.0):
        self.ranks = ranks
        self.barrier = threading.Barrier(ranks, timeout=timeout)
        self.slots = [None] * ranks

    def for_rank(self, rank: int) -> "ThreadComm.Rank":
        return ThreadComm.Rank(self, rank)

    class Rank:
        def __init__(self, comm, rank):
            self.c, self.rank, self.ranks = comm, rank, comm.ranks

        def allreduce(self, v: np.ndarray) -> None:
            c = self.c
            c.slots[self.rank] = np.array(v, np.float64)
            c.barrier.wait()
            s = np.zeros_like(c.slots[self.rank])
            for r in range(c.ranks):  # the same order on every rank: identical sums
                s += c.slots[r]
            c.barrier.wait()
            v[:] = s

        def exchange(self, lo, hi):
            c = self.c
            c.slots[self.rank] = (lo, hi)
            c.barrier.wait()
            halo_lo = c.slots[self.rank - 1][1].clone() if self.rank > 0 else None
            halo_hi = c.slots[self.rank + 1][0].clone() if self.rank < c.ranks - 1 else None
            c.barrier.wait()
            return halo_lo, halo_hi


class SlabSolver:
    """One rank's share of a sharded stage: `stage` holds slab `rank` of
    `comm.ranks` (built from split_scan's rows).  prepare() and iterate()
    drive it and keep the halos current."""

    def __init__(self, stage, comm):
        self.stage, self.comm = stage, comm
        self.rank, self.ranks = comm.rank, comm.ranks
        stage.set_z_slab(self.rank, self.ranks, comm.allreduce)

    def exchange(self) -> None:
        lo, hi = self.stage.slab_faces()
        halo_lo, halo_hi = self.comm.exchange(lo, hi)
        if self.ranks > 1:
            if lo.is_cuda:  # the stage copies the halos on its own stream
                import torch
                torch.cuda.current_stream().synchronize()
            self.stage.set_slab_halo(halo_lo, halo_hi)

    def prepare(self, obj=None, offset=None) -> None:
        self.stage.prepare(obj, offset)
        self.exchange()

    def iterate(self, it: int) -> bool:
        converged = self.stage.iterate(it)
        self.exchange()
        return converged

    def cost(self):
        """The whole volume's MAP cost (every rank gets the same)."""
        return self.stage.cost()
