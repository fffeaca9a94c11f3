"""z-slab sharding's host logic on CPU (timbir_b200/slab.py): the slab split
and its preconditions (XT_Engine.c:101-104), and the driver with its two
communicators -- torch.distributed over gloo with two processes, and threads
of one process -- around a stand-in stage that has the sharded stage's
interface and the same coupling (a quadratic data term per slice, a
quadratic prior between neighbouring slices, Gauss-Seidel sweeps over the
slab's slices, halo slices from the neighbours, cost and convergence sums
through the all-reduce).  A 2-rank solve must reach the whole-volume
solution and cost."""
import os
import socket
import threading

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from timbir_b200 import slab, synth  # noqa: E402

BETA = 0.7


class ChainStage:
    """Stand-in for a sharded Stage: per (frame, y, x) a chain over z with
    cost sum_z w (x - y)^2 + BETA sum_z (x_z - x_{z+1})^2, updated voxel by
    voxel in slice order (ICD), the neighbouring slabs' boundary slices as
    read-only halo neighbours."""

    def __init__(self, y, w):
        self.y, self.w = y.astype(np.float64), w.astype(np.float64)
        self.x = np.zeros_like(self.y)
        self.rank, self.ranks, self.red = 0, 1, None
        T, Z, Y, X = y.shape
        self.halo = [None, None]

    def set_z_slab(self, rank, ranks, allreduce):
        self.rank, self.ranks, self.red = rank, ranks, allreduce

    def _sum(self, v):
        v = np.asarray(v, np.float64)
        if self.ranks > 1:
            self.red(v)
        return v

    def slab_faces(self):
        return torch.from_numpy(self.x[:, 0].copy()), torch.from_numpy(self.x[:, -1].copy())

    def set_slab_halo(self, lo, hi):
        if lo is not None:
            self.halo[0] = lo.numpy().astype(np.float64)
        if hi is not None:
            self.halo[1] = hi.numpy().astype(np.float64)

    def prepare(self, obj=None, offset=None):
        if obj is not None:
            self.x = np.array(obj, np.float64)

    def iterate(self, it):
        Z = self.x.shape[1]
        dx = 0.0
        for z in range(Z):
            nb, cnt = np.zeros_like(self.x[:, z]), 0
            for zz in (z - 1, z + 1):
                if 0 <= zz < Z:
                    nb += self.x[:, zz]
                    cnt += 1
                elif zz < 0 and self.rank > 0:
                    nb += self.halo[0]
                    cnt += 1
                elif zz >= Z and self.rank < self.ranks - 1:
                    nb += self.halo[1]
                    cnt += 1
            new = (self.w[:, z] * self.y[:, z] + BETA * nb) / (self.w[:, z] + BETA * cnt)
            dx += float(np.abs(new - self.x[:, z]).sum())
            self.x[:, z] = new
        s = self._sum([dx, float(np.abs(self.x).sum())])
        return bool(s[0] / max(s[1], 1e-300) < 1e-12)

    def cost(self):
        c = float((self.w * (self.x - self.y) ** 2).sum())
        c += BETA * float(((self.x[:, 1:] - self.x[:, :-1]) ** 2).sum())
        if self.rank < self.ranks - 1:
            c += BETA * float(((self.x[:, -1] - self.halo[1]) ** 2).sum())
        return float(self._sum([c])[0])


def problem(seed=0, shape=(2, 8, 5, 6)):
    rng = np.random.default_rng(seed)
    return rng.normal(size=shape), rng.uniform(0.5, 2.0, size=shape)


def whole_solution(y, w, iters=400):
    st = ChainStage(y, w)
    for it in range(1, iters + 1):
        st.iterate(it)
    return st.x, st.cost()


def test_split_scan_and_preconditions():
    sc = synth.Scan(np.arange(3 * 8 * 4, dtype=np.float32).reshape(3, 8, 4), np.ones((3, 8, 4), np.float32),
                    np.zeros(3, np.float32), np.arange(3, dtype=np.float32), np.array([0, 3], np.float32),
                    8, 4, 3, 1, 1.0, 2.0, np.zeros((1, 8, 4, 4), np.float32))
    parts = [slab.split_scan(sc, r, 2) for r in range(2)]
    assert all(p.proj_rows == 4 and p.projections.shape == (3, 4, 4) for p in parts)
    assert np.array_equal(np.concatenate([p.projections for p in parts], axis=1), sc.projections)
    assert parts[1].phantom.shape == (1, 4, 4, 4)
    assert slab.check_slab_split(8, 4) == 2
    for rows, ranks in ((8, 3), (6, 2), (8, 8)):  # not divisible, odd rows per slab, fewer than 2
        with pytest.raises(ValueError):
            slab.check_slab_split(rows, ranks)


def test_threads_reach_the_whole_volume_solution():
    y, w = problem(1)
    x_ref, c_ref = whole_solution(y, w)
    comm = slab.ThreadComm(2, timeout=30)
    out, costs = [None, None], [None, None]

    def run(rank):
        st = ChainStage(slab.split_volume(y, rank, 2), slab.split_volume(w, rank, 2))
        s = slab.SlabSolver(st, comm.for_rank(rank))
        s.prepare()
        for it in range(1, 401):
            s.iterate(it)
        out[rank], costs[rank] = st.x, s.cost()

    th = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert np.allclose(np.concatenate(out, axis=1), x_ref, atol=1e-9)
    assert costs[0] == costs[1]
    assert abs(costs[0] - c_ref) <= 1e-9 * c_ref


def _gloo_rank(rank, port, y, w, result_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        comm = slab.TorchComm("cpu")
        st = ChainStage(slab.split_volume(y, rank, 2), slab.split_volume(w, rank, 2))
        s = slab.SlabSolver(st, comm)
        s.prepare()
        for it in range(1, 401):
            s.iterate(it)
        c = s.cost()
        parts = [torch.zeros(st.x.shape, dtype=torch.float64) for _ in range(2)]
        dist.all_gather(parts, torch.from_numpy(st.x))
        if rank == 0:
            np.savez(result_path, x=np.concatenate([p.numpy() for p in parts], axis=1), cost=c)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gloo_two_ranks_reach_the_whole_volume_solution(tmp_path):
    import torch.multiprocessing as mp
    y, w = problem(2)
    x_ref, c_ref = whole_solution(y, w)
    path = str(tmp_path / "slab.npz")
    mp.start_processes(_gloo_rank, args=(_free_port(), y, w, path), nprocs=2, join=True, start_method="spawn")
    r = np.load(path)
    assert np.allclose(r["x"], x_ref, atol=1e-9)
    assert abs(float(r["cost"]) - c_ref) <= 1e-9 * c_ref


def test_gloo_exchange_directions(tmp_path):
    import torch.multiprocessing as mp
    path = str(tmp_path / "ex.npz")
    mp.start_processes(_gloo_exchange, args=(_free_port(), path), nprocs=3, join=True, start_method="spawn")
    r = np.load(path)
    # rank r's faces are filled with 10 r (bottom) and 10 r + 1 (top)
    assert r["lo"].tolist() == [-1, 1, 11]   # halo_lo of rank r = rank r - 1's top face
    assert r["hi"].tolist() == [10, 20, -1]  # halo_hi of rank r = rank r + 1's bottom face
    assert r["sum"].tolist() == [3.0, 30.0]


def _gloo_exchange(rank, port, path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=3)
    try:
        comm = slab.TorchComm("cpu")
        lo = torch.full((2, 3), 10.0 * rank)
        hi = torch.full((2, 3), 10.0 * rank + 1)
        hl, hh = comm.exchange(lo, hi)
        v = np.array([1.0, 10.0 * rank])
        comm.allreduce(v)
        got = torch.tensor([hl[0, 0].item() if hl is not None else -1, hh[0, 0].item() if hh is not None else -1])
        allg = [torch.zeros(2) for _ in range(3)]
        dist.all_gather(allg, got)
        if rank == 0:
            a = torch.stack(allg).numpy()
            np.savez(path, lo=a[:, 0].astype(int), hi=a[:, 1].astype(int), sum=v)
    finally:
        dist.destroy_process_group()
