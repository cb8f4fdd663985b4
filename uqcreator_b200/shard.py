"""Spatial sharding of one mesh: a rank per GPU, each with its own block of
cells and a one-ring halo (uqc_partition).

The reference runs its time loop on every MPI rank over all cells: each rank
solves the duals of its round-robin cells, broadcasts every cell's duals,
reduces the moments of its slice of quadrature nodes onto the cell's owner
and takes the step as an all-reduce MIN (MomentSolver::Solve,
code/src/momentsolver.cpp:83-152). That is O(cells) collectives per step.
Here a rank keeps only its cells and their halo, and a time step is

    closure of the owned cells                 uqc_step_phase(h, 0)
    all-reduce MIN of the step (8 bytes)       dt bits as int64
    halo exchange of the nodal states          uqc_halo_pack + send / recv
    flux and update of the owned cells         uqc_step_phase(h, 1)

with the residual all-reduced (SUM) only where the minResidual stopping rule
needs it. Everything is issued on the handle's stream, so the collectives of
NCCL order themselves after the closure and before the update without a host
synchronisation.

Two drivers share the Shard class:
  ShardedSolver   one shard per process over torch.distributed (NCCL on GPUs;
                  gloo works for the exchange of host tensors);
  LocalShards     several shards of one mesh in one process, exchanging by
                  device copies (one GPU standing in for several ranks; the
                  kernels never wait on one another).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from ._lib import ShardInfo, StepInfo, check
from .solver import Solver

__all__ = ["Shard", "ShardedSolver", "LocalShards", "shard_plan", "exchange"]


def shard_plan(solver: Solver) -> dict:
    """The shard plan of a (partitioned) handle: uqc_get_shard as numpy arrays."""
    info = ShardInfo()
    lib = solver.lib
    check(solver.h, lib.uqc_get_shard(solver.h, C.byref(info), None, None, None, None, None))
    n_local = info.n_owned + info.n_halo
    gid = np.zeros(n_local, dtype=np.int32)
    peers = np.zeros(info.n_peers, dtype=np.int32)
    sc = np.zeros(info.n_peers, dtype=np.int32)
    rc = np.zeros(info.n_peers, dtype=np.int32)
    cells = np.zeros(info.n_send, dtype=np.int32)
    check(solver.h, lib.uqc_get_shard(solver.h, C.byref(info), L.ptr(gid, L._ip), L.ptr(peers, L._ip),
                                      L.ptr(sc, L._ip), L.ptr(rc, L._ip), L.ptr(cells, L._ip)))
    d = info.as_dict()
    d.update(global_ids=gid, peers=peers, send_counts=sc, recv_counts=rc, send_cells=cells)
    return d


def _device_view(ptr: int, n: int, typestr: str):
    import torch

    class _Mem:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False), "version": 2,
                                    "strides": None}

    return torch.as_tensor(_Mem(), device="cuda")


def exchange(dist, group, peers, sends, recvs):
    """Point-to-point exchange with each peer (global ranks of `group`): sends[i]
    goes to peers[i], recvs[i] is filled from it. Empty tensors are skipped."""
    ops = []
    for p, s, r in zip(peers, sends, recvs):
        g = int(p) if group is None else dist.get_global_rank(group, int(p))
        if s.numel():
            ops.append(dist.P2POp(dist.isend, s, g, group))
        if r.numel():
            ops.append(dist.P2POp(dist.irecv, r, g, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class Shard:
    """One rank's part of a mesh: a partitioned Solver handle plus device views
    of its exchange buffers (set up by init_state)."""

    def __init__(self, settings, rank: int, n_ranks: int, stream=None, precision: int | None = None):
        self.solver = s = Solver(settings, stream)
        check(s.h, s.lib.uqc_partition(s.h, int(rank), int(n_ranks)))
        self.plan = shard_plan(s)
        s.n_cells = self.plan["n_owned"] + self.plan["n_halo"]
        self.rank, self.n_ranks = int(rank), int(n_ranks)
        self.n_owned = self.plan["n_owned"]
        self._precision = precision
        self.send = None

    # ---- set-up
    def init_state(self):
        import torch
        s = self.solver
        if self._precision is not None:
            s.set_precision(self._precision)
        s.init_state()
        row = self.plan["row_doubles"]
        halo, dtb, res = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(s.h, s.lib.uqc_shard_buffers(s.h, C.byref(halo), C.byref(dtb), C.byref(res)))
        self.dt_bits = _device_view(dtb.value, 1, "<i8")
        self.residual = _device_view(res.value, 1, "<f8")
        n_halo = self.plan["n_halo"]
        self.halo = _device_view(halo.value, n_halo * row, "<f8") if n_halo else torch.zeros(0, dtype=torch.float64,
                                                                                               device="cuda")
        self.send = torch.empty(self.plan["n_send"] * row, dtype=torch.float64, device="cuda")
        so = np.concatenate([[0], np.cumsum(self.plan["send_counts"])]) * row
        ro = np.concatenate([[0], np.cumsum(self.plan["recv_counts"])]) * row
        self.send_parts = [self.send[so[i]:so[i + 1]] for i in range(len(self.plan["peers"]))]
        self.recv_parts = [self.halo[ro[i]:ro[i + 1]] for i in range(len(self.plan["peers"]))]
        self.stream = torch.cuda.ExternalStream(s.stream())

    # ---- the halves of a step
    def closure(self):
        s = self.solver
        check(s.h, s.lib.uqc_step_phase(s.h, 0, None))

    def pack(self):
        s = self.solver
        if self.send.numel():
            check(s.h, s.lib.uqc_halo_pack(s.h, C.c_void_p(self.send.data_ptr())))

    def update(self, info: StepInfo | None = None):
        s = self.solver
        rc = s.lib.uqc_step_phase(s.h, 1, None if info is None else C.byref(info))
        check(s.h, rc)

    def close(self):
        self.send = None
        self.solver.close()

    # ---- results
    def owned_mean_var(self):
        """(global ids, E and Var per state) of the owned cells."""
        mv = self.solver.mean_var()
        return self.plan["global_ids"][: self.n_owned], mv[: self.n_owned]

    def owned_state(self):
        """(global ids, u, lambda) of the owned cells (state-major)."""
        u, lam, _ = self.solver.download_state()
        n = self.n_owned
        return self.plan["global_ids"][:n], u[:n], lam[:n]


class ShardedSolver:
    """This process's shard of a mesh split over the ranks of a torch.distributed
    process group (NCCL over NVLink for GPU ranks). All ranks call every method
    in the same order."""

    def __init__(self, settings, group=None, stream=None, precision: int | None = None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        rank, n = dist.get_rank(group), dist.get_world_size(group)
        self.shard = Shard(settings, rank, n, stream, precision)

    def init_state(self):
        self.shard.init_state()

    def step(self, n_steps: int = 1, with_info: bool = False):
        """n_steps time steps with no host synchronisation; with_info: wait for
        the last one and return this rank's step info (uqc_step_info; its
        residual is the rank's part)."""
        import torch
        sh, dist = self.shard, self.dist
        info = StepInfo() if with_info else None
        with torch.cuda.stream(sh.stream):
            for k in range(n_steps):
                sh.closure()
                dist.all_reduce(sh.dt_bits, op=dist.ReduceOp.MIN, group=self.group)
                sh.pack()
                exchange(dist, self.group, sh.plan["peers"], sh.send_parts, sh.recv_parts)
                sh.update(info if k == n_steps - 1 else None)
        return None if info is None else info.as_dict()

    def close(self):
        self.shard.close()

    def residual(self) -> float:
        """The last step's residual summed over the ranks (momentsolver.cpp:149-152)."""
        import torch
        with torch.cuda.stream(self.shard.stream):
            r = self.shard.residual.clone()
            self.dist.all_reduce(r, op=self.dist.ReduceOp.SUM, group=self.group)
        return float(r.item())

    def gather_mean_var(self, dst: int = 0):
        """E and Var of every cell in global order on rank dst (None elsewhere)."""
        import torch
        gid, mv = self.shard.owned_mean_var()
        parts = [None] * self.dist.get_world_size(self.group)
        self.dist.all_gather_object(parts, (gid, mv), group=self.group)
        if self.dist.get_rank(self.group) != dst:
            return None
        n = self.shard.plan["n_global"]
        out = np.zeros((n, mv.shape[1]))
        for g, m in parts:
            out[g] = m
        return out


class LocalShards:
    """n_shards shards of one mesh in this process, on one stream of the
    current device, stepped in lockstep: each step runs every shard's closure,
    takes the smallest step of all, copies the halo rows between shards and
    runs every shard's update. For a mesh split over more ranks than there
    are GPUs, and for checking a partition against the unsplit mesh."""

    def __init__(self, settings, n_shards: int, precision: int | None = None):
        import torch
        self.stream = torch.cuda.Stream()
        self.shards = [Shard(settings, r, n_shards, self.stream.cuda_stream, precision) for r in range(n_shards)]

    def init_state(self):
        for sh in self.shards:
            sh.init_state()

    def step(self, n_steps: int = 1, with_info: bool = False):
        """n_steps lockstep time steps (waits for them); with_info: the step
        info of every shard's last step."""
        import torch
        infos = [StepInfo() for _ in self.shards] if with_info else None
        with torch.cuda.stream(self.stream):
            for k in range(n_steps):
                for sh in self.shards:
                    sh.closure()
                dt = torch.stack([sh.dt_bits for sh in self.shards]).min()
                for sh in self.shards:
                    sh.dt_bits.copy_(dt.reshape(1))
                    sh.pack()
                for sh in self.shards:
                    for p, r in zip(sh.plan["peers"], sh.recv_parts):
                        src = self.shards[int(p)]
                        i = int(np.nonzero(src.plan["peers"] == sh.rank)[0][0])
                        r.copy_(src.send_parts[i])
                for i, sh in enumerate(self.shards):
                    sh.update(infos[i] if infos is not None and k == n_steps - 1 else None)
        self.stream.synchronize()
        return None if infos is None else [i.as_dict() for i in infos]

    def mean_var(self):
        """E and Var of every cell in global order."""
        n = self.shards[0].plan["n_global"]
        out = None
        for sh in self.shards:
            g, m = sh.owned_mean_var()
            if out is None:
                out = np.zeros((n, m.shape[1]))
            out[g] = m
        return out

    def state(self):
        """(u, lambda) of every cell in global order (state-major)."""
        out = None
        for sh in self.shards:
            g, u, lam = sh.owned_state()
            if out is None:
                n = sh.plan["n_global"]
                out = (np.zeros((n,) + u.shape[1:]), np.zeros((n,) + lam.shape[1:]))
            out[0][g] = u
            out[1][g] = lam
        return out

    def residual(self) -> float:
        return float(sum(sh.residual.item() for sh in self.shards))
