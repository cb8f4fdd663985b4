"""Spatial sharding on the host: the partition, the local meshes and the halo
exchange (uqc_partition / uqc_get_shard, uqcreator_b200/shard.py).

The partition and each rank's local mesh are built on the host when a handle
is partitioned, so these checks need no GPU:
- the owned cells of the ranks partition the mesh, in balanced blocks;
- each rank's halo is exactly the set of neighbours of its cells owned
  elsewhere, grouped by owner in global order;
- the local geometry is the global geometry of the local cells, with the
  neighbours renumbered (ghost faces keep the ghost index);
- what a rank sends to a peer is what the peer stores in its halo, in order.
The exchange itself (uqcreator_b200.shard.exchange, and the MIN / SUM
all-reduces of the step and the residual) runs over torch.distributed with
the gloo backend on world sizes 2 and 3 as separate processes.
"""
import os
import socket

import numpy as np
import pytest

from uqcreator_b200 import Solver, workloads as W
from uqcreator_b200.shard import shard_plan

CASES = {
    "euler2d": W.euler2d(nx=12, ny=5, degree=2, nquad=4),
    "burgers1d": W.burgers1d(ncells=50, degree=2, nquad=6),
    "sw1d": W.shallow_water1d(ncells=40),
}


def _shards(toml, n):
    out = []
    for r in range(n):
        s = Solver(toml)
        check = s.lib.uqc_partition(s.h, r, n)
        assert check == 0, s.lib.uqc_last_error(s.h)
        p = shard_plan(s)
        s.n_cells = p["n_owned"] + p["n_halo"]
        out.append((s, p))
    return out


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_partition_local_meshes_and_plans(case, n):
    toml = CASES[case]
    full = Solver(toml)
    g = full.geometry()
    N, F = full.n_cells, full.n_faces
    shards = _shards(toml, n)
    owner = np.full(N, -1)
    for r, (s, p) in enumerate(shards):
        assert p["rank"] == r and p["n_ranks"] == n and p["n_global"] == N
        own = p["global_ids"][: p["n_owned"]]
        assert np.all(np.diff(own) > 0)                      # owned cells in global order
        assert np.all(owner[own] == -1)
        owner[own] = r
    assert np.all(owner >= 0)                                # every cell has one owner
    sizes = np.bincount(owner, minlength=n)
    assert sizes.max() - sizes.min() <= 1
    for r, (s, p) in enumerate(shards):
        gid = p["global_ids"]
        no, nh = p["n_owned"], p["n_halo"]
        own = gid[:no]
        nb = g["nbr"][own]
        real = nb[nb < N]
        want = np.unique(real[owner[real] != r])
        halo = gid[no:]
        assert sorted(halo.tolist()) == want.tolist()
        # grouped by owner, global order within a group
        key = list(zip(owner[halo], halo))
        assert key == sorted(key)
        # local geometry = global geometry of the local cells
        lg = s.geometry()
        for k in ("area", "max_edge", "center", "unit_normal", "scaled_normal", "boundary"):
            np.testing.assert_array_equal(lg[k], g[k][gid])
        lnb = lg["nbr"][:no]
        gl = np.where(lnb < no + nh, gid[np.minimum(lnb, no + nh - 1)], N)
        np.testing.assert_array_equal(gl, np.where(nb < N, nb, N))
        # peers, receive counts and what each peer sends
        peers = p["peers"].tolist()
        assert peers == sorted(set(owner[halo].tolist()) | {q for q in range(n) if q != r and
                                                             np.isin(shards[q][1]["global_ids"][shards[q][1]["n_owned"]:], own).any()})
        off = 0
        for i, q in enumerate(peers):
            assert p["recv_counts"][i] == int(np.count_nonzero(owner[halo] == q))
            sent = gid[p["send_cells"][off:off + p["send_counts"][i]]]
            off += p["send_counts"][i]
            sq, pq = shards[q]
            qh = pq["global_ids"][pq["n_owned"]:]
            assert sent.tolist() == qh[owner[qh] == r].tolist()
        assert off == p["n_send"]
        assert p["row_doubles"] == full.n_states * full.n_quad


def test_partition_before_device_and_once():
    s = Solver(CASES["euler2d"])
    assert s.lib.uqc_partition(s.h, 2, 2) == -1        # rank out of range
    assert s.lib.uqc_partition(s.h, 0, 0) == -1
    assert s.lib.uqc_partition(s.h, 1, 3) == 0
    assert s.lib.uqc_partition(s.h, 0, 3) == -6        # already sharded


def test_single_rank_plan_is_the_mesh():
    s, p = _shards(CASES["burgers1d"], 1)[0]
    assert p["n_owned"] == 50 and p["n_halo"] == 0 and p["n_peers"] == 0 and p["n_send"] == 0
    np.testing.assert_array_equal(p["global_ids"], np.arange(50))


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _exchange_worker(rank, world, port, toml, q):
    import torch
    import torch.distributed as dist
    from uqcreator_b200.shard import exchange
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
        s = Solver(toml)
        assert s.lib.uqc_partition(s.h, rank, world) == 0
        p = shard_plan(s)
        row = p["row_doubles"]
        no, nh = p["n_owned"], p["n_halo"]
        gid = p["global_ids"]
        value = lambda ids: torch.tensor((ids[:, None] * 1000.0 + np.arange(row)[None, :]).ravel(), dtype=torch.float64)
        local = torch.zeros((no + nh) * row, dtype=torch.float64)
        local[: no * row] = value(gid[:no])
        send = local.view(no + nh, row)[torch.as_tensor(p["send_cells"], dtype=torch.long)].reshape(-1)
        so = np.concatenate([[0], np.cumsum(p["send_counts"])]) * row
        ro = np.concatenate([[0], np.cumsum(p["recv_counts"])]) * row
        halo = local[no * row:]
        exchange(dist, None, p["peers"], [send[so[i]:so[i + 1]] for i in range(p["n_peers"])],
                 [halo[ro[i]:ro[i + 1]] for i in range(p["n_peers"])])
        ok_halo = bool(torch.equal(halo, value(gid[no:]))) if nh else True
        # the step: MIN of positive doubles as int64 bits; the residual: SUM
        dt = torch.tensor([np.float64(0.5 + rank).view(np.int64)], dtype=torch.int64)
        dist.all_reduce(dt, op=dist.ReduceOp.MIN)
        res = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(res, op=dist.ReduceOp.SUM)
        ok_dt = dt.numpy().view(np.float64)[0] == 0.5
        ok_res = res.item() == world * (world + 1) / 2
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, ok_halo, ok_dt, ok_res, nh, p["n_peers"]))
    except Exception as e:    # reported to the parent
        q.put((rank, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", ["euler2d", "burgers1d"])
def test_halo_exchange_over_gloo(world, case):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, CASES[case], q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = {}
    try:
        for _ in range(world):
            item = q.get(timeout=120)
            got[item[0]] = item
    finally:
        for pr in procs:
            pr.join(timeout=30)
            if pr.is_alive():
                pr.kill()
    for r in range(world):
        assert len(got[r]) == 6, got[r]
        _, ok_halo, ok_dt, ok_res, nh, npeers = got[r]
        assert ok_halo and ok_dt and ok_res
        assert nh > 0 and npeers >= 1
