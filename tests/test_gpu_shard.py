"""Sharded time steps on the GPU against the unsharded solver (needs a B200).

A mesh split into 2 or 3 shards (uqc_partition), stepped in lockstep in one
process on one GPU (uqcreator_b200.shard.LocalShards: closure of every shard,
the smallest step of all, halo rows copied between shards, update of every
shard) must give the unsharded handle's moments, duals and time bit for bit:
every cell's closure and update do the same arithmetic on the same inputs, and
the step is the same minimum. Covered: 2-D Euler (FP64 and the mixed form),
1-D Burgers with Dirichlet end cells, adaptive 1-D shallow water (several
refinement levels) and the SU2 channel with no-slip and shallow-water walls.
Also: a sharded handle refuses the unsharded time loop, and a one-shard
partition is the unsharded run.
"""
import shutil
from pathlib import Path

import numpy as np
import pytest

from uqcreator_b200 import MIXED, Solver, UqcError, workloads as W
from uqcreator_b200.shard import LocalShards, Shard

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"

CASES = {
    "euler2d": W.euler2d(nx=24, ny=8, degree=3, nquad=6),
    "burgers1d": W.burgers1d(ncells=120, degree=4, nquad=20),
    "sw1d_adaptive": W.shallow_water1d(ncells=150),
}


def _unsharded(toml, steps, precision=None):
    s = Solver(toml)
    if precision is not None:
        s.set_precision(precision)
    s.init_state()
    info = s.step(steps)
    u, lam, _ = s.download_state()
    return u, lam, info["t"]


def _compare(toml, n, steps, precision=None):
    u0, l0, t0 = _unsharded(toml, steps, precision)
    ls = LocalShards(toml, n, precision)
    ls.init_state()
    infos = ls.step(steps, with_info=True)
    u, lam = ls.state()
    np.testing.assert_array_equal(u, u0)
    np.testing.assert_array_equal(lam, l0)
    assert [i["t"] for i in infos] == [t0] * n
    assert all(i["failed_cells"] == 0 for i in infos)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("n", [2, 3])
def test_shards_match_unsharded_fp64(case, n):
    _compare(CASES[case], n, 6)


@pytest.mark.parametrize("n", [2, 3])
def test_shards_match_unsharded_mixed(n):
    _compare(CASES["euler2d"], n, 6, MIXED)


def test_shards_match_unsharded_walls(tmp_path):
    g = np.load(GOLD / "su2_steps.npz")
    shutil.copy(GOLD / "su2_channel.su2", tmp_path / "su2_channel.su2")
    cfg = tmp_path / "c.toml"
    cfg.write_text(str(g["toml"]))
    _compare(str(cfg), 3, int(g["steps"]))


def test_one_shard_is_the_unsharded_run():
    _compare(CASES["euler2d"], 1, 4)


def test_sharded_handle_refuses_the_unsharded_loop():
    sh = Shard(CASES["burgers1d"], 0, 2)
    sh.init_state()
    with pytest.raises(UqcError):
        sh.solver.step(1)
    with pytest.raises(UqcError):
        sh.solver.run()


def test_sharded_solver_one_rank_over_nccl():
    """ShardedSolver on a one-rank NCCL group: the step's all-reduce runs on the
    library's own device memory on the handle's stream; the result is the
    unsharded run's (a single process and GPU: nothing waits on another rank)."""
    import socket
    import torch.distributed as dist
    from uqcreator_b200.shard import ShardedSolver
    toml = CASES["euler2d"]
    u0, l0, t0 = _unsharded(toml, 5)
    ref = Solver(toml)
    ref.init_state()
    rinfo = ref.step(5)
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("cpu:gloo,cuda:nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        ss = ShardedSolver(toml)
        ss.init_state()
        info = ss.step(5, with_info=True)
        assert info["t"] == t0
        u, lam, _ = ss.shard.solver.download_state()
        np.testing.assert_array_equal(u, u0)
        np.testing.assert_array_equal(lam, l0)
        np.testing.assert_array_equal(ss.gather_mean_var(), ref.mean_var())
        assert abs(ss.residual() - rinfo["residual"]) <= 1e-12 * abs(rinfo["residual"])
        ss.close()
    finally:
        dist.destroy_process_group()
