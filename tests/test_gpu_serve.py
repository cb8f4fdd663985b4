"""Asynchronous stepping and the request server (needs a B200).

A request's result must not depend on what else runs: the kernels of one
handle use only that handle's buffers and reduce in a fixed order, so the
mean and variance of a request served in a mix equal those of the same
request solved alone, bit for bit.
"""
import time

import numpy as np
import pytest

from uqcreator_b200 import Solver, workloads as W, FP64, MIXED
from uqcreator_b200.serve import Server, latency_percentiles

pytestmark = pytest.mark.gpu


def _requests():
    return [
        W.burgers1d(ncells=400, degree=3, nquad=16, tend=0.004, x0=0.6),
        W.euler2d(nx=16, ny=8, degree=2, nquad=4, tend=0.01, xs=0.4),
        W.burgers1d(ncells=900, degree=5, nquad=24, tend=0.002, x0=0.7),
        W.euler2d(nx=24, ny=10, degree=3, nquad=6, tend=0.006, xs=0.3),
        W.shallow_water1d(ncells=2000, max_degree=4, nquad=12, tend=0.002),
    ]


def _alone(toml, precision=FP64):
    s = Solver(toml)
    s.init_state()
    if precision == MIXED:
        s.set_precision(MIXED)
    info = s.run()
    return s.mean_var(), info


def test_step_async_matches_step():
    toml = W.euler2d(nx=16, ny=8, degree=3, nquad=6)
    a = Solver(toml); a.init_state()
    b = Solver(toml); b.init_state()
    ia = a.step(5)
    b.step_async(5)
    ib = None
    t0 = time.time()
    while ib is None and time.time() - t0 < 60:
        ib = b.step_query()
    assert ib is not None
    for k in ("t", "dt", "residual", "steps", "newton_iterations", "running"):
        assert ia[k] == ib[k], k
    ua, la, _ = a.download_state()
    ub, lb, _ = b.download_state()
    np.testing.assert_array_equal(ua, ub)
    np.testing.assert_array_equal(la, lb)


def test_server_results_same_alone_and_in_mix():
    reqs = _requests()
    alone = [_alone(t)[0] for t in reqs]
    srv = Server(budget_bytes=8 << 30, max_active=len(reqs), steps_per_slice=2)
    ids = [srv.submit(t) for t in reqs]
    srv.drain()
    for rid, ref in zip(ids, alone):
        r = srv.result(rid)
        assert r["state"] == "done" and r["status"] == 0, r
        assert r["latency_ms"] >= 0 and r["steps"] > 0
        np.testing.assert_array_equal(r["mean_var"], ref)
    srv.close()


def test_server_submissions_from_another_thread():
    """A front-end thread submits while the main thread runs the scheduling
    passes: every request finishes with its result alone, bit for bit."""
    import threading
    reqs = _requests()
    alone = [_alone(t)[0] for t in reqs]
    srv = Server(budget_bytes=8 << 30, max_active=3, steps_per_slice=2)
    ids = [None] * len(reqs)

    def front_end():
        for k, t in enumerate(reqs):
            ids[k] = srv.submit(t)
            time.sleep(0.002)

    th = threading.Thread(target=front_end)
    th.start()
    deadline = time.monotonic() + 120.0
    while True:
        alive = th.is_alive()
        q, r, _ = srv.progress()
        if not alive and q == 0 and r == 0:
            break
        assert time.monotonic() < deadline
    th.join()
    for rid, ref in zip(ids, alone):
        res = srv.result(rid)
        assert res["state"] == "done" and res["status"] == 0, res
        np.testing.assert_array_equal(res["mean_var"], ref)
    srv.close()


def test_server_mixed_precision_request_within_tolerance():
    toml = W.euler2d(nx=16, ny=8, degree=3, nquad=6, tend=0.01)
    ref, _ = _alone(toml)
    srv = Server(budget_bytes=4 << 30, max_active=2, steps_per_slice=3)
    rid = srv.submit(toml, precision=MIXED)
    other = srv.submit(_requests()[0])
    srv.drain()
    r = srv.result(rid)
    assert r["state"] == "done"
    assert np.abs(r["mean_var"] - ref).sum() / np.abs(ref).sum() <= 1e-6
    assert srv.result(other)["state"] == "done"


def test_server_admits_by_device_budget():
    reqs = _requests()
    sizes = []
    for t in reqs:
        s = Solver(t)
        sizes.append(s.device_bytes())
        s.close()
    budget = sum(sorted(sizes)[-2:])    # room for the two largest at once, not for all
    srv = Server(budget_bytes=budget, max_active=len(reqs), steps_per_slice=1)
    ids = [srv.submit(t) for t in reqs]
    peak = 0
    while True:
        q, r, d = srv.progress()
        used = sum(srv.info(i)["device_bytes"] for i in ids if srv.info(i)["state"] == "running")
        assert used <= budget
        peak = max(peak, r)
        if q == 0 and r == 0:
            break
    assert peak < len(reqs)
    lat = [srv.result(i, mean_var=False)["latency_ms"] for i in ids]
    assert all(srv.info(i)["state"] == "done" for i in ids)
    p = latency_percentiles(lat)
    assert p["p50_ms"] <= p["p99_ms"]


def test_handles_with_different_shared_memory_needs_coexist():
    """Kernel launch limits are process-wide: a handle with a small workspace
    set up after one with a large workspace must not break the latter."""
    big = Solver(W.euler2d(nx=8, ny=4, degree=5, nquad=10)); big.init_state(); big.step(1)
    small = Solver(W.euler2d(nx=8, ny=4, degree=2, nquad=4)); small.init_state(); small.step(1)
    assert big.step(2)["steps"] == 2
    assert small.step(2)["steps"] == 2


def test_graph_replay_matches_direct_launches():
    """uqc_run through cached CUDA graphs gives the same state as direct launches."""
    toml = W.burgers1d(ncells=500, tend=0.02)
    a = Solver(toml); a.init_state(); a.set_option("graphs", 0)
    b = Solver(toml); b.init_state()
    ia, ib = a.run(), b.run()
    assert ia["steps"] == ib["steps"] and ia["t"] == ib["t"]
    np.testing.assert_array_equal(a.download_state()[0], b.download_state()[0])
    # a settings change between runs re-captures the graph
    b.set_newton(1000, 1e-11, 0)
    a.set_newton(1000, 1e-11, 0)
    ja, jb = a.run(0.03), b.run(0.03)
    assert ja["newton_iterations"] == jb["newton_iterations"]
    np.testing.assert_array_equal(a.download_state()[1], b.download_state()[1])


def test_autotune_picks_a_valid_shape_and_keeps_results(tmp_path):
    from uqcreator_b200.autotune import autotune
    from oracle.oracle import Oracle
    from ._util import rel_l1
    toml = W.euler2d(nx=16, ny=6, degree=4, nquad=8)
    s = Solver(toml); s.init_state(); s.step(2)
    r = autotune(s, steps=1, repeats=1, cache=tmp_path / "tune.json")
    assert r["best"]["closure_group"] in (32, 64, 256) and not r["cached"]
    assert min(v for v in r["ms_per_step"].values() if v is not None) > 0
    s.step(2)
    o = Oracle(toml, W.mesh_for(toml)); o.init_state(); o.step(4)
    err = rel_l1(s.mean_var(), o.mean_var(), o.geometry()["area"])
    assert (err <= 1e-10).all(), err
    s2 = Solver(toml); s2.init_state()
    assert autotune(s2, cache=tmp_path / "tune.json")["cached"]


@pytest.mark.parametrize("toml,steps", [
    (W.euler2d(nx=24, ny=8), 6),
    (W.shallow_water1d(ncells=400), 12),
    (W.burgers1d(ncells=300), 20),
])
def test_update_side_convergence_test_matches_check_kernel(toml, steps):
    """k_update's test of the next step's convergence (cells that pass keep
    their moments and skip the closure) against k_check testing every cell:
    the same Newton work and the same results up to rounding of the
    re-projection."""
    a = Solver(toml); a.init_state()
    b = Solver(toml); b.init_state()
    a.set_option("update_test", 1)    # also with refinement levels (automatic: off there)
    b.set_option("update_test", 0)
    ia = a.step(steps)
    ib = b.step(steps)
    assert ia["newton_iterations"] == ib["newton_iterations"]
    assert ia["failed_cells"] == ib["failed_cells"] == 0
    ua, la, va = a.download_state()
    ub, lb, vb = b.download_state()
    np.testing.assert_array_equal(va, vb)
    np.testing.assert_allclose(ua, ub, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(la, lb, rtol=1e-10, atol=1e-12)
    assert abs(ia["t"] - ib["t"]) <= 1e-14 * ib["t"]


@pytest.mark.parametrize("policy", [0, 1])
def test_scheduling_policies_give_the_same_results(policy):
    """Round robin and shortest-remaining-work-first order the slices
    differently; each request's result is still the one it has alone."""
    reqs = _requests()
    alone = [_alone(t)[0] for t in reqs]
    srv = Server(budget_bytes=8 << 30, max_active=len(reqs), steps_per_slice=2, policy=policy, max_stepping=2)
    ids = [srv.submit(t) for t in reqs]
    srv.drain()
    for rid, ref in zip(ids, alone):
        r = srv.result(rid)
        assert r["state"] == "done", r
        assert r["queue_ms"] >= 0 and r["service_ms"] >= 0
        np.testing.assert_array_equal(r["mean_var"], ref)


def test_shortest_remaining_work_goes_first():
    """With one request stepping at a time, a short request submitted after a
    long one finishes first; under round robin the long one is not held back."""
    long_req = W.euler2d(nx=40, ny=20, degree=4, nquad=8, tend=10.0, steps=30)
    short_req = W.burgers1d(ncells=300, degree=3, nquad=16, tend=10.0, steps=4)
    srv = Server(budget_bytes=8 << 30, max_active=4, steps_per_slice=2, policy=1, max_stepping=1)
    a = srv.submit(long_req)
    b = srv.submit(short_req)
    srv.drain()
    ra, rb = srv.result(a, mean_var=False), srv.result(b, mean_var=False)
    assert ra["state"] == rb["state"] == "done"
    assert ra["steps"] == 30 and rb["steps"] == 4
    assert rb["done_ms"] < ra["done_ms"]
