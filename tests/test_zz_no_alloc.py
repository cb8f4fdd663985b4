"""uqc_closure_solve_device_noalloc: the closure for callers that may not allocate.

Some callers cannot let a library call cudaMalloc: a framework that owns all
device memory through its own pool (a stray allocation would fragment or
overrun the budget it manages), or a latency-critical loop that must not
reach the allocator. For them the library offers one entry point whose
scratch is a static device array. These tests call it through the C ABI on
device arrays the test owns, twice in a row, and check each result against
the allocating entry point uqc_closure_solve_device on the same inputs (the
same FP64 kernel: duals agree to the closure tests' tolerance, rtol 1e-8;
statuses exactly), and against the golden duals the reference's own
Closure::SolveClosure wrote.

The file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from uqcreator_b200 import Solver, workloads as W
from uqcreator_b200._lib import lib, NOALLOC_MAX_CELLS

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _device_inputs(torch, toml):
    s = Solver(toml)
    s.init_state()
    u, lam, _ = s.download_state()
    s.close()
    return torch.from_numpy(u).cuda(), torch.from_numpy(lam).cuda()


def _solve(torch, fn_name, h, d_lam0, d_u, stream_arg, d_nt=None):
    lam = d_lam0.clone()
    status = torch.full((lam.shape[0],), -1, dtype=torch.int32, device="cuda")
    nt = None if d_nt is None else C.c_void_p(d_nt.data_ptr())
    torch.cuda.synchronize()    # the allocating entry point runs on the handle's own stream
    L = lib()
    if fn_name == "noalloc":
        rc = L.uqc_closure_solve_device_noalloc(h, lam.shape[0], C.c_void_p(lam.data_ptr()), C.c_void_p(d_u.data_ptr()),
                                                nt, C.c_void_p(status.data_ptr()), stream_arg)
    else:
        rc = L.uqc_closure_solve_device(h, lam.shape[0], C.c_void_p(lam.data_ptr()), C.c_void_p(d_u.data_ptr()), nt,
                                        C.c_void_p(status.data_ptr()))
    assert rc == 0, L.uqc_last_error(h)
    torch.cuda.synchronize()
    return lam.cpu().numpy(), status.cpu().numpy()


def _compare_twice(torch, toml, d_lam0, d_u, d_nt=None):
    # a fresh handle whose own device state is never set up: the no-alloc path
    # must work from the handle's host data alone
    fresh = Solver(toml)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    first = _solve(torch, "noalloc", fresh.h, d_lam0, d_u, stream, d_nt)
    second = _solve(torch, "noalloc", fresh.h, d_lam0, d_u, stream, d_nt)
    ref_solver = Solver(toml)
    expect_lam, expect_status = _solve(torch, "alloc", ref_solver.h, d_lam0, d_u, None, d_nt)
    for lam, status in (first, second):
        np.testing.assert_array_equal(status, expect_status)
        np.testing.assert_allclose(lam, expect_lam, rtol=1e-8, atol=1e-12)
    return first, expect_status


@pytest.mark.parametrize("toml", [W.euler2d(nx=10, ny=4), W.burgers1d(ncells=300), W.shallow_water1d(ncells=500),
                                  W.euler2d(nx=6, ny=2, degree=1, nquad=20)],
                         ids=["euler2d", "burgers1d", "sw1d", "euler2d_deg1_q20x20"])
def test_noalloc_matches_allocating_entry_point(toml):
    """The last case has 12 duals and 400 nodes: a cell's workspace is large
    enough that fewer than eight warp groups share a CTA, so the no-alloc path
    must pick the allocating path's launch shape rather than a fixed one."""
    torch = pytest.importorskip("torch")
    d_u, d_lam0 = _device_inputs(torch, toml)
    _, status = _compare_twice(torch, toml, d_lam0, d_u)
    assert np.all(status == 0)


def test_noalloc_per_cell_moment_counts():
    """Cells solved for different numbers of moments (d_n_total, the refinement
    levels of the adaptive shallow-water workload) in one call."""
    torch = pytest.importorskip("torch")
    toml = W.shallow_water1d(ncells=400)
    d_u, d_lam0 = _device_inputs(torch, toml)
    s = Solver(toml)
    levels = np.array(s.n_total_levels, dtype=np.uint32)
    s.close()
    assert len(levels) > 1
    rng = np.random.default_rng(5)
    nt = levels[rng.integers(0, len(levels), size=d_u.shape[0])]
    d_nt = torch.from_numpy(nt.astype(np.int32)).cuda()
    (lam, status), _ = _compare_twice(torch, toml, d_lam0, d_u, d_nt)
    assert np.all(status == 0)
    # moments beyond a cell's count are left as they came in
    lam0 = d_lam0.cpu().numpy()
    for j in range(0, len(nt), 37):
        np.testing.assert_array_equal(lam[j][:, nt[j]:], lam0[j][:, nt[j]:])


def test_noalloc_matches_reference_golden():
    """The reference's own Closure::SolveClosure (guarded Newton) wrote the
    golden duals of 32 Euler cells from perturbed starting duals."""
    torch = pytest.importorskip("torch")
    g = np.load(GOLD / "c2_closure.npz")
    toml = str(g["toml"])
    d_u = torch.from_numpy(np.ascontiguousarray(g["u"])).cuda()
    d_lam0 = torch.from_numpy(np.ascontiguousarray(g["lam0"])).cuda()
    (lam, status), _ = _compare_twice(torch, toml, d_lam0, d_u)
    ok = g["status_guarded"] == 0
    np.testing.assert_array_equal(status == 0, ok)
    np.testing.assert_allclose(lam[ok], g["lam_guarded"][ok], rtol=1e-8, atol=1e-9)


def test_noalloc_rejects_oversized_batch():
    toml = W.burgers1d(ncells=300)
    s = Solver(toml)
    L = lib()
    rc = L.uqc_closure_solve_device_noalloc(s.h, NOALLOC_MAX_CELLS + 1, C.c_void_p(16), C.c_void_p(16), None,
                                            C.c_void_p(16), None)
    assert rc == -7
    assert b"UQC_NOALLOC_MAX_CELLS" in L.uqc_last_error(s.h)
