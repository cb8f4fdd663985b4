"""uqc_closure_solve_device_noalloc: the closure for callers that may not allocate.

Some callers cannot let a library call cudaMalloc: a framework that owns all
device memory through its own pool, code enqueued while a CUDA graph is being
captured in global mode, latency-critical loops that must not reach the
allocator. For them the library offers one entry point whose scratch is a
static device array. This test calls it through the C ABI on device arrays the
test owns, twice in a row, and checks each result against the allocating
entry point uqc_closure_solve_device on the same inputs (same kernel: the
duals must agree to the closure tests' tolerance, rtol 1e-8; statuses exactly).

The file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from uqcreator_b200 import Solver, workloads as W
from uqcreator_b200._lib import lib, NOALLOC_MAX_CELLS

pytestmark = pytest.mark.gpu


def _device_inputs(torch, toml):
    s = Solver(toml)
    s.init_state()
    u, lam, _ = s.download_state()
    s.close()
    return torch.from_numpy(u).cuda(), torch.from_numpy(lam).cuda()


def _solve(torch, fn_name, h, d_lam0, d_u, stream_arg):
    lam = d_lam0.clone()
    status = torch.full((lam.shape[0],), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()    # the allocating entry point runs on the handle's own stream
    L = lib()
    if fn_name == "noalloc":
        rc = L.uqc_closure_solve_device_noalloc(h, lam.shape[0], C.c_void_p(lam.data_ptr()), C.c_void_p(d_u.data_ptr()),
                                                None, C.c_void_p(status.data_ptr()), stream_arg)
    else:
        rc = L.uqc_closure_solve_device(h, lam.shape[0], C.c_void_p(lam.data_ptr()), C.c_void_p(d_u.data_ptr()), None,
                                        C.c_void_p(status.data_ptr()))
    assert rc == 0, L.uqc_last_error(h)
    torch.cuda.synchronize()
    return lam.cpu().numpy(), status.cpu().numpy()


@pytest.mark.parametrize("toml", [W.euler2d(nx=10, ny=4), W.burgers1d(ncells=300), W.shallow_water1d(ncells=500)],
                         ids=["euler2d", "burgers1d", "sw1d"])
def test_noalloc_matches_allocating_entry_point(toml):
    torch = pytest.importorskip("torch")
    d_u, d_lam0 = _device_inputs(torch, toml)
    # a fresh handle whose own device state is never set up: the no-alloc path
    # must work from the handle's host data alone
    fresh = Solver(toml)
    stream = torch.cuda.current_stream().cuda_stream
    first = _solve(torch, "noalloc", fresh.h, d_lam0, d_u, C.c_void_p(stream))
    second = _solve(torch, "noalloc", fresh.h, d_lam0, d_u, C.c_void_p(stream))
    ref_solver = Solver(toml)
    torch.cuda.synchronize()
    expect_lam, expect_status = _solve(torch, "alloc", ref_solver.h, d_lam0, d_u, None)
    for lam, status in (first, second):
        np.testing.assert_array_equal(status, expect_status)
        np.testing.assert_allclose(lam, expect_lam, rtol=1e-8, atol=1e-12)
    assert np.all(expect_status == 0)


def test_noalloc_rejects_oversized_batch():
    toml = W.burgers1d(ncells=300)
    s = Solver(toml)
    L = lib()
    rc = L.uqc_closure_solve_device_noalloc(s.h, NOALLOC_MAX_CELLS + 1, C.c_void_p(16), C.c_void_p(16), None,
                                            C.c_void_p(16), None)
    assert rc == -7
    assert b"UQC_NOALLOC_MAX_CELLS" in L.uqc_last_error(s.h)
