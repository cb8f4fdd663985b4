"""uqc_step_host (one step from host state to host state, the copies beside
the kernels) against uqc_upload_state + uqc_step + uqc_download_state on the
same state (needs a B200).

The chunked closure and update and the overlapped copies change nothing a
cell computes, so the two paths agree bit for bit in moments, duals, levels,
time and time step; the residual sums the same terms in another order
(relative 1e-12). Cases: 2-D Euler (FP64 and the mixed form),
1-D Burgers (register Newton), adaptive shallow water (levels; both forms),
1-D Euler, and the output written over the input arrays.
"""
import numpy as np
import pytest

from uqcreator_b200 import MIXED, Solver, workloads as W

pytestmark = pytest.mark.gpu

CASES = {
    "euler2d_fp64": (lambda: W.euler2d(nx=40, ny=16), False),
    "euler2d_mixed": (lambda: W.euler2d(nx=40, ny=16), True),
    "burgers1d": (lambda: W.burgers1d(ncells=300), False),
    "sw_levels": (lambda: W.shallow_water1d(ncells=3000), False),
    "sw_levels_mixed": (lambda: W.shallow_water1d(ncells=3000), True),
    "euler1d": (lambda: W.euler1d(ncells=400), False),
}


def _pinned(a):
    import torch
    p = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32, pin_memory=True).numpy()
    if a.dtype == np.uint32:
        p = p.view(np.uint32)
    p[...] = a
    return p


@pytest.mark.parametrize("case", list(CASES))
def test_step_host_matches_upload_step_download(case):
    make, mixed = CASES[case]
    toml = make()
    s = Solver(toml)
    if mixed:
        s.set_precision(MIXED)
    s.init_state()
    s.step(3)    # some cells need Newton from here on
    u0, l0, v0 = s.download_state()
    t0 = s.step(0)["t"]
    for k in range(3):
        # reference path: upload, step, download
        s.upload_state(u0, l0, v0, t=t0)
        a = s.step(1)
        ua, la, va = s.download_state()
        # host-step path, from pinned copies of the same state
        hu, hl, hv = _pinned(u0), _pinned(l0), _pinned(v0)
        ub, lb, vb, b = s.step_host(hu, hl, hv, t=t0)
        np.testing.assert_array_equal(ub, ua)
        np.testing.assert_array_equal(lb, la)
        np.testing.assert_array_equal(vb, va)
        for key in ("t", "dt", "newton_iterations", "active_cells", "failed_cells"):
            assert b[key] == a[key], (key, a[key], b[key])
        assert b["residual"] == pytest.approx(a["residual"], rel=1e-12, abs=1e-300)
        # in place: the outputs over the inputs
        uc, lc, vc, c = s.step_host(hu, hl, hv, t=t0, out=(hu, hl, hv))
        assert uc is hu
        np.testing.assert_array_equal(hu, ua)
        np.testing.assert_array_equal(hl, la)
        np.testing.assert_array_equal(hv, va)
        assert c["t"] == a["t"]
        u0, l0, v0, t0 = ua, la, va, a["t"]


def test_step_host_first_state_and_levels_kept():
    """A handle without state takes its first state from uqc_step_host; NULL
    levels keep the resident ones (the finest level on a fresh handle)."""
    toml = W.euler2d(nx=20, ny=10)
    s = Solver(toml)
    s.init_state()
    u0, l0, v0 = s.download_state()
    s.step(1)
    ua, la, va = s.download_state()
    s2 = Solver(toml)
    ub, lb, vb, info = s2.step_host(_pinned(u0), _pinned(l0), None, t=0.0)
    np.testing.assert_array_equal(ub, ua)
    np.testing.assert_array_equal(lb, la)
    np.testing.assert_array_equal(vb, va)
    assert info["steps"] == 1


@pytest.mark.parametrize("chunks", [1, 3, 13, 32])
def test_step_host_chunk_counts(chunks):
    """Any chunk count (option host_chunks, here more chunks than some meshes
    have cells per chunk) gives the three calls' result."""
    toml = W.euler2d(nx=12, ny=5)
    s = Solver(toml)
    s.set_precision(MIXED)
    s.init_state()
    s.step(2)
    u0, l0, v0 = s.download_state()
    t0 = s.step(0)["t"]
    s.upload_state(u0, l0, v0, t=t0)
    a = s.step(1)
    ua, la, va = s.download_state()
    s.set_option("host_chunks", chunks)
    ub, lb, vb, b = s.step_host(_pinned(u0), _pinned(l0), _pinned(v0), t=t0)
    np.testing.assert_array_equal(ub, ua)
    np.testing.assert_array_equal(lb, la)
    np.testing.assert_array_equal(vb, va)
    assert b["t"] == a["t"] and b["dt"] == a["dt"]


def test_step_host_refused_while_async_steps_run():
    """A uqc_step_async batch in flight owns the control block: uqc_step_host
    is refused until the batch has been queried to completion."""
    from uqcreator_b200._lib import UqcError
    toml = W.euler2d(nx=12, ny=5)
    s = Solver(toml)
    s.init_state()
    u0, l0, v0 = s.download_state()
    s.step_async(2)
    with pytest.raises(UqcError):
        s.step_host(_pinned(u0), _pinned(l0), _pinned(v0), t=0.0)
    import time
    deadline = time.monotonic() + 60.0
    while s.step_query() is None:
        assert time.monotonic() < deadline
        time.sleep(0.001)
    s.step_host(_pinned(u0), _pinned(l0), _pinned(v0), t=0.0)
