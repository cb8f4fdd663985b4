"""Mixed form (FP32 Hessian, factor and solves; FP64 gradient, tests and
update) vs the FP64 oracle, through the C ABI (needs a B200).

Bound: moments and E/Var within relative L1 1e-6 of the FP64 oracle after
several time steps. The convergence test is the FP64 one (||g||_2 < eps), so a
converged mixed cell sits within the same tolerance of the exact duals as an
FP64 cell; the bound leaves room for the different path the iterates take.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from uqcreator_b200 import Solver, workloads as W, MIXED, FP64

from ._util import rel_l1

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _moment_err(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


@pytest.mark.parametrize("toml,steps", [
    (W.burgers1d(ncells=200), 20),
    (W.euler2d(nx=16, ny=4), 4),
    (W.shallow_water1d(ncells=300), 10),
    (W.euler2d_3u(nx=4, ny=2), 2),
])
def test_mixed_steps_match_oracle(toml, steps):
    s = Solver(toml)
    s.set_precision(MIXED)
    o = Oracle(toml, W.mesh_for(toml))
    s.init_state(); o.init_state()
    info = s.step(steps)
    o.step(steps)
    assert info["failed_cells"] == 0 and info["steps"] == steps
    us, _, vs = s.download_state()
    uo, _, vo = o.get_state()
    np.testing.assert_array_equal(vs, vo)
    assert _moment_err(us, uo) <= TOL
    err = rel_l1(s.mean_var(), o.mean_var(), o.geometry()["area"])
    assert np.all(err <= TOL), err


def test_mixed_batched_closure_meets_fp64_tolerance():
    """Batched closure from perturbed duals: mixed and FP64 reach duals whose
    moments agree to the Newton tolerance."""
    toml = W.euler2d(nx=16, ny=4)
    a = Solver(toml); b = Solver(toml)
    a.init_state(); b.init_state()
    b.set_precision(MIXED)
    u, lam, lev = a.download_state()
    rng = np.random.default_rng(3)
    lam2 = lam * (1 + 1e-3 * rng.standard_normal(lam.shape))
    la, sa = a.closure_solve_host(lam2, u)
    lb, sb = b.closure_solve_host(lam2, u)
    assert np.all(sa == 0) and np.all(sb == 0)
    assert _moment_err(lb, la) <= 1e-6


def test_mixed_fallback_to_fp64():
    """With an FP32 iteration budget of 2, cells that need more go to the FP64
    form, which finishes them from the last accepted duals."""
    toml = W.euler2d(nx=16, ny=4)
    ref = Solver(toml); ref.init_state()
    ref.step(3)
    s = Solver(toml); s.init_state()
    s.set_precision(MIXED)
    s.set_option("mixed_max_iterations", 2)
    info = s.step(3)
    assert info["fallback_cells"] > 0
    assert info["failed_cells"] == 0
    ur, _, _ = ref.download_state()
    um, _, _ = s.download_state()
    assert _moment_err(um, ur) <= TOL


def test_fp64_and_mixed_switch_on_one_handle():
    toml = W.euler2d(nx=8, ny=3)
    s = Solver(toml); s.init_state()
    s.set_precision(MIXED); s.step(2)
    s.set_precision(FP64); b = s.step(2)
    assert b["fallback_cells"] == 0 and b["failed_cells"] == 0


def test_chord_newton_reuses_factors_reproducibly():
    """The inexact (chord) Newton of the mixed form keeps each cell's factor
    between steps; results stay within the mixed bound of the FP64 form, and a
    state uploaded again starts without stored factors, so the same steps give
    the same result."""
    toml = W.euler2d(nx=16, ny=6)
    ref = Solver(toml); ref.init_state(); ref.step(4)
    s = Solver(toml); s.init_state(); s.set_precision(MIXED)
    u0, l0, v0 = s.download_state()
    a = s.step(4)
    ua = s.download_state()[0]
    s.upload_state(u0, l0, v0)
    b = s.step(4)
    ub = s.download_state()[0]
    assert a["newton_iterations"] == b["newton_iterations"]
    np.testing.assert_array_equal(ua, ub)
    assert _moment_err(ua, ref.download_state()[0]) <= TOL
    s.set_option("mixed_chord", 0)
    s.upload_state(u0, l0, v0)
    c = s.step(4)
    assert _moment_err(s.download_state()[0], ref.download_state()[0]) <= TOL
    assert c["newton_iterations"] <= a["newton_iterations"]
