"""Linear closures on the GPU against the reference itself (needs a B200).

Stochastic Galerkin, the L2 filter and the Lasso filter (stochasticgalerkin.cpp,
l2filter.cpp, lassofilter.cpp) take the duals from the moments without a
Newton solve; the kernels run them as closure kinds 3-5 (the states of
Burgers, 2-D Euler, shallow water). The check is against the reference's own
closure classes and time loop, compiled from its sources (oracle/_ref, the
exact build): the mean and variance within relative L1 1e-10, the moments
and duals elementwise within 1e-10 relative. The Lasso filter runs on a 2-D
case of total degree 4 (in one uncertain dimension the reference's Lasso
divides by zero: index_0 of the last basis function is 0). The exponential
filter is refused (the reference reads an uninitialised order and time step).
"""
import numpy as np
import pytest

from oracle import refharness
from uqcreator_b200 import MIXED, Solver, UqcError, workloads as W

from ._util import rel_l1

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refharness.available("exact"), reason="oracle/_ref/libuqcref.so not built")]


def _with_closure(toml, closure, old):
    return toml.replace(f'closure = "{old}"', f'closure = "{closure}"')


EULER_WEAK = [0.5, 1.0, 1.0, 0.8, 0.8]


def _weak(toml):
    out = toml.replace("ic = [0.5,1.0,1.0,0.125,0.1]", "ic = [0.5,1.0,1.0,0.8,0.8]")
    assert out != toml
    return out


CASES = {
    "burgers_sg": (lambda: _with_closure(W.burgers1d(ncells=300, degree=5, nquad=16, tend=0.05), "StochasticGalerkin", "BoundedBarrier"),
                   ("Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5), False), 25),
    "burgers_l2": (lambda: _with_closure(W.burgers1d(ncells=300, degree=5, nquad=16, tend=0.05), "L2Filter", "BoundedBarrier"),
                   ("Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5), False), 25),
    "sw_sg_adaptive": (lambda: _with_closure(W.shallow_water1d(ncells=400, max_degree=5, nquad=12), "StochasticGalerkin", "ShallowWater"),
                       ("ShallowWater1D", [0.5, 1.0, 0.5], (3.0, 12.0), False), 20),
    # a weak interface (right state 0.8 / 0.8): the polynomial ansatz of Sod's
    # jump oscillates into negative densities, in the reference as here
    "euler_l2": (lambda: _weak(_with_closure(W.euler2d(nx=12, ny=4, degree=4, nquad=8, newton="reference"), "L2Filter", "Euler2D")),
                 ("Euler2D", EULER_WEAK, (3, 12), True), 6),
    "euler_lasso": (lambda: _weak(_with_closure(W.euler2d(nx=12, ny=4, degree=4, nquad=8, newton="reference"), "LassoFilter", "Euler2D")),
                    ("Euler2D", EULER_WEAK, (3, 12), True), 6),
    "euler_sg": (lambda: _weak(_with_closure(W.euler2d(nx=12, ny=4, degree=3, nquad=6, newton="reference"), "StochasticGalerkin", "Euler2D")),
                 ("Euler2D", EULER_WEAK, (3, 12), True), 6),
}


@pytest.mark.parametrize("case", list(CASES))
def test_linear_closure_steps_match_reference(case):
    make, (problem, ic, bounds, two_d), steps = CASES[case]
    toml = make()
    s = Solver(toml)
    r = refharness.RefSolver(toml, problem, ic, bounds=bounds, mesh2d=W.mesh_for(toml) if two_d else None, variant="exact")
    s.init_state(); r.init_state()
    a = s.step(steps)
    b = r.step(steps)
    assert a["failed_cells"] == 0
    assert abs(a["t"] - b["t"]) <= 1e-10 * b["t"]
    us, ls, vs = s.download_state()
    ur, lr, vr = r.get_state()
    assert np.isfinite(us).all() and np.isfinite(ls).all()
    np.testing.assert_array_equal(vs, vr)
    np.testing.assert_allclose(us, ur, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(ls, lr, rtol=1e-10, atol=1e-12)
    area = r.geometry(3 if two_d else 2)["area"]
    err = rel_l1(s.mean_var(), r.mean_var(), area)
    assert np.all(err <= 1e-10), err


def test_linear_closure_refuses_the_mixed_form_and_the_exponential_filter():
    toml = CASES["burgers_sg"][0]()
    s = Solver(toml)
    s.init_state()
    with pytest.raises(UqcError):
        s.set_precision(MIXED)
    with pytest.raises(UqcError):
        Solver(_with_closure(W.burgers1d(ncells=50), "ExponentialFilter", "BoundedBarrier"))
