"""1-D Euler on the GPU against the reference itself (needs a B200).

The reference's Euler1D problem (euler.cpp: HLL flux, CFL rule, its fixed Sod
state) with its entropy closure EulerClosure (eulerclosure.cpp, three states)
runs as closure kind 6; with a linear closure as kind 7. The check is against
the reference's own classes and time loop compiled from its sources
(oracle/_ref, the exact build): FP64 mean and variance within relative L1
1e-10 and moments within 1e-8 elementwise, the simulated time within 1e-8;
the mixed form within 1e-6; the
register Newton (degree 1: six duals) and the general kernel (degree 4: 15
duals) both.
"""
import numpy as np
import pytest

from oracle import refharness
from uqcreator_b200 import MIXED, Solver, workloads as W

from ._util import rel_l1

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refharness.available("exact"), reason="oracle/_ref/libuqcref.so not built")]

# Newton to |g| < 1e-12: two FP64 closures (here and the reference) that stop
# at |g| < eps leave duals that differ by up to H^-1 eps, which at 1e-10 shows
# in the small momentum moments at a few 1e-9
CASES = {
    "deg4": (W.euler1d(ncells=400, degree=4, nquad=10, tend=0.1, eps=1e-12), "guarded", 30),
    "deg1_register_newton": (W.euler1d(ncells=300, degree=1, nquad=6, tend=0.1, eps=1e-12), "guarded", 30),
    "deg3_two_uncertainties": (W.euler1d(ncells=200, degree=3, nquad=6, tend=0.1, sigmas=[0.05, 0.05], eps=1e-12), "guarded", 15),
    "sg": (W.euler1d(ncells=300, degree=3, nquad=8, tend=0.1).replace('closure = "Euler"', 'closure = "StochasticGalerkin"'),
           "reference", 20),
}


@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
@pytest.mark.parametrize("case", list(CASES))
def test_euler1d_steps_match_reference(case, mixed):
    toml, newton, steps = CASES[case]
    s = Solver(toml)
    if mixed:
        if case == "sg":
            pytest.skip("a linear closure has no Newton system to run in FP32")
        s.set_precision(MIXED)
    r = refharness.RefSolver(toml, "Euler1D", [], bounds=(3, 12), variant="exact", newton=newton)
    s.init_state(); r.init_state()
    a = s.step(steps)
    b = r.step(steps)
    assert a["failed_cells"] == 0 and b["failures"] == 0
    # the steps are minima of the CFL rule over nodes whose states come from
    # exp / log of the duals: CUDA's and glibc's last bits accumulate over the steps
    assert abs(a["t"] - b["t"]) <= 1e-8 * b["t"]
    assert s.n_states == 3
    us, ls, _ = s.download_state()
    ur, lr, _ = r.get_state()
    area = r.geometry(2)["area"]
    err = rel_l1(s.mean_var(), r.mean_var(), area)
    assert np.all(err <= (1e-6 if mixed else 1e-10)), err
    if not mixed:
        np.testing.assert_allclose(us, ur, rtol=1e-8, atol=1e-10)
