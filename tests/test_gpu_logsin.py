"""LogSin closure on the GPU against the reference itself (needs a B200).

LogSin (logsin.cpp: U = ((u+ - u-) / PI)(PI / 2 + atan Lambda) + u-, one state,
bounds fixed by the number of uncertain dimensions) runs as closure kind 8
with the Burgers problem. The check is against the reference's own closure
and time loop compiled from its sources (oracle/_ref, the exact build), in
one and two uncertain dimensions: FP64 mean and variance within relative L1
1e-10 and moments within 1e-8 elementwise (Newton to |g| < 1e-12); the mixed
form within 1e-6.
"""
import numpy as np
import pytest

from oracle import refharness
from uqcreator_b200 import MIXED, Solver, workloads as W

from ._util import rel_l1

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refharness.available("exact"), reason="oracle/_ref/libuqcref.so not built")]


def _logsin(dims):
    t = W.burgers1d(ncells=300, degree=4, nquad=12, tend=0.05, eps=1e-12).replace('closure = "BoundedBarrier"', 'closure = "LogSin"')
    if dims == 2:
        t2 = t.replace('distribution = [["Legendre"],[0.2]]', 'distribution = [["Legendre","Legendre"],[0.2,0.1]]')
        assert t2 != t
        t = t2
    return t


@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
@pytest.mark.parametrize("dims", [1, 2])
def test_logsin_steps_match_reference(dims, mixed):
    toml = _logsin(dims)
    s = Solver(toml)
    if mixed:
        s.set_precision(MIXED)
    r = refharness.RefSolver(toml, "Burgers1D", [12.0, 3.0, 0.5, 0.6], bounds=(2.5, 12.5), variant="exact", newton="reference")
    s.init_state(); r.init_state()
    a = s.step(20)
    b = r.step(20)
    assert a["failed_cells"] == 0 and b["failures"] == 0
    assert a["newton_iterations"] > 0
    assert abs(a["t"] - b["t"]) <= 1e-8 * b["t"]
    area = r.geometry(2)["area"]
    err = rel_l1(s.mean_var(), r.mean_var(), area)
    assert np.all(err <= (1e-6 if mixed else 1e-10)), err
    if not mixed:
        np.testing.assert_allclose(s.download_state()[0], r.get_state()[0], rtol=1e-8, atol=1e-10)
