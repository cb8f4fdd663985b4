"""The drop-in proof: UQCreator's own MomentSolver::Solve() with its closure
on the GPU (needs a B200).

oracle/_ref/libuqcref_gpu.so is the reference's code/src compiled from its
sources (the oracle harness) with one change a maintainer would make:
Closure::Create returns GpuClosure (oracle/ref/gpuclosure.cpp), which
overrides SolveClosure with a call to uqc_closure_solve_host on the cell's
Matrix storage. Everything else is the reference's: the time loop of
momentsolver.cpp:79-162, ExplicitEuler, the Burgers flux of the workload, the
ansatz, re-projection, mean and variance. The Burgers workload (500 cells,
T = 0.11, 459 steps) must reproduce the mean and variance that the
reference's unmodified Solve() wrote (tests/golden/c1_solve.npz) within
relative L1 1e-10, the bound of the FP64 form.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import refharness

from ._util import rel_l1

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.skipif(not refharness.available("gpu"), reason="oracle/_ref/libuqcref_gpu.so not built (make -C oracle/ref)")
def test_reference_moment_solver_with_gpu_closure():
    g = np.load(GOLD / "c1_solve.npz")
    r = refharness.RefSolver(str(g["toml"]), "Burgers1D", [12.0, 3.0, 0.5, 0.6], bounds=(2.5, 12.5), variant="gpu",
                             newton="reference")
    mv, lam15 = r.full_solve()
    area = r.geometry(2)["area"]
    err = rel_l1(mv, g["mean_var"], area)
    assert np.all(err <= 1e-10), err
    np.testing.assert_allclose(lam15, g["lambda15"], rtol=1e-9, atol=1e-9)
