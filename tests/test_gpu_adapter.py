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


@pytest.mark.skipif(not refharness.available("gpu"), reason="oracle/_ref/libuqcref_gpu.so not built (make -C oracle/ref)")
@pytest.mark.parametrize("case", ["burgers", "euler2d"])
def test_gpu_moment_solver_drop_in(case, tmp_path):
    """GpuMomentSolver (oracle/ref/gpumomentsolver.cpp): MomentSolver's
    constructor and Solve() over the C ABI, writing through the reference's own
    Mesh::Export and "moments"/"duals" loggers. Its final mean and variance,
    moments and duals match what the reference's unmodified Solve() writes
    from the same input (relative L1 1e-10 on E/Var, 1e-9 on the moments)."""
    from uqcreator_b200 import workloads as W
    if case == "burgers":
        toml = W.burgers1d(ncells=200, tend=0.05)
        args = ("Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5), None, "reference")
    else:
        # a case the reference's own Newton (no finiteness guard) solves to the end
        toml = W.euler2d(nx=12, ny=4, degree=2, nquad=4, tend=0.02, newton="reference")
        args = ("Euler2D", [0.5, 1.0, 1.0, 0.125, 0.1], (3, 12), W.mesh_for(toml), "reference")
    problem, ic, bounds, mesh, newton = args
    ref = refharness.RefSolver(toml, problem, ic, bounds=bounds, mesh2d=mesh, variant="exact", newton=newton)
    mv_ref = ref.full_solve_export(str(tmp_path / "ref"))
    gpu = refharness.RefSolver(toml, problem, ic, bounds=bounds, mesh2d=mesh, variant="gpu", newton=newton)
    mv_gpu = gpu.full_solve_gpu(str(tmp_path / "gpu"))
    area = ref.geometry(2 if mesh is None else 3)["area"]
    err = rel_l1(mv_gpu, mv_ref, area)
    assert np.all(err <= 1e-10), err
    def lines(path):    # MomentSolver::Export: comma after every value
        return np.array([[float(v) for v in ln.rstrip().rstrip(",").split(",")] for ln in open(path) if ln.strip()])

    for kind, tol in (("_moments", 1e-9), ("_duals", 1e-6)):
        a, b = lines(tmp_path / ("gpu" + kind)), lines(tmp_path / ("ref" + kind))
        assert a.shape == b.shape == (ref.n_cells, ref.n_states * ref.n_total)
        np.testing.assert_allclose(a, b, rtol=tol, atol=tol)
