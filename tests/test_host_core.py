"""The product's host-side tables and geometry pinned to the reference's own.

uqc_get_tables returns the basis tables the kernels use (phiTilde, phiTildeWf,
quadrature nodes and weights of Closure::Closure, closure.cpp:16-84, built by
uqcreator_b200/csrc/tables.cpp) and uqc_get_geometry the mesh geometry
(Line/Triangle, built by csrc/mesh.cpp). Both are built on the host when a
handle is created, so these checks need no GPU. They are compared bit for bit
with what the reference's own Closure and Cell classes compute (oracle/_ref,
the reference compiled from its sources), for the shapes of every workload:
1-D Burgers (degree 4, 20 nodes), 2-D Euler (total degree 5, 10 x 10 nodes),
adaptive shallow water (degrees 1..9, 30 nodes), 2-D Euler with three
uncertainties (total degree 4, 8^3 nodes) and the serving stream's small
shapes (Burgers degree 9 with 40 nodes, Euler total degree 2 with 4 x 4).
"""
import numpy as np
import pytest

from oracle import refharness
from uqcreator_b200 import Solver, workloads as W

pytestmark = pytest.mark.skipif(not refharness.available(), reason="reference harness oracle/_ref not built")

EULER_IC = [0.5, 1.0, 1.0, 0.125, 0.1]
CASES = {
    "burgers1d": (W.burgers1d(ncells=60), "Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5)),
    "euler2d": (W.euler2d(nx=9, ny=4), "Euler2D", EULER_IC, (3, 12)),
    "sw1d_adaptive": (W.shallow_water1d(ncells=80), "ShallowWater1D", [0.5, 1.0, 0.5], (3, 12)),
    "euler2d_3u": (W.euler2d_3u(nx=5, ny=3), "Euler2D", EULER_IC, (3, 12)),
    "burgers1d_deg9": (W.burgers1d(ncells=40, degree=9, nquad=40), "Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5)),
    "euler2d_deg2": (W.euler2d(nx=7, ny=5, degree=2, nquad=4, seed=3), "Euler2D", EULER_IC, (3, 12)),
    "euler1d": (W.euler1d(ncells=40, degree=4, nquad=10), "Euler1D", [], (3, 12)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_tables_and_geometry_bit_identical_to_reference(case):
    toml, problem, ic, bounds = CASES[case]
    s = Solver(toml)
    r = refharness.RefSolver(toml, problem, ic, bounds=bounds, mesh2d=W.mesh_for(toml))
    assert (s.n_cells, s.n_states, s.n_total, s.n_quad) == (r.n_cells, r.n_states, r.n_total, r.n_q)
    assert s.n_total_levels == r.n_total_levels
    for name, a, b in zip(("phi", "phi_wf", "xi", "w"), s.tables(), r.tables()):
        np.testing.assert_array_equal(a, b, err_msg=name)
    gs, gr = s.geometry(), r.geometry(s.n_faces)
    for k in ("area", "max_edge", "center", "unit_normal", "scaled_normal"):
        np.testing.assert_array_equal(gs[k], gr[k], err_msg=k)
    # neighbour ids: the product gives a missing neighbour the ghost id n_cells;
    # the reference leaves that slot unset (1-D end cells, mesh1d.cpp:38-47), so
    # only the slots with a real neighbour are compared
    real = gs["nbr"] < s.n_cells
    np.testing.assert_array_equal(gs["nbr"][real], gr["nbr"][real])
    assert real[gs["boundary"] == 0].all()
    # the product marks Dirichlet cells 1 (walls 2, 3); these meshes have Dirichlet boundaries only
    np.testing.assert_array_equal(gs["boundary"] != 0, gr["boundary"] != 0)
