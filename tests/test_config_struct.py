"""uqc_create_from_config: the input file's settings as a C struct.

A handle made from a uqc_config struct must be the handle made from the
equivalent input file: same sizes, basis tables, quadrature and mesh geometry
(bit for bit; host-side, no GPU needed), for a 1-D Burgers, an adaptive
shallow-water and a 2-D Euler configuration; invalid structs are refused.
"""
import ctypes as C

import numpy as np
import pytest

from uqcreator_b200 import Solver, UqcError, workloads as W
from uqcreator_b200._lib import Config, lib


def _cfg(problem, closure, **kw):
    c = Config()
    lib().uqc_config_defaults(C.byref(c))
    c.problem, c.closure = problem.encode(), closure.encode()
    for k, v in kw.items():
        if k in ("sigma", "degree", "quad_points", "ic", "bounds"):
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = x
            if k == "ic":
                c.n_ic = len(v)
            if k == "degree":
                c.n_levels = len(v)
        else:
            setattr(c, k, v)
    return c


CASES = {
    "burgers": (W.burgers1d(ncells=60, degree=4, nquad=20),
                dict(problem="Burgers1D", closure="BoundedBarrier", mesh_dimension=1, n_cells=60, a=0.0, b=3.0, dim_xi=1,
                     sigma=[0.2], cfl=0.5, t_end=0.11, degree=[4], quad_points=[20], max_iterations=1000, epsilon=1e-10,
                     ic=[12.0, 3.0, 0.5, 0.6], bounds=[2.5, 12.5])),
    "sw_adaptive": (W.shallow_water1d(ncells=80),
                    dict(problem="ShallowWater1D", closure="ShallowWater", mesh_dimension=1, n_cells=80, a=0.0, b=1.0,
                         dim_xi=1, sigma=[0.2], cfl=0.5, t_end=0.05, degree=list(range(1, 10)), quad_points=[30] * 9,
                         max_iterations=1000, epsilon=1e-10, ic=[0.5, 1.0, 0.5])),
    "euler2d": (W.euler2d(nx=7, ny=3, degree=3, nquad=6),
                dict(problem="Euler2D", closure="Euler2D", mesh_dimension=2, dim_xi=2, sigma=[0.05, 0.1], cfl=0.5, t_end=0.2,
                     gamma=1.4, degree=[3], quad_points=[6], max_iterations=1000, epsilon=1e-10,
                     ic=[0.5, 1.0, 1.0, 0.125, 0.1], nx=7, ny=3, jitter=0.2, seed=7, newton_mode=1)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_struct_handle_equals_file_handle(case):
    toml, kw = CASES[case]
    a = Solver(toml)
    b = Solver.from_config(_cfg(**kw))
    assert (a.n_cells, a.n_states, a.n_total, a.n_quad, a.n_levels, a.dim_xi) == \
           (b.n_cells, b.n_states, b.n_total, b.n_quad, b.n_levels, b.dim_xi)
    assert a.n_total_levels == b.n_total_levels
    for x, y in zip(a.tables(), b.tables()):
        np.testing.assert_array_equal(x, y)
    ga, gb = a.geometry(), b.geometry()
    for k in ga:
        np.testing.assert_array_equal(ga[k], gb[k])


def test_invalid_structs_are_refused():
    _, kw = CASES["burgers"]
    for bad in (dict(kw, problem="Euler1D"), dict(kw, n_cells=0), dict(kw, newton_mode=5)):
        with pytest.raises(UqcError):
            Solver.from_config(_cfg(**bad))
    c = _cfg(**kw)
    c.problem = None
    with pytest.raises(UqcError):
        Solver.from_config(c)
