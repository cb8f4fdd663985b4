"""Refinement-level machinery on the host: the S_l indicator, the level-rule
bounds and the retardation schedule (configuration, tables, oracle).

The paper's indicator S_l = <(u_l - u_{l-1})^2> / <u_l^2> (Paper1/adaptivity.tex:
12-14) is evaluated from the moments as the added moments' squares over all
squares. That is the quadrature form exactly when the basis tables are
orthonormal under the quadrature, which is checked here for every workload
shape, together with the two forms on random moment vectors. The oracle's
retardation schedule (Paper1/results.tex:179,241) is checked on the adaptive
shallow-water workload: the level cap starts at the first entry and rises once
the residual falls below a threshold. Invalid [uqc] keys are refused.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from uqcreator_b200 import Solver, UqcError, workloads as W

SHAPES = [W.burgers1d(ncells=10), W.euler2d(nx=3, ny=2), W.shallow_water1d(ncells=10), W.euler2d_3u(nx=3, ny=2),
          W.burgers1d(ncells=10, degree=9, nquad=40)]


@pytest.mark.parametrize("toml", SHAPES)
def test_basis_tables_are_orthonormal_under_the_quadrature(toml):
    s = Solver(toml)
    phi, pwf, _, _ = s.tables()
    np.testing.assert_allclose(phi.T @ pwf, np.eye(s.n_total), atol=1e-12)


def test_energy_indicator_coefficient_form_equals_quadrature_form():
    s = Solver(W.shallow_water1d(ncells=10))
    phi, pwf, _, _ = s.tables()
    wt = pwf[:, 0] / phi[:, 0]
    nt = s.n_total_levels
    rng = np.random.default_rng(5)
    for lev in range(len(nt)):
        prev = 1 if lev == 0 else nt[lev - 1]
        for _ in range(5):
            u = rng.normal(size=s.n_total) * 0.5 ** np.arange(s.n_total)
            ul = phi[:, : nt[lev]] @ u[: nt[lev]]
            up = phi[:, :prev] @ u[:prev]
            quad = np.sum((ul - up) ** 2 * wt) / np.sum(ul ** 2 * wt)
            coef = np.sum(u[prev: nt[lev]] ** 2) / np.sum(u[: nt[lev]] ** 2)
            assert abs(quad - coef) <= 1e-12 * max(coef, 1e-300)


def test_oracle_retardation_caps_the_levels():
    ex = ('refinementIndicator = "energy"\nrefinementBounds = [1e-10, 1e-8]\n'
          'retardationLevels = [0, 2, 8]\nretardationResiduals = [1.0, 1e-9]\n')
    o = Oracle(W.shallow_water1d(ncells=400, uqc_extra=ex), None)
    o.init_state()
    o.step(1)
    assert o.get_state()[2].max() == 0          # the first step's rule runs under the first cap
    seen = 0
    for _ in range(30):
        o.step(1)
        lev = o.get_state()[2]
        assert lev.max() <= 2                   # the residual never reaches 1e-9
        seen = max(seen, int(lev.max()))
    assert seen == 2


def test_oracle_energy_indicator_changes_levels():
    ex = 'refinementIndicator = "energy"\nrefinementBounds = [1e-8, 1e-6]\n'
    o = Oracle(W.shallow_water1d(ncells=400, uqc_extra=ex), None)
    d = Oracle(W.shallow_water1d(ncells=400), None)
    o.init_state(); d.init_state()
    o.step(10); d.step(10)
    assert not np.array_equal(o.get_state()[2], d.get_state()[2])


@pytest.mark.parametrize("extra", [
    'refinementIndicator = "variance"\n',
    'refinementBounds = [0.02, 0.004]\n',
    'retardationLevels = [2, 1]\nretardationResiduals = [1e-3]\n',
    'retardationLevels = [0, 1, 2]\nretardationResiduals = [1e-3]\n',
    'retardationLevels = [0, 1, 2]\nretardationResiduals = [1e-4, 1e-3]\n',
])
def test_invalid_level_options_are_refused(extra):
    with pytest.raises(UqcError):
        Solver(W.shallow_water1d(ncells=10, uqc_extra=extra))
