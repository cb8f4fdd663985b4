"""The oracle (C restatement, oracle/uqc_oracle.c) pinned to the reference.

1. Against the committed golden vectors made by UQCreator's own code
   (tests/golden/make_golden.py, MomentSolver::Solve included): always runs.
2. Bit for bit against the reference harness itself (oracle/_ref), when that
   build is present.
All comparisons are exact: both sides are IEEE double arithmetic in the same
operation order with the same libm.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import refharness
from oracle.oracle import Oracle
from uqcreator_b200 import workloads as W

GOLD = Path(__file__).resolve().parent / "golden"


def _oracle_for(npz, newton=None):
    toml = str(npz["toml"])
    if newton is not None:
        toml = toml.replace('newton = "reference"', f'newton = "{newton}"').replace('newton = "guarded"', f'newton = "{newton}"')
    return Oracle(toml, W.mesh_for(toml))


def test_c1_full_solve_matches_reference_solve():
    """MomentSolver::Solve (500 cells, T=0.11, 459 steps) vs the oracle's time loop."""
    g = np.load(GOLD / "c1_solve.npz")
    o = _oracle_for(g)
    o.init_state()
    tend = W.parse(str(g["toml"]))["problem"]["tEnd"]
    steps = 0
    while True:
        r = o.step(1)
        steps += 1
        if r["t"] >= tend:
            break
    assert steps == 459
    mv = o.mean_var()
    np.testing.assert_array_equal(mv, g["mean_var"])
    _, lam, _ = o.get_state()
    np.testing.assert_allclose(lam, g["lambda15"], rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("case", ["c1", "c2", "c3", "c5"])
def test_steps_match_golden(case):
    g = np.load(GOLD / f"{case}_steps.npz")
    o = _oracle_for(g)
    o.init_state()
    r = o.step(int(g["steps"]))
    u, lam, lev = o.get_state()
    np.testing.assert_array_equal(u, g["u"])
    np.testing.assert_array_equal(lam, g["lam"])
    np.testing.assert_array_equal(lev, g["level"])
    assert r["t"] == float(g["t"]) and r["dt"] == float(g["dt"]) and r["residual"] == float(g["residual"])
    np.testing.assert_array_equal(o.mean_var(), g["mean_var"])


@pytest.mark.parametrize("mode", ["reference", "guarded", "safe"])
def test_batched_closure_matches_golden(mode):
    g = np.load(GOLD / "c2_closure.npz")
    o = _oracle_for(g, newton=mode)
    lam, st, it = o.solve_closure(g["lam0"], g["u"])
    ok = g[f"status_{mode}"] == 0
    np.testing.assert_array_equal((st == 0), ok)
    np.testing.assert_array_equal(lam[ok], g[f"lam_{mode}"][ok])


@pytest.mark.skipif(not refharness.available(), reason="reference harness oracle/_ref not built")
@pytest.mark.parametrize("case,steps,newton", [("burgers", 7, "reference"), ("euler2u", 2, "guarded"),
                                               ("sw", 6, "reference"), ("euler2u", 2, "safe")])
def test_bit_exact_against_reference_harness(case, steps, newton):
    if case == "burgers":
        toml, prob, ic, b = W.burgers1d(ncells=120), "Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5)
    elif case == "euler2u":
        toml, prob, ic, b = W.euler2d(nx=10, ny=3, newton=newton), "Euler2D", [0.5, 1.0, 1.0, 0.125, 0.1], (3, 12)
    else:
        toml, prob, ic, b = W.shallow_water1d(ncells=150), "ShallowWater1D", [0.5, 1.0, 0.5], (3, 12)
    mesh = W.mesh_for(toml)
    r = refharness.RefSolver(toml, prob, ic, bounds=b, mesh2d=mesh, newton=newton)
    o = Oracle(toml, mesh)
    for a, c in zip(r.tables(), o.tables()):
        np.testing.assert_array_equal(a, c)
    gr, go = r.geometry(o.n_faces), o.geometry()
    for k in ("area", "max_edge", "center", "unit_normal", "scaled_normal", "boundary"):
        np.testing.assert_array_equal(gr[k], go[k])
    r.init_state(); o.init_state()
    a, c = r.step(steps), o.step(steps)
    assert a == c
    for x, y in zip(r.get_state(), o.get_state()):
        np.testing.assert_array_equal(x, y)
