"""Generates the golden vectors in tests/golden/*.npz from the reference itself.

Runs UQCreator's own C++ (code/src, built against project shims into
oracle/_ref/libuqcref.so by `make -C oracle/ref`, which needs the reference
sources) on small cases of every workload:

  c1_solve.npz       Burgers (the Burgers workload at full size: 500 cells, T = 0.11)
                     through MomentSolver::Solve() itself: final mean/variance
                     (full precision) and duals (15 digits, MomentSolver::Export).
  c1_steps.npz       same workload, 25 steps of the harness loop: u, lambda.
  c2_steps.npz       2-D Euler, 2 uncertainties, degree 5, 10x10 nodes, 8x2x2 mesh,
                     guarded Newton, 3 steps: u, lambda, t.
  c3_steps.npz       shallow water, adaptive degree 1..9, 30 nodes, 100 cells, 12 steps.
  c5_steps.npz       2-D Euler, 3 uncertainties, degree 4, 8^3 nodes, 6x2x2 mesh, 1 step.
  c2_closure.npz     batched SolveClosure / SolveClosureSafe from the initial state.
  su2_steps.npz      2-D Euler on the SU2 channel mesh su2_channel.su2 (6x4x2 cells,
                     leaning right wall; written by workloads.su2_channel(6, 4)):
                     Dirichlet inlet, no-slip outlet wall, shallow-water walls
                     top and bottom, 6 steps: u, lambda, t.

    python tests/golden/make_golden.py          # every case
    python tests/golden/make_golden.py su2      # only the named cases
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import su2  # noqa: E402
from oracle.refharness import RefSolver  # noqa: E402
from uqcreator_b200 import workloads as W  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    "c1": dict(toml=W.burgers1d(), problem="Burgers1D", ic=[12.0, 3.0, 0.5, 0.6], bounds=(2.5, 12.5), newton="reference"),
    "c2": dict(toml=W.euler2d(nx=8, ny=2), problem="Euler2D", ic=[0.5, 1.0, 1.0, 0.125, 0.1], bounds=(3, 12), newton="guarded"),
    "c3": dict(toml=W.shallow_water1d(ncells=100), problem="ShallowWater1D", ic=[0.5, 1.0, 0.5], bounds=(3, 12),
               newton="reference"),
    "c5": dict(toml=W.euler2d_3u(nx=6, ny=2), problem="Euler2D", ic=[0.5, 1.0, 1.0, 0.125, 0.1], bounds=(3, 12),
               newton="guarded"),
}
STEPS = {"c1": 25, "c2": 3, "c3": 12, "c5": 1, "su2": 6}
SU2_FILE = OUT / "su2_channel.su2"
SU2_BC = [["inlet", "dirichlet"], ["outlet", "noslip"], ["bottom", "swwall"], ["top", "swwall"]]
CASES["su2"] = dict(toml=W.euler2d_su2("su2_channel.su2", bcs=SU2_BC), problem="Euler2D", ic=[0.7, 1.0, 1.0, 0.125, 0.1],
                    bounds=(3, 12), newton="guarded")


def su2_mesh():
    return su2.read_su2(str(SU2_FILE), su2.bc_table(SU2_BC))


def ref(name, variant="exact", newton=None):
    c = CASES[name]
    mesh = su2_mesh() if name == "su2" else W.mesh_for(c["toml"])
    return RefSolver(c["toml"], c["problem"], c["ic"], bounds=c["bounds"], mesh2d=mesh,
                     variant=variant, newton=newton or c["newton"])


def main(only=()):
    SU2_FILE.write_text(W.su2_channel(6, 4))
    if not only:
        r = ref("c1")
        mv, lam15 = r.full_solve()
        np.savez_compressed(OUT / "c1_solve.npz", mean_var=mv, lambda15=lam15, toml=CASES["c1"]["toml"])
    for name, n in STEPS.items():
        if only and name not in only:
            continue
        r = ref(name)
        r.init_state()
        out = r.step(n)
        u, lam, lev = r.get_state()
        np.savez_compressed(OUT / f"{name}_steps.npz", u=u, lam=lam, level=lev, t=out["t"], dt=out["dt"],
                            residual=out["residual"], steps=n, mean_var=r.mean_var(), toml=CASES[name]["toml"],
                            newton=CASES[name]["newton"])
    if only:
        return
    res = {}
    for mode in ("reference", "guarded", "safe"):
        r = ref("c2", newton=mode)
        r.init_state()
        u, lam, _ = r.get_state()
        lam2, st = r.solve_closure(lam, u)
        res[f"lam_{mode}"] = lam2
        res[f"status_{mode}"] = st
        res["u"], res["lam0"] = u, lam
    np.savez_compressed(OUT / "c2_closure.npz", toml=CASES["c2"]["toml"], **res)
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))    # case names (e.g. su2) regenerate only those
