"""Autotuner of the time step's launch shapes and schedules.

What it chooses, per configuration shape:
- closure (FP64 form): a cell on one warp, two warps (several cells per CTA,
  named barriers) or a whole CTA, with the basis tables staged in shared memory
  or read through L1 (which leaves room for more cells per SM);
- chord schedule of the single mixed kernel: theta and whether the held FP32
  factor is kept as its packed inverse;
- chord schedule (mixed form in rounds, 2-D Euler): theta, the contraction
  below which a cell's held inverse is re-formed (more re-factorisations mean
  fewer, dearer iterations), and the re-factorisation rounds per step before
  the FP64 form takes the remaining cells;
- where the next step's convergence test runs: in the update kernel, which
  then lists the cells that need Newton or a level change (update_test 1), or
  in the check kernel over every cell (0);
- CTA sizes: cells (warps) per CTA of the chord kernel, the convergence-check
  kernel and the update kernel (occupancy against shared memory and
  registers, and the grain of the work stealing).

Which is fastest depends on the moments per cell, the node count, the
precision and the state. `autotune(solver)` times the candidates on a few time
steps of the solver's own state (after untimed warm-up steps, so held inverses
are in their steady state) by coordinate descent: the groups above in turn,
each candidate with the best of the groups before it applied. It restores the
state, applies the best options through uqc_set_option and returns the
timings. Results are cached per configuration shape (states, moments, nodes,
levels, uncertain dimensions, precision, mixed form) in a JSON file, so a shape
is tuned once per machine.

    s = Solver(toml); s.init_state(); s.step(3)     # tune on a representative state
    best = autotune(s)
"""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path

from ._lib import UqcError, Info, lib, check

__all__ = ["autotune", "candidates", "groups", "DEFAULT_CACHE"]

DEFAULT_CACHE = Path(os.environ.get("UQC_AUTOTUNE_CACHE", Path.home() / ".cache" / "uqcreator_b200" / "autotune.json"))


THETAS = (0.05, 0.1, 0.2, 0.35, 0.5)
ROUNDS = (2, 3)


def candidates(n_per_cell: int, mixed_form: int = 0):
    """Options of the first group: launch shapes of the FP64 closure kernel for
    n = states x moments duals per cell, or (mixed form in rounds) the chord
    schedule: theta x re-factorisation rounds."""
    if mixed_form >= 1:
        return [{"mixed_chord_theta": t, "mixed_rounds": r} for t in THETAS for r in ROUNDS]
    groups = [32, 64, 256] if n_per_cell <= 64 else [64, 256]
    return [{"closure_group": g, "closure_tables_smem": t} for g in groups for t in (1, 0)]


def groups(n_per_cell: int, mixed_form: int = 0, mixed: bool = False):
    """The option groups of the coordinate descent, in order: (name, candidates).
    mixed: the handle runs UQC_MIXED (with mixed_form 0: the single mixed kernel,
    whose chord schedule is theta and whether the held factor is kept as its
    inverse)."""
    out = [("closure" if mixed_form == 0 else "schedule", candidates(n_per_cell, mixed_form))]
    if mixed and mixed_form == 0:
        out.append(("single_schedule", [{"mixed_chord_theta": t, "mixed_chord_inverse": ci}
                                        for t in (0.05, 0.1, 0.2, 0.35) for ci in (1, 0)]))
    if mixed_form >= 1:
        out.append(("chord_cta", [{"chord_warps": w} for w in (8, 12, 16)]))
    out.append(("update_test", [{"update_test": v} for v in (1, 0)]))
    out.append(("check_cta", [{"check_warps": w} for w in (8, 16)]))
    out.append(("update_cta", [{"update_warps": w} for w in (4, 8, 16)]))
    return out


def _key(solver, precision, mixed_form):
    return (f"v4_s{solver.n_states}_t{solver.n_total}_q{solver.n_quad}_l{solver.n_levels}_d{solver.dim_xi}_p{precision}"
            f"_m{mixed_form if precision else 0}")


def autotune(solver, steps: int = 2, repeats: int = 2, cache: Path | None = DEFAULT_CACHE, verbose: bool = False,
             warmup: int = 2) -> dict:
    """Times each candidate for `steps` steps (best of `repeats`, each after
    `warmup` untimed steps) from the solver's current state, restores that
    state and applies the fastest.
    Returns {"best": options, "ms_per_step": {name: ms or None}, "cached": bool}."""
    info = Info()
    check(solver.h, lib().uqc_get_info(solver.h, C.byref(info)))
    mixed_form = info.mixed_form if info.precision == 1 else 0
    key = _key(solver, info.precision, mixed_form)
    table = {}
    if cache is not None and Path(cache).exists():
        try:
            table = json.loads(Path(cache).read_text())
        except (OSError, ValueError):
            table = {}
    if key in table:
        best = table[key]["best"]
        for k, v in best.items():
            solver.set_option(k, v)
        return {"best": best, "ms_per_step": table[key]["ms_per_step"], "cached": True}
    u0, l0, v0 = solver.download_state()
    t0 = info.t
    timings = {}
    best = {}

    def time_options(opts):
        for k, v in opts.items():
            solver.set_option(k, v)
        best_ms = None
        for _ in range(repeats):
            solver.upload_state(u0, l0, v0, t=t0)
            if warmup:
                solver.step(warmup)
            solver.step(steps)
            ms = solver.last_timing()[2] / steps
            best_ms = ms if best_ms is None or ms < best_ms else best_ms
        return best_ms

    for gname, cands in groups(solver.n_states * solver.n_total, mixed_form, info.precision == 1):
        group_best, group_ms = None, None
        for opts in cands:
            name = ",".join(f"{k}={v}" for k, v in opts.items())
            try:
                ms = time_options(opts)
            except UqcError as e:    # a shape that does not fit this configuration
                ms = None
                if verbose:
                    print("autotune: skip", name, e)
            timings[name] = ms
            if verbose:
                print("autotune:", gname, name, ms)
            if ms is not None and (group_ms is None or ms < group_ms):
                group_best, group_ms = opts, ms
        if group_best is None:
            raise UqcError(-2, f"no {gname} option fits this configuration")
        best.update(group_best)
        for k, v in group_best.items():
            solver.set_option(k, v)
    for k, v in best.items():
        solver.set_option(k, v)
    solver.upload_state(u0, l0, v0, t=t0)
    if cache is not None:
        try:
            Path(cache).parent.mkdir(parents=True, exist_ok=True)
            table[key] = {"best": best, "ms_per_step": timings}
            Path(cache).write_text(json.dumps(table, indent=1))
        except OSError:
            pass
    return {"best": best, "ms_per_step": timings, "cached": False}
