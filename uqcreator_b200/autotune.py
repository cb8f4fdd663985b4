"""Autotuner of the closure kernel's launch shape.

The closure kernel can run a cell on one warp, two warps (several cells per
CTA, named barriers) or a whole CTA, and can stage the basis tables in shared
memory or read them through L1 (which leaves room for more cells per SM).
Which is fastest depends on the moments per cell, the node count and the
precision. `autotune(solver)` times every candidate on a few time steps of the
solver's own state, restores the state, applies the fastest through
uqc_set_option and returns the timings. Results are cached per configuration
shape (states, moments, nodes, levels, uncertain dimensions, precision) in a
JSON file, so a shape is tuned once per machine.

    s = Solver(toml); s.init_state(); s.step(3)     # tune on a representative state
    best = autotune(s)
"""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path

from ._lib import UqcError, Info, lib, check

__all__ = ["autotune", "candidates", "DEFAULT_CACHE"]

DEFAULT_CACHE = Path(os.environ.get("UQC_AUTOTUNE_CACHE", Path.home() / ".cache" / "uqcreator_b200" / "autotune.json"))


def candidates(n_per_cell: int):
    """Launch shapes worth timing for n = states x moments duals per cell."""
    groups = [32, 64, 256] if n_per_cell <= 64 else [64, 256]
    return [{"closure_group": g, "closure_tables_smem": t} for g in groups for t in (1, 0)]


def _key(solver, precision):
    return f"s{solver.n_states}_t{solver.n_total}_q{solver.n_quad}_l{solver.n_levels}_d{solver.dim_xi}_p{precision}"


def autotune(solver, steps: int = 2, repeats: int = 2, cache: Path | None = DEFAULT_CACHE, verbose: bool = False) -> dict:
    """Times each candidate for `steps` steps (best of `repeats`) from the
    solver's current state, restores that state and applies the fastest.
    Returns {"best": options, "ms_per_step": {name: ms or None}, "cached": bool}."""
    info = Info()
    check(solver.h, lib().uqc_get_info(solver.h, C.byref(info)))
    key = _key(solver, info.precision)
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
    for opts in candidates(solver.n_states * solver.n_total):
        name = ",".join(f"{k}={v}" for k, v in opts.items())
        try:
            for k, v in opts.items():
                solver.set_option(k, v)
            best_ms = None
            for _ in range(repeats):
                solver.upload_state(u0, l0, v0, t=t0)
                solver.step(steps)
                ms = solver.last_timing()[2] / steps
                best_ms = ms if best_ms is None or ms < best_ms else best_ms
            timings[name] = best_ms
        except UqcError as e:    # a shape that does not fit this configuration
            timings[name] = None
            if verbose:
                print("autotune: skip", name, e)
        if verbose:
            print("autotune:", name, timings[name])
    valid = {k: v for k, v in timings.items() if v is not None}
    if not valid:
        raise UqcError(-2, "no launch shape fits this configuration")
    best_name = min(valid, key=valid.get)
    best = {kv.split("=")[0]: int(kv.split("=")[1]) for kv in best_name.split(",")}
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
