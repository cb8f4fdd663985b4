"""Python mirror of UQCreator's operator surface for the IPM hot path.

Same names, argument meaning and error behaviour as the reference's C++
classes (code/src/settings.h, closure.h, momentsolver.h), backed by the CUDA
kernels through the C ABI (include/uqc.h). Errors raise UqcError instead of
exiting the process, and Newton failures are reported per cell.

    s = Settings(toml_path)                 # Settings::Settings (settings.h:103)
    solver = MomentSolver(s)                # MomentSolver(settings, mesh, problem)
    solver.Solve()                          # MomentSolver::Solve (momentsolver.cpp:37-162)
    mv = solver.mean_var()                  # WriteMeanAndVar (momentsolver.cpp:302-328)

    closure = Closure.Create(s)             # Closure::Create (closure.cpp:94-131)
    closure.SolveClosure(lam, u, nTotal, nQTotal)   # in place, batched over cells
"""
from __future__ import annotations

import ctypes as C
import os
import tomllib

import numpy as np

from . import _lib as L
from ._lib import UqcError, StepInfo, Info, ptr, check

__all__ = ["Settings", "Solver", "Closure", "MomentSolver", "UqcError"]


class Settings:
    """The input file: reference TOML schema plus an optional [uqc] table."""

    def __init__(self, toml_path_or_text: str):
        if os.path.exists(toml_path_or_text):
            with open(toml_path_or_text) as f:
                self.text = f.read()
            self.path = toml_path_or_text
        else:
            self.text = toml_path_or_text
            self.path = None
        self.doc = tomllib.loads(self.text)

    # getters named as in settings.h:107-183 (subset read by the hot path)
    def GetProblemType(self):
        return self.doc["general"]["problem"]

    def GetClosureType(self):
        return self.doc["moment_system"]["closure"]

    def GetCFL(self):
        return float(self.doc["problem"]["CFL"])

    def GetTEnd(self):
        return float(self.doc["problem"]["tEnd"])

    def GetEpsilon(self):
        return float(self.doc["moment_system"].get("epsilon", 5e-5))

    def GetMaxIterations(self):
        return int(self.doc["moment_system"].get("maxIterations", 1000))

    def GetNDimXi(self):
        return len(self.doc["problem"]["distribution"][0])


class Solver:
    """Owns one uqc_solver handle: settings, mesh, tables and device state."""

    def __init__(self, settings: Settings | str, stream=None):
        if isinstance(settings, str):
            settings = Settings(settings)
        self.settings = settings
        self.lib = L.lib()
        h = C.c_void_p()
        err = C.create_string_buffer(1024)
        s = None if stream is None else C.c_void_p(int(stream))
        if settings.path is not None:    # files the config names are relative to its directory
            rc = self.lib.uqc_create_from_file(os.fsencode(settings.path), s, C.byref(h), err, 1024)
        else:
            rc = self.lib.uqc_create_from_string(settings.text.encode(), s, C.byref(h), err, 1024)
        if rc != 0:
            raise UqcError(rc, err.value.decode())
        self.h = h
        info = Info()
        check(h, self.lib.uqc_get_info(h, C.byref(info)))
        self.n_cells, self.n_states, self.n_total, self.n_quad = info.n_cells, info.n_states, info.n_total, info.n_quad
        self.n_levels, self.dim_xi, self.n_faces = info.n_levels, info.dim_xi, info.n_faces
        self.n_total_levels = list(info.n_total_level)[: info.n_levels]

    @classmethod
    def from_config(cls, cfg, stream=None) -> "Solver":
        """A solver from a uqc_config struct (uqcreator_b200._lib.Config) instead
        of an input file (uqc_create_from_config)."""
        self = cls.__new__(cls)
        self.settings = None
        self.lib = L.lib()
        h = C.c_void_p()
        err = C.create_string_buffer(1024)
        s = None if stream is None else C.c_void_p(int(stream))
        rc = self.lib.uqc_create_from_config(C.byref(cfg), s, C.byref(h), err, 1024)
        if rc != 0:
            raise UqcError(rc, err.value.decode())
        self.h = h
        info = Info()
        check(h, self.lib.uqc_get_info(h, C.byref(info)))
        self.n_cells, self.n_states, self.n_total, self.n_quad = info.n_cells, info.n_states, info.n_total, info.n_quad
        self.n_levels, self.dim_xi, self.n_faces = info.n_levels, info.dim_xi, info.n_faces
        self.n_total_levels = list(info.n_total_level)[: info.n_levels]
        return self

    def form(self):
        """Precision in use and how UQC_MIXED steps run the closure (uqc_info:
        mixed_form 0 single kernel, 1 rounds with the CUDA-core Hessian, 2 with
        the tensor-core Hessian; -1 before the device side is set up)."""
        info = Info()
        check(self.h, self.lib.uqc_get_info(self.h, C.byref(info)))
        return dict(precision=info.precision, mixed_form=info.mixed_form, mixed_rounds=info.mixed_rounds)

    def debug_mixed_inverse(self, cells, form):
        """H^-1 (FP32) of the mixed form's re-factorisation for the given cells of
        the resident state; form 1: Hessian on CUDA cores, 2: on the tensor cores."""
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        n = self.n_states * self.n_total
        out = np.zeros((len(cells), n, n), dtype=np.float32)
        check(self.h, self.lib.uqc_debug_mixed_inverse(self.h, len(cells), ptr(cells, L._ip), form,
                                                       out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.uqc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- tables / geometry
    def tables(self):
        nq, nt = self.n_quad, self.n_total
        phi = np.zeros((nq, nt)); pwf = np.zeros((nq, nt)); xi = np.zeros((nq, self.dim_xi)); w = np.zeros(nq)
        check(self.h, self.lib.uqc_get_tables(self.h, ptr(phi), ptr(pwf), ptr(xi), ptr(w)))
        return phi, pwf, xi, w

    def geometry(self):
        n, f = self.n_cells, self.n_faces
        g = dict(area=np.zeros(n), max_edge=np.zeros(n), center=np.zeros((n, 2)), unit_normal=np.zeros((n, f, 2)),
                 scaled_normal=np.zeros((n, f, 2)), nbr=np.zeros((n, f), dtype=np.int32),
                 boundary=np.zeros(n, dtype=np.int32))
        check(self.h, self.lib.uqc_get_geometry(self.h, ptr(g["area"]), ptr(g["max_edge"]), ptr(g["center"]),
                                                ptr(g["unit_normal"]), ptr(g["scaled_normal"]),
                                                ptr(g["nbr"], L._ip), ptr(g["boundary"], L._ip)))
        return g

    # ---- state
    def init_state(self):
        check(self.h, self.lib.uqc_init_state(self.h))

    def upload_state(self, u, lam, level=None, t=0.0, layout=L.LAYOUT_STATE_MAJOR):
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        lev = None if level is None else np.ascontiguousarray(level, dtype=np.uint32)
        check(self.h, self.lib.uqc_upload_state(self.h, ptr(u), ptr(lam), ptr(lev, L._up), layout, t))

    def download_state(self, layout=L.LAYOUT_STATE_MAJOR, out=None):
        """(u, lambda, level); out = caller-owned (e.g. pinned) arrays to fill."""
        shape = (self.n_cells, self.n_states, self.n_total)
        if out is not None:
            u, lam, lev = out
            assert u.shape == shape and lam.shape == shape and lev.dtype == np.uint32 and u.flags.c_contiguous
        else:
            u = np.zeros(shape); lam = np.zeros(shape); lev = np.zeros(self.n_cells, dtype=np.uint32)
        check(self.h, self.lib.uqc_download_state(self.h, ptr(u), ptr(lam), ptr(lev, L._up), layout))
        return u, lam, lev

    def export_state(self, path_prefix: str):
        """MomentSolver::Export: <prefix>_moments and <prefix>_duals, the reference's restart files."""
        check(self.h, self.lib.uqc_export_state(self.h, str(path_prefix).encode()))

    def write_vtk(self, path: str):
        """Mesh::Export: legacy VTK file of the mean and variance (cell and point data)."""
        check(self.h, self.lib.uqc_write_vtk(self.h, str(path).encode()))

    def set_precision(self, precision: int):
        check(self.h, self.lib.uqc_set_precision(self.h, precision))

    def set_option(self, key: str, value: float):
        check(self.h, self.lib.uqc_set_option(self.h, key.encode(), float(value)))

    def set_newton(self, max_iterations: int, epsilon: float, mode: int):
        check(self.h, self.lib.uqc_set_newton(self.h, max_iterations, epsilon, mode))

    # ---- hot path
    def solve_closure(self, raise_on_failure=True):
        info = StepInfo()
        rc = self.lib.uqc_solve_closure(self.h, C.byref(info))
        if rc != 0 and (raise_on_failure or rc != -4):
            check(self.h, rc)
        return info.as_dict()

    def solve_closure_cells(self, cells=None, tol=0.0, max_iter=0, raise_on_failure=True):
        """Closure on a subset of the resident cells (None: all) with this call's
        tolerance and iteration limit (0: the configured ones)."""
        info = StepInfo()
        if cells is None:
            rc = self.lib.uqc_solve_closure_cells(self.h, None, 0, float(tol), int(max_iter), C.byref(info))
        else:
            c = np.ascontiguousarray(cells, dtype=np.uint32)
            rc = self.lib.uqc_solve_closure_cells(self.h, ptr(c, L._up), len(c), float(tol), int(max_iter), C.byref(info))
        if rc != 0 and (raise_on_failure or rc != -4):
            check(self.h, rc)
        return info.as_dict()

    def cell_status(self):
        st = np.zeros(self.n_cells, dtype=np.int32); it = np.zeros(self.n_cells, dtype=np.int32)
        check(self.h, self.lib.uqc_cell_status(self.h, ptr(st, L._ip), ptr(it, L._ip)))
        return st, it

    def step(self, n_steps=1, raise_on_failure=True):
        info = StepInfo()
        rc = self.lib.uqc_step(self.h, n_steps, C.byref(info))
        if rc != 0 and (raise_on_failure or rc != -4):
            check(self.h, rc)
        return info.as_dict()

    def step_host(self, u, lam, level=None, t=0.0, out=None, raise_on_failure=True):
        """One step from host state to host state (uqc_step_host): upload, step
        and download with the copies beside the kernels. u, lam: (n_cells,
        n_states, n_total) float64, C-contiguous (pinned memory for overlap);
        out = (u, lam, level) arrays to fill (may be the inputs), else new ones.
        Returns (u, lam, level, info)."""
        shape = (self.n_cells, self.n_states, self.n_total)
        for a in (u, lam):
            assert a.shape == shape and a.dtype == np.float64 and a.flags.c_contiguous
        lev = None if level is None else np.ascontiguousarray(level, dtype=np.uint32)
        if out is None:
            out = (np.empty(shape), np.empty(shape), np.empty(self.n_cells, dtype=np.uint32))
        uo, lo, vo = out
        for a in (uo, lo):
            assert a.shape == shape and a.dtype == np.float64 and a.flags.c_contiguous
        assert vo is None or (vo.dtype == np.uint32 and vo.shape == (self.n_cells,))
        info = StepInfo()
        rc = self.lib.uqc_step_host(self.h, ptr(u), ptr(lam), ptr(lev, L._up), float(t), ptr(uo), ptr(lo), ptr(vo, L._up),
                                    C.byref(info))
        if rc != 0 and (raise_on_failure or rc != -4):
            check(self.h, rc)
        return uo, lo, vo, info.as_dict()

    def step_async(self, n_steps=1):
        """Enqueues n_steps steps and returns at once (uqc_step_async)."""
        check(self.h, self.lib.uqc_step_async(self.h, n_steps))

    def step_query(self):
        """None while the last step_async runs, else its step info."""
        info = StepInfo()
        rc = self.lib.uqc_step_query(self.h, C.byref(info))
        if rc == 0:
            return None
        if rc < 0:
            check(self.h, rc)
        return info.as_dict()

    def device_bytes(self):
        b = C.c_ulonglong()
        check(self.h, self.lib.uqc_device_bytes(self.h, C.byref(b)))
        return b.value

    def run(self, t_end=0.0, raise_on_failure=True):
        info = StepInfo()
        rc = self.lib.uqc_run(self.h, t_end, C.byref(info))
        if rc != 0 and (raise_on_failure or rc != -4):
            check(self.h, rc)
        return info.as_dict()

    def mean_var(self):
        out = np.zeros((self.n_cells, 2 * self.n_states))
        check(self.h, self.lib.uqc_mean_var(self.h, ptr(out)))
        return out

    def closure_solve_host(self, lam, u, n_total=None, layout=L.LAYOUT_STATE_MAJOR):
        lam = np.ascontiguousarray(lam, dtype=np.float64).copy()
        u = np.ascontiguousarray(u, dtype=np.float64)
        n = lam.shape[0]
        st = np.zeros(n, dtype=np.int32)
        nt = None if n_total is None else np.ascontiguousarray(n_total, dtype=np.uint32)
        rc = self.lib.uqc_closure_solve_host(self.h, n, ptr(lam), ptr(u), ptr(nt, L._up), layout, ptr(st, L._ip))
        if rc not in (0, -4):
            check(self.h, rc)
        return lam, st

    def last_timing(self):
        ms = (C.c_float * 3)()
        check(self.h, self.lib.uqc_last_timing(self.h, ms))
        return list(ms)

    def last_launch_count(self):
        return int(self.lib.uqc_last_launch_count(self.h))

    def stream(self):
        return self.lib.uqc_stream(self.h)

    def device_state(self):
        du, dl = C.c_void_p(), C.c_void_p()
        check(self.h, self.lib.uqc_device_state(self.h, C.byref(du), C.byref(dl)))
        return du.value, dl.value


class Closure:
    """Closure operator (closure.h:13-119): batched SolveClosure on the GPU."""

    def __init__(self, solver: Solver):
        self.solver = solver

    @staticmethod
    def Create(settings: Settings | str) -> "Closure":
        return Closure(Solver(settings))

    def GetPhiTilde(self):
        return self.solver.tables()[0]

    def GetPhiTildeWf(self):
        return self.solver.tables()[1]

    def SolveClosure(self, lam, u, nTotal=None, nQTotal=None):
        """In place on lam (cells, nStates, nTotal) state-major, or a single cell
        (nStates, nTotal). Raises UqcError if any cell fails, like the reference
        exits (closure.cpp:180-192)."""
        single = np.asarray(lam).ndim == 2
        L3 = np.asarray(lam)[None] if single else np.asarray(lam)
        U3 = np.asarray(u)[None] if single else np.asarray(u)
        nt = None if nTotal is None else np.full(L3.shape[0], int(nTotal), dtype=np.uint32)
        out, st = self.solver.closure_solve_host(L3, U3, nt)
        if np.any(st != 0):
            bad = int(np.count_nonzero(st))
            raise UqcError(-4, f"[closure] Newton failed in {bad} cells ({L.CELL_CODES[int(st[st != 0][0])]})")
        if single:
            lam[...] = out[0]
        else:
            lam[...] = out
        return lam

    SolveClosureSafe = SolveClosure


class MomentSolver:
    """MomentSolver (momentsolver.h:139-147): the time loop on the GPU."""

    def __init__(self, settings: Settings | str, stream=None):
        self.solver = Solver(settings, stream)
        self.solver.init_state()

    def Solve(self):
        return self.solver.run()

    def step(self, n=1):
        return self.solver.step(n)

    def mean_var(self):
        return self.solver.mean_var()
