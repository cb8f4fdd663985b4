"""ctypes binding of the reference harness (oracle/_ref/libuqcref*.so).

TEST INFRASTRUCTURE ONLY. The harness is UQCreator's own C++ (code/src) built
against project shims by oracle/ref/Makefile; it runs the reference's
Closure::SolveClosure, ExplicitEuler::Advance, Problem fluxes and, for small
cases, MomentSolver::Solve itself. Tests, the golden-vector script and the
CPU-baseline leg of bench.py use it as the checker / baseline; the product
never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIBS: dict[str, C.CDLL] = {}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_uint)


def lib_path(variant: str = "exact") -> Path:
    """exact: the parity build; omp: the timed OpenMP build; gpu: the parity
    build with GpuClosure (oracle/ref/gpuclosure.cpp) selected by Closure::Create."""
    name = {"exact": "libuqcref.so", "omp": "libuqcref_omp.so", "gpu": "libuqcref_gpu.so"}[variant]
    return _HERE / "_ref" / name


def available(variant: str = "exact") -> bool:
    return lib_path(variant).exists()


def _lib(variant: str = "exact") -> C.CDLL:
    if variant in _LIBS:
        return _LIBS[variant]
    path = lib_path(variant)
    if not path.exists():
        raise FileNotFoundError(f"{path} not built (make -C oracle/ref)")
    lib = C.CDLL(str(path))
    lib.uqcref_create.restype = C.c_int
    lib.uqcref_create.argtypes = [C.c_char_p, C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_int, _dp, _ip,
                                  C.c_int, _ip, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
    lib.uqcref_destroy.argtypes = [C.c_void_p]
    lib.uqcref_set_cell_bc.argtypes = [C.c_void_p, _ip]
    lib.uqcref_boundary_normals.argtypes = [C.c_void_p, _dp]
    lib.uqcref_sizes.argtypes = [C.c_void_p, _ip]
    lib.uqcref_tables.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
    lib.uqcref_geometry.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _ip, _ip]
    lib.uqcref_init_state.argtypes = [C.c_void_p]
    lib.uqcref_get_state.argtypes = [C.c_void_p, _dp, _dp, _up]
    lib.uqcref_set_state.argtypes = [C.c_void_p, _dp, _dp, _up, C.c_double]
    lib.uqcref_solve_closure.restype = C.c_int
    lib.uqcref_solve_closure.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _up, _ip]
    lib.uqcref_step.restype = C.c_int
    lib.uqcref_step.argtypes = [C.c_void_p, C.c_int, _dp]
    lib.uqcref_mean_var.argtypes = [C.c_void_p, _dp]
    lib.uqcref_full_solve.restype = C.c_int
    lib.uqcref_full_solve.argtypes = [C.c_void_p, _dp, _dp, C.c_char_p, C.c_int]
    lib.uqcref_full_solve_export.restype = C.c_int
    lib.uqcref_full_solve_export.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_char_p, C.c_int]
    lib.uqcref_full_solve_gpu.restype = C.c_int
    lib.uqcref_full_solve_gpu.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_char_p, C.c_int]
    _LIBS[variant] = lib
    return lib


def _p(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


PROBLEM_KIND = {"Burgers1D": 1, "Euler2D": 2, "ShallowWater1D": 3, "Euler1D": 4}
NEWTON_MODE = {"reference": 0, "guarded": 1, "safe": 2}


class RefSolver:
    """One reference solver instance (settings + mesh + problem + closure)."""

    def __init__(self, toml_text: str, problem: str, params, bounds=(3.0, 12.0), mesh2d=None,
                 variant: str = "exact", newton: str = "reference"):
        self.lib = _lib(variant)
        self._dir = tempfile.mkdtemp(prefix="uqcref_")
        self.toml_path = os.path.join(self._dir, "config.toml")
        with open(self.toml_path, "w") as f:
            f.write(toml_text)
        prm = np.ascontiguousarray(params, dtype=np.float64)
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        if mesh2d is not None:
            xy = np.ascontiguousarray(mesh2d["xy"], dtype=np.float64)
            bnd = np.ascontiguousarray(mesh2d["node_boundary"], dtype=np.int32)
            tri = np.ascontiguousarray(mesh2d["tri"], dtype=np.int32)
            rc = self.lib.uqcref_create(self.toml_path.encode(), PROBLEM_KIND[problem], NEWTON_MODE[newton], _p(prm), bounds[0], bounds[1],
                                        len(bnd), _p(xy), _p(bnd, _ip), len(tri), _p(tri, _ip), C.byref(h), err, 512)
            if rc == 0 and mesh2d.get("cell_bc") is not None:    # SU2 boundary types (oracle/su2.py)
                self.lib.uqcref_set_cell_bc(h, _p(np.ascontiguousarray(mesh2d["cell_bc"], dtype=np.int32), _ip))
        else:
            rc = self.lib.uqcref_create(self.toml_path.encode(), PROBLEM_KIND[problem], NEWTON_MODE[newton], _p(prm), bounds[0], bounds[1],
                                        0, None, None, 0, None, C.byref(h), err, 512)
        if rc != 0:
            raise RuntimeError("reference harness: " + err.value.decode())
        self.h = h
        sz = np.zeros(22, dtype=np.int32)
        self.lib.uqcref_sizes(h, _p(sz, _ip))
        self.n_cells, self.n_states, self.n_total, self.n_q, self.n_levels, self.dim_xi = (int(v) for v in sz[:6])
        self.n_total_levels = [int(v) for v in sz[6:6 + self.n_levels]]

    def close(self):
        if self.h:
            self.lib.uqcref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        nq, nt, d = self.n_q, self.n_total, self.dim_xi
        phi = np.zeros((nt, nq)); phiwf = np.zeros((nt, nq)); xi = np.zeros((nq, d)); w = np.zeros(nq)
        self.lib.uqcref_tables(self.h, _p(phi), _p(phiwf), _p(xi), _p(w))
        # returned as (nQ, nT) arrays: phi[k, i]
        return phi.T.copy(), phiwf.T.copy(), xi, w

    def geometry(self, n_faces):
        n = self.n_cells
        area = np.zeros(n); maxe = np.zeros(n); cen = np.zeros((n, 2))
        un = np.zeros((n, n_faces, 2)); sn = np.zeros((n, n_faces, 2))
        nbr = np.zeros((n, n_faces), dtype=np.int32); bnd = np.zeros(n, dtype=np.int32)
        self.lib.uqcref_geometry(self.h, _p(area), _p(maxe), _p(cen), _p(un), _p(sn), _p(nbr, _ip), _p(bnd, _ip))
        bn = np.zeros((n, 2))
        self.lib.uqcref_boundary_normals(self.h, _p(bn))
        return dict(area=area, max_edge=maxe, center=cen, unit_normal=un, scaled_normal=sn, nbr=nbr, boundary=bnd,
                    boundary_normal=bn)

    def init_state(self):
        self.lib.uqcref_init_state(self.h)

    def get_state(self):
        """u, lambda as (nCells, nStates, nTotal) arrays; refinement level per cell."""
        n = self.n_states * self.n_total
        u = np.zeros(self.n_cells * n); lam = np.zeros(self.n_cells * n)
        lev = np.zeros(self.n_cells, dtype=np.uint32)
        self.lib.uqcref_get_state(self.h, _p(u), _p(lam), _p(lev, _up))
        shape = (self.n_cells, self.n_total, self.n_states)
        return (u.reshape(shape).transpose(0, 2, 1).copy(), lam.reshape(shape).transpose(0, 2, 1).copy(), lev)

    def set_state(self, u, lam, level=None, t=0.0):
        u = np.ascontiguousarray(np.asarray(u).transpose(0, 2, 1), dtype=np.float64)
        lam = np.ascontiguousarray(np.asarray(lam).transpose(0, 2, 1), dtype=np.float64)
        lev = None if level is None else np.ascontiguousarray(level, dtype=np.uint32)
        self.lib.uqcref_set_state(self.h, _p(u), _p(lam), _p(lev, _up), t)

    def solve_closure(self, lam, u, n_total_cell=None):
        """Batched Closure::SolveClosure; lam/u are (cells, nStates, nTotal). Returns (lam, status)."""
        cells = lam.shape[0]
        lam_r = np.ascontiguousarray(np.asarray(lam).transpose(0, 2, 1), dtype=np.float64)
        u_r = np.ascontiguousarray(np.asarray(u).transpose(0, 2, 1), dtype=np.float64)
        st = np.zeros(cells, dtype=np.int32)
        ntc = None if n_total_cell is None else np.ascontiguousarray(n_total_cell, dtype=np.uint32)
        self.lib.uqcref_solve_closure(self.h, cells, _p(lam_r), _p(u_r), _p(ntc, _up), _p(st, _ip))
        return lam_r.transpose(0, 2, 1).copy(), st

    def step(self, n_steps=1):
        out = np.zeros(4)
        self.lib.uqcref_step(self.h, n_steps, _p(out))
        return dict(t=out[0], dt=out[1], residual=out[2], failures=int(out[3]))

    def mean_var(self):
        out = np.zeros(self.n_cells * 2 * self.n_states)
        self.lib.uqcref_mean_var(self.h, _p(out))
        return out.reshape(self.n_cells, 2 * self.n_states)

    def full_solve_export(self, prefix):
        """MomentSolver::Solve(), writing <prefix>_moments / <prefix>_duals (the
        reference's Export) and the log <prefix> with its configuration echo;
        returns the final meanVar (cells, 2 nS)."""
        mv = np.zeros(self.n_cells * 2 * self.n_states)
        err = C.create_string_buffer(512)
        rc = self.lib.uqcref_full_solve_export(self.h, os.fsencode(prefix), _p(mv), err, 512)
        if rc != 0:
            raise RuntimeError("reference Solve: " + err.value.decode())
        return mv.reshape(self.n_cells, 2 * self.n_states)

    def full_solve_gpu(self, prefix):
        """As full_solve_export with GpuMomentSolver (the "gpu" variant only):
        the product's time loop behind MomentSolver's constructor and Solve(),
        writing through the reference's Mesh::Export and loggers."""
        mv = np.zeros(self.n_cells * 2 * self.n_states)
        err = C.create_string_buffer(512)
        rc = self.lib.uqcref_full_solve_gpu(self.h, os.fsencode(prefix), _p(mv), err, 512)
        if rc != 0:
            raise RuntimeError("GpuMomentSolver: " + err.value.decode())
        return mv.reshape(self.n_cells, 2 * self.n_states)

    def full_solve(self):
        """Runs MomentSolver::Solve(); returns (meanVar (cells, 2nS), lambda at 15 digits)."""
        mv = np.zeros(self.n_cells * 2 * self.n_states)
        lam = np.zeros(self.n_cells * self.n_states * self.n_total)
        err = C.create_string_buffer(512)
        rc = self.lib.uqcref_full_solve(self.h, _p(mv), _p(lam), err, 512)
        if rc != 0:
            raise RuntimeError("reference Solve: " + err.value.decode())
        shape = (self.n_cells, self.n_total, self.n_states)
        return mv.reshape(self.n_cells, 2 * self.n_states), lam.reshape(shape).transpose(0, 2, 1).copy()
