"""ctypes binding of the FP64 CPU restatement (oracle/uqc_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Imported by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg; never by the product.
Build: `make -C oracle` (also done by __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
import subprocess
import tomllib
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB = _HERE / "liboracle.so"
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_up = C.POINTER(C.c_uint)

CLOSURES = {"BoundedBarrier": 0, "Euler2D": 1, "ShallowWater": 2}
PROBLEMS = {"Burgers1D": 0, "Euler2D": 1, "ShallowWater1D": 2}


class Config(C.Structure):
    _fields_ = [("closure", C.c_int), ("problem", C.c_int), ("dim_xi", C.c_int), ("max_degree", C.c_int),
                ("n_levels", C.c_int), ("degree", C.c_int * 16), ("n_quad", C.c_int), ("sigma", C.c_double * 4),
                ("cfl", C.c_double), ("epsilon", C.c_double), ("max_iterations", C.c_int), ("newton_mode", C.c_int), ("gamma", C.c_double),
                ("bb_minus", C.c_double), ("bb_plus", C.c_double), ("ic", C.c_double * 8), ("mesh_dim", C.c_int),
                ("n_cells_1d", C.c_int), ("a", C.c_double), ("b", C.c_double),
                ("ref_indicator", C.c_int), ("ref_down", C.c_double), ("ref_up", C.c_double),
                ("n_ret_levels", C.c_int), ("ret_res", C.c_double * 8), ("ret_lev", C.c_int * 9)]


def build():
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.uqco_create.restype = C.c_int
        L.uqco_create.argtypes = [C.POINTER(Config), C.c_int, _dp, _ip, C.c_int, _ip, C.POINTER(C.c_void_p)]
        L.uqco_destroy.argtypes = [C.c_void_p]
        L.uqco_set_cell_bc.argtypes = [C.c_void_p, _ip]
        L.uqco_sizes.argtypes = [C.c_void_p, _ip]
        L.uqco_tables.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.uqco_geometry.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _ip, _ip]
        L.uqco_init_state.argtypes = [C.c_void_p]
        L.uqco_get_state.argtypes = [C.c_void_p, _dp, _dp, _up]
        L.uqco_set_state.argtypes = [C.c_void_p, _dp, _dp, _up, C.c_double]
        L.uqco_solve_closure.restype = C.c_int
        L.uqco_solve_closure.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _up, _ip, _ip]
        L.uqco_step.restype = C.c_int
        L.uqco_step.argtypes = [C.c_void_p, C.c_int, _dp]
        L.uqco_mean_var.argtypes = [C.c_void_p, _dp]
        L.uqco_ansatz.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int]
        L.uqco_entropy_grad.argtypes = [C.c_void_p, _dp, _dp]
        _lib = L
    return _lib


def _p(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def config_from_toml(toml_text: str) -> Config:
    """Maps the reference's TOML keys (code/src/settings.cpp:22-323) plus the [uqc] table."""
    d = tomllib.loads(toml_text)
    ms, pr, me, uq = d["moment_system"], d["problem"], d["mesh"], d.get("uqc", {})
    c = Config()
    c.closure = CLOSURES[ms["closure"]]
    c.problem = PROBLEMS[d["general"]["problem"]]
    dist = pr["distribution"]
    c.dim_xi = len(dist[0])
    for i, s in enumerate(dist[1]):
        c.sigma[i] = float(s)
    c.max_degree = 1 if ms["moments"][0][0] == "maxDegree" else 0
    degs = ms["moments"][1]
    c.n_levels = len(degs)
    for i, v in enumerate(degs):
        c.degree[i] = int(v)
    c.n_quad = int(ms["quadPoints"][1][-1])
    c.cfl = float(pr["CFL"])
    c.epsilon = float(ms.get("epsilon", 5e-5))
    c.max_iterations = int(ms.get("maxIterations", 1000))
    c.newton_mode = {"reference": 0, "guarded": 1, "safe": 2}[uq.get("newton", "reference")]
    c.gamma = float(pr.get("gamma", 1.4))
    b = uq.get("bounds", [3.0, 12.0])
    c.bb_minus, c.bb_plus = float(b[0]), float(b[1])
    for i, v in enumerate(uq.get("ic", [])):
        c.ic[i] = float(v)
    c.mesh_dim = int(me["dimension"])
    c.n_cells_1d = int(me.get("numberOfCells", 0))
    c.a = float(me.get("a", 0.0))
    c.b = float(me.get("b", 0.0))
    c.ref_indicator = {"moments": 0, "energy": 1}[uq.get("refinementIndicator", "moments")]
    c.ref_down, c.ref_up = (float(v) for v in uq.get("refinementBounds", [0.004, 0.02]))
    lev = uq.get("retardationLevels", [])
    res = uq.get("retardationResiduals", [])
    c.n_ret_levels = len(lev)
    for i, v in enumerate(lev):
        c.ret_lev[i] = int(v)
    for i, v in enumerate(res):
        c.ret_res[i] = float(v)
    return c


class Oracle:
    """FP64 oracle instance for one workload (state-major per-cell layout)."""

    def __init__(self, toml_text: str, mesh2d: dict | None = None):
        self.L = lib()
        self.cfg = config_from_toml(toml_text)
        h = C.c_void_p()
        if mesh2d is not None:
            xy = np.ascontiguousarray(mesh2d["xy"], dtype=np.float64)
            bnd = np.ascontiguousarray(mesh2d["node_boundary"], dtype=np.int32)
            tri = np.ascontiguousarray(mesh2d["tri"], dtype=np.int32)
            self.L.uqco_create(C.byref(self.cfg), len(bnd), _p(xy), _p(bnd, _ip), len(tri), _p(tri, _ip), C.byref(h))
            if mesh2d.get("cell_bc") is not None:    # SU2 boundary types (oracle/su2.py)
                self.L.uqco_set_cell_bc(h, _p(np.ascontiguousarray(mesh2d["cell_bc"], dtype=np.int32), _ip))
        else:
            self.L.uqco_create(C.byref(self.cfg), 0, None, None, 0, None, C.byref(h))
        self.h = h
        sz = np.zeros(24, dtype=np.int32)
        self.L.uqco_sizes(h, _p(sz, _ip))
        (self.n_cells, self.n_states, self.n_total, self.n_q, self.n_levels, self.dim_xi,
         self.n_faces) = (int(v) for v in sz[:7])
        self.n_total_levels = [int(v) for v in sz[7:7 + self.n_levels]]

    def close(self):
        if self.h:
            self.L.uqco_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        nq, nt = self.n_q, self.n_total
        phi = np.zeros((nq, nt)); phiwf = np.zeros((nq, nt)); xi = np.zeros((nq, self.dim_xi)); w = np.zeros(nq)
        self.L.uqco_tables(self.h, _p(phi), _p(phiwf), _p(xi), _p(w))
        return phi, phiwf, xi, w

    def geometry(self):
        n, f = self.n_cells, self.n_faces
        area = np.zeros(n); maxe = np.zeros(n); cen = np.zeros((n, 2))
        un = np.zeros((n, f, 2)); sn = np.zeros((n, f, 2))
        nbr = np.zeros((n, f), dtype=np.int32); bnd = np.zeros(n, dtype=np.int32)
        self.L.uqco_geometry(self.h, _p(area), _p(maxe), _p(cen), _p(un), _p(sn), _p(nbr, _ip), _p(bnd, _ip))
        return dict(area=area, max_edge=maxe, center=cen, unit_normal=un, scaled_normal=sn, nbr=nbr, boundary=bnd)

    def init_state(self):
        self.L.uqco_init_state(self.h)

    def get_state(self):
        shape = (self.n_cells, self.n_states, self.n_total)
        u = np.zeros(shape); lam = np.zeros(shape); lev = np.zeros(self.n_cells, dtype=np.uint32)
        self.L.uqco_get_state(self.h, _p(u), _p(lam), _p(lev, _up))
        return u, lam, lev

    def set_state(self, u, lam, level=None, t=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        lev = None if level is None else np.ascontiguousarray(level, dtype=np.uint32)
        self.L.uqco_set_state(self.h, _p(u), _p(lam), _p(lev, _up), t)

    def solve_closure(self, lam, u, n_total_cell=None):
        lam = np.ascontiguousarray(lam, dtype=np.float64).copy()
        u = np.ascontiguousarray(u, dtype=np.float64)
        n = lam.shape[0]
        st = np.zeros(n, dtype=np.int32); it = np.zeros(n, dtype=np.int32)
        ntc = None if n_total_cell is None else np.ascontiguousarray(n_total_cell, dtype=np.uint32)
        self.L.uqco_solve_closure(self.h, n, _p(lam), _p(u), _p(ntc, _up), _p(st, _ip), _p(it, _ip))
        return lam, st, it

    def step(self, n_steps=1):
        out = np.zeros(4)
        self.L.uqco_step(self.h, n_steps, _p(out))
        return dict(t=out[0], dt=out[1], residual=out[2], failures=int(out[3]))

    def mean_var(self):
        out = np.zeros((self.n_cells, 2 * self.n_states))
        self.L.uqco_mean_var(self.h, _p(out))
        return out

    def ansatz(self, Lam, matrix_form=False):
        Lam = np.ascontiguousarray(Lam, dtype=np.float64)
        u = np.zeros(self.n_states); du = np.zeros(self.n_states * self.n_states)
        self.L.uqco_ansatz(self.h, _p(Lam), _p(u), _p(du), int(matrix_form))
        return u, du.reshape(self.n_states, self.n_states)
