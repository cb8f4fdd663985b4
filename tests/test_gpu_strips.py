"""Parity at the resolution that is benchmarked (needs a B200).

The benchmark configurations run 200k-1M cells; the oracle cannot. These
tests run samples of the same mesh construction at the same resolution, so the
uncertain interface covers the same share of cells and the hard Newton cells
appear in the same proportion:

  C2  2-D Euler, total degree 5, 10 x 10 nodes: a 400 x 10 x 2 = 8,000-cell
      strip of the 400 x 250 x 2 benchmark mesh (same x spacing), 5 steps from
      the initial state (the CPU baseline's sample);
  C5  2-D Euler, 3 uncertainties, total degree 4, 8^3 nodes: a 512 x 2 x 2 =
      2,048-cell strip of the 512 x 256 x 2 mesh, 2 steps;
  C3  adaptive shallow water, degrees 1..9, 30 nodes: 50,000 cells (the
      benchmark's dx is 1e-6 on 1M cells; the sample keeps the dam break and
      the adaptive levels), 10 steps.

Bounds: the plain FP64 form reproduces the FP64 oracle's mean and variance of
every state within relative L1 1e-10 (and the moments elementwise to 1e-8,
levels exactly); the mixed form stays within relative L1 1e-6 of the oracle's
moments and mean/variance.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from uqcreator_b200 import Solver, workloads as W, MIXED

from ._util import rel_l1

pytestmark = pytest.mark.gpu

STRIPS = {
    "c2_strip_8000": (lambda: W.euler2d(nx=400, ny=10), 5),
    "c5_strip_2048": (lambda: W.euler2d_3u(nx=512, ny=2), 2),
    "c3_sample_50000": (lambda: W.shallow_water1d(ncells=50_000), 10),
}
_ORACLE = {}


def _oracle(name):
    if name not in _ORACLE:
        mk, steps = STRIPS[name]
        toml = mk()
        o = Oracle(toml, W.mesh_for(toml))
        o.init_state()
        r = o.step(steps)
        assert r["failures"] == 0
        u, lam, lev = o.get_state()
        _ORACLE[name] = dict(toml=toml, steps=steps, r=r, u=u, lev=lev, mv=o.mean_var(), area=o.geometry()["area"])
    return _ORACLE[name]


def _moment_err(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


@pytest.mark.parametrize("name", list(STRIPS))
@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_benchmark_resolution_matches_oracle(name, form):
    ref = _oracle(name)
    s = Solver(ref["toml"])
    if form == "mixed":
        s.set_precision(MIXED)
    s.init_state()
    info = s.step(ref["steps"])
    assert info["failed_cells"] == 0 and info["steps"] == ref["steps"]
    u, _, lev = s.download_state()
    np.testing.assert_array_equal(lev, ref["lev"])
    mv_err = rel_l1(s.mean_var(), ref["mv"], ref["area"])
    if form == "fp64":
        assert abs(info["t"] - ref["r"]["t"]) <= 1e-12 * ref["r"]["t"]
        assert np.all(mv_err <= 1e-10), mv_err
        np.testing.assert_allclose(u, ref["u"], rtol=1e-8, atol=1e-10)
    else:
        assert np.all(mv_err <= 1e-6), mv_err
        assert _moment_err(u, ref["u"]) <= 1e-6
