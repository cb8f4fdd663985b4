"""State export and restart in the reference's file format (needs a B200).

uqc_export_state writes what a run of the reference leaves behind:
<prefix>_moments and <prefix>_duals as MomentSolver::Export writes them (a line
per cell, values with 15 significant digits, each followed by a comma) and the
log <prefix> with the configuration echo of main.cpp's PrintInit, which
MomentSolver::ImportPrevSettings reads back. A configuration with
[general] restartFile = "<prefix>" continues from them in uqc_init_state: at the
previous run's tEnd, with the duals too when importDualState = true, and onto
another number of moments as MomentSolver::SetDuals does (momentsolver.cpp:463-523).
The reference itself (oracle/_ref) writes the files of the last tests and runs
the same restarts, so both sides are checked against each other.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle import refharness
from uqcreator_b200 import Solver, workloads as W

from ._util import rel_l1

pytestmark = pytest.mark.gpu
BURGERS = ("Burgers1D", [12.0, 3.0, 0.5, 0.6], (2.5, 12.5))


def _restart_toml(toml, prefix, duals, tend=None):
    extra = f'restartFile = "{prefix}"\nimportDualState = {"true" if duals else "false"}\n'
    out = toml.replace("[general]\n", "[general]\n" + extra, 1)
    if tend is not None:
        import re
        out = re.sub(r"tEnd = [0-9.e+-]+", f"tEnd = {tend!r}", out, count=1)
    return out


def test_export_format_and_restart_with_duals(tmp_path):
    toml = W.euler2d(nx=12, ny=4, degree=3, nquad=6, tend=0.5)
    a = Solver(toml); a.init_state(); a.step(3)
    prefix = tmp_path / "run"
    a.export_state(prefix)
    u, lam, _ = a.download_state()
    lines = (tmp_path / "run_moments").read_text().splitlines()
    assert len(lines) == a.n_cells
    assert lines[0] == "".join("%.15g," % v for v in u[0].reshape(-1))
    assert "Config file" in (tmp_path / "run").read_text()
    b = Solver(_restart_toml(toml, prefix, True, tend=1.0)); b.init_state()
    ub, lb, _ = b.download_state()
    np.testing.assert_allclose(ub, u, rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(lb, lam, rtol=1e-14, atol=1e-300)
    assert b.step(1)["t"] > 0.5    # the time continues from the previous run's tEnd
    a.step(1)
    np.testing.assert_allclose(b.download_state()[0], a.download_state()[0], rtol=1e-11, atol=1e-14)


def test_restart_without_duals_recovers_them(tmp_path):
    toml = W.burgers1d(ncells=200, tend=0.02)
    a = Solver(toml); a.init_state(); a.step(10)
    a.export_state(tmp_path / "b")
    b = Solver(_restart_toml(toml, tmp_path / "b", False, tend=0.5)); b.init_state()
    info = b.step(1)
    assert info["failed_cells"] == 0
    a.step(1)
    np.testing.assert_allclose(b.download_state()[0], a.download_state()[0], rtol=1e-9, atol=1e-10)


def _reference_run(toml, prefix_name):
    """The reference's Solve() on toml in its own directory; returns the
    directory and the final mean/variance. It leaves <dir>/<prefix_name>*."""
    r = refharness.RefSolver(toml, *BURGERS[:2], bounds=BURGERS[2])
    mv = r.full_solve_export(os.path.join(r._dir, prefix_name))
    return r, mv


def _gpu_in_dir(toml):
    d = tempfile.mkdtemp(prefix="uqcgpu_")
    path = os.path.join(d, "config.toml")
    with open(path, "w") as f:
        f.write(toml)
    return Solver(path)


@pytest.mark.skipif(not refharness.available(), reason="oracle/_ref not built")
def test_restart_from_files_the_reference_wrote():
    """The reference runs to T = 0.02 and leaves its files; the GPU restarts
    from them (same moments, duals imported) and both continue to T = 0.04:
    mean and variance within relative L1 1e-10. The GPU's export of the
    imported state is byte-identical to the reference's files."""
    ta = W.burgers1d(ncells=200, degree=4, nquad=16, tend=0.02)
    ra, _ = _reference_run(ta, "runA")
    rel = "../" + os.path.basename(ra._dir) + "/runA"
    tb = _restart_toml(ta, rel, True, tend=0.04)
    rb, mv_ref = _reference_run(tb, "runB")
    g = _gpu_in_dir(tb)
    g.init_state()
    d = tempfile.mkdtemp(prefix="uqcexp_")
    g.export_state(os.path.join(d, "same"))
    for suffix in ("_moments", "_duals"):
        with open(os.path.join(ra._dir, "runA" + suffix), "rb") as f1, open(os.path.join(d, "same" + suffix), "rb") as f2:
            assert f1.read() == f2.read(), suffix
    info = g.run()
    assert info["failed_cells"] == 0 and abs(info["t"] - 0.04) < 1e-3
    err = rel_l1(g.mean_var(), mv_ref, g.geometry()["area"])
    assert np.all(err <= 1e-10), err


@pytest.mark.skipif(not refharness.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("duals", [False, True])
def test_restart_onto_more_moments_matches_the_reference(duals):
    """Degree 3 to T = 0.02, then degree 5 from those files to T = 0.04: the
    previous order's duals (imported, or solved from DS with the previous basis),
    U at the new quadrature from the previous basis, projection onto the new
    basis, duals padded and solved (momentsolver.cpp:463-523); the reference's
    own Solve() does the same. Mean and variance within relative L1 1e-10."""
    ta = W.burgers1d(ncells=200, degree=3, nquad=16, tend=0.02)
    ra, _ = _reference_run(ta, "runA")
    rel = "../" + os.path.basename(ra._dir) + "/runA"
    tb = _restart_toml(W.burgers1d(ncells=200, degree=5, nquad=16, tend=0.04), rel, duals)
    rb, mv_ref = _reference_run(tb, "runB")
    g = _gpu_in_dir(tb)
    g.init_state()
    info = g.run()
    assert info["failed_cells"] == 0
    err = rel_l1(g.mean_var(), mv_ref, g.geometry()["area"])
    assert np.all(err <= 1e-10), err


def _read_vtk_fields(path, section):
    lines = path.read_text(encoding="utf-8").splitlines()
    i = next(k for k, l in enumerate(lines) if l.startswith(section))
    n = int(lines[i].split()[1]); nf = int(lines[i + 1].split()[2])
    k = i + 2; out = {}
    for _ in range(nf):
        name, comps, cnt, _t = lines[k].split(); comps, cnt = int(comps), int(cnt)
        out[name] = np.array([[float(x) for x in lines[k + 1 + r].split()] for r in range(cnt)])
        k += 1 + cnt
    return n, out


@pytest.mark.parametrize("toml,dim", [(W.burgers1d(ncells=60), 1), (W.euler2d(nx=6, ny=3, degree=2, nquad=4), 2)])
def test_vtk_output_holds_mean_and_variance(tmp_path, toml, dim):
    s = Solver(toml); s.init_state(); s.step(2)
    s.write_vtk(tmp_path / "out")
    mv = s.mean_var()
    n, cell = _read_vtk_fields(tmp_path / "out.vtk", "CELL_DATA")
    assert n == s.n_cells
    if dim == 1:
        np.testing.assert_allclose(cell["E(u)"][:, 0], mv[:, 0], rtol=1e-15)
        np.testing.assert_allclose(cell["Var(u)"][:, 0], mv[:, 1], rtol=1e-15)
        ev = np.loadtxt(tmp_path / "outExpectedValue")
        assert ev.shape == (s.n_cells, 2)
        np.testing.assert_allclose(ev[:, 1], mv[:, 0], rtol=1e-5)
    else:
        np.testing.assert_allclose(cell["E(ρ)"][:, 0], mv[:, 0], rtol=1e-15)
        np.testing.assert_allclose(cell["E(ρU)"][:, :2], mv[:, 1:3], rtol=1e-15)
        np.testing.assert_allclose(cell["Var(ρE)"][:, 0], mv[:, 7], rtol=1e-15)
    npts, pt = _read_vtk_fields(tmp_path / "out.vtk", "POINT_DATA")
    assert npts > 0 and all(v.shape[0] == npts for v in pt.values())
