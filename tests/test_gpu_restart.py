"""State export and restart in the reference's file format (needs a B200).

uqc_export_state writes what MomentSolver::Export writes (a line per cell,
values with 15 significant digits, each followed by a comma); a configuration
with [general] restartFile = "<prefix>" reads them back in uqc_init_state,
with the duals too when importDualState = true."""
import numpy as np
import pytest

from uqcreator_b200 import Solver, workloads as W

pytestmark = pytest.mark.gpu


def _restart_toml(toml, prefix, duals):
    extra = f'restartFile = "{prefix}"\nimportDualState = {"true" if duals else "false"}\n'
    return toml.replace("[general]\n", "[general]\n" + extra, 1)


def test_export_format_and_restart_with_duals(tmp_path):
    toml = W.euler2d(nx=12, ny=4, degree=3, nquad=6)
    a = Solver(toml); a.init_state(); a.step(3)
    prefix = tmp_path / "run"
    a.export_state(prefix)
    u, lam, _ = a.download_state()
    lines = (tmp_path / "run_moments").read_text().splitlines()
    assert len(lines) == a.n_cells
    assert lines[0] == "".join("%.15g," % v for v in u[0].reshape(-1))
    b = Solver(_restart_toml(toml, prefix, True)); b.init_state()
    ub, lb, _ = b.download_state()
    np.testing.assert_allclose(ub, u, rtol=1e-14, atol=1e-300)
    np.testing.assert_allclose(lb, lam, rtol=1e-14, atol=1e-300)
    a.step(3); b.step(3)
    np.testing.assert_allclose(b.download_state()[0], a.download_state()[0], rtol=1e-11, atol=1e-14)


def test_restart_without_duals_recovers_them(tmp_path):
    toml = W.burgers1d(ncells=200, tend=0.02)
    a = Solver(toml); a.init_state(); a.step(10)
    a.export_state(tmp_path / "b")
    b = Solver(_restart_toml(toml, tmp_path / "b", False)); b.init_state()
    info = b.step(1)
    assert info["failed_cells"] == 0
    a.step(1)
    np.testing.assert_allclose(b.download_state()[0], a.download_state()[0], rtol=1e-9, atol=1e-10)


def test_restart_with_other_moment_count_is_refused(tmp_path):
    a = Solver(W.burgers1d(ncells=50, degree=3)); a.init_state()
    a.export_state(tmp_path / "c")
    b = Solver(_restart_toml(W.burgers1d(ncells=50, degree=4), tmp_path / "c", True))
    with pytest.raises(Exception) as e:
        b.init_state()
    assert "moments" in str(e.value)


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
