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
