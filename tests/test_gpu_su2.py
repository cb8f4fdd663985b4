"""SU2 mesh with wall boundaries on the GPU vs the reference (needs a B200).

The channel of tests/golden/su2_channel.su2: Dirichlet inlet, no-slip ghost
states on the leaning outlet wall, shallow-water wall ghost states top and
bottom (expliciteuler.cpp:24-70). FP64: moments elementwise at 1e-9 relative
and E/Var within relative L1 1e-10 of the reference's own ExplicitEuler
(golden su2_steps.npz); mixed form: within 1e-6 of the FP64 oracle.
"""
import shutil
from pathlib import Path

import numpy as np
import pytest

from oracle import su2
from oracle.oracle import Oracle
from uqcreator_b200 import Solver, MIXED

from ._util import rel_l1

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
BC = [["inlet", "dirichlet"], ["outlet", "noslip"], ["bottom", "swwall"], ["top", "swwall"]]


def _config(tmp_path):
    g = np.load(GOLD / "su2_steps.npz")
    shutil.copy(GOLD / "su2_channel.su2", tmp_path / "su2_channel.su2")
    cfg = tmp_path / "c.toml"
    cfg.write_text(str(g["toml"]))
    return g, cfg


def test_su2_walls_match_reference(tmp_path):
    g, cfg = _config(tmp_path)
    s = Solver(str(cfg))
    s.init_state()
    info = s.step(int(g["steps"]))
    assert info["failed_cells"] == 0
    assert abs(info["t"] - float(g["t"])) <= 1e-12 * abs(float(g["t"]))
    u, lam, lev = s.download_state()
    np.testing.assert_allclose(u, g["u"], rtol=1e-9, atol=1e-11)
    err = rel_l1(s.mean_var(), g["mean_var"], s.geometry()["area"])
    assert np.all(err <= 1e-10), err


def test_su2_walls_mixed_matches_oracle(tmp_path):
    g, cfg = _config(tmp_path)
    s = Solver(str(cfg))
    s.set_precision(MIXED)
    o = Oracle(str(g["toml"]), su2.read_su2(str(GOLD / "su2_channel.su2"), su2.bc_table(BC)))
    s.init_state(); o.init_state()
    n = 2 * int(g["steps"])
    assert s.step(n)["failed_cells"] == 0
    o.step(n)
    us = s.download_state()[0]
    uo = o.get_state()[0]
    assert np.abs(us - uo).sum() / np.abs(uo).sum() <= 1e-6
