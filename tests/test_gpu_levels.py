"""Level-rule options on the GPU vs the oracle (needs a B200).

Adaptive shallow water (degrees 1..9, 2,000 cells) with the paper's S_l
indicator and its own bounds, and with a retardation schedule on top (the
level cap starts at 0 and rises to 2 after the first step; a threshold that is
never reached keeps it there). FP64: refinement levels identical to the
oracle's after every 10 steps, mean and variance within relative L1 1e-10.
Mixed form: mean and variance within 1e-6 and at most 0.5 % of the levels
different (a moment at a bound may fall either side of it).
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from uqcreator_b200 import MIXED, Solver, workloads as W

from ._util import rel_l1

pytestmark = pytest.mark.gpu
EX_E = 'refinementIndicator = "energy"\nrefinementBounds = [1e-10, 1e-8]\n'
EX_R = EX_E + 'retardationLevels = [0, 2, 8]\nretardationResiduals = [1.0, 1e-9]\n'


@pytest.mark.parametrize("extra", [EX_E, EX_R], ids=["energy", "retardation"])
@pytest.mark.parametrize("mixed", [False, True], ids=["fp64", "mixed"])
def test_level_options_match_oracle(extra, mixed):
    toml = W.shallow_water1d(ncells=2000, uqc_extra=extra)
    s = Solver(toml)
    if mixed:
        s.set_precision(MIXED)
    o = Oracle(toml, None)
    s.init_state(); o.init_state()
    area = o.geometry()["area"]
    top = 0
    for chunk in range(4):
        a = s.step(10)
        b = o.step(10)
        assert a["failed_cells"] == 0 and b["failures"] == 0
        vs, vo = s.download_state()[2], o.get_state()[2]
        if mixed:
            assert np.count_nonzero(vs != vo) <= 0.005 * len(vo)
        else:
            np.testing.assert_array_equal(vs, vo)
        err = rel_l1(s.mean_var(), o.mean_var(), area)
        assert np.all(err <= (1e-6 if mixed else 1e-10)), err
        top = max(top, int(vs.max()))
    if extra == EX_R:
        assert top == 2
    else:
        assert top >= 2
