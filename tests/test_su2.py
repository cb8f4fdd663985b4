"""SU2 mesh ingestion and wall boundary types, host side (no GPU).

1. The product's reader (uqcreator_b200/csrc/mesh.cpp, through uqc_get_geometry,
   which needs no device) and the oracle's (oracle/su2.py) give the same
   geometry, neighbours and boundary types, bit for bit.
2. The boundary-type rule of Mesh2D::LoadSU2MeshFromFile (mesh2d.cpp:199-214:
   per cell node, per marker, per marker element, the last match wins) on a
   hand-derived case.
3. Refused configurations: neumann / periodic markers (the reference's
   ExplicitEuler has no ghost state for them), unknown types, markers without
   an SU2BC entry, quadrangles, a missing file.
4. The oracle's wall ghost states against the reference's own
   ExplicitEuler::Advance (golden su2_steps.npz; bit for bit against the
   harness when oracle/_ref is built).
"""
import shutil
from pathlib import Path

import numpy as np
import pytest

from oracle import refharness, su2
from oracle.oracle import Oracle
from uqcreator_b200 import Solver, UqcError, workloads as W

GOLD = Path(__file__).resolve().parent / "golden"
BC = [["inlet", "dirichlet"], ["outlet", "noslip"], ["bottom", "swwall"], ["top", "swwall"]]

# unit square, centre node 4, four triangles; every cell has two boundary nodes
SQUARE = """NDIME= 2
NELEM= 4
5 0 1 4 0
5 1 2 4 1
5 2 3 4 2
5 3 0 4 3
NPOIN= 5
0.5 0.5 4
0.0 0.0 0
1.0 0.0 1
1.0 1.0 2
0.0 1.0 3
NMARK= 4
MARKER_TAG= bottom
MARKER_ELEMS= 1
3 0 1
MARKER_TAG= right
MARKER_ELEMS= 1
3 1 2
MARKER_TAG= top
MARKER_ELEMS= 1
3 2 3
MARKER_TAG= left
MARKER_ELEMS= 1
3 3 0
"""
SQUARE_BC = [["bottom", "noslip"], ["right", "swwall"], ["top", "dirichlet"], ["left", "noslip"]]


def _case(tmp_path, mesh_text, bcs, name="m.su2"):
    (tmp_path / name).write_text(mesh_text)
    cfg = tmp_path / "c.toml"
    cfg.write_text(W.euler2d_su2(name, bcs=[tuple(b) for b in bcs], degree=2, nquad=4))
    return cfg


def test_committed_channel_is_the_generator_output():
    assert (GOLD / "su2_channel.su2").read_text() == W.su2_channel(6, 4)


def test_product_reader_matches_oracle_reader(tmp_path):
    cfg = _case(tmp_path, W.su2_channel(7, 5, seed=3), BC)
    g = Solver(str(cfg)).geometry()
    m = su2.read_su2(str(tmp_path / "m.su2"), su2.bc_table(BC))
    go = Oracle(cfg.read_text(), m).geometry()
    for k, v in go.items():
        np.testing.assert_array_equal(np.asarray(g[k]).reshape(np.shape(v)), v, err_msg=k)
    np.testing.assert_array_equal(g["boundary"], m["cell_bc"])
    assert set(np.unique(m["cell_bc"])) == {0, 1, 2, 3}


def test_boundary_type_rule_last_match_wins(tmp_path):
    # cell (0,1,4): node 0 -> bottom, left (noslip); node 1 -> bottom, right: swwall (3)
    # cell (1,2,4): node 1 -> ..., right; node 2 -> right, top: dirichlet (1)
    # cell (2,3,4): node 3 -> top, left: noslip (2); cell (3,0,4): node 0 -> bottom, left: noslip
    expected = [3, 1, 2, 2]
    cfg = _case(tmp_path, SQUARE, SQUARE_BC)
    m = su2.read_su2(str(tmp_path / "m.su2"), su2.bc_table(SQUARE_BC))
    np.testing.assert_array_equal(m["cell_bc"], expected)
    g = Solver(str(cfg)).geometry()
    np.testing.assert_array_equal(g["boundary"], expected)
    # nodes are sorted by id, whatever the file order
    np.testing.assert_array_equal(m["xy"][4], [0.5, 0.5])


@pytest.mark.parametrize("bcs,text,msg", [
    ([["bottom", "neumann"], ["right", "swwall"], ["top", "dirichlet"], ["left", "noslip"]], SQUARE, "not supported"),
    ([["bottom", "periodic"], ["right", "swwall"], ["top", "dirichlet"], ["left", "noslip"]], SQUARE, "not supported"),
    ([["bottom", "slip"], ["right", "swwall"], ["top", "dirichlet"], ["left", "noslip"]], SQUARE, "Invalid boundary condition"),
    ([["bottom", "noslip"], ["right", "swwall"], ["top", "dirichlet"]], SQUARE, "no SU2BC entry for marker 'left'"),
    (SQUARE_BC, SQUARE.replace("5 3 0 4 3", "9 3 0 4 1 3"), "triangles only"),
])
def test_refused_configurations(tmp_path, bcs, text, msg):
    cfg = _case(tmp_path, text, bcs)
    with pytest.raises(UqcError) as e:
        Solver(str(cfg))
    assert msg in str(e.value)


def test_missing_mesh_file_and_relative_paths(tmp_path):
    cfg = _case(tmp_path, SQUARE, SQUARE_BC)
    (tmp_path / "m.su2").unlink()
    with pytest.raises(UqcError) as e:
        Solver(str(cfg))
    assert "File not found" in str(e.value)
    # the mesh file is found next to the config, not in the working directory
    sub = tmp_path / "sub"
    sub.mkdir()
    (sub / "m.su2").write_text(SQUARE)
    shutil.move(str(cfg), str(sub / "c.toml"))
    assert Solver(str(sub / "c.toml")).geometry()["area"].shape == (4,)


def test_oracle_walls_match_reference_golden():
    g = np.load(GOLD / "su2_steps.npz")
    m = su2.read_su2(str(GOLD / "su2_channel.su2"), su2.bc_table(BC))
    o = Oracle(str(g["toml"]), m)
    o.init_state()
    out = o.step(int(g["steps"]))
    u, lam, lev = o.get_state()
    assert out["t"] == float(g["t"])
    np.testing.assert_array_equal(u, g["u"])
    np.testing.assert_array_equal(lam, g["lam"])


@pytest.mark.skipif(not refharness.available(), reason="reference harness not built")
def test_harness_boundary_normals_match_product_rule():
    """Cell::UpdateBoundaryNormal of the reference vs the oracle's rule (face of
    the largest neighbour id) through the unit normals of that face."""
    g = np.load(GOLD / "su2_steps.npz")
    m = su2.read_su2(str(GOLD / "su2_channel.su2"), su2.bc_table(BC))
    r = refharness.RefSolver(str(g["toml"]), "Euler2D", [0.7, 1.0, 1.0, 0.125, 0.1], bounds=(3, 12), mesh2d=m,
                             newton="guarded")
    geo = r.geometry(3)
    idx = np.argmax(geo["nbr"], axis=1)
    rule = geo["unit_normal"][np.arange(len(idx)), idx]
    wall = m["cell_bc"] > 0
    np.testing.assert_array_equal(geo["boundary_normal"][wall], rule[wall])
