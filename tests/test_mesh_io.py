"""Mesh files and raw snapshots, the reference's formats (no GPU).

Meshes are written in the reference's Mesh2D::from_file layout (info.txt, coordinates.txt,
elements.txt) and read three ways: by the library (wdg_mesh_from_file), by the reference's own
reader compiled from its sources (oracle/_ref, where the sources were present at build time),
and by the oracle's restatement.  The connectivity, min_h and boundary midpoints must agree
exactly.  Snapshots follow dg::to_file: raw native-order doubles.
"""
import os

import numpy as np
import pytest

from conftest import require_reference_build
from oracle import cpu


@pytest.fixture(scope="module")
def W():
    from wavedg_b200 import build

    build.build()
    import wavedg_b200

    return wavedg_b200


def _meshes():
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(7, 0.2, seed=5)
    out = {"rect": mg.uniform_rect(5, -1.0, 1.0, 4, 0.0, 2.0), "perturbed": mg.scrambled(v, q, seed=6),
           "l_shape": mg.l_shape(6)}
    return out


@pytest.mark.parametrize("name", ["rect", "perturbed", "l_shape"])
def test_from_file_matches_the_reference_reader(W, tmp_path, name):
    v, q = _meshes()[name]
    d = str(tmp_path / name)
    W.Mesh2D.from_vertices(v, q).to_file(d)
    m = W.Mesh2D.from_file(d)
    direct = W.Mesh2D.from_vertices(v, q)
    for t in (0, 1):
        np.testing.assert_array_equal(m.edges(t), direct.edges(t))
    assert m.min_h() == direct.min_h()
    r = cpu.Mesh.from_file(d, "oracle")
    assert r is not None and r.n_elem == len(q)
    for t in (0, 1):
        np.testing.assert_array_equal(m.edges(t), r.edges(t))
    assert m.min_h() == r.min_h()
    np.testing.assert_array_equal(m.boundary_midpoints(), r.boundary_midpoints())
    require_reference_build()
    g = cpu.reference_mesh_from_file(d)
    assert g is not None and g["n_elem"] == len(q)
    np.testing.assert_array_equal(m.edges(0), g["edges_interior"])
    np.testing.assert_array_equal(m.edges(1), g["edges_boundary"])
    assert m.min_h() == g["min_h"]
    np.testing.assert_array_equal(m.boundary_midpoints(), g["midpoints"])


def test_file_text_is_read_as_the_reference_reads_it(W, tmp_path):
    """Whitespace and line breaks are free-form (stream extraction), indices 0-based."""
    d = tmp_path / "hand"
    d.mkdir()
    (d / "info.txt").write_text("6 2\n")
    (d / "coordinates.txt").write_text("0 0\n1 0 2 0\n\n0 1 1 1\n2 1\n")
    (d / "elements.txt").write_text("0 1 4 3\n1 2 5 4\n")
    m = W.Mesh2D.from_file(str(d))
    assert m.n_edges(0) == 1 and m.n_edges(1) == 6
    r = cpu.Mesh.from_file(str(d), "oracle")
    for t in (0, 1):
        np.testing.assert_array_equal(m.edges(t), r.edges(t))
    require_reference_build()
    g = cpu.reference_mesh_from_file(str(d))
    np.testing.assert_array_equal(m.edges(0), g["edges_interior"])
    np.testing.assert_array_equal(m.edges(1), g["edges_boundary"])


def test_bad_mesh_files_are_errors(W, tmp_path):
    with pytest.raises(W.WdgError, match="cannot open"):
        W.Mesh2D.from_file(str(tmp_path / "missing"))
    d = tmp_path / "short"
    d.mkdir()
    (d / "info.txt").write_text("4 1\n")
    (d / "coordinates.txt").write_text("0 0\n1 0\n1 1\n")  # one point short
    (d / "elements.txt").write_text("0 1 2 3\n")
    with pytest.raises(W.WdgError, match="fewer than 4 points"):
        W.Mesh2D.from_file(str(d))
    (d / "coordinates.txt").write_text("0 0\n1 0\n1 1\n0 1\n")
    (d / "elements.txt").write_text("0 1 2\n")
    with pytest.raises(W.WdgError, match="fewer than 1 elements"):
        W.Mesh2D.from_file(str(d))
    (d / "elements.txt").write_text("0 1 2 9\n")
    with pytest.raises(W.WdgError, match="out of range"):
        W.Mesh2D.from_file(str(d))


def test_snapshot_bytes_and_round_trip(W, tmp_path):
    u = np.random.default_rng(2).standard_normal(1234)
    f = str(tmp_path / "u00000.00000")
    W.to_file(f, u)
    with open(f, "rb") as fh:
        assert fh.read() == u.tobytes()  # dg::to_file: the array's bytes, nothing else
    back = np.zeros_like(u)
    W.read_file(f, back)
    np.testing.assert_array_equal(back, u)
    with pytest.raises(W.WdgError, match="expected"):
        W.read_file(f, np.zeros(1233))
    W.to_file(str(tmp_path / "empty"), np.zeros(0))
    assert os.path.getsize(tmp_path / "empty") == 0


@pytest.mark.parametrize("name", ["Square", "L", "skew"])
def test_reference_mesh_files(W, name):
    """The reference's own mesh files (copied into tests/golden/meshes/ by make_golden.py
    --reference-meshes): the library's reader must build exactly the connectivity, min_h and
    boundary midpoints that the reference's Mesh2D::from_file built from the same files
    (fixture), and the oracle's reader the same."""
    from conftest import GOLDEN, golden

    d = os.path.join(GOLDEN, "meshes", name)
    g = golden(f"mesh_file_{name}.npz")
    m = W.Mesh2D.from_file(d)
    assert m.n_elem() == len(g["quads"])
    np.testing.assert_array_equal(m.edges(0), g["edges_interior"])
    np.testing.assert_array_equal(m.edges(1), g["edges_boundary"])
    assert m.min_h() == float(g["min_h"])
    np.testing.assert_array_equal(m.boundary_midpoints(), g["midpoints"])
    np.testing.assert_array_equal(W.Mesh2D.from_vertices(g["verts"], g["quads"]).edges(0), g["edges_interior"])
    r = cpu.Mesh.from_file(d, "oracle")
    for t in (0, 1):
        np.testing.assert_array_equal(r.edges(t), m.edges(t))
