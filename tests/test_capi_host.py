"""The C-ABI library without a GPU: it loads, exports every declared symbol,
and its host-side set-up (mesh connectivity, quadrature) matches the
reference's golden vectors.  No compute entry point is called here."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden, golden_files


@pytest.fixture(scope="module")
def L():
    from wavedg_b200 import build, lib

    build.build()
    return lib()


def test_exports_every_declared_symbol(L):
    from wavedg_b200._lib import SIGNATURES, header_symbols

    declared = header_symbols()
    assert len(declared) >= 45
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
        assert name in SIGNATURES, f"{name} has no ctypes signature"


def test_header_has_no_torch_types():
    import os

    from wavedg_b200._lib import HEADER

    txt = open(HEADER).read()
    for bad in ("torch", "at::", "Tensor", "c10"):
        assert bad not in txt
    assert os.path.exists(HEADER)


def test_basis_matches_reference(L):
    import wavedg_b200 as W

    g = golden("basis.npz")
    for n in range(2, 10):
        q = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
        assert np.abs(q.x - g[f"x{n}"]).max() < 1e-15
        assert np.abs(q.w - g[f"w{n}"]).max() < 1e-15
        D = q.derivative_matrix()
        assert np.linalg.norm(D - g[f"D{n}"]) / np.linalg.norm(g[f"D{n}"]) < 1e-14


@pytest.mark.parametrize("fname", golden_files("mesh_"))
def test_mesh_tables_match_reference(L, fname):
    import wavedg_b200 as W

    g = golden(fname)
    m = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    np.testing.assert_array_equal(m.edges(0), g["edges_interior"])
    np.testing.assert_array_equal(m.edges(1), g["edges_boundary"])
    assert m.min_h() == g["min_h"]
    np.testing.assert_array_equal(m.boundary_midpoints(), g["midpoints"])
    # adopting the reference's own tables gives the same mesh
    corners = g["verts"][g["quads"]].reshape(-1, 8)
    m2 = W.Mesh2D.from_tables(corners, g["edges_interior"], g["edges_boundary"])
    np.testing.assert_array_equal(m2.edges(0), g["edges_interior"])
    assert m2.min_h() == g["min_h"]


def test_uniform_rect_numbering(L):
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    g = golden("mesh_rect4x3.npz")
    v, q = mg.uniform_rect(4, -1.0, 1.0, 3, 0.0, 2.0)
    np.testing.assert_array_equal(v, g["verts"])
    np.testing.assert_array_equal(q, g["quads"])
    m = W.Mesh2D.uniform_rect(4, -1.0, 1.0, 3, 0.0, 2.0)
    np.testing.assert_array_equal(m.edges(0), g["edges_interior"])
    # 2n(n-1) interior and 4n boundary edges on an n x n grid
    m = W.Mesh2D.uniform_rect(64, -1, 1, 64, -1, 1)
    assert m.n_edges(0) == 2 * 64 * 63 and m.n_edges(1) == 4 * 64


def test_large_mesh_64bit_edge_keys(L):
    """More vertices than the reference's int edge key can hold (~46k): counts must still hold."""
    import wavedg_b200 as W

    m = W.Mesh2D.uniform_rect(300, -1, 1, 300, -1, 1)  # 90601 vertices
    assert m.n_edges(0) == 2 * 300 * 299 and m.n_edges(1) == 4 * 300


def test_large_scrambled_mesh_edge_tables_equal_the_oracle(L):
    """Past the int key's range, on a perturbed mesh with scrambled vertex and element numbers
    (so vertex pairs with large ids meet in every order): the whole interior and boundary edge
    tables, in the reference's edge order, equal the oracle's (64-bit keys too), element by
    element and side by side."""
    import wavedg_b200 as W
    from oracle import cpu
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(240, 0.2, seed=17)  # 58081 vertices
    v, q = mg.scrambled(v, q, seed=18)
    assert len(v) > 46341  # sqrt(2^31): the reference's int key i + nx j overflows from here
    m = W.Mesh2D.from_vertices(v, q)
    o = cpu.Mesh(v, q, "oracle")
    for t in (0, 1):
        np.testing.assert_array_equal(m.edges(t), o.edges(t))


def test_errors_are_reported(L):
    import wavedg_b200 as W

    with pytest.raises(W.WdgError):
        W.Mesh2D.from_vertices(np.zeros((3, 2)), np.array([[0, 1, 2, 7]]))  # vertex out of range
    h = C.c_void_p()
    assert L.wdg_mesh_uniform_rect(0, -1, 1, 4, -1, 1, C.byref(h)) == W._lib.WDG_ERR_ARG
    assert b"bad arguments" in L.wdg_last_error()
    with pytest.raises(W.WdgError):
        # exact quadrature with a caller-chosen rule: only the reference's default rules are built
        W.WaveEquation(W.Mesh2D.uniform_rect(2, -1, 1, 2, -1, 1), W.QuadratureRule.quadrature_rule(4, 1), False,
                       quad=W.QuadratureRule.quadrature_rule(7, 0))
    with pytest.raises(W.WdgError):  # Gauss-Legendre bases are not the Lobatto path
        W.WaveEquation(W.Mesh2D.uniform_rect(2, -1, 1, 2, -1, 1), W.QuadratureRule.quadrature_rule(4, 0), True)


def test_meshgen_properties():
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(16, 0.2, seed=3)
    v0, _ = mg.uniform_rect(16, -1, 1, 16, -1, 1)
    h = 2 / 16
    d = np.abs(v - v0)
    assert d.max() <= 0.2 * h + 1e-15
    boundary = (np.abs(v0[:, 0]) == 1) | (np.abs(v0[:, 1]) == 1)
    assert (d[boundary] == 0).all()
    # counter-clockwise elements after scrambling
    vs, qs = mg.scrambled(v, q, seed=4)
    p = vs[qs]
    area = 0.5 * np.sum(p[:, :, 0] * np.roll(p[:, :, 1], -1, 1) - np.roll(p[:, :, 0], -1, 1) * p[:, :, 1], axis=1)
    assert (area > 0).all()


def test_argument_errors_before_any_device_work(L):
    """Argument checks of the exact-quadrature, advection and decomposition front ends raise
    before anything touches a GPU."""
    import wavedg_b200 as W
    from wavedg_b200 import decomp

    mesh = W.Mesh2D.uniform_rect(3, -1, 1, 3, -1, 1)
    basis = W.QuadratureRule.quadrature_rule(4, W.QuadratureRule.GaussLobatto)
    with pytest.raises(W.WdgError, match="default rules"):
        W.ExactDiscretisation(mesh, 4, quad=W.QuadratureRule.quadrature_rule(6, 0))
    with pytest.raises(W.WdgError, match="2 n_var"):
        W.AdvectionSystem(2, mesh, basis, np.zeros(5))
    with pytest.raises(W.WdgError, match="n_elem coefficients"):
        W.Advection(1, mesh, basis, [1.0, 0.0], constant_coefficient=False)
    with pytest.raises(W.WdgError, match="2 n_var"):
        W.Advection(1, mesh, basis, [1.0, 0.0, 3.0], approx_quad=False)
    # a spatially varying coefficient whose n.A is not symmetric: refused at set-up, on the host
    a = np.zeros((mesh.n_elem(), 4, 4, 2, 2, 2))
    a[..., 0, 0, 1] = 1.0  # A_0 = [[0, 0], [1, 0]]
    with pytest.raises(W.WdgError, match="symmetric"):
        W.VariableAdvectionSystem(2, mesh, basis, a.reshape(-1), True)
    with pytest.raises(ValueError, match="one rank per element"):
        decomp.Plan(mesh, 4, None, np.zeros(5, dtype=np.int32), 0)
    with pytest.raises(ValueError):
        decomp.partition(10, 0)
    # the C entry points reject bad arguments with a status, not a crash
    h = C.c_void_p()
    assert L.wdg_waveq_create(None, 4, None, 0, C.byref(h)) == W._lib.WDG_ERR_ARG
    assert L.wdg_advect_create(mesh._h, 4, 9, C.c_void_p(np.zeros(162).ctypes.data), 0, C.byref(h)) == \
        W._lib.WDG_ERR_UNSUPPORTED
    assert L.wdg_mesh_partner_table(mesh._h, 1, None, None, None) == W._lib.WDG_ERR_ARG
    # the Gauss-Legendre set-up and variable-coefficient handles check basis type and degree
    # before any device work
    a = np.zeros(2 * 16 * mesh.n_elem())
    assert L.wdg_massmatrix_create(mesh._h, 4, 7, 1, 0, C.byref(h)) == W._lib.WDG_ERR_ARG
    assert L.wdg_massmatrix_create(mesh._h, 12, 0, 1, 0, C.byref(h)) == W._lib.WDG_ERR_UNSUPPORTED
    assert L.wdg_vadvect_create(mesh._h, 4, 7, 1, C.c_void_p(a.ctypes.data), 1, 0, C.byref(h)) == W._lib.WDG_ERR_ARG
    assert L.wdg_vadvect_create(mesh._h, 4, 0, 9, C.c_void_p(a.ctypes.data), 1, 0, C.byref(h)) == \
        W._lib.WDG_ERR_UNSUPPORTED
