"""MassMatrix<AQ> and LinearFunctional2D on Gauss-Legendre and Gauss-Lobatto bases
(wdg_massmatrix_*, dg.BasisMassMatrix, and the mirror classes for Gauss-Legendre bases) against
the compiled reference (tests/golden/massb_*.npz, make_golden.py --vadvection): M x, M^{-1} x,
the load vector's sample points, (f, phi) of examples/advec2d.cpp's coefficient r (y, -x) and
its projection M^{-1} (f, phi).  Bars: 1e-13 relative for M x and (f, phi), 1e-12 for the
inverses, 1e-14 absolute for the points."""
import numpy as np
import pytest

from conftest import golden, golden_files, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fname", golden_files("massb_"))
def test_mass_and_load_match_the_reference(gpu_lib, fname):
    import wavedg_b200 as W

    g = golden(fname)
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    n, approx = int(g["n"]), bool(int(g["approx"]))
    basis = W.QuadratureRule.quadrature_rule(n, int(g["basis_type"]))
    m = W.BasisMassMatrix(mesh, basis, approx)
    y = np.zeros_like(g["x"])
    m.action(2, g["x"], y)
    assert rel(y, g["action"]) < 1e-13
    z = g["x"].copy()
    m.inv(2, z)
    assert rel(z, g["inv"]) < 1e-12
    assert np.abs(m.points().reshape(-1) - g["points"]).max() < 1e-14
    F = np.zeros_like(g["load"])
    m.load(2, g["fq"], F)
    assert rel(F, g["load"]) < 1e-13
    m.inv(2, F)
    assert rel(F, g["projection"]) < 1e-12


@pytest.mark.parametrize("fname", [f for f in golden_files("massb_") if "_gl_" in f])
def test_mirror_classes_on_gauss_legendre_bases(gpu_lib, fname):
    """The reference-shaped classes route Gauss-Legendre bases to the same handle: the
    coefficient set-up of examples/advec2d.cpp, LF.action then m.inv, on device arrays."""
    import torch

    import wavedg_b200 as W

    g = golden(fname)
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    n, approx = int(g["n"]), bool(int(g["approx"]))
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLegendre)
    lf = W.LinearFunctional2D(mesh, basis)
    mm = W.MassMatrix(mesh, basis, approx_quad=approx)
    c = torch.zeros(g["load"].size, dtype=torch.float64, device="cuda")
    lf.action(2, lambda x, y: np.stack([np.hypot(x, y) * y, -np.hypot(x, y) * x]), c)
    assert rel(c.cpu().numpy(), g["load"]) < 1e-12
    mm.inv(2, c)
    torch.cuda.synchronize()
    assert rel(c.cpu().numpy(), g["projection"]) < 1e-12
