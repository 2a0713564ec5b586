"""Linear advection with constant coefficients on the GPU against the reference.

tests/golden/adv_*.npz hold the reference's Advection<true> and AdvectionHomogeneousBC<true>
(n_var = 1, 2, 4; symmetric A_0, A_1), the RHS with MassMatrix<true>, and five RK4 steps, on
the perturbed + scrambled and L-shaped meshes.  1e-12 per operator, 1e-11 after the steps."""
import numpy as np
import pytest

from conftest import golden, golden_files, rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("fname", golden_files("adv_"))
def test_advection_matches_reference(gpu_lib, fname):
    import wavedg_b200 as W

    g = golden(fname)
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    n, nv = int(g["n"]), int(g["nv"])
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
    s = W.AdvectionSystem(nv, mesh, basis, g["a"])
    u = g["u"]
    r = g["action_in"].copy()
    W.Advection(nv, mesh, basis, g["a"]).action(u, r)
    assert rel(r, g["action"]) < TOL
    r = g["bc_action_in"].copy()
    W.AdvectionHomogeneousBC(nv, mesh, basis, g["a"]).action(u, r)
    assert rel(r, g["bc_action"]) < TOL
    du = np.zeros_like(u)
    s.rhs(u, du)
    assert rel(du, g["rhs"]) < TOL
    un = u.copy()
    s.rk4_steps(un, float(g["dt"]), 0.0, 5)
    assert rel(un, g["rk4_5"]) < 1e-11


def test_nonsymmetric_coefficients_are_rejected(gpu_lib):
    import wavedg_b200 as W

    mesh = W.Mesh2D.uniform_rect(3, -1, 1, 3, -1, 1)
    basis = W.QuadratureRule.quadrature_rule(4, W.QuadratureRule.GaussLobatto)
    a = np.zeros(8)
    a[1] = 1.0  # a(1, 0, 0) = 1, a(0, 1, 0) = 0
    with pytest.raises(W.WdgError, match="symmetric"):
        W.AdvectionSystem(2, mesh, basis, a)


def test_scalar_advection_conserves_with_reflection_free_outflow(gpu_lib):
    """Scalar transport of a bump by a constant velocity: the discrete mass sum_i m_i u_i only
    decreases (outflow through the boundary, nothing enters), and a long run moves the bump."""
    import torch

    import wavedg_b200 as W

    mesh = W.Mesh2D.uniform_rect(32, -1, 1, 32, -1, 1)
    basis = W.QuadratureRule.quadrature_rule(5, W.QuadratureRule.GaussLobatto)
    s = W.AdvectionSystem(1, mesh, basis, [0.5, 0.0])
    lf = W.WaveSystem(mesh, basis)
    F = np.zeros(3 * s.ndof)
    lf.load_gaussians([[-0.3, 0.0]], [0.1], [1.0], 1.0, 0, True, out=F)  # p component of a 3-field load
    u = np.ascontiguousarray(F[0::3])
    m = W.MassMatrix(mesh, basis)
    ones = np.ones_like(u)
    w = np.zeros_like(u)
    m.action(1, ones, w)
    mass0 = float(w @ u)
    dt = 0.1 * mesh.min_h() / 25
    s.rk4_steps(u, dt, 0.0, 200)
    mass1 = float(w @ u)
    assert mass1 <= mass0 * (1 + 1e-12) and mass1 > 0.5 * mass0
    torch.cuda.synchronize()


@pytest.mark.parametrize("fname", golden_files("vadv_"))
def test_variable_coefficient_advection_matches_reference(gpu_lib, fname):
    """Advection<AQ> / AdvectionHomogeneousBC<AQ> with constant_coefficient = false
    (tests/golden/vadv_*.npz: the compiled reference's outputs for n_var = 1 with the rotating
    velocity of examples/advec2d.cpp and n_var = 2, 3 with symmetric matrices varying in
    space; approx_quad true (_aq) and false (_ex); Gauss-Lobatto bases, and Gauss-Legendre
    (_gl) as examples/advec2d.cpp uses): the actions and the RHS to 1e-12, three RK4 and
    SSPRK3 steps to 1e-11, host and device arrays alike."""
    import torch

    import wavedg_b200 as W

    g = golden(fname)
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    n, nv, approx = int(g["n"]), int(g["nv"]), bool(int(g["approx"]))
    basis = W.QuadratureRule.quadrature_rule(n, int(g["basis_type"]))
    u = g["u"]
    r = g["action_in"].copy()
    W.Advection(nv, mesh, basis, g["a"], False, approx_quad=approx).action(u, r)
    assert rel(r, g["action"]) < TOL
    r = g["bc_action_in"].copy()
    W.AdvectionHomogeneousBC(nv, mesh, basis, g["a"], False, approx_quad=approx).action(u, r)
    assert rel(r, g["bc_action"]) < TOL
    s = W.VariableAdvectionSystem(nv, mesh, basis, g["a"], approx)
    r = np.zeros_like(u)
    s.rhs(u, r)
    e = rel(r, g["rhs"])
    print(f"{fname}: rhs rel err {e:.2e}")
    assert e < TOL
    dt = float(g["dt"])
    for method, key in (("rk4", "rk4_3"), ("ssprk3", "ssprk3_3")):
        v = u.copy()
        t = s.steps(v, dt, 0.0, 3, method)
        assert abs(t - 3 * dt) < 1e-15
        assert rel(v, g[key]) < 1e-11, method
        vd = torch.from_numpy(u.copy()).cuda()
        s.steps(vd, dt, 0.0, 3, method)
        s.sync()
        np.testing.assert_array_equal(vd.cpu().numpy(), v)



@pytest.mark.parametrize("fname", golden_files("adv_"))
def test_constant_coefficient_through_the_table_path(gpu_lib, fname):
    """A constant coefficient spread to the nodes through the variable-coefficient kernel gives
    the reference's constant-coefficient Advection<true> results (the route the mirror classes
    take for exact quadrature and Gauss-Legendre bases)."""
    import wavedg_b200 as W

    g = golden(fname)
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    n, nv = int(g["n"]), int(g["nv"])
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
    s = W.VariableAdvectionSystem(nv, mesh, basis, np.tile(g["a"], n * n * mesh.n_elem()), True)
    r = np.zeros_like(g["u"])
    s.rhs(g["u"], r)
    assert rel(r, g["rhs"]) < TOL
    r = g["action_in"].copy()
    s.action(g["u"], r)
    assert rel(r, g["action"]) < TOL
