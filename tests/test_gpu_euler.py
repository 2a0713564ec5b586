"""The nonlinear conservation-law path (the compressible Euler system of examples/cl2d.cpp)
against the reference library compiled from its sources (written by make_golden.py --euler:
tests/golden/euler_*.npz with approx_quad = true, DivF2D<true> and EdgeFluxF2D<true>;
tests/golden/eulerq_*.npz with approx_quad = false, as the example ships, DivF2D<false>,
EdgeFluxF2D<false> and MassMatrix<false>; both with the example's local Lax-Friedrichs flux,
its time derivative, ode::RungeKutta4 and ode::SSPRK3), and the fused advection path against
the Advection fixtures.

Bars: 1e-12 relative (2-norm) per operator and RHS; 1e-11 after three RK4 or SSPRK3 steps.
"""
import numpy as np
import pytest

from conftest import golden, golden_files, rel

pytestmark = pytest.mark.gpu


def _system(g):
    import wavedg_b200 as W

    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    basis = W.QuadratureRule.quadrature_rule(int(g["n"]), W.QuadratureRule.GaussLobatto)
    return W, mesh, W.EulerSystem(mesh, basis, approx_quad=not fname_exact(g))


def fname_exact(g):
    return bool(g.get("exact", False))


EULER_FILES = golden_files("euler_") + golden_files("eulerq_")


def _load(fname):
    g = dict(golden(fname))
    g["exact"] = fname.startswith("eulerq_")
    return g


@pytest.mark.parametrize("fname", EULER_FILES)
def test_euler_operators_match_the_reference(gpu_lib, fname):
    g = _load(fname)
    W, mesh, s = _system(g)
    u = g["u"]
    d = g["div_in"].copy()
    s.div(u, d)
    assert rel(d, g["div"]) < 1e-12
    for k in (0, 1):
        fb = np.zeros_like(g[f"flux{k}_in"])
        s.flux(k, g[f"flux{k}_in"], fb)
        assert rel(fb, g[f"flux{k}"]) < 1e-12, k
        inplace = g[f"flux{k}_in"].copy()
        s.flux(k, inplace, inplace)
        np.testing.assert_array_equal(inplace, fb)
    r = np.zeros_like(u)
    s.rhs(u, r)
    e = rel(r, g["rhs"])
    print(f"{fname}: rhs rel err {e:.2e}")
    assert e < 1e-12


@pytest.mark.parametrize("fname", EULER_FILES)
@pytest.mark.parametrize("method", ["rk4", "ssprk3"])
def test_euler_steps_match_the_reference(gpu_lib, fname, method):
    import torch

    g = _load(fname)
    W, mesh, s = _system(g)
    want = g["rk4_3" if method == "rk4" else "ssprk3_3"]
    u = g["u"].copy()
    t = s.steps(u, float(g["dt"]), 0.0, 3, method)  # host array
    assert abs(t - 3 * float(g["dt"])) < 1e-15
    assert rel(u, want) < 1e-11
    ud = torch.from_numpy(g["u"].copy()).cuda()  # device array: the same result
    s.steps(ud, float(g["dt"]), 0.0, 3, method)
    s.sync()
    np.testing.assert_array_equal(ud.cpu().numpy(), u)


def test_euler_mass_changes_only_through_the_boundary(gpu_lib):
    """Total mass sum_i m_i rho_i changes only through boundary fluxes: for a state that is
    uniform (to rounding) near the boundary, sum_i m_i (rho_t)_i vanishes to rounding (a
    derived property; the masses m_i = w_i w_j det J are formed here from the corners)."""
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    n = 5
    v, q = mg.perturbed_rect(10, 0.2, seed=4)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
    s = W.EulerSystem(mesh, basis)
    xg, wg = np.asarray(basis.x), np.asarray(basis.w)
    c = v[q]  # (nel, 4, 2)
    xi, eta = xg[None, None, :], xg[None, :, None]  # node (i, j) at [.., j, i]
    X = lambda k, a, b: c[:, a, k][:, None, None] - c[:, b, k][:, None, None]  # noqa: E731
    Xx = 0.25 * ((1 - eta) * X(0, 1, 0) + (1 + eta) * X(0, 2, 3))
    Yx = 0.25 * ((1 - eta) * X(1, 1, 0) + (1 + eta) * X(1, 2, 3))
    Xe = 0.25 * ((1 - xi) * X(0, 3, 0) + (1 + xi) * X(0, 2, 1))
    Ye = 0.25 * ((1 - xi) * X(1, 3, 0) + (1 + xi) * X(1, 2, 1))
    m = (wg[None, :, None] * wg[None, None, :] * (Xx * Ye - Yx * Xe)).ravel()
    phi = lambda a, b: 0.25 * ((1 - xi) * (1 - eta) * c[:, 0, a][:, None, None] + (1 + xi) * (1 - eta) *  # noqa: E731
                               c[:, 1, a][:, None, None] + (1 + xi) * (1 + eta) * c[:, 2, a][:, None, None] +
                               (1 - xi) * (1 + eta) * c[:, 3, a][:, None, None])
    x, y = phi(0, 0).ravel(), phi(1, 1).ravel()
    bump = np.exp(-((x ** 2 + y ** 2) / 0.05))  # below 1e-30 at the boundary
    rho, p = 1.0 + 0.3 * bump, 1.0 + 0.2 * bump
    uu, vv = 0.2 * bump, -0.1 * bump
    U = np.stack([rho, rho * uu, rho * vv, p / 0.4 + 0.5 * rho * (uu * uu + vv * vv)], axis=1).ravel()
    r = np.zeros_like(U)
    s.rhs(U, r)
    total = np.sum(m * r[0::4])
    assert abs(total) < 1e-12 * np.sum(np.abs(m * r[0::4]))


@pytest.mark.parametrize("fname", golden_files("adv_"))
def test_fused_advection_rhs_and_rk4(gpu_lib, fname):
    """Advection's RHS and RK4 now run through the fused kernel: the same bars as before."""
    import wavedg_b200 as W

    g = golden(fname)
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    basis = W.QuadratureRule.quadrature_rule(int(g["n"]), W.QuadratureRule.GaussLobatto)
    s = W.AdvectionSystem(int(g["nv"]), mesh, basis, g["a"])
    r = np.zeros_like(g["u"])
    s.rhs(g["u"], r)
    assert rel(r, g["rhs"]) < 1e-12
    u = g["u"].copy()
    s.rk4_steps(u, float(g["dt"]), 0.0, 5)
    assert rel(u, g["rk4_5"]) < 1e-11
