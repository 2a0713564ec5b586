"""The oracle (oracle/wdg_oracle.cpp) against the reference's golden vectors.

Every fixture in tests/golden/ was produced by the reference library compiled
from its own sources (tests/golden/make_golden.py).  The oracle restates the
algorithm independently (64-bit edge keys, Newton-computed GLL nodes, Jacobi
eigen-decomposition for the flux matrices), so agreement here pins it.
"""
import numpy as np
import pytest

from conftest import golden, golden_files, rel, require_reference_build
from oracle import cpu

TOL = 1e-13  # FP64 restatement vs reference: only rounding order differs


def test_basis_matches_reference():
    g = golden("basis.npz")
    for n in range(2, 10):
        x, w, D = cpu.basis(n, "oracle")
        assert np.abs(x - g[f"x{n}"]).max() < 1e-15
        assert np.abs(w - g[f"w{n}"]).max() < 1e-15
        assert rel(D, g[f"D{n}"]) < 1e-14


@pytest.mark.parametrize("fname", golden_files("mesh_"))
def test_mesh_connectivity(fname):
    g = golden(fname)
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    np.testing.assert_array_equal(m.edges(0), g["edges_interior"])
    np.testing.assert_array_equal(m.edges(1), g["edges_boundary"])
    assert m.min_h() == g["min_h"]
    np.testing.assert_array_equal(m.boundary_midpoints(), g["midpoints"])


@pytest.mark.parametrize("fname", golden_files("op_"))
def test_operators(fname):
    g = golden(fname)
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    op = cpu.Op(m, int(g["n"]), g["bc"])
    u = g["u"]
    for nm in ("div", "wave_action", "bc_action"):
        r = g[f"{nm}_in"].copy()
        getattr(op, nm)(u, r)
        assert rel(r, g[nm]) < TOL, nm
    assert rel(op.rhs(u), g["rhs"]) < TOL
    assert rel(op.rhs(u, g["F"], 0.37), g["rhs_forced"]) < TOL
    for k in (0, 1):
        assert rel(op.prolong(k, u), g[f"prolong{k}"]) == 0.0
        assert rel(op.flux(k, g[f"flux{k}_in"]), g[f"flux{k}"]) < TOL
        r = g[f"prolong_t{k}_in"].copy()
        op.prolong_t(k, g[f"flux{k}_in"], r)
        assert rel(r, g[f"prolong_t{k}"]) < 1e-15
    uB = g["apply_bc_in"].copy()
    op.apply_bc(uB)
    assert rel(uB, g["apply_bc"]) < TOL
    x = u.copy()
    op.mass_inv(3, x)
    assert rel(x, g["mass_inv"]) < TOL
    assert rel(op.mass_action(3, u), g["mass_action"]) < TOL
    un, _ = op.rk4(u, float(g["rk4_dt"]), 3)
    assert rel(un, g["rk4"]) < TOL
    assert rel(op.node_coords(), g["node_coords"]) < 1e-15
    cen = np.array([[0.1, 0.2], [-0.3, 0.4]])
    assert rel(op.load_gaussians(cen, [0.3, 0.2], [1.0, -0.5], 2.0, 0, False), g["load"]) < 1e-13
    assert rel(op.load_gaussians(cen, [0.3, 0.2], [1.0, -0.5], 2.0, 1, True), g["load_minv"]) < 1e-13


@pytest.mark.parametrize("fname", golden_files("opq_"))
def test_exact_quadrature_operators(fname):
    """approx_quad = false: the oracle's Div<false>, EdgeFlux<false>, MassMatrix<false> and the
    operators built from them against the reference's."""
    g = golden(fname)
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    op = cpu.OpQ(m, int(g["n"]), g["bc"])
    u = g["u"]
    for nm in ("div", "wave_action", "bc_action"):
        r = g[f"{nm}_in"].copy()
        getattr(op, nm)(u, r)
        assert rel(r, g[nm]) < TOL, nm
    for k, tag in ((0, "interior"), (1, "boundary")):
        assert rel(op.flux(k, g[f"flux_{tag}_in"]), g[f"flux_{tag}"]) < TOL, tag
    x = u.copy()
    op.mass_inv(3, x)
    assert rel(x, g["mass_inv"]) < TOL
    assert rel(op.mass_action(3, u), g["mass_action"]) < TOL
    assert rel(op.rhs(u), g["rhs"]) < TOL
    un, _ = op.rk4(u, float(g["dt"]), 5)
    assert rel(un, g["rk4_5"]) < TOL


@pytest.mark.parametrize("fname", golden_files("adv_"))
def test_advection_operators(fname):
    """Advection<true> and AdvectionHomogeneousBC<true> (constant coefficients, any n_var)."""
    g = golden(fname)
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    op = cpu.OpA(m, int(g["n"]), int(g["nv"]), g["a"])
    u = g["u"]
    for nm in ("action", "bc_action"):
        r = g[f"{nm}_in"].copy()
        getattr(op, nm)(u, r)
        assert rel(r, g[nm]) < TOL, nm
    assert rel(op.rhs(u), g["rhs"]) < TOL
    un, _ = op.rk4(u, float(g["dt"]), 5)
    assert rel(un, g["rk4_5"]) < TOL


def test_config1_trajectory():
    g = golden("config1_32x32_P3.npz")
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    op = cpu.Op(m, int(g["n"]), g["bc"])
    u0 = op.load_gaussians([[0.0, 0.0]], [np.sqrt(0.005)], [1.0], 1.0, 0, True)
    assert rel(u0, g["u0"]) < 1e-13
    assert rel(op.rhs(g["u0"]), g["rhs0"]) < TOL
    u1, _ = op.rk4(g["u0"], float(g["dt"]), 1)
    assert rel(u1, g["u1"]) < TOL
    u200, t = op.rk4(g["u0"], float(g["dt"]), 200)
    assert rel(u200, g["u200"]) < 1e-12
    assert t == g["t200"]


def test_waveholtz():
    g = golden("waveholtz_5x5_P3.npz")
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    op = cpu.Op(m, int(g["n"]), g["bc"])
    wh = cpu.WaveHoltz(op, float(g["omega"]))
    assert (wh.T, wh.dt, wh.nt) == (g["T"], g["dt"], g["nt"])
    pi0 = wh.pi0(g["F"])
    assert rel(pi0, g["pi0"]) < 1e-13
    assert rel(wh.S(g["pi0"]), g["S_pi0"]) < 1e-13
    W, it, err = wh.solve(g["pi0"], 1e-6, 200)
    assert it == g["iters"]
    assert rel(W, g["W"]) < 1e-12
    assert rel(wh.postprocess(g["W"]), g["H"]) < 1e-13


def test_waveholtz_reflecting_uses_reference_class():
    g = golden("waveholtz_reflect_5x5_P3.npz")
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    op = cpu.Op(m, int(g["n"]), g["bc"])
    wh = cpu.WaveHoltz(op, float(g["omega"]))
    assert rel(wh.pi0(g["F"]), g["pi0"]) < 1e-13
    assert rel(wh.S(g["pi0"]), g["S_pi0"]) < 1e-13


def test_waveholtz_exact_quadrature():
    """approx_quad = false: the reference's own WaveHoltz class (all-reflecting walls) and the
    restated loop over the exact operators (mixed walls, solve to 1e-6)."""
    g = golden("waveholtz_exact_5x5_P3.npz")
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    n, om = int(g["n"]), float(g["omega"])
    wh1 = cpu.WaveHoltz(cpu.OpQ(m, n, g["bc_reflect"]), om)
    assert rel(wh1.pi0(g["F"]), g["pi0_reflect"]) < 1e-13
    assert rel(wh1.S(g["pi0_reflect"]), g["S_pi0_reflect"]) < 1e-13
    wh = cpu.WaveHoltz(cpu.OpQ(m, n, g["bc"]), om)
    assert (wh.T, wh.dt, wh.nt) == (g["T"], g["dt"], g["nt"])
    assert rel(wh.pi0(g["F"]), g["pi0"]) < 1e-13
    assert rel(wh.S(g["pi0"]), g["S_pi0"]) < 1e-13
    W, it, err = wh.solve(g["pi0"], 1e-6, 200)
    assert it == g["iters"]
    assert rel(W, g["W"]) < 1e-12


def test_oracle_catches_planted_error():
    """A mistake planted in the oracle's inputs must show up as a parity failure."""
    g = golden("op_scrambled6_n5.npz")
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    bc = g["bc"].copy()
    bc[0] = (bc[0] + 1) % 3  # wrong boundary code on one edge
    op = cpu.Op(m, int(g["n"]), bc)
    assert rel(op.rhs(g["u"]), g["rhs"]) > 1e-6


@pytest.mark.parametrize("n", range(2, 10))
def test_exact_quadrature_every_degree_against_the_reference(n):
    """The oracle's exact-quadrature restatement against the compiled reference for every
    degree the GPU path builds (n = 2..9), all operators, one seeded state."""
    from wavedg_b200 import meshgen as mg

    require_reference_build()
    v, q = mg.perturbed_rect(4, 0.2, seed=n)
    v, q = mg.scrambled(v, q, seed=n + 1)
    rng = np.random.default_rng(n)
    mo, mr = cpu.Mesh(v, q, "oracle"), cpu.Mesh(v, q, "reference")
    bc = rng.integers(0, 3, size=mo.n_edges(1)).astype(np.int32)
    o, r = cpu.OpQ(mo, n, bc), cpu.OpQ(mr, n, bc)
    u = rng.standard_normal(o.ndof)
    assert rel(o.rhs(u), r.rhs(u)) < 1e-12
    for k in (0, 1):
        uf = rng.standard_normal(n * 6 * mo.n_edges(k))
        assert rel(o.flux(k, uf), r.flux(k, uf)) < 1e-12
    x1, x2 = u.copy(), u.copy()
    o.mass_inv(3, x1)
    r.mass_inv(3, x2)
    assert rel(x1, x2) < 1e-12


@pytest.mark.parametrize("nv", range(1, 9))
def test_advection_every_variable_count_against_the_reference(nv):
    """The oracle's constant-coefficient advection against the compiled reference for every
    n_var the GPU path builds (1..8), random symmetric coefficients."""
    from wavedg_b200 import meshgen as mg

    require_reference_build()
    v, q = mg.perturbed_rect(4, 0.2, seed=nv)
    rng = np.random.default_rng(100 + nv)
    A = rng.standard_normal((2, nv, nv))
    A = A + A.transpose(0, 2, 1)
    a = np.concatenate([A[0].reshape(-1, order="F"), A[1].reshape(-1, order="F")])
    o = cpu.OpA(cpu.Mesh(v, q, "oracle"), 4, nv, a)
    r = cpu.OpA(cpu.Mesh(v, q, "reference"), 4, nv, a)
    u = rng.standard_normal(o.ndof)
    assert rel(o.rhs(u), r.rhs(u)) < 1e-12


@pytest.mark.parametrize("fname", golden_files("euler_"))
def test_oracle_euler_against_reference_fixtures(fname):
    """The oracle's restatement of DivF2D<true>, EdgeFluxF2D<true> with the local
    Lax-Friedrichs flux, the cl2d time derivative, RK4 and SSPRK3 against the reference's
    own outputs."""
    g = golden(fname)
    m = cpu.Mesh(g["verts"], g["quads"], "oracle")
    op = cpu.OpE(m, int(g["n"]))
    d = g["div_in"].copy()
    op.div(g["u"], d)
    assert rel(d, g["div"]) < 1e-13
    for k in (0, 1):
        np.testing.assert_array_equal(op.prolong(k, g["u"]), g[f"prolong{k}"])
        assert rel(op.flux(k, g[f"flux{k}_in"]), g[f"flux{k}"]) < 1e-13
    assert rel(op.rhs(g["u"]), g["rhs"]) < 1e-13
    assert rel(op.steps(g["u"], float(g["dt"]), 3, "rk4")[0], g["rk4_3"]) < 1e-13
    assert rel(op.steps(g["u"], float(g["dt"]), 3, "ssprk3")[0], g["ssprk3_3"]) < 1e-13


@pytest.mark.parametrize("fname", golden_files("eulerq_"))
def test_reference_exact_euler_fixtures_reproduce(fname):
    """The approx_quad = false Euler fixtures (DivF2D<false>, EdgeFluxF2D<false>,
    MassMatrix<false>) are what the compiled reference computes on their inputs; the GPU
    tests compare the CUDA path with these reference outputs directly."""
    require_reference_build()
    g = golden(fname)
    op = cpu.OpEQ(cpu.Mesh(g["verts"], g["quads"], "reference"), int(g["n"]))
    d = g["div_in"].copy()
    op.div(g["u"], d)
    np.testing.assert_array_equal(d, g["div"])
    for k in (0, 1):
        np.testing.assert_array_equal(op.flux(k, g[f"flux{k}_in"]), g[f"flux{k}"])
    np.testing.assert_array_equal(op.rhs(g["u"]), g["rhs"])
    np.testing.assert_array_equal(op.steps(g["u"], float(g["dt"]), 3, "rk4")[0], g["rk4_3"])
    np.testing.assert_array_equal(op.steps(g["u"], float(g["dt"]), 3, "ssprk3")[0], g["ssprk3_3"])


@pytest.mark.parametrize("fname", golden_files("vadv_"))
def test_reference_variable_advection_fixtures_reproduce(fname):
    """The variable-coefficient advection fixtures (Advection<AQ>, AdvectionHomogeneousBC<AQ>
    with constant_coefficient = false, MassMatrix<AQ>) are what the compiled reference computes
    on their inputs; the GPU tests compare the CUDA path with them directly."""
    require_reference_build()
    g = golden(fname)
    op = cpu.OpV(cpu.Mesh(g["verts"], g["quads"], "reference"), int(g["n"]), int(g["nv"]), g["a"],
                 bool(int(g["approx"])), int(g["basis_type"]))
    for nm in ("action", "bc_action"):
        r = g[f"{nm}_in"].copy()
        getattr(op, nm)(g["u"], r)
        np.testing.assert_array_equal(r, g[nm])
    np.testing.assert_array_equal(op.rhs(g["u"]), g["rhs"])
    np.testing.assert_array_equal(op.steps(g["u"], float(g["dt"]), 3, "rk4")[0], g["rk4_3"])
    np.testing.assert_array_equal(op.steps(g["u"], float(g["dt"]), 3, "ssprk3")[0], g["ssprk3_3"])
