"""Exact quadrature (approx_quad = false) on the GPU against the reference and the oracle.

The fixtures tests/golden/opq_*.npz hold the reference's own Div<false>, EdgeFlux<false>,
MassMatrix<false>, WaveEquation / boundary operator, RHS and five RK4 steps on seeded
inputs (perturbed + scrambled and L-shaped meshes, every boundary code).  Tolerances as
for the collocation path: 1e-12 relative per operator, 1e-11 after the RK4 steps.
"""
import numpy as np
import pytest

from conftest import golden, golden_files, rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _disc(g):
    import wavedg_b200 as W

    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    return W, mesh, W.ExactDiscretisation(mesh, int(g["n"]), g["bc"])


@pytest.mark.parametrize("fname", golden_files("opq_"))
def test_operators_match_reference(gpu_lib, fname):
    g = golden(fname)
    W, mesh, d = _disc(g)
    u = g["u"]
    for nm, fn in (("div", d.div_action), ("wave_action", d.wave_action), ("bc_action", d.wavebc_action)):
        r = g[f"{nm}_in"].copy()
        fn(u, r)
        assert rel(r, g[nm]) < TOL, nm
    for k, tag in ((0, "interior"), (1, "boundary")):
        ub = g[f"flux_{tag}_in"]
        fb = np.zeros_like(ub)
        d.edge_flux(k, ub, fb)
        assert rel(fb, g[f"flux_{tag}"]) < TOL, tag
        inplace = ub.copy()
        d.edge_flux(k, inplace, inplace)
        assert rel(inplace, g[f"flux_{tag}"]) < TOL, tag
    x = u.copy()
    d.mass_inv(3, x)
    assert rel(x, g["mass_inv"]) < TOL
    y = np.zeros_like(u)
    d.mass_action(3, u, y)
    assert rel(y, g["mass_action"]) < TOL
    du = np.zeros_like(u)
    d.rhs(u, du)
    assert rel(du, g["rhs"]) < TOL
    un = u.copy()
    t = d.rk4_steps(un, float(g["dt"]), 0.0, 5)
    assert rel(un, g["rk4_5"]) < 1e-11
    assert abs(t - 5 * float(g["dt"])) < 1e-15


def test_reference_classes_with_approx_quad_false(gpu_lib):
    """The mirror classes route approx_quad=False to the exact operators; device arrays too."""
    import torch

    g = golden("opq_scrambled6_n5.npz")
    W, mesh, d = _disc(g)
    basis = W.QuadratureRule.quadrature_rule(int(g["n"]), W.QuadratureRule.GaussLobatto)
    u = g["u"]
    a = W.WaveEquation(mesh, basis, False)
    b = W.WaveBC(mesh, g["bc"], basis, False)
    m = W.MassMatrix(mesh, basis, approx_quad=False)
    du = torch.zeros(len(u), dtype=torch.float64, device="cuda")
    ud = torch.from_numpy(u).cuda()
    a.action(ud, du)
    b.action(ud, du)
    m.inv(3, du)
    torch.cuda.synchronize()
    assert rel(du.cpu().numpy(), g["rhs"]) < TOL
    assert d.rules() == (5, 6, 6)  # Div 1 + (3 + 4 + 1)//2; EdgeFlux and MassMatrix 1 + (8 + 2)//2


def test_larger_mesh_against_oracle(gpu_lib):
    """A 24 x 24 perturbed mesh, P = 4 and P = 6: RHS against the oracle's restatement."""
    import wavedg_b200 as W
    from oracle import cpu
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(24, 0.2, seed=8)
    mesh = W.Mesh2D.from_vertices(v, q)
    om = cpu.Mesh(v, q, "oracle")
    rng = np.random.default_rng(9)
    bc = rng.integers(0, 3, size=mesh.n_edges(1)).astype(np.int32)
    for n in (5, 7):
        d = W.ExactDiscretisation(mesh, n, bc)
        op = cpu.OpQ(om, n, bc)
        u = rng.standard_normal(d.ndof)
        du = np.zeros_like(u)
        d.rhs(u, du)
        assert rel(du, op.rhs(u)) < TOL, n


def test_waveholtz_exact_quadrature(gpu_lib):
    """WaveHoltz(..., approx_quad=False): pi0 and S against the reference's own WaveHoltz class
    (all-reflecting walls) and against the restated loop (mixed walls); the solve takes the
    reference's iteration count; postprocess against the oracle."""
    import wavedg_b200 as W
    from oracle import cpu

    g = golden("waveholtz_exact_5x5_P3.npz")
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    n, om = int(g["n"]), float(g["omega"])
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
    wr = W.WaveHoltz(om, mesh, basis, g["bc_reflect"], False)
    p = np.zeros_like(g["F"])
    wr.pi0(p, g["F"])
    assert rel(p, g["pi0_reflect"]) < 1e-12
    s = g["pi0_reflect"].copy()
    wr.S(s)
    assert rel(s, g["S_pi0_reflect"]) < 1e-12
    wh = W.WaveHoltz(om, mesh, basis, g["bc"], False)
    assert (wh.T, wh.dt, wh.nt) == (g["T"], g["dt"], g["nt"])
    p = np.zeros_like(g["F"])
    wh.pi0(p, g["F"])
    assert rel(p, g["pi0"]) < 1e-12
    s = g["pi0"].copy()
    wh.S(s)
    assert rel(s, g["S_pi0"]) < 1e-12
    Wx, it, res = wh.solve(g["F"], 1e-6, 200)
    assert it == int(g["iters"])
    assert rel(Wx, g["W"]) < 1e-10
    H = np.zeros(2 * len(g["W"]) // 3)
    wh.postprocess(H, g["W"])
    ref = cpu.WaveHoltz(cpu.OpQ(cpu.Mesh(g["verts"], g["quads"], "oracle"), n, g["bc"]), om).postprocess(g["W"])
    assert rel(H, ref) < TOL
