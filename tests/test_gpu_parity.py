"""CUDA path vs the reference's golden vectors, through the C ABI.

Tolerances (FP64): 1e-12 relative (2-norm) per operator / RHS application, the
bar the drop-in must meet; trajectories of many steps are held to the bound
stated at each test.
"""
import numpy as np
import pytest

from conftest import golden, golden_files, rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _torch_cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


def _setup(g, precision="fp64"):
    import wavedg_b200 as W

    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    basis = W.QuadratureRule.quadrature_rule(int(g["n"]), W.QuadratureRule.GaussLobatto)
    return W, mesh, basis


@pytest.mark.parametrize("fname", golden_files("op_"))
def test_operators_host_arrays(gpu_lib, fname):
    g = golden(fname)
    W, mesh, basis = _setup(g)
    u = g["u"]
    ops = {
        "div": W.Div(mesh, basis),
        "wave_action": W.WaveEquation(mesh, basis, True),
        "bc_action": W.WaveBC(mesh, g["bc"], basis, True),
    }
    for nm, op in ops.items():
        r = g[f"{nm}_in"].copy()
        op.action(u, r)
        assert rel(r, g[nm]) < TOL, nm
    sys = W.WaveSystem(mesh, basis, g["bc"])
    du = np.zeros_like(u)
    sys.rhs(u, du)
    assert rel(du, g["rhs"]) < TOL
    sys.rhs(u, du, g["F"], 0.37)
    assert rel(du, g["rhs_forced"]) < TOL
    for k in (0, 1):
        P = W.make_face_prolongator(mesh, basis, k)
        uf = np.zeros(P.size())
        P.action(3, u, uf)
        assert rel(uf, g[f"prolong{k}"]) == 0.0
        r = g[f"prolong_t{k}_in"].copy()
        P.t(3, g[f"flux{k}_in"], r)
        assert rel(r, g[f"prolong_t{k}"]) < 1e-15
        flx = W.EdgeFlux(mesh, k, basis)
        fb = np.zeros_like(uf)
        flx.action(g[f"flux{k}_in"], fb)
        assert rel(fb, g[f"flux{k}"]) < TOL
        inplace = g[f"flux{k}_in"].copy()
        flx.action(inplace, inplace)  # EdgeFlux allows fb == ub
        assert rel(inplace, g[f"flux{k}"]) < TOL
    uB = g["apply_bc_in"].copy()
    ops["bc_action"].apply_bc(uB)
    assert rel(uB, g["apply_bc"]) < TOL
    M = W.MassMatrix(mesh, basis)
    x = u.copy()
    M.inv(3, x)
    assert rel(x, g["mass_inv"]) < TOL
    y = np.zeros_like(u)
    M.action(3, u, y)
    assert rel(y, g["mass_action"]) < TOL
    un = u.copy()
    t = sys.rk4_steps(un, float(g["rk4_dt"]), 0.0, 3)
    assert rel(un, g["rk4"]) < TOL
    assert abs(t - 3 * float(g["rk4_dt"])) < 1e-15
    assert rel(sys.node_coordinates(), g["node_coords"]) < 1e-15
    cen = np.array([[0.1, 0.2], [-0.3, 0.4]])
    assert rel(sys.load_gaussians(cen, [0.3, 0.2], [1.0, -0.5], 2.0, 0, False), g["load"]) < 1e-13
    assert rel(sys.load_gaussians(cen, [0.3, 0.2], [1.0, -0.5], 2.0, 1, True), g["load_minv"]) < 1e-13


@pytest.mark.parametrize("fname", ["op_scrambled6_n5.npz", "op_lshape3_n5.npz", "op_rect4x3_n6.npz"])
def test_operators_device_arrays(gpu_lib, fname):
    torch = _torch_cuda()
    g = golden(fname)
    W, mesh, basis = _setup(g)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    u = dev(g["u"])
    sys = W.WaveSystem(mesh, basis, g["bc"])
    du = torch.zeros_like(u)
    sys.rhs(u, du)
    sys.sync()
    assert rel(du.cpu().numpy(), g["rhs"]) < TOL
    r = dev(g["wave_action_in"])
    W.WaveEquation(mesh, basis, True).action(u, r)
    torch.cuda.synchronize()
    assert rel(r.cpu().numpy(), g["wave_action"]) < TOL
    un = u.clone()
    sys.rk4_steps(un, float(g["rk4_dt"]), 0.0, 3)
    sys.sync()
    assert rel(un.cpu().numpy(), g["rk4"]) < TOL
    # a misaligned (8-byte offset) device view takes the non-TMA load path
    buf = torch.zeros(u.numel() + 1, dtype=torch.float64, device="cuda")
    buf[1:].copy_(u)
    du2 = torch.zeros_like(u)
    sys.rhs(buf[1:], du2)
    sys.sync()
    assert rel(du2.cpu().numpy(), g["rhs"]) < TOL


@pytest.mark.parametrize("tile", [0, 4, 8, 12, 16, 20])
def test_tile_sizes_agree(gpu_lib, tile):
    g = golden("op_scrambled6_n5.npz")
    W, mesh, basis = _setup(g)
    sys = W.WaveSystem(mesh, basis, g["bc"])
    if tile == 0:
        sys.set_kernel(0)
    else:
        sys.set_kernel(1)
        sys.tile = tile
    un = g["u"].copy()
    sys.rk4_steps(un, float(g["rk4_dt"]), 0.0, 3)
    assert rel(un, g["rk4"]) < TOL


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_many_tiles_per_cta(gpu_lib, precision):
    """Few CTAs on a 48 x 48 scrambled mesh: every CTA walks dozens of tiles through the
    double-buffered pipeline (tile sizes 4..24, stage 0 and stages 1-4, tail tiles)."""
    from oracle import cpu
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(48, 0.2, seed=5)
    v, q = mg.scrambled(v, q, seed=6)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(5, W.QuadratureRule.GaussLobatto)
    bc = np.random.default_rng(7).integers(0, 3, size=mesh.n_edges(1)).astype(np.int32)
    op = cpu.Op(cpu.Mesh(v, q, "oracle"), 5, bc)
    u = np.random.default_rng(8).standard_normal(op.ndof)
    ref_rhs = op.rhs(u)
    ref_rk, _ = op.rk4(u, 1e-3, 2)
    sys = W.WaveSystem(mesh, basis, bc, precision=precision)
    tol = TOL if precision == "fp64" else 2e-5
    sys.set_kernel(0)  # warp per element
    un = u.copy()
    sys.rk4_steps(un, 1e-3, 0.0, 2)
    assert rel(un, ref_rk) < tol, ("warp", rel(un, ref_rk))
    if precision == "fp64":
        du = np.zeros_like(u)
        sys.rhs(u, du)
        assert rel(du, ref_rhs) < TOL
    sys.set_kernel(1)  # tiled pipeline
    for stages in (2, 3, 4):
      sys.set_stages(stages)
      for tile in (4, 8, 12, 16, 20):
        for ctas in (1, 3, 7):
            try:
                sys.tile = tile
            except W.WdgError:
                continue  # does not fit shared memory at this depth
            sys.set_max_ctas(ctas)
            un = u.copy()
            sys.rk4_steps(un, 1e-3, 0.0, 2)
            assert rel(un, ref_rk) < tol, (tile, ctas, rel(un, ref_rk))
            if precision == "fp64":
                du = np.zeros_like(u)
                sys.rhs(u, du)
                assert rel(du, ref_rhs) < TOL, (tile, ctas)
    sys.set_max_ctas(0)
    sys.set_stages(0)
    sys.tile = 0
    sys.set_kernel(-1)
    ms = sys.autotune(2)
    cfg = sys.launch_config()
    assert ms > 0 and cfg["stages"] in (2, 3, 4, 5, 6)
    un = u.copy()
    sys.rk4_steps(un, 1e-3, 0.0, 2)
    assert rel(un, ref_rk) < tol


def test_config1_trajectory(gpu_lib):
    """32 x 32, P = 3, Dirichlet p = 0, 200 RK4 steps: state vs the reference at steps 1 and 200."""
    g = golden("config1_32x32_P3.npz")
    W, mesh, basis = _setup(g)
    sys = W.WaveSystem(mesh, basis, g["bc"])
    u0 = sys.load_gaussians([[0.0, 0.0]], [np.sqrt(0.005)], [1.0], 1.0, 0, True)
    assert rel(u0, g["u0"]) < 1e-13
    du = np.zeros_like(u0)
    sys.rhs(g["u0"], du)
    assert rel(du, g["rhs0"]) < TOL
    u = g["u0"].copy()
    t = sys.rk4_steps(u, float(g["dt"]), 0.0, 1)
    assert rel(u, g["u1"]) < TOL
    t = sys.rk4_steps(u, float(g["dt"]), t, 199)
    assert rel(u, g["u200"]) < 1e-11  # 200 steps x 5 stages of 1e-16 rounding
    assert t == pytest.approx(float(g["t200"]), abs=1e-14)


def test_config1_fp32_error_stated(gpu_lib):
    """FP32 stepping: error vs the FP64 reference after 200 steps (stated, bounded)."""
    g = golden("config1_32x32_P3.npz")
    W, mesh, basis = _setup(g)
    sys = W.WaveSystem(mesh, basis, g["bc"], precision="fp32")
    u = g["u0"].copy()
    sys.rk4_steps(u, float(g["dt"]), 0.0, 200)
    err = rel(u, g["u200"])
    print(f"config1 FP32 relative error after 200 steps: {err:.3e}")
    assert err < 1e-5


def test_waveholtz_fp64(gpu_lib):
    g = golden("waveholtz_5x5_P3.npz")
    W, mesh, basis = _setup(g)
    wh = W.WaveHoltz(float(g["omega"]), mesh, basis, g["bc"], True)
    assert (wh.T, wh.dt, wh.nt) == (g["T"], g["dt"], g["nt"])
    p0 = np.zeros_like(g["F"])
    wh.pi0(p0, g["F"])
    assert rel(p0, g["pi0"]) < 1e-12
    s = g["pi0"].copy()
    wh.S(s)
    assert rel(s, g["S_pi0"]) < 1e-12
    Wx, it, res = wh.solve(g["F"], 1e-6, 200)
    assert it == int(g["iters"])
    assert rel(Wx, g["W"]) < 1e-10
    H = np.zeros(2 * len(g["W"]) // 3)
    wh.postprocess(H, g["W"])
    assert rel(H, g["H"]) < TOL


def test_waveholtz_reflecting(gpu_lib):
    g = golden("waveholtz_reflect_5x5_P3.npz")
    W, mesh, basis = _setup(g)
    wh = W.WaveHoltz(float(g["omega"]), mesh, basis, g["bc"], True)
    p0 = np.zeros_like(g["F"])
    wh.pi0(p0, g["F"])
    assert rel(p0, g["pi0"]) < 1e-12
    s = g["pi0"].copy()
    wh.S(s)
    assert rel(s, g["S_pi0"]) < 1e-12


def test_waveholtz_fp32_error_stated(gpu_lib):
    g = golden("waveholtz_5x5_P3.npz")
    W, mesh, basis = _setup(g)
    wh = W.WaveHoltz(float(g["omega"]), mesh, basis, g["bc"], True, precision="fp32")
    Wx, it, res = wh.solve(g["F"], 1e-6, 200)
    err = rel(Wx, g["W"])
    print(f"WaveHoltz FP32 stepping: {it} iterations (FP64 reference {int(g['iters'])}), "
          f"residual {res:.2e}, error vs FP64 reference {err:.2e}")
    assert err < 1e-4
