"""The warp-specialised RK stage kernel (family 2) against the oracle.

Covers every supported degree (element-per-warp packing for n <= 5 differs from
the several-nodes-per-lane layout for n >= 6), both stepping precisions, ring
depths 2..6, chunk sizes with and without a ragged last chunk, few CTAs (each
walks many chunks round the ring), forcing and the FP64 filter (WaveHoltz),
and the fall-back to the tiled kernel for misaligned arrays.
Tolerances: 1e-12 relative (FP64) after two RK4 steps; 2e-5 (FP32).
"""
import numpy as np
import pytest

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _problem(n, nx, seed):
    from oracle import cpu
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(nx, 0.2, seed=seed)
    v, q = mg.scrambled(v, q, seed=seed + 1)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
    bc = np.random.default_rng(seed + 2).integers(0, 3, size=mesh.n_edges(1)).astype(np.int32)
    op = cpu.Op(cpu.Mesh(v, q, "oracle"), n, bc)
    u = np.random.default_rng(seed + 3).standard_normal(op.ndof)
    return W, mesh, basis, bc, op, u


def _valid_chunks(sys, W, count):
    """The smallest `count` chunk sizes the warp-specialised kernel accepts at the current ring."""
    out = []
    for c in range(4, 1025, 4):
        try:
            sys.tile = c
        except W.WdgError:
            continue
        out.append(c)
        if len(out) == count:
            break
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [2, 3, 4, 5, 6, 7, 8, 9])
def test_all_degrees(gpu_lib, n, precision):
    W, mesh, basis, bc, op, u = _problem(n, 13, 40 + n)  # 169 elements: a ragged last chunk for every unit
    ref, _ = op.rk4(u, 1e-3, 2)
    sys = W.WaveSystem(mesh, basis, bc, precision=precision)
    sys.set_kernel(2)
    assert sys.launch_config()["kernel"] == "ws"
    tol = 1e-12 if precision == "fp64" else 2e-5
    for ring in (2, 4, 6):
        try:
            sys.set_stages(ring)
        except W.WdgError:
            continue  # no chunk fits shared memory at this depth
        for chunk in _valid_chunks(sys, W, 2):
            sys.tile = chunk
            for ctas in (0, 1, 3):
                sys.set_max_ctas(ctas)
                un = u.copy()
                sys.rk4_steps(un, 1e-3, 0.0, 2)
                assert rel(un, ref) < tol, (ring, chunk, ctas, rel(un, ref))
    sys.set_max_ctas(0)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_chunks_and_rings_n5(gpu_lib, precision):
    """47 x 47 mesh (a prime count of elements per row, so chunks leave a ragged tail), P = 4:
    the four smallest chunk sizes at every ring depth that fits."""
    W, mesh, basis, bc, op, u = _problem(5, 47, 5)
    ref, _ = op.rk4(u, 1e-3, 2)
    sys = W.WaveSystem(mesh, basis, bc, precision=precision)
    sys.set_kernel(2)
    tol = 1e-12 if precision == "fp64" else 2e-5
    tried = 0
    for ring in (2, 3, 4, 5, 6):
        try:
            sys.set_stages(ring)
        except W.WdgError:
            continue
        for chunk in _valid_chunks(sys, W, 4):
            sys.tile = chunk
            for ctas in (0, 1, 7):
                sys.set_max_ctas(ctas)
                un = u.copy()
                sys.rk4_steps(un, 1e-3, 0.0, 2)
                assert rel(un, ref) < tol, (ring, chunk, ctas, rel(un, ref))
                tried += 1
    assert tried >= 6
    # the operator-mode RHS and a misaligned state take the tiled kernel
    if precision == "fp64":
        du = np.zeros_like(u)
        sys.rhs(u, du)
        assert rel(du, op.rhs(u)) < 1e-12
    sys.set_max_ctas(0)


def test_misaligned_state_falls_back(gpu_lib):
    import torch

    W, mesh, basis, bc, op, u = _problem(5, 12, 60)
    ref, _ = op.rk4(u, 1e-3, 1)
    sys = W.WaveSystem(mesh, basis, bc)
    sys.set_kernel(2)
    buf = torch.zeros(u.size + 1, dtype=torch.float64, device="cuda")
    view = buf[1:]
    view.copy_(torch.from_numpy(u))
    sys.rk4_steps(view, 1e-3, 0.0, 1)
    sys.sync()
    assert rel(view.cpu().numpy(), ref) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_waveholtz_forcing_and_filter(gpu_lib, precision):
    """WaveHoltz periods run the forcing + FP64 filter variant of the kernel."""
    import wavedg_b200 as W

    g = golden("waveholtz_5x5_P3.npz")
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    basis = W.QuadratureRule.quadrature_rule(int(g["n"]), W.QuadratureRule.GaussLobatto)
    sys = W.WaveSystem(mesh, basis, g["bc"], precision=precision)
    sys.set_kernel(2)
    wh = W.WaveHoltz(float(g["omega"]), mesh, basis, g["bc"], True, precision=precision, system=sys)
    s = g["pi0"].copy()
    wh.S(s)
    Wx, it, res = wh.solve(g["F"], 1e-6, 200)
    if precision == "fp64":
        assert rel(s, g["S_pi0"]) < 1e-12
        assert it == int(g["iters"])
        assert rel(Wx, g["W"]) < 1e-10
    else:
        assert rel(s, g["S_pi0"]) < 1e-4
        assert rel(Wx, g["W"]) < 1e-4
