"""Full-size checks at the 512 x 512, P = 4 workload (19.7M DOF), where the
oracle is only run once: one RHS against the oracle, and size-independent
properties (linearity, free-stream preservation, energy decay under upwind
fluxes, agreement of the host- and device-pointer paths)."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(512, 0.2, seed=2024)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(5, W.QuadratureRule.GaussLobatto)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)  # outflow everywhere
    return W, v, q, mesh, basis, bc


def test_rhs_vs_oracle_full_size(gpu_lib, big):
    from oracle import cpu

    W, v, q, mesh, basis, bc = big
    sys = W.WaveSystem(mesh, basis, bc)
    rng = np.random.default_rng(7)
    u = rng.standard_normal(sys.ndof)
    du = np.zeros_like(u)
    sys.rhs(u, du)
    om = cpu.Mesh(v, q, "oracle")
    op = cpu.Op(om, 5, bc)
    ref = op.rhs(u)
    assert rel(du, ref) < 1e-12


def test_rk4_step_vs_oracle_full_size(gpu_lib, big):
    """One RK4 step (5 fused stages) at full size against the oracle."""
    from oracle import cpu

    W, v, q, mesh, basis, bc = big
    sys = W.WaveSystem(mesh, basis, bc)
    xy = sys.node_coordinates().reshape(-1, 2)
    rng = np.random.default_rng(9)
    u = rng.standard_normal(sys.ndof) * 0.1
    u[0::3] += np.exp(-((xy[:, 0] - 0.3) ** 2 + xy[:, 1] ** 2) / (2 * 0.1**2))
    dt = 0.1 * mesh.min_h() / 25.0
    un = u.copy()
    sys.rk4_steps(un, dt, 0.0, 1)
    op = cpu.Op(cpu.Mesh(v, q, "oracle"), 5, bc)
    ref, _ = op.rk4(u, dt, 1)
    assert rel(un, ref) < 1e-12
    # both kernel families and several tile sizes agree at full size
    for family, tile in ((0, 0), (1, 8), (1, 12), (1, 16), (2, 0)):
        sys.set_kernel(family)
        if tile:
            sys.tile = tile
        u2 = u.copy()
        sys.rk4_steps(u2, dt, 0.0, 1)
        assert rel(u2, ref) < 1e-12, (family, tile)
    sys.set_kernel(-1)
    sys.tile = 0


def test_linearity(gpu_lib, big):
    torch = pytest.importorskip("torch")
    W, v, q, mesh, basis, bc = big
    sys = W.WaveSystem(mesh, basis, bc)
    g = torch.Generator(device="cuda").manual_seed(3)
    a = torch.randn(sys.ndof, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(sys.ndof, dtype=torch.float64, device="cuda", generator=g)
    ra, rb, rc = (torch.zeros_like(a) for _ in range(3))
    sys.rhs(a, ra)
    sys.rhs(b, rb)
    sys.rhs(2.5 * a - 0.75 * b, rc)
    sys.sync()
    lhs = rc
    rhs = 2.5 * ra - 0.75 * rb
    assert (torch.linalg.norm(lhs - rhs) / torch.linalg.norm(rhs)).item() < 1e-13


def test_free_stream_with_reflecting_walls(gpu_lib, big):
    """Constant pressure, zero velocity, reflecting walls: the discrete RHS vanishes."""
    W, v, q, mesh, basis, bc = big
    refl = np.ones_like(bc)
    nd = 3 * 25 * mesh.n_elem()
    u = np.zeros(nd)
    u[0::3] = 1.7
    r = np.zeros_like(u)
    W.WaveEquation(mesh, basis, True).action(u, r)
    W.WaveBC(mesh, refl, basis, True).action(u, r)
    dv = np.zeros_like(u)
    W.Div(mesh, basis).action(u, dv)  # the size of the terms that cancel
    assert np.abs(r).max() < 1e-12 * np.abs(dv).max()


def test_energy_decays_and_paths_agree(gpu_lib, big):
    W, v, q, mesh, basis, bc = big
    sys = W.WaveSystem(mesh, basis, bc)
    xy = sys.node_coordinates().reshape(-1, 2)
    u0 = np.zeros(sys.ndof)
    u0[0::3] = np.exp(-((xy[:, 0] - 0.1) ** 2 + (xy[:, 1] + 0.2) ** 2) / (2 * 0.05**2))
    dt = 0.1 * mesh.min_h() / 25.0
    sys.upload(u0)
    e = [sys.energy()]
    t = 0.0
    for _ in range(5):
        t = sys.step_state(dt, t, 4)
        e.append(sys.energy())
    assert all(e[k + 1] <= e[k] * (1 + 1e-13) for k in range(len(e) - 1)), e
    resident = sys.download()
    host = u0.copy()
    sys.rk4_steps(host, dt, 0.0, 20)
    assert rel(host, resident) < 1e-14
