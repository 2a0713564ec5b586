"""The symmetries the learned warm start trains on, checked on the CPU oracle.

The warm-start family (uniform mesh of [-1, 1]^2, one boundary code on every wall) is
invariant under the eight symmetries of the square; training uses them to get eight pairs
from one solve.  These tests pin the field convention (p, v_x, v_y) and the node order: the
oracle's right-hand side commutes with each symmetry, and the load vector of a source moved
by a symmetry is the moved load vector.
"""
import numpy as np
import pytest

from oracle import cpu
from wavedg_b200 import meshgen
from wavedg_b200 import warmstart as ws

NE, N = 4, 3


def _op():
    verts, quads = meshgen.uniform_rect(NE, -1.0, 1.0, NE, -1.0, 1.0)
    m = cpu.Mesh(verts, quads, "oracle")
    return cpu.Op(m, N, np.zeros(m.n_edges(1), dtype=np.int32))


@pytest.mark.parametrize("k", range(8))
def test_rhs_commutes_with_the_symmetries(k):
    op = _op()
    u = np.random.default_rng(k).standard_normal(op.ndof)
    lhs = op.rhs(ws.sym_nodes(u, NE, N, k))
    rhs = ws.sym_nodes(op.rhs(u), NE, N, k)
    assert np.abs(lhs - rhs).max() <= 1e-12 * np.abs(rhs).max()


@pytest.mark.parametrize("k", range(8))
def test_moved_source_gives_the_moved_load(k):
    op = _op()
    c = np.array([[0.31, -0.17]])
    F = op.load_gaussians(c, [0.2], [1.0])
    Fk = op.load_gaussians(ws.sym_centers(c, k), [0.2], [1.0])
    assert np.abs(Fk - ws.sym_nodes(F, NE, N, k)).max() <= 1e-13 * np.abs(F).max()


def test_grid_and_node_symmetries_agree():
    """sym_grid on the cell-centred grid matches sym_nodes: a field sampled at grid points,
    moved either way, is the same (exact for the nearest-node sampling used here)."""
    import torch

    G = 2 * NE * N  # grid points at cell centres, symmetric about 0
    rng = np.random.default_rng(3)
    u = rng.standard_normal(3 * NE * NE * N * N)
    # nearest-node sampling (a symmetric map between the node set and the grid)
    x = np.polynomial.legendre.leggauss(N)[0]  # any symmetric node set works for this check
    xs = -1.0 + (np.arange(G) + 0.5) * 2.0 / G

    def sample(v):
        q = v.reshape(NE, NE, N, N, 3)
        g = np.zeros((3, G, G))
        h = 2.0 / NE
        for iy, y in enumerate(xs):
            for ix, xx in enumerate(xs):
                ex, ey = min(int((xx + 1) / h), NE - 1), min(int((y + 1) / h), NE - 1)
                xi = 2 * (xx - (-1 + ex * h)) / h - 1
                eta = 2 * (y - (-1 + ey * h)) / h - 1
                a, b = int(np.argmin(np.abs(x - xi))), int(np.argmin(np.abs(x - eta)))
                g[:, iy, ix] = q[ey, ex, b, a, :]
        return g

    for k in range(8):
        a = ws.sym_grid(torch.from_numpy(sample(u)), k).numpy()
        b = sample(ws.sym_nodes(u, NE, N, k))
        assert np.array_equal(a, b), k


def test_shipped_weights_record_their_training():
    """The network the bench's learned warm start loads: the shipped shape (4 Fourier layers,
    32 channels, 16 modes, hidden 64, 512 grid), trained on 2000 generated solutions of the
    128 x 128, P = 4, omega = 20 family, with every spectral tensor stored as float16 and a
    power-of-two scale."""
    import json

    path = ws.PACKAGED_WEIGHTS
    z = np.load(path)
    meta = json.loads(str(z["__meta__"]))
    assert meta["fno"] == {"layers": 4, "width": 32, "modes": 16, "hidden": 64}
    assert meta["grid"] == 512 and meta["family"] == "waveholtz_128x128_P4_omega20_outflow"
    assert meta["data"]["solutions"] == 2000 and meta["data"]["symmetries"] == 8
    assert meta["final_rel_rms_error"] < 1e-2
    spectral = [k for k in z.files if k.startswith("R") and not k.endswith(".exp2")]
    assert spectral and all(z[k].dtype == np.float16 and k + ".exp2" in z.files for k in spectral)
    assert float(z["__scale__"]) > 0
