"""The single WaveHoltz solve at full size (128 x 128 uniform quads, P = 4, outflow, omega = 20,
one Gaussian source) against the reference library's own solve of the same problem
(tests/golden/waveholtz_c3_128x128_P4.npz, written by make_c3_waveholtz.py from the reference
compiled from its sources: its operators, its RK4, the WaveHoltz loop of
source/WaveHoltz.cpp:55-121 and the fixed-point loop of examples/waveholtz2d.cpp:165-185).

The fixture keeps, per vector, its 2-norm, 8192 seeded entries and its inner products with
four seeded normal vectors.  A GPU vector x is compared with the reference's r by
  sampled:  |x[idx] - r[idx]| / |r[idx]|   (2-norms over the sampled entries)
  proj:     max_k |p_k . (x - r)| / |r|
  norm:     | |x| - |r| | / |r|
Bars: F (the load vector) 1e-13; pi0 and one fixed-point update W_2 = S(pi0) + pi0 in FP64
1e-12; the converged W in FP64 1e-10 with the same iteration count; FP32 stepping with the
FP64 filter and an FP64 finish: stated (its error against the reference is printed and held
under 1e-5).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
FIXTURE = os.path.join(GOLDEN, "waveholtz_c3_128x128_P4.npz")


def compare(x, g, name):
    """(sampled, proj, norm) relative differences of x (numpy) from the fixture's `name`."""
    idx = g["sample_index"]
    r = g[f"{name}_samples"]
    sampled = np.linalg.norm(x[idx] - r) / np.linalg.norm(r)
    nr = float(g[f"{name}_norm"])
    proj = max(abs(np.random.default_rng(int(g["proj_seed"]) + k).standard_normal(x.size) @ x - g[f"{name}_proj"][k])
               for k in range(int(g["nproj"]))) / nr
    return sampled, proj, abs(np.linalg.norm(x) - nr) / nr


@pytest.fixture(scope="module")
def c3(gpu_lib):
    import torch

    import wavedg_b200 as W

    g = dict(np.load(FIXTURE))
    ne, n, om = int(g["ne"]), int(g["n"]), float(g["omega"])
    mesh = W.Mesh2D.uniform_rect(ne, -1.0, 1.0, ne, -1.0, 1.0)
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
    s64 = W.WaveSystem(mesh, basis, bc, precision="fp64")
    F = torch.zeros(s64.ndof, dtype=torch.float64, device="cuda")
    s64.load_gaussians([g["x0"]], [float(g["sigma"])], [float(g["amp"])], 1.0, 0, False, out=F)
    return W, torch, g, mesh, basis, bc, s64, F, om


def test_load_vector_and_period_parameters(c3):
    W, torch, g, mesh, basis, bc, s64, F, om = c3
    assert max(compare(F.cpu().numpy(), g, "F")) < 1e-13
    wh = W.WaveHoltz(om, mesh, basis, bc, True, system=s64)
    assert wh.nt == int(g["nt"]) and wh.dt == float(g["dt"]) and wh.T == float(g["T"])


def test_pi0_and_one_update_fp64(c3):
    W, torch, g, mesh, basis, bc, s64, F, om = c3
    wh = W.WaveHoltz(om, mesh, basis, bc, True, system=s64)
    p = torch.zeros_like(F)
    wh.pi0(p, F)
    e = compare(p.cpu().numpy(), g, "pi0")
    print("pi0 vs reference (sampled, proj, norm):", e)
    assert max(e) < 1e-12
    w2 = p.clone()
    wh.S(w2)
    w2 += p
    e = compare(w2.cpu().numpy(), g, "W2")
    print("W2 vs reference:", e)
    assert max(e) < 1e-12


def test_converged_solution_fp64_and_fp32(c3):
    W, torch, g, mesh, basis, bc, s64, F, om = c3
    wh = W.WaveHoltz(om, mesh, basis, bc, True, system=s64)
    w = torch.zeros_like(F)
    _, it, res = wh.solve(F, float(g["tol"]), 1000, W=w)
    assert it == int(g["iterations"]), (it, int(g["iterations"]))
    e64 = compare(w.cpu().numpy(), g, "W")
    s32 = W.WaveSystem(mesh, basis, bc, precision="fp32")
    wh32 = W.WaveHoltz(om, mesh, basis, bc, True, precision="fp32", system=s32)
    w32 = torch.zeros_like(F)
    wh32.solve(F, 3e-6, 1000, W=w32)
    _, it64, res64 = wh.solve(F, float(g["tol"]), 1000, W=w32)
    e32 = compare(w32.cpu().numpy(), g, "W")
    print(f"converged W vs reference: FP64 {e64} ({it} iterations), FP32 + FP64 finish {e32} ({it64} FP64 iterations)")
    assert max(e64) < 1e-10
    assert res64 < float(g["tol"]) and max(e32) < 1e-5
