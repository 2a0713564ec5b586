"""Batched WaveHoltz (wdg_whbatch_*) against single WaveHoltz solves.

The batch runs several solves of different degree, mesh and frequency through one
persistent launch per RK stage.  FP64 batch: every solve must take the same number of
iterations as the single-solve path (itself pinned to the reference by the golden
fixture) and agree with its iterate within 1e-10 relative; the golden solve is also
checked against the reference's own W.  Warm starts, launch shapes, FP32 stepping with
the stall rule, and the FP32 -> FP64 finish are covered too.
"""
import numpy as np
import pytest

from conftest import golden, rel

pytestmark = pytest.mark.gpu


def _batch_problems(precision="fp64"):
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    g = golden("waveholtz_5x5_P3.npz")
    probs = []
    # the golden problem (reference W, iteration count)
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    probs.append((mesh, int(g["n"]), g["bc"], float(g["omega"]), g["F"], g))
    # two more: other degrees, meshes, frequencies, boundary codes
    for (nx, n, omega, seed) in ((6, 5, 6.0, 11), (4, 7, 4.5, 12)):
        v, q = mg.perturbed_rect(nx, 0.2, seed=seed)
        mesh = W.Mesh2D.from_vertices(v, q)
        bc = np.random.default_rng(seed).integers(0, 2, size=mesh.n_edges(1)).astype(np.int32)
        probs.append((mesh, n, bc, omega, None, None))
    systems, Fs = [], []
    for (mesh, n, bc, omega, F, _) in probs:
        basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
        sys = W.WaveSystem(mesh, basis, bc, precision=precision)
        if F is None:
            F = sys.load_gaussians([[0.2, -0.1]], [0.15], [omega ** 2], 1.0, 0, False)
        systems.append(sys)
        Fs.append(np.ascontiguousarray(F))
    return W, probs, systems, Fs


def _single(W, mesh, n, bc, omega, F, tol, maxit=300):
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLobatto)
    wh = W.WaveHoltz(omega, mesh, basis, bc, True)
    Wx, it, res = wh.solve(F, tol, maxit)
    return Wx, it, res, wh


def test_batch_fp64_matches_single_solves(gpu_lib):
    W, probs, systems, Fs = _batch_problems()
    b = W.WaveHoltzBatch(systems, [p[3] for p in probs])
    Ws, its, res, st = b.solve(Fs, 1e-6, 300)
    g = probs[0][5]
    assert its[0] == int(g["iters"]) and rel(Ws[0], g["W"]) < 1e-10
    for s, (mesh, n, bc, omega, _, _) in enumerate(probs):
        Wx, it, r, wh = _single(W, mesh, n, bc, omega, Fs[s], 1e-6)
        assert (wh.T, wh.dt, wh.nt) == b.params(s)
        assert st[s] == 0 and res[s] < 1e-6
        assert its[s] == it, (s, its[s], it)
        assert rel(Ws[s], Wx) < 1e-10, (s, rel(Ws[s], Wx))


def test_launch_shapes_agree(gpu_lib):
    W, probs, systems, Fs = _batch_problems()
    b = W.WaveHoltzBatch(systems, [p[3] for p in probs])
    ref, its0, _, _ = b.solve(Fs, 1e-6, 300)
    ref = [x.copy() for x in ref]
    tried = 0
    for rounds, ring in ((2, 2), (1, 3), (1, 4), (3, 2)):
        try:
            b.set_launch(rounds, ring)
        except W.WdgError:
            continue  # does not fit shared memory with the degree-7 solve
        tried += 1
        assert b.launch_config()["ring"] == ring
        Ws, its, _, _ = b.solve(Fs, 1e-6, 300)
        assert (its == its0).all()
        for s in range(len(Ws)):
            assert rel(Ws[s], ref[s]) < 1e-12
    assert tried >= 2
    ms = b.autotune(64)
    assert ms > 0
    Ws, its, _, _ = b.solve(Fs, 1e-6, 300)
    assert (its == its0).all()


def test_warm_start_and_early_exit(gpu_lib):
    """A warm start near the solution converges in fewer iterations to the same answer; a
    solve that finishes early stops taking steps while the others run on."""
    W, probs, systems, Fs = _batch_problems()
    b = W.WaveHoltzBatch(systems, [p[3] for p in probs])
    W0, its0, _, _ = b.solve(Fs, 1e-8, 400)
    W0 = [x.copy() for x in W0]
    rng = np.random.default_rng(1)
    guess = [x + 1e-4 * np.linalg.norm(x) / np.sqrt(x.size) * rng.standard_normal(x.size) for x in W0]
    warm = [1, 0, 1]
    Ws, its, res, st = b.solve(Fs, 1e-8, 400, W=[x.copy() for x in guess], warm=warm)
    assert (st == 0).all()
    assert its[0] < its0[0] and its[2] < its0[2] and its[1] == its0[1]
    for s in range(3):
        assert rel(Ws[s], W0[s]) < 1e-6


def test_known_pi0_skips_the_extra_period(gpu_lib):
    """A warm start given |pi0| starts from W at once and follows the same iterates as one
    that measures |pi0| first; the norms reported match the zero start's first period."""
    W, probs, systems, Fs = _batch_problems()
    b = W.WaveHoltzBatch(systems, [p[3] for p in probs])
    W0, _, _, _ = b.solve(Fs, 1e-8, 400)
    p0 = b.pi0_norm.copy()
    assert (p0 > 0).all()
    rng = np.random.default_rng(2)
    guess = [x + 1e-4 * np.linalg.norm(x) / np.sqrt(x.size) * rng.standard_normal(x.size) for x in W0]
    Wa, ita, ra, sa = b.solve(Fs, 1e-8, 400, W=[x.copy() for x in guess], warm=[1, 1, 1])
    assert np.array_equal(b.pi0_norm, p0)
    Wb, itb, rb, sb = b.solve(Fs, 1e-8, 400, W=[x.copy() for x in guess], warm=[1, 1, 1], pi0_norm=p0)
    assert np.array_equal(b.pi0_norm, p0)
    assert (sa == 0).all() and (sb == 0).all() and (ita == itb).all()
    for s in range(3):
        assert rel(Wb[s], Wa[s]) < 1e-13
        assert abs(rb[s] - ra[s]) <= 1e-12 * ra[s]


def test_device_inputs_written_just_before_the_solve(gpu_lib):
    """Warm starts and forcing written on the caller's stream right before solve() are read
    only once complete (the batch orders its own stream after the solves' streams)."""
    import torch

    W, probs, systems, Fs = _batch_problems()
    b = W.WaveHoltzBatch(systems, [p[3] for p in probs])
    ref, its0, _, _ = b.solve(Fs, 1e-8, 400)
    ref = [x.copy() for x in ref]
    for _ in range(2):
        Fd, W0 = [], []
        for s in range(3):
            # a long chain of queued work (exact: powers of two) ending in the inputs' values
            f = torch.from_numpy(Fs[s]).cuda()
            w = torch.from_numpy(ref[s]).cuda()
            for _ in range(200):
                f.mul_(2.0).mul_(0.5)
                w.mul_(2.0).mul_(0.5)
            Fd.append(f)
            W0.append(w)
        Ws, its, res, st = b.solve(Fd, 1e-8, 400, W=W0, warm=[1, 1, 1])
        assert (st == 0).all() and (its <= 2).all(), its
        for s in range(3):
            assert rel(Ws[s].cpu().numpy(), ref[s]) < 1e-7


def test_fp32_batch_and_fp64_finish(gpu_lib):
    """FP32 stepping stops on the stall rule or at tol; an FP64 batch warm-started from its
    iterates then meets the FP64 tolerance (the plain iteration decides convergence)."""
    W, probs, systems32, Fs = _batch_problems("fp32")
    b32 = W.WaveHoltzBatch(systems32, [p[3] for p in probs])
    W32, it32, res32, st32 = b32.solve(Fs, 1e-6, 300, stall_limit=3)
    assert set(st32.tolist()) <= {0, 2}
    print("FP32 batch: iterations", it32.tolist(), "residuals", res32.tolist(), "status", st32.tolist())
    _, _, systems64, _ = _batch_problems("fp64")
    b64 = W.WaveHoltzBatch(systems64, [p[3] for p in probs])
    p32 = b32.pi0_norm.copy()
    Wf, itf, resf, stf = b64.solve(Fs, 1e-6, 300, W=[x.copy() for x in W32], warm=[1, 1, 1])
    assert (stf == 0).all() and (resf < 1e-6).all()
    p64 = b64.pi0_norm.copy()
    # the FP32 batch's |pi0| serves the FP64 finish in place of its own pi0 period
    assert np.allclose(p32, p64, rtol=1e-5, atol=0)
    Wk, itk, resk, stk = b64.solve(Fs, 1e-6, 300, W=[x.copy() for x in W32], warm=[1, 1, 1], pi0_norm=p32)
    assert (stk == 0).all() and (resk < 1e-6).all() and (np.abs(itk - itf) <= 1).all()
    Wd, itd, _, _ = b64.solve(Fs, 1e-6, 300)
    for s in range(3):
        err32 = rel(W32[s], Wd[s])
        print(f"solve {s}: FP32 iterate vs FP64 {err32:.2e}; FP64 finish {itf[s]} iterations (plain {itd[s]})")
        assert err32 < 1e-4
        assert rel(Wf[s], Wd[s]) < 1e-5
        assert itf[s] < itd[s]


def test_rejects_bad_batches(gpu_lib):
    import wavedg_b200 as W

    W_, probs, systems, Fs = _batch_problems()
    with pytest.raises(W.WdgError):
        W.WaveHoltzBatch([systems[0], systems[0]], [1.0, 2.0])
    with pytest.raises(W.WdgError):
        W.WaveHoltzBatch(systems, [1.0, -1.0, 2.0])
    _, _, sys32, _ = _batch_problems("fp32")
    with pytest.raises(W.WdgError):
        W.WaveHoltzBatch([systems[0], sys32[1]], [1.0, 2.0])
