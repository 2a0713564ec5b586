"""A decomposed mesh steps exactly like the undivided one (ranks emulated on one GPU).

Each rank's Domain holds its elements and a halo; the ranks run one after another in one
process, exchanging halo traces by device copies before every RK stage (no kernel waits on
another).  Every element's arithmetic is the undivided mesh's, so the states must agree
bit for bit after several RK4 steps, for contiguous and scattered partitions, FP64 and FP32.
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _setup(precision):
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(20, 0.2, seed=5)
    v, q = mg.scrambled(v, q, seed=6)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(5, W.QuadratureRule.GaussLobatto)
    bc = np.random.default_rng(7).integers(0, 3, size=mesh.n_edges(1)).astype(np.int32)
    whole = W.WaveSystem(mesh, basis, bc, precision=precision)
    u0 = np.random.default_rng(8).standard_normal(whole.ndof)
    return W, mesh, basis, bc, whole, u0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("world,kind", [(3, "blocks"), (3, "rcb"), (4, "random")])
def test_decomposed_steps_match_undivided(gpu_lib, precision, world, kind):
    from wavedg_b200 import decomp

    W, mesh, basis, bc, whole, u0 = _setup(precision)
    dt = 0.1 * mesh.min_h() / 25
    nsteps = 4
    ref = u0.copy()
    whole.rk4_steps(ref, dt, 0.0, nsteps)
    nel = mesh.n_elem()
    if kind == "blocks":  # contiguous element ids: spatially scattered on this scrambled mesh
        part = decomp.partition(nel, world)
    elif kind == "rcb":
        part = decomp.partition_mesh(mesh, world, "rcb")
    else:
        part = np.random.default_rng(9).integers(0, world, size=nel).astype(np.int32)
    doms = [decomp.Domain(mesh, basis, bc, part, r, precision=precision) for r in range(world)]
    assert all(d.halo > 0 for d in doms)
    if kind == "rcb":  # coordinate bisection leaves elements that read no halo trace
        assert all(d.split > 0 for d in doms)
    for overlap in (True, False):
        for d in doms:
            d.upload(u0)
        # with overlap every stage runs the halo-free elements before the halo is filled
        decomp.step_all(doms, dt, nsteps, overlap=overlap)
        out = np.zeros_like(u0)
        for d in doms:
            d.sync()
            d.download(out)
        diff = np.abs(out - ref).max()
        print(f"{precision} {kind} x{world} overlap {overlap}: max |decomposed - undivided| = {diff:.3e}")
        assert diff == 0.0


def test_whole_mesh_calls_are_refused(gpu_lib):
    """A domain steps stage by stage with its halo filled; whole-step and operator calls, which
    would take its cut sides for boundary sides, are refused with an error."""
    import ctypes as C

    import wavedg_b200 as W
    from wavedg_b200 import decomp

    _, mesh, basis, bc, whole, u0 = _setup("fp64")
    d = decomp.Domain(mesh, basis, bc, decomp.partition(mesh.n_elem(), 2), 0)
    u = np.zeros(d.ndof)
    t = C.c_double(0.0)
    rc = W.lib().wdg_rk4_steps(d._h, C.c_void_p(u.ctypes.data), 1e-3, C.byref(t), 1)
    assert rc == W._lib.WDG_ERR_UNSUPPORTED
    assert b"decomposed" in W.lib().wdg_last_error()
    du = np.zeros(d.ndof)
    rc = W.lib().wdg_rhs(d._h, C.c_void_p(u.ctypes.data), C.c_void_p(du.ctypes.data), None, 0.0)
    assert rc == W._lib.WDG_ERR_UNSUPPORTED


def _waveholtz_fixture():
    from conftest import golden

    return golden("waveholtz_5x5_P3.npz")


@pytest.mark.parametrize("world,method", [(3, "rcb"), (4, "rcm")])
def test_decomposed_waveholtz_matches_the_reference(gpu_lib, world, method):
    """The reference's WaveHoltz solve (5 x 5 perturbed mesh, P = 3, omega = 2, reflecting and
    absorbing walls) on a mesh split over `world` emulated ranks: the halo exchange before every
    stage, the filter per step and the norms summed over the ranks give the reference's
    iteration count and iterate."""
    import torch

    import wavedg_b200 as W
    from wavedg_b200 import decomp

    g = _waveholtz_fixture()
    mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
    basis = W.QuadratureRule.quadrature_rule(int(g["n"]), W.QuadratureRule.GaussLobatto)
    part = decomp.partition_mesh(mesh, world, method)
    doms = [decomp.Domain(mesh, basis, g["bc"], part, r) for r in range(world)]
    whs = [decomp.DomainWaveHoltz(d, float(g["omega"]), mesh.min_h()) for d in doms]
    assert whs[0].nt == int(g["nt"]) and whs[0].dt == float(g["dt"])
    Fs = [torch.from_numpy(d.local(g["F"])).cuda() for d in doms]
    Ws, it, res = decomp.waveholtz_solve(whs, Fs, 1e-6, 200, decomp.local_exchange(doms), lambda v: v)
    out = np.zeros_like(g["W"])
    for d, w in zip(doms, Ws):
        out.reshape(-1, d.plan.nd)[d.plan.local] = w.cpu().numpy().reshape(-1, d.plan.nd)
    print(f"{method} x{world}: {it} iterations (reference {int(g['iters'])}), W rel diff {rel(out, g['W']):.2e}")
    assert it == int(g["iters"])
    assert rel(out, g["W"]) < 1e-10


def test_decomposed_waveholtz_two_processes(gpu_lib, tmp_path):
    """The same solve by two processes over a gloo process group (halo traces and norm sums
    through host buffers; both processes on this GPU, no kernel waits on the other process)."""
    import os
    import socket
    import subprocess
    import sys

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    here = os.path.dirname(os.path.abspath(__file__))
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, os.path.join(here, "dist_waveholtz_worker.py"),
                                       str(tmp_path / f"r{r}.npz")], env=env))
    for p in procs:
        assert p.wait(timeout=600) == 0
    g = _waveholtz_fixture()
    out = np.full_like(g["W"], np.nan)
    nd = 3 * int(g["n"]) ** 2
    its = set()
    for r in range(2):
        z = np.load(tmp_path / f"r{r}.npz")
        out.reshape(-1, nd)[z["elems"]] = z["W"].reshape(-1, nd)
        its.add(int(z["iters"]))
    assert its == {int(g["iters"])}
    assert np.isfinite(out).all() and rel(out, g["W"]) < 1e-10
