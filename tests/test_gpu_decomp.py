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
@pytest.mark.parametrize("world,kind", [(3, "blocks"), (4, "random")])
def test_decomposed_steps_match_undivided(gpu_lib, precision, world, kind):
    from wavedg_b200 import decomp

    W, mesh, basis, bc, whole, u0 = _setup(precision)
    dt = 0.1 * mesh.min_h() / 25
    nsteps = 4
    ref = u0.copy()
    whole.rk4_steps(ref, dt, 0.0, nsteps)
    nel = mesh.n_elem()
    part = decomp.partition(nel, world) if kind == "blocks" else \
        np.random.default_rng(9).integers(0, world, size=nel).astype(np.int32)
    doms = [decomp.Domain(mesh, basis, bc, part, r, precision=precision) for r in range(world)]
    assert all(d.halo > 0 for d in doms)
    for d in doms:
        d.upload(u0)
    decomp.step_all(doms, dt, nsteps)
    out = np.zeros_like(u0)
    for d in doms:
        d.sync()
        d.download(out)
    diff = np.abs(out - ref).max()
    print(f"{precision} {kind} x{world}: max |decomposed - undivided| = {diff:.3e}, rel {rel(out, ref):.3e}")
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
