"""Failure detection on the GPU, exercised without faulting it.

Every wait of the fused stage kernels on a copy completion is bounded: past the handle's
limit (wdg_wave_set_wait_limit) the waiting warps record it in the device error word, wait
(bounded) for their own copies in flight and return, and the next synchronising call reports
WDG_ERR_TIMEOUT.  The test makes a wait run out on purpose: the test hook wdg_test_skip_chunk
has every CTA leave one chunk unloaded, so nothing ever completes the barrier its consumers
wait on.  The neighbour-offset check is exercised by overwriting one partner offset with a
value outside the state (wdg_test_set_partner): the kernel must skip that trace and report
it, not read it.  After either failure the same handle must give correct results again.
"""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case():
    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(48, 0.2, seed=41)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(5, W.QuadratureRule.GaussLobatto)
    bc = np.random.default_rng(42).integers(0, 3, size=mesh.n_edges(1)).astype(np.int32)
    u0 = np.random.default_rng(43).standard_normal(3 * 25 * mesh.n_elem())
    dt = 0.1 * mesh.min_h() / 25
    return W, mesh, basis, bc, u0, dt


def _reference_step(W, mesh, basis, bc, u0, dt):
    s = W.WaveSystem(mesh, basis, bc)
    u = u0.copy()
    s.rk4_steps(u, dt, 0.0, 1)
    return u


def test_expired_wait_is_reported_and_the_handle_recovers(gpu_lib):
    W, mesh, basis, bc, u0, dt = _case()
    want = _reference_step(W, mesh, basis, bc, u0, dt)
    s = W.WaveSystem(mesh, basis, bc)
    assert s.launch_config()["kernel"] == "ws"
    L = W.lib()
    assert L.wdg_wave_set_wait_limit(s._h, 0.005) == 0
    assert L.wdg_test_skip_chunk(s._h, 0) == 0
    u = u0.copy()
    t0 = time.perf_counter()
    with pytest.raises(W.WdgError) as e:
        s.rk4_steps(u, dt, 0.0, 1)
    took = time.perf_counter() - t0
    assert e.value.code == W._lib.WDG_ERR_TIMEOUT, e.value
    assert "bounded device-side wait" in str(e.value)
    # the 5 ms limit, not the 2 s default, ended the waits (a few waits in a row at most)
    assert took < 1.0, took
    # the error word was cleared and the hook was one-shot: the same handle steps correctly
    assert L.wdg_wave_sync(s._h) == 0
    assert L.wdg_wave_set_wait_limit(s._h, 2.0) == 0
    u = u0.copy()
    s.rk4_steps(u, dt, 0.0, 1)
    np.testing.assert_array_equal(u, want)
    assert L.wdg_wave_set_wait_limit(s._h, 0.0) == W._lib.WDG_ERR_ARG
    assert L.wdg_test_skip_chunk(s._h, -2) == W._lib.WDG_ERR_ARG


@pytest.mark.parametrize("bad", [10 ** 9, -7])
def test_neighbour_offset_outside_the_state_is_reported_not_read(gpu_lib, bad):
    W, mesh, basis, bc, u0, dt = _case()
    want = _reference_step(W, mesh, basis, bc, u0, dt)
    s = W.WaveSystem(mesh, basis, bc)
    L = W.lib()
    el, side = (int(x) for x in mesh.edges(0)[7][:2])  # one side of an interior edge
    prev = C.c_int()
    assert L.wdg_test_set_partner(s._h, el, side, bad, C.byref(prev)) == 0
    assert prev.value >= 0
    u = u0.copy()
    with pytest.raises(W.WdgError) as e:
        s.rk4_steps(u, dt, 0.0, 1)
    assert e.value.code == W._lib.WDG_ERR_ARG and "neighbour index" in str(e.value)
    assert L.wdg_test_set_partner(s._h, el, side, prev.value, None) == 0
    u = u0.copy()
    s.rk4_steps(u, dt, 0.0, 1)
    np.testing.assert_array_equal(u, want)
    assert L.wdg_test_set_partner(s._h, mesh.n_elem(), 0, 0, None) == W._lib.WDG_ERR_ARG
