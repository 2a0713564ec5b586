"""wdg_load_gaussians_noalloc: the load-vector entry point for callers that cannot
allocate device memory (real-time loops whose memory is fixed before they start,
hosts whose own allocator has reserved the GPU).  It must give the same load
vector as wdg_load_gaussians, call after call, while keeping its source table in
the library's fixed-size array.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
    import torch

    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(24, 0.2, seed=31)
    v, q = mg.scrambled(v, q, seed=32)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(5, W.QuadratureRule.GaussLobatto)
    sys = W.WaveSystem(mesh, basis, None)
    return torch, W, sys


def _sources(rng, k):
    c = rng.uniform(-0.8, 0.8, size=(k, 2))
    return (np.ascontiguousarray(c[:, 0]), np.ascontiguousarray(c[:, 1]),
            rng.uniform(0.05, 0.3, size=k), rng.standard_normal(k))


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def test_noalloc_matches_allocating_entry_point_twice():
    torch, W, sys = _setup()
    L = W.lib()
    rng = np.random.default_rng(33)
    for call, (k, comp, minv) in enumerate([(7, 0, 0), (3, 2, 1)]):
        cx, cy, sg, am = _sources(rng, k)
        ref = torch.zeros(sys.ndof, dtype=torch.float64, device="cuda")
        out = torch.full((sys.ndof,), float("nan"), dtype=torch.float64, device="cuda")
        st = L.wdg_load_gaussians(sys._h, k, _ptr(cx), _ptr(cy), _ptr(sg), _ptr(am), 1.5, comp, minv,
                                  C.c_void_p(ref.data_ptr()))
        assert st == 0, L.wdg_last_error()
        st = L.wdg_load_gaussians_noalloc(sys._h, k, _ptr(cx), _ptr(cy), _ptr(sg), _ptr(am), 1.5, comp, minv,
                                          C.c_void_p(out.data_ptr()))
        assert st == 0, L.wdg_last_error()
        sys.sync()
        r, o = ref.cpu().numpy(), out.cpu().numpy()
        assert np.isfinite(o).all()
        assert np.linalg.norm(o - r) <= 1e-13 * np.linalg.norm(r), call


def test_noalloc_limits_are_reported():
    torch, W, sys = _setup()
    L = W.lib()
    k = 1025
    cx = np.zeros(k)
    out = torch.zeros(sys.ndof, dtype=torch.float64, device="cuda")
    st = L.wdg_load_gaussians_noalloc(sys._h, k, _ptr(cx), _ptr(cx), _ptr(cx + 0.1), _ptr(cx), 1.0, 0, 0,
                                      C.c_void_p(out.data_ptr()))
    assert st == W._lib.WDG_ERR_ARG and b"1024" in L.wdg_last_error()
    host = np.zeros(sys.ndof)
    st = L.wdg_load_gaussians_noalloc(sys._h, 1, _ptr(cx), _ptr(cx), _ptr(cx + 0.1), _ptr(cx), 1.0, 0, 0,
                                      _ptr(host))
    assert st == W._lib.WDG_ERR_ARG and b"device memory" in L.wdg_last_error()
