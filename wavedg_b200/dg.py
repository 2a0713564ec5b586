"""Python mirror of the reference's `dg::` interface over the C ABI.

Class and method names, argument meaning and accumulate-into-output semantics
follow waveDG (arotem3/waveDG):

    Mesh2D.uniform_rect / from_vertices / from_file   source/Mesh2D.cpp:5-163
    QuadratureRule.quadrature_rule                    wavedg/QuadratureRule.hpp:77
    WaveEquation(mesh, basis, approx_quad).action     source/WaveEquation.cpp:5-68
    WaveBC(mesh, bc, basis, approx_quad).action       source/WaveEquation.cpp:70-215
    MassMatrix(mesh, basis).action / .inv             source/MassMatrix.cpp:6-82
    Div, make_face_prolongator, EdgeFlux              source/Div.cpp, FaceProlongator.cpp, EdgeFlux.cpp
    LinearFunctional2D(mesh, basis).action            wavedg/LinearFunctional.hpp:61-202
    RungeKutta4(n).step(dt, f, t, u)                  wavedg/ode.hpp:46-94
    WaveHoltz(omega, mesh, basis, bc, approx_quad)    source/WaveHoltz.cpp
    norm / error                                      source/linalg.cpp:102-131

Arrays are numpy float64 (host memory; results are back when the call
returns) or CUDA float64 torch tensors (device memory; asynchronous on the
handle's stream).  Errors raise WdgError, as the reference's wdg_error throws.
Gauss-Lobatto bases.  approx_quad=True is the fused hot path; approx_quad=False (exact
quadrature with the reference's default rules, FP64) goes through ExactDiscretisation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import WDG_FP32, WDG_FP64, WdgError, check, lib



def _destroy(name: str, h) -> None:
    """Release a handle from a finaliser.  At interpreter exit the loader's module state may
    already be torn down; the process is ending and its device memory goes with it."""
    try:
        getattr(lib(), name)(h)
    except Exception:
        pass

class FaceType:
    INTERIOR = 0
    BOUNDARY = 1


def _precision(p) -> int:
    if p in (WDG_FP64, "fp64", "float64", np.float64):
        return WDG_FP64
    if p in (WDG_FP32, "fp32", "float32", np.float32):
        return WDG_FP32
    raise ValueError(f"precision must be 'fp64' or 'fp32', not {p!r}")


def _ptr(a, writable: bool = False, name: str = "array"):
    """(c_void_p, keepalive) for a float64 numpy array or CUDA torch tensor."""
    if a is None:
        return None, None
    mod = type(a).__module__
    if mod.startswith("torch"):
        if a.dtype.__repr__() != "torch.float64":
            raise TypeError(f"{name}: torch tensors must be float64")
        if not a.is_contiguous():
            raise ValueError(f"{name}: tensor must be contiguous")
        return C.c_void_p(a.data_ptr()), a
    if not isinstance(a, np.ndarray):
        raise TypeError(f"{name}: expected a numpy array or a CUDA torch tensor")
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        if writable:
            raise TypeError(f"{name}: output arrays must be C-contiguous float64")
        a = np.ascontiguousarray(a, dtype=np.float64)
    if writable and not a.flags.writeable:
        raise ValueError(f"{name}: array is read-only")
    return C.c_void_p(a.ctypes.data), a


def _size(a) -> int:
    return int(a.numel()) if type(a).__module__.startswith("torch") else int(np.asarray(a).size)


# ------------------------------------------------------------------ quadrature
class QuadratureRule:
    """Quadrature rule on [-1, 1]; the GPU operators take Gauss-Lobatto rules."""

    GaussLegendre = 0
    GaussLobatto = 1
    _cache: dict = {}

    def __init__(self, n: int, type_: int):
        self.n, self.type = int(n), type_
        if type_ == self.GaussLobatto:
            x, w = np.zeros(n), np.zeros(n)
            check(lib().wdg_gauss_lobatto(n, C.c_void_p(x.ctypes.data), C.c_void_p(w.ctypes.data), None),
                  "gauss_lobatto")
        else:
            x, w = np.polynomial.legendre.leggauss(n)
        self.x, self.w = x, w

    @classmethod
    def quadrature_rule(cls, n: int, rule: int = GaussLegendre) -> "QuadratureRule":
        key = (int(n), rule)
        if key not in cls._cache:
            cls._cache[key] = cls(n, rule)
        return cls._cache[key]

    def derivative_matrix(self) -> np.ndarray:
        """D[l, j] = phi_j'(x_l) (lagrange_basis_deriv at the nodes)."""
        if self.type != self.GaussLobatto:
            raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "derivative matrix only for Gauss-Lobatto rules")
        x, w, D = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n * self.n)
        check(lib().wdg_gauss_lobatto(self.n, C.c_void_p(x.ctypes.data), C.c_void_p(w.ctypes.data),
                                      C.c_void_p(D.ctypes.data)))
        return D.reshape(self.n, self.n, order="F")


def _gll_n(basis) -> int:
    if isinstance(basis, QuadratureRule):
        if basis.type != QuadratureRule.GaussLobatto:
            raise WdgError(_lib.WDG_ERR_UNSUPPORTED,
                           "the GPU operators are built for Gauss-Lobatto bases (LobattoFaceProlongator path)")
        return basis.n
    return int(basis)


# ------------------------------------------------------------------------ mesh
class Mesh2D:
    """Quad mesh; same element and edge numbering as dg::Mesh2D."""

    def __init__(self, handle, verts=None, quads=None):
        self._h = handle
        self.verts, self.quads = verts, quads

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_mesh_destroy", h)
            self._h = None

    @staticmethod
    def from_vertices(x, elems) -> "Mesh2D":
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 2)
        q = np.ascontiguousarray(elems, dtype=np.int32).reshape(-1, 4)
        h = C.c_void_p()
        check(lib().wdg_mesh_from_vertices(len(x), C.c_void_p(x.ctypes.data), len(q), C.c_void_p(q.ctypes.data),
                                           C.byref(h)), "Mesh2D.from_vertices")
        return Mesh2D(h, x, q)

    @staticmethod
    def uniform_rect(nx: int, ax: float, bx: float, ny: int, ay: float, by: float) -> "Mesh2D":
        from .meshgen import uniform_rect

        v, q = uniform_rect(nx, ax, bx, ny, ay, by)
        return Mesh2D.from_vertices(v, q)

    @staticmethod
    def from_file(directory: str) -> "Mesh2D":
        """Mesh2D::from_file (wdg_mesh_from_file): directory/info.txt (n_pts n_elem),
        coordinates.txt (x y per point), elements.txt (four 0-based point indices per element)."""
        h = C.c_void_p()
        check(lib().wdg_mesh_from_file(os.fsencode(directory), C.byref(h)), "Mesh2D.from_file")
        return Mesh2D(h)

    def to_file(self, directory: str) -> None:
        """Write a mesh built from vertices in the from_file format (the inverse of from_file)."""
        if self.verts is None:
            raise WdgError(_lib.WDG_ERR_ARG, "Mesh2D.to_file: only meshes built from vertices keep their points")
        os.makedirs(directory, exist_ok=True)
        with open(os.path.join(directory, "info.txt"), "w") as f:
            f.write(f"{len(self.verts)} {len(self.quads)}\n")
        np.savetxt(os.path.join(directory, "coordinates.txt"), self.verts, fmt="%.18e")
        np.savetxt(os.path.join(directory, "elements.txt"), self.quads, fmt="%d")

    @staticmethod
    def from_tables(corners, interior_edges, boundary_edges) -> "Mesh2D":
        c = np.ascontiguousarray(corners, dtype=np.float64).reshape(-1, 8)
        ie = np.ascontiguousarray(interior_edges, dtype=np.int32).reshape(-1, 5)
        be = np.ascontiguousarray(boundary_edges, dtype=np.int32).reshape(-1, 5)
        h = C.c_void_p()
        check(lib().wdg_mesh_from_tables(len(c), C.c_void_p(c.ctypes.data), len(ie), C.c_void_p(ie.ctypes.data),
                                         len(be), C.c_void_p(be.ctypes.data), C.byref(h)), "Mesh2D.from_tables")
        return Mesh2D(h)

    def n_elem(self) -> int:
        return check(lib().wdg_mesh_n_elem(self._h))

    def n_edges(self, face_type: int) -> int:
        return check(lib().wdg_mesh_n_edges(self._h, face_type))

    def edges(self, face_type: int) -> np.ndarray:
        out = np.zeros((self.n_edges(face_type), 5), dtype=np.int32)
        check(lib().wdg_mesh_edges(self._h, face_type, C.c_void_p(out.ctypes.data)))
        return out

    def min_h(self) -> float:
        h = C.c_double()
        check(lib().wdg_mesh_min_h(self._h, C.byref(h)))
        return h.value

    def boundary_midpoints(self) -> np.ndarray:
        out = np.zeros((self.n_edges(FaceType.BOUNDARY), 2))
        check(lib().wdg_mesh_boundary_midpoints(self._h, C.c_void_p(out.ctypes.data)))
        return out


# ---------------------------------------------------------- discretisation
class Discretisation:
    """One wdg_wave handle: geometry of `mesh` on the GPU for n GLL nodes."""

    def __init__(self, mesh: Mesh2D, n: int, bc=None, precision="fp64", device: int = -1):
        self.mesh, self.n = mesh, int(n)
        self.precision = _precision(precision)
        codes = None
        if bc is not None:
            codes = np.ascontiguousarray(bc, dtype=np.int32)
            if codes.size != mesh.n_edges(FaceType.BOUNDARY):
                raise WdgError(_lib.WDG_ERR_ARG, "bc needs one code per boundary edge")
        self._codes = codes
        h = C.c_void_p()
        check(lib().wdg_wave_create(mesh._h, self.n, None if codes is None else C.c_void_p(codes.ctypes.data),
                                    self.precision, device, C.byref(h)), "wdg_wave_create")
        self._h = h
        nd = C.c_longlong()
        check(lib().wdg_wave_info(h, None, None, C.byref(nd), None))
        self.ndof = nd.value
        self.n_elem = mesh.n_elem()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_wave_destroy", h)
            self._h = None

    def set_stream(self, stream) -> None:
        """A torch.cuda.Stream, a raw cudaStream_t int, or None (legacy default stream)."""
        raw = getattr(stream, "cuda_stream", stream)
        check(lib().wdg_wave_set_stream(self._h, C.c_void_p(raw or 0)))

    def sync(self) -> None:
        check(lib().wdg_wave_sync(self._h))

    @property
    def tile(self) -> int:
        t = C.c_int()
        check(lib().wdg_wave_get_tile(self._h, C.byref(t)))
        return t.value

    @tile.setter
    def tile(self, v: int) -> None:
        check(lib().wdg_wave_set_tile(self._h, int(v)), "set_tile")

    def set_stages(self, stages: int) -> None:
        """Depth of the bulk-copy pipeline: 2-4 for the tiled kernel, 2-6 chunk slots for
        the warp-specialised one; 0 = default."""
        check(lib().wdg_wave_set_stages(self._h, int(stages)), "set_stages")

    def set_kernel(self, family: int) -> None:
        """0: warp per element, 1: tiled TMA pipeline, 2: warp-specialised TMA ring,
        -1: default for this degree."""
        check(lib().wdg_wave_set_kernel(self._h, int(family)), "set_kernel")

    def launch_config(self) -> dict:
        f, t, st, mc = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().wdg_wave_get_launch(self._h, C.byref(f), C.byref(t), C.byref(st), C.byref(mc)))
        return {"kernel": ("warp", "tiled", "ws")[f.value], "tile": t.value, "stages": st.value, "max_ctas": mc.value}

    def autotune(self, steps: int = 5) -> float:
        """Pick elements-per-block and pipeline depth by timing; returns the best ms per RK4 step."""
        ms = C.c_float()
        check(lib().wdg_wave_autotune(self._h, int(steps), C.byref(ms)), "autotune")
        return ms.value

    def set_max_ctas(self, n: int) -> None:
        """Cap the persistent CTAs of the fused kernels (0 = one full wave)."""
        check(lib().wdg_wave_set_max_ctas(self._h, int(n)), "set_max_ctas")

    def zeros(self) -> np.ndarray:
        return np.zeros(self.ndof)

    def node_coordinates(self) -> np.ndarray:
        """element_metrics(basis).physical_coordinates(): (2, n, n, n_elem) flattened."""
        xy = np.zeros(2 * self.ndof // 3)
        check(lib().wdg_wave_node_coords(self._h, C.c_void_p(xy.ctypes.data)))
        return xy

    def quad_points(self) -> np.ndarray:
        xy = np.zeros(2 * self.ndof // 3)
        check(lib().wdg_quad_points(self._h, C.c_void_p(xy.ctypes.data)))
        return xy

    def _call(self, fn, *arrays, what=""):
        check(fn(self._h, *arrays), what)

    # fused hot path ---------------------------------------------------------
    def rhs(self, u, dudt, F=None, s: float = 0.0) -> None:
        """dudt <- M^{-1}(A u + B u + s F), one fused kernel."""
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(dudt, True, "dudt")
        pF, _kF = _ptr(F, name="F")
        check(lib().wdg_rhs(self._h, pu, pd, pF, float(s)), "rhs")

    def rk4_steps(self, u, dt: float, t: float, nsteps: int) -> float:
        """nsteps of low-storage RK4 in place; returns the new time."""
        pu, _k = _ptr(u, True, "u")
        tt = C.c_double(t)
        check(lib().wdg_rk4_steps(self._h, pu, float(dt), C.byref(tt), int(nsteps)), "rk4_steps")
        return tt.value

    # resident state -----------------------------------------------------------
    def upload(self, u) -> None:
        p, _k = _ptr(u, name="u")
        check(lib().wdg_state_upload(self._h, p), "state_upload")

    def download(self, u=None):
        if u is None:
            u = np.zeros(self.ndof)
        p, _k = _ptr(u, True, "u")
        check(lib().wdg_state_download(self._h, p), "state_download")
        return u

    def state_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().wdg_state_device_ptr(self._h, C.byref(p)))
        return p.value

    def step_state(self, dt: float, t: float, nsteps: int) -> float:
        tt = C.c_double(t)
        check(lib().wdg_state_rk4_steps(self._h, float(dt), C.byref(tt), int(nsteps)), "state_rk4_steps")
        return tt.value

    def energy(self) -> float:
        e = C.c_double()
        check(lib().wdg_state_energy(self._h, C.byref(e)), "state_energy")
        return e.value

    def load_gaussians(self, centers, sigmas, amps, scale=1.0, comp=0, mass_inv=False, out=None):
        c = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 2)
        cx, cy = np.ascontiguousarray(c[:, 0]), np.ascontiguousarray(c[:, 1])
        sg = np.ascontiguousarray(np.broadcast_to(np.asarray(sigmas, dtype=np.float64), (len(c),)))
        am = np.ascontiguousarray(np.broadcast_to(np.asarray(amps, dtype=np.float64), (len(c),)))
        F = np.zeros(self.ndof) if out is None else out
        pF, _k = _ptr(F, True, "F")
        check(lib().wdg_load_gaussians(self._h, len(c), C.c_void_p(cx.ctypes.data), C.c_void_p(cy.ctypes.data),
                                       C.c_void_p(sg.ctypes.data), C.c_void_p(am.ctypes.data), float(scale),
                                       int(comp), 1 if mass_inv else 0, pF), "load_gaussians")
        return F

    def norm(self, x) -> float:
        r = C.c_double()
        px, _k = _ptr(x, name="x")
        check(lib().wdg_norm(self._h, px, C.byref(r)))
        return r.value

    def error(self, x, y) -> float:
        r = C.c_double()
        px, _kx = _ptr(x, name="x")
        py, _ky = _ptr(y, name="y")
        check(lib().wdg_error(self._h, px, py, C.byref(r)))
        return r.value


def _require_approx(approx_quad: bool) -> None:
    if not approx_quad:
        raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "this operator is built for approx_quad=True only")


class ExactDiscretisation:
    """One wdg_waveq handle: the wave system with approx_quad = false (Div<false>,
    EdgeFlux<false>, MassMatrix<false>; the reference's default Gauss-Legendre rules), FP64."""

    def __init__(self, mesh: Mesh2D, n: int, bc=None, device: int = -1, quad=None):
        if quad is not None:
            raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "exact quadrature is built for the default rules (quad=None)")
        self.mesh, self.n = mesh, int(n)
        codes = None
        if bc is not None:
            codes = np.ascontiguousarray(bc, dtype=np.int32)
            if codes.size != mesh.n_edges(FaceType.BOUNDARY):
                raise WdgError(_lib.WDG_ERR_ARG, "bc needs one code per boundary edge")
        self._codes = codes
        h = C.c_void_p()
        check(lib().wdg_waveq_create(mesh._h, self.n, None if codes is None else C.c_void_p(codes.ctypes.data),
                                     device, C.byref(h)), "wdg_waveq_create")
        self._h = h
        self.ndof = 3 * self.n * self.n * mesh.n_elem()
        self.n_elem = mesh.n_elem()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_waveq_destroy", h)
            self._h = None

    def rules(self) -> tuple:
        """(Div, EdgeFlux, MassMatrix) points per direction."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().wdg_waveq_rules(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def _acc(self, fn, u, du, what):
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(du, True, "du")
        check(getattr(lib(), fn)(self._h, pu, pd), what)

    def div_action(self, u, du) -> None:
        self._acc("wdg_waveq_div_action", u, du, "Div<false>.action")

    def wave_action(self, u, du) -> None:
        self._acc("wdg_waveq_wave_action", u, du, "WaveEquation.action")

    def wavebc_action(self, u, du) -> None:
        self._acc("wdg_waveq_wavebc_action", u, du, "WaveBC.action")

    def edge_flux(self, face_type: int, ub, fb) -> None:
        pu, _ku = _ptr(ub, name="ub")
        pf, _kf = _ptr(fb, True, "fb")
        check(lib().wdg_waveq_edge_flux(self._h, int(face_type), pu, pf), "EdgeFlux<false>.action")

    def mass_action(self, n_var: int, x, y) -> None:
        px, _kx = _ptr(x, name="x")
        py, _ky = _ptr(y, True, "y")
        check(lib().wdg_waveq_mass_action(self._h, int(n_var), px, py), "MassMatrix<false>.action")

    def mass_inv(self, n_var: int, x) -> None:
        px, _kx = _ptr(x, True, "x")
        check(lib().wdg_waveq_mass_inv(self._h, int(n_var), px), "MassMatrix<false>.inv")

    def rhs(self, u, dudt, F=None, s: float = 0.0) -> None:
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(dudt, True, "dudt")
        pf, _kf = _ptr(F, name="F")
        check(lib().wdg_waveq_rhs(self._h, pu, pd, pf, float(s)), "rhs")

    def rk4_steps(self, u, dt: float, t: float, nsteps: int) -> float:
        pu, _ku = _ptr(u, True, "u")
        tt = C.c_double(t)
        check(lib().wdg_waveq_rk4_steps(self._h, pu, float(dt), C.byref(tt), int(nsteps)), "rk4_steps")
        return tt.value


class Operator:
    """dg::Operator: action(x, y) accumulates y += A x, like the reference's operators."""

    def action(self, *args):  # pragma: no cover - interface
        raise NotImplementedError


class WaveEquation(Operator):
    """du += Div(u) + P^T Flux(P u) over interior edges (source/WaveEquation.cpp:54-68)."""

    def __init__(self, mesh: Mesh2D, basis, approx_quad: bool = False, quad=None, precision="fp64"):
        self.exact = not approx_quad
        if self.exact:
            if precision != "fp64":
                raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "exact quadrature is built in FP64")
            self.disc = ExactDiscretisation(mesh, _gll_n(basis), None, quad=quad)
        else:
            self.disc = Discretisation(mesh, _gll_n(basis), None, precision)

    def action(self, *args) -> None:
        u, du = args[-2], args[-1]  # action(u, du) or action(n_var, u, du); n_var is ignored
        if self.exact:
            return self.disc.wave_action(u, du)
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(du, True, "du")
        check(lib().wdg_wave_action(self.disc._h, pu, pd), "WaveEquation.action")


class WaveBC(Operator):
    """du += boundary flux with exterior states from bc (source/WaveEquation.cpp:190-215)."""

    def __init__(self, mesh: Mesh2D, bc, basis, approx_quad: bool = False, quad=None):
        self.exact = not approx_quad
        self.disc = (ExactDiscretisation(mesh, _gll_n(basis), bc, quad=quad) if self.exact
                     else Discretisation(mesh, _gll_n(basis), bc))

    def action(self, *args) -> None:
        u, du = args[-2], args[-1]
        if self.exact:
            return self.disc.wavebc_action(u, du)
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(du, True, "du")
        check(lib().wdg_wavebc_action(self.disc._h, pu, pd), "WaveBC.action")

    def apply_bc(self, uB) -> None:
        """apply_bc_2d on boundary traces (n, 3, 2, n_boundary): side 1 <- exterior state."""
        p, _k = _ptr(uB, True, "uB")
        h = self.disc._h
        if self.exact:
            w = C.c_void_p()
            check(lib().wdg_waveq_wave(h, C.byref(w)))
            h = w
        check(lib().wdg_apply_bc(h, p), "apply_bc")


class Div(Operator):
    """Div<true> of the wave system: du += (F(u), grad phi) (source/Div.cpp:131-196)."""

    def __init__(self, mesh: Mesh2D, basis, approx_quad: bool = True):
        self.exact = not approx_quad
        self.disc = ExactDiscretisation(mesh, _gll_n(basis)) if self.exact else Discretisation(mesh, _gll_n(basis))

    def action(self, *args) -> None:
        u, du = args[-2], args[-1]
        if self.exact:
            return self.disc.div_action(u, du)
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(du, True, "du")
        check(lib().wdg_div_action(self.disc._h, pu, pd), "Div.action")


class FaceProlongator:
    """LobattoFaceProlongator for n_var = 3 (source/FaceProlongator.cpp:497-714)."""

    def __init__(self, mesh: Mesh2D, basis, face_type: int, bc=None):
        self.disc = Discretisation(mesh, _gll_n(basis), bc)
        self.face_type = face_type
        self.n_faces = mesh.n_edges(face_type)

    def size(self) -> int:
        return self.disc.n * 3 * 2 * self.n_faces

    def action(self, n_var: int, u, uf) -> None:
        if n_var != 3:
            raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "the GPU prolongator is built for the wave system (n_var = 3)")
        pu, _ku = _ptr(u, name="u")
        pf, _kf = _ptr(uf, True, "uf")
        check(lib().wdg_face_prolong(self.disc._h, self.face_type, pu, pf), "FaceProlongator.action")

    def t(self, n_var: int, uf, u) -> None:
        if n_var != 3:
            raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "the GPU prolongator is built for the wave system (n_var = 3)")
        pf, _kf = _ptr(uf, name="uf")
        pu, _ku = _ptr(u, True, "u")
        check(lib().wdg_face_prolong_t(self.disc._h, self.face_type, pf, pu), "FaceProlongator.t")


def make_face_prolongator(mesh: Mesh2D, basis, face_type: int) -> FaceProlongator:
    return FaceProlongator(mesh, basis, face_type)


class EdgeFlux(Operator):
    """EdgeFlux<true> of the wave system with the upwind defaults a = -1, b = -1/2."""

    def __init__(self, mesh: Mesh2D, face_type: int, basis, approx_quad: bool = True):
        self.exact = not approx_quad
        self.disc = ExactDiscretisation(mesh, _gll_n(basis)) if self.exact else Discretisation(mesh, _gll_n(basis))
        self.face_type = face_type

    def action(self, *args) -> None:
        ub, fb = args[-2], args[-1]
        if self.exact:
            return self.disc.edge_flux(self.face_type, ub, fb)
        pu, _ku = _ptr(ub, name="ub")
        pf, _kf = _ptr(fb, True, "fb")
        check(lib().wdg_edge_flux(self.disc._h, self.face_type, pu, pf), "EdgeFlux.action")


class BasisMassMatrix:
    """MassMatrix<AQ> and LinearFunctional2D on a basis of either type (wdg_massmatrix_*): the
    set-up operators for Gauss-Legendre bases (examples/advec2d.cpp)."""

    def __init__(self, mesh: Mesh2D, basis, approx_quad: bool = True, device: int = -1):
        n, bt = (basis.n, basis.type) if isinstance(basis, QuadratureRule) else (int(basis), QuadratureRule.GaussLobatto)
        self.mesh, self.n = mesh, n
        h = C.c_void_p()
        check(lib().wdg_massmatrix_create(mesh._h, n, int(bt), int(bool(approx_quad)), device, C.byref(h)),
              "wdg_massmatrix_create")
        self._h = h
        self.npts = n * n * mesh.n_elem()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_massmatrix_destroy", h)
            self._h = None

    def action(self, n_var, x, y) -> None:
        px, _kx = _ptr(x, name="x")
        py, _ky = _ptr(y, True, "y")
        check(lib().wdg_massmatrix_action(self._h, int(n_var), px, py), "MassMatrix.action")

    def inv(self, n_var, x) -> None:
        px, _kx = _ptr(x, True, "x")
        check(lib().wdg_massmatrix_inv(self._h, int(n_var), px), "MassMatrix.inv")

    def points(self) -> np.ndarray:
        """(npts, 2): where LinearFunctional2D samples f (its default n-point rule)."""
        xy = np.zeros(2 * self.npts)
        check(lib().wdg_massmatrix_points(self._h, C.c_void_p(xy.ctypes.data)), "points")
        return xy.reshape(-1, 2)

    def load(self, n_var, fq, F) -> None:
        fq = np.ascontiguousarray(fq, dtype=np.float64).reshape(-1)
        if fq.size != int(n_var) * self.npts:
            raise WdgError(_lib.WDG_ERR_ARG, "fq must hold n_var values per point")
        pF, _kF = _ptr(F, True, "F")
        check(lib().wdg_massmatrix_load(self._h, int(n_var), C.c_void_p(fq.ctypes.data), pF),
              "LinearFunctional2D.action")


def _legendre(basis) -> bool:
    return isinstance(basis, QuadratureRule) and basis.type == QuadratureRule.GaussLegendre


class MassMatrix:
    """MassMatrix<true>: diagonal w_i w_j detJ (source/MassMatrix.cpp:6-82); with
    approx_quad=False MassMatrix<false>: block Cholesky of the exact element mass matrices.
    Gauss-Legendre bases through BasisMassMatrix."""

    def __init__(self, mesh: Mesh2D, basis, quad=None, approx_quad: bool = True):
        self.exact = not approx_quad
        self.basis_mm = None
        if _legendre(basis):
            if quad is not None:
                raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "only the default rules are built for Gauss-Legendre bases")
            self.basis_mm = BasisMassMatrix(mesh, basis, approx_quad)
            return
        self.disc = (ExactDiscretisation(mesh, _gll_n(basis), quad=quad) if self.exact
                     else Discretisation(mesh, _gll_n(basis)))

    def action(self, *args) -> None:
        n_var, x, y = (args if len(args) == 3 else (1, *args))
        if self.basis_mm is not None:
            return self.basis_mm.action(n_var, x, y)
        if self.exact:
            return self.disc.mass_action(n_var, x, y)
        px, _kx = _ptr(x, name="x")
        py, _ky = _ptr(y, True, "y")
        check(lib().wdg_mass_action(self.disc._h, int(n_var), px, py), "MassMatrix.action")

    def inv(self, *args) -> None:
        n_var, x = (args if len(args) == 2 else (1, *args))
        if self.basis_mm is not None:
            return self.basis_mm.inv(n_var, x)
        if self.exact:
            return self.disc.mass_inv(n_var, x)
        px, _kx = _ptr(x, True, "x")
        check(lib().wdg_mass_inv(self.disc._h, int(n_var), px), "MassMatrix.inv")


class WaveSystem(Discretisation):
    """The examples' time derivative M^{-1}(A + B) u (+ s F) as one fused GPU operator."""

    def __init__(self, mesh: Mesh2D, basis, bc=None, precision="fp64", device: int = -1):
        super().__init__(mesh, _gll_n(basis), bc, precision, device)

    def __call__(self, dudt, t, u) -> None:  # f(F, t, u) as ode::RungeKutta4 calls it
        self.rhs(u, dudt)


class LinearFunctional2D:
    """(f, phi) with the n-point Gauss-Legendre rule (wavedg/LinearFunctional.hpp:136-202), on a
    Gauss-Lobatto or Gauss-Legendre basis."""

    def __init__(self, mesh: Mesh2D, basis, quad=None):
        self.basis_mm = None
        n = basis.n if isinstance(basis, QuadratureRule) else int(basis)
        if quad is not None and quad.n != n:
            raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "only the default n-point quadrature is built")
        if _legendre(basis):
            self.basis_mm = BasisMassMatrix(mesh, basis, True)
            return
        self.disc = Discretisation(mesh, _gll_n(basis))

    def action(self, n_var: int, f, F) -> None:
        """f(x, y) -> array (n_var, npts) (vectorised over quadrature points)."""
        if self.basis_mm is not None:
            xy = self.basis_mm.points()
            vals = np.asarray(f(xy[:, 0], xy[:, 1]), dtype=np.float64).reshape(n_var, -1)
            return self.basis_mm.load(n_var, np.ascontiguousarray(vals.T), F)
        xy = self.disc.quad_points().reshape(-1, 2)
        vals = np.asarray(f(xy[:, 0], xy[:, 1]), dtype=np.float64).reshape(n_var, -1)
        fq = np.ascontiguousarray(vals.T)
        pF, _k = _ptr(F, True, "F")
        check(lib().wdg_linear_functional(self.disc._h, int(n_var), C.c_void_p(fq.ctypes.data), pF),
              "LinearFunctional2D.action")


class RungeKutta4:
    """ode::RungeKutta4 (wavedg/ode.hpp:46-94).  f must be a WaveSystem: the whole step
    (five fused stages) runs on the GPU."""

    def __init__(self, n: int):
        self.n = int(n)

    def step(self, dt: float, f: WaveSystem, t: float, u) -> float:
        if not isinstance(f, WaveSystem):
            raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "RungeKutta4.step needs a WaveSystem (fused GPU RHS)")
        if _size(u) != self.n or f.ndof != self.n:
            raise WdgError(_lib.WDG_ERR_ARG, "state length does not match RungeKutta4(n)")
        return f.rk4_steps(u, dt, t, 1)


class WaveHoltz:
    """dg::WaveHoltz on the GPU (source/WaveHoltz.cpp)."""

    def __init__(self, omega: float, mesh: Mesh2D, basis, bc, approx_quad: bool = False, precision="fp64",
                 device: int = -1, system: WaveSystem | None = None):
        self.omega = float(omega)
        h = C.c_void_p()
        if not approx_quad:
            # exact quadrature (Div<false>, EdgeFlux<false>, MassMatrix<false>), FP64
            if precision != "fp64" or system is not None:
                raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "exact-quadrature WaveHoltz is FP64 on its own operators")
            self.system = ExactDiscretisation(mesh, _gll_n(basis), bc, device)
            check(lib().wdg_waveholtz_create_exact(self.system._h, self.omega, C.byref(h)), "WaveHoltz")
        else:
            self.system = system if system is not None else WaveSystem(mesh, basis, bc, precision, device)
            check(lib().wdg_waveholtz_create(self.system._h, self.omega, C.byref(h)), "WaveHoltz")
        self._h = h
        T, dt, nt = C.c_double(), C.c_double(), C.c_int()
        check(lib().wdg_waveholtz_params(h, C.byref(T), C.byref(dt), C.byref(nt)))
        self.T, self.dt, self.nt = T.value, dt.value, nt.value
        self.ndof = self.system.ndof

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_waveholtz_destroy", h)
            self._h = None

    def K(self, t: float) -> float:
        return self.omega / np.pi * (np.cos(self.omega * t) - 0.25)

    def pi0(self, w, F) -> None:
        pw, _kw = _ptr(w, True, "w")
        pF, _kF = _ptr(F, name="F")
        check(lib().wdg_waveholtz_pi0(self._h, pw, pF), "WaveHoltz.pi0")

    def S(self, w) -> None:
        pw, _k = _ptr(w, True, "w")
        check(lib().wdg_waveholtz_S(self._h, pw), "WaveHoltz.S")

    def postprocess(self, H, w) -> None:
        pH, _kH = _ptr(H, True, "H")
        pw, _kw = _ptr(w, name="w")
        check(lib().wdg_waveholtz_postprocess(self._h, pH, pw), "WaveHoltz.postprocess")

    def solve(self, F, tol: float = 1e-6, maxit: int = 1000, W=None, raise_on_stall: bool = False):
        """pi0, then W <- S W + pi0 until ||W - W_prev|| / ||pi0|| < tol.  Returns (W, iters, residual)."""
        if W is None:
            W = np.zeros(self.ndof)
        pW, _kW = _ptr(W, True, "W")
        pF, _kF = _ptr(F, name="F")
        it, res = C.c_int(), C.c_double()
        st = lib().wdg_waveholtz_solve(self._h, pF, float(tol), int(maxit), pW, C.byref(it), C.byref(res))
        if st != _lib.WDG_ERR_NOT_CONVERGED or raise_on_stall:
            check(st, "WaveHoltz.solve")
        return W, it.value, res.value


class WaveHoltzBatch:
    """Many independent WaveHoltz solves advanced together (wdg_whbatch_*): each solve has its
    own WaveSystem (mesh, degree; all of one precision and device) and its own omega.  One
    persistent kernel launch per RK stage covers every running solve."""

    STATUS = {0: "converged", 1: "iteration limit", 2: "stalled", -1: "running"}

    def __init__(self, systems, omegas):
        self.systems = list(systems)
        n = len(self.systems)
        om = np.ascontiguousarray(np.broadcast_to(np.asarray(omegas, dtype=np.float64), (n,)))
        hs = (C.c_void_p * n)(*[s._h for s in self.systems])
        h = C.c_void_p()
        check(lib().wdg_whbatch_create(n, hs, C.c_void_p(om.ctypes.data), C.byref(h)), "WaveHoltzBatch")
        self._h = h
        self.omegas = om
        self.n = n
        self.pi0_norm = None  # |pi0| per solve, after a solve

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_whbatch_destroy", h)
            self._h = None

    def params(self, solve: int):
        T, dt, nt = C.c_double(), C.c_double(), C.c_int()
        check(lib().wdg_whbatch_params(self._h, int(solve), C.byref(T), C.byref(dt), C.byref(nt)))
        return T.value, dt.value, nt.value

    def set_launch(self, rounds: int, ring: int) -> None:
        check(lib().wdg_whbatch_set_launch(self._h, int(rounds), int(ring)), "WaveHoltzBatch.set_launch")

    def launch_config(self) -> dict:
        r, g, grid = C.c_int(), C.c_int(), C.c_int()
        check(lib().wdg_whbatch_get_launch(self._h, C.byref(r), C.byref(g), C.byref(grid)))
        return {"rounds": r.value, "ring": g.value, "grid": grid.value}

    def autotune(self, steps: int = 64) -> float:
        ms = C.c_float()
        check(lib().wdg_whbatch_autotune(self._h, int(steps), C.byref(ms)), "WaveHoltzBatch.autotune")
        return ms.value

    def solve(self, F, tol: float = 1e-6, maxit: int = 1000, W=None, warm=None, stall_limit: int = 0,
              pi0_norm=None):
        """Solve every problem.  F, W: one float64 array per solve (numpy or CUDA tensors);
        W (optional) holds initial guesses where warm[s] is true and receives the iterates.
        pi0_norm (optional): per solve a known |pi0| (> 0) that lets a warm-started solve skip
        the period that measures it.  After the call `self.pi0_norm` holds the |pi0| each solve
        used.  Returns (W, iters, residuals, status)."""
        n = self.n
        if len(F) != n:
            raise ValueError("one forcing per solve")
        if W is None:
            W = [np.zeros(s.ndof) for s in self.systems]
        keep = []
        fp, wp = (C.c_void_p * n)(), (C.c_void_p * n)()
        for s in range(n):
            pf, kf = _ptr(F[s], name="F")
            pw, kw = _ptr(W[s], True, "W")
            keep += [kf, kw]
            fp[s], wp[s] = pf, pw
        wm = None
        if warm is not None:
            wm = np.ascontiguousarray(np.broadcast_to(np.asarray(warm, dtype=np.int32), (n,)))
        it = np.zeros(n, dtype=np.int32)
        res = np.zeros(n)
        stt = np.zeros(n, dtype=np.int32)
        p0 = np.zeros(n) if pi0_norm is None else np.array(np.broadcast_to(np.asarray(pi0_norm, dtype=np.float64), (n,)))
        check(lib().wdg_whbatch_solve(self._h, fp, float(tol), int(maxit), int(stall_limit), wp,
                                      None if wm is None else C.c_void_p(wm.ctypes.data),
                                      C.c_void_p(p0.ctypes.data),
                                      C.c_void_p(it.ctypes.data), C.c_void_p(res.ctypes.data),
                                      C.c_void_p(stt.ctypes.data)), "WaveHoltzBatch.solve")
        self.pi0_norm = p0
        return W, it, res, stt


class AdvectionSystem:
    """Linear advection with constant coefficients (wdg_advect_*): Advection<true>,
    AdvectionHomogeneousBC<true> and MassMatrix<true> for n_var variables; a = (A_0, A_1) as
    a(d, c, k) = a[d + n_var (c + n_var k)] (the reference's (n_var, n_var, 2) layout), both
    symmetric.  FP64."""

    def __init__(self, n_var: int, mesh: Mesh2D, basis, a, device: int = -1):
        self.n_var, self.mesh, self.n = int(n_var), mesh, _gll_n(basis)
        av = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if av.size != 2 * self.n_var ** 2:
            raise WdgError(_lib.WDG_ERR_ARG, "a must hold 2 n_var^2 coefficients")
        self._a = av
        h = C.c_void_p()
        check(lib().wdg_advect_create(mesh._h, self.n, self.n_var, C.c_void_p(av.ctypes.data), device, C.byref(h)),
              "wdg_advect_create")
        self._h = h
        self.ndof = self.n_var * self.n * self.n * mesh.n_elem()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_advect_destroy", h)
            self._h = None

    def _call(self, fn, u, du, what):
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(du, True, "du")
        check(getattr(lib(), fn)(self._h, pu, pd), what)

    def action(self, u, du) -> None:
        self._call("wdg_advect_action", u, du, "Advection.action")

    def bc_action(self, u, du) -> None:
        self._call("wdg_advect_bc_action", u, du, "AdvectionHomogeneousBC.action")

    def rhs(self, u, dudt) -> None:
        self._call("wdg_advect_rhs", u, dudt, "rhs")

    def rk4_steps(self, u, dt: float, t: float, nsteps: int) -> float:
        pu, _ku = _ptr(u, True, "u")
        tt = C.c_double(t)
        check(lib().wdg_advect_rk4_steps(self._h, pu, float(dt), C.byref(tt), int(nsteps)), "rk4_steps")
        return tt.value


class VariableAdvectionSystem:
    """Linear advection with a spatially varying coefficient (wdg_vadvect_*): Advection<AQ>,
    AdvectionHomogeneousBC<AQ> (constant_coefficient = false) and MassMatrix<AQ> for n_var
    variables on a Gauss-Lobatto or Gauss-Legendre basis (a QuadratureRule; an int means
    Gauss-Lobatto); a in the reference's (n_var, n_var, 2, n, n, n_elem) layout (a host array);
    approx_quad False selects the Gauss-Legendre rules of Div<false> / EdgeFlux<false> and the
    dense mass matrix.  examples/advec2d.cpp uses a Gauss-Legendre basis with approx_quad False.
    One variable, or symmetric coefficient matrices.  FP64."""

    def __init__(self, n_var: int, mesh: Mesh2D, basis, a, approx_quad: bool = True, device: int = -1):
        if isinstance(basis, QuadratureRule):
            self.n, self.basis_type = basis.n, basis.type
        else:
            self.n, self.basis_type = int(basis), QuadratureRule.GaussLobatto
        self.n_var, self.mesh = int(n_var), mesh
        self.approx_quad = bool(approx_quad)
        av = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        if av.size != 2 * self.n_var ** 2 * self.n ** 2 * mesh.n_elem():
            raise WdgError(_lib.WDG_ERR_ARG, "a must hold 2 n_var^2 n^2 n_elem coefficients")
        h = C.c_void_p()
        check(lib().wdg_vadvect_create(mesh._h, self.n, int(self.basis_type), self.n_var, C.c_void_p(av.ctypes.data),
                                       int(self.approx_quad), device, C.byref(h)), "wdg_vadvect_create")
        self._h = h
        self.ndof = self.n_var * self.n * self.n * mesh.n_elem()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_vadvect_destroy", h)
            self._h = None

    def _call(self, fn, u, du, what):
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(du, True, "du")
        check(getattr(lib(), fn)(self._h, pu, pd), what)

    def set_stream(self, stream) -> None:
        check(lib().wdg_vadvect_set_stream(self._h, C.c_void_p(getattr(stream, "cuda_stream", stream))))

    def sync(self) -> None:
        check(lib().wdg_vadvect_sync(self._h))

    def action(self, u, du) -> None:
        self._call("wdg_vadvect_action", u, du, "Advection.action")

    def bc_action(self, u, du) -> None:
        self._call("wdg_vadvect_bc_action", u, du, "AdvectionHomogeneousBC.action")

    def rhs(self, u, dudt) -> None:
        self._call("wdg_vadvect_rhs", u, dudt, "rhs")

    def steps(self, u, dt: float, t: float, nsteps: int, method: str = "ssprk3") -> float:
        """nsteps of ode::SSPRK3 ("ssprk3", examples/advec2d.cpp's stepper) or ode::RungeKutta4
        ("rk4") on u in place; returns the new time."""
        pu, _ku = _ptr(u, True, "u")
        tt = C.c_double(t)
        check(lib().wdg_vadvect_steps(self._h, {"rk4": 0, "ssprk3": 1}[method], pu, float(dt), C.byref(tt),
                                      int(nsteps)), "steps")
        return tt.value


class EulerSystem:
    """The compressible Euler system of examples/cl2d.cpp (wdg_euler_create[_exact], wdg_claw_*):
    state u(d, i, j, el) with d = density, x-momentum, y-momentum, energy, gamma = 1.4; DivF2D
    with the example's flux, EdgeFluxF2D with its local Lax-Friedrichs flux (exterior boundary
    state = interior state) and MassMatrix on GLL nodes, with the example's approx_quad switch:
    True for the collocation rule, False (as the example ships) for the 2n-point Gauss-Legendre
    rules and the dense inverse mass matrix.  FP64."""

    n_var = 4

    def __init__(self, mesh: Mesh2D, basis, device: int = -1, approx_quad: bool = True):
        self.mesh, self.n, self.approx_quad = mesh, _gll_n(basis), bool(approx_quad)
        name = "wdg_euler_create" if self.approx_quad else "wdg_euler_create_exact"
        h = C.c_void_p()
        check(getattr(lib(), name)(mesh._h, self.n, device, C.byref(h)), name)
        self._h = h
        self.ndof = 4 * self.n * self.n * mesh.n_elem()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _destroy("wdg_claw_destroy", h)
            self._h = None

    def set_stream(self, stream) -> None:
        check(lib().wdg_claw_set_stream(self._h, C.c_void_p(getattr(stream, "cuda_stream", stream))))

    def sync(self) -> None:
        check(lib().wdg_claw_sync(self._h))

    def div(self, u, divF) -> None:
        """DivF2D::action: divF += (F(u), grad v)."""
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(divF, True, "divF")
        check(lib().wdg_claw_div(self._h, pu, pd), "DivF2D.action")

    def flux(self, face_type: int, uB, fB) -> None:
        """EdgeFluxF2D::action on nodal face traces (n, 4, 2, n_edges); fB may be uB."""
        pu, _ku = _ptr(uB, name="uB")
        pf, _kf = _ptr(fB, True, "fB")
        check(lib().wdg_claw_flux(self._h, int(face_type), pu, pf), "EdgeFluxF2D.action")

    def rhs(self, u, dudt) -> None:
        """The time derivative of examples/cl2d.cpp."""
        pu, _ku = _ptr(u, name="u")
        pd, _kd = _ptr(dudt, True, "dudt")
        check(lib().wdg_claw_rhs(self._h, pu, pd), "rhs")

    def steps(self, u, dt: float, t: float, nsteps: int, method: str = "ssprk3") -> float:
        """nsteps of ode::SSPRK3 ("ssprk3", the example's stepper) or ode::RungeKutta4 ("rk4")
        on u in place; returns the new time."""
        pu, _ku = _ptr(u, True, "u")
        tt = C.c_double(t)
        check(lib().wdg_claw_steps(self._h, {"rk4": 0, "ssprk3": 1}[method], pu, float(dt), C.byref(tt),
                                   int(nsteps)), "steps")
        return tt.value


def _advection_system(n_var, mesh, basis, a, constant_coefficient, quad, approx_quad):
    """The fused constant-coefficient path for GLL bases with approx_quad; every other case
    (a varying coefficient, exact quadrature, a Gauss-Legendre basis) through the table-driven
    path, a constant coefficient spread to the nodes."""
    if quad is not None:
        raise WdgError(_lib.WDG_ERR_UNSUPPORTED, "advection is built for the default quadrature rules")
    legendre = isinstance(basis, QuadratureRule) and basis.type == QuadratureRule.GaussLegendre
    if constant_coefficient and approx_quad and not legendre:
        return AdvectionSystem(n_var, mesh, basis, a)
    if constant_coefficient:
        n = basis.n if isinstance(basis, QuadratureRule) else int(basis)
        av = np.asarray(a, dtype=np.float64).reshape(-1)
        if av.size != 2 * int(n_var) ** 2:
            raise WdgError(_lib.WDG_ERR_ARG, "a must hold 2 n_var^2 coefficients")
        a = np.tile(av, n * n * mesh.n_elem())
    return VariableAdvectionSystem(n_var, mesh, basis, a, approx_quad)


class Advection(Operator):
    """Advection<AQ>(n_var, mesh, basis, a, constant_coefficient): du += (A u, grad v) + upwind
    flux over interior edges (wavedg/Advection.hpp:17-142).  Constant symmetric coefficients
    (approx_quad = True), or a spatially varying coefficient with either quadrature."""

    def __init__(self, n_var: int, mesh: Mesh2D, basis, a, constant_coefficient: bool = True, quad=None,
                 approx_quad: bool = True):
        self.sys = _advection_system(n_var, mesh, basis, a, constant_coefficient, quad, approx_quad)

    def action(self, *args) -> None:
        self.sys.action(args[-2], args[-1])


class AdvectionHomogeneousBC(Operator):
    """AdvectionHomogeneousBC<AQ>: du += boundary flux with u = 0 outside (wavedg/Advection.hpp:144-273)."""

    def __init__(self, n_var: int, mesh: Mesh2D, basis, a, constant_coefficient: bool = True, quad=None,
                 approx_quad: bool = True):
        self.sys = _advection_system(n_var, mesh, basis, a, constant_coefficient, quad, approx_quad)

    def action(self, *args) -> None:
        self.sys.bc_action(args[-2], args[-1])


def to_file(fname: str, u) -> None:
    """dg::to_file (examples/examples.hpp:14-19): a float64 array (numpy or CUDA tensor) as raw
    native-order bytes."""
    p, keep = _ptr(u, name="u")
    check(lib().wdg_write_raw(os.fsencode(fname), _size(u), p), "to_file")


def read_file(fname: str, out) -> None:
    """Read a to_file snapshot into `out` (float64 numpy array or CUDA tensor of the right size)."""
    p, keep = _ptr(out, True, "out")
    check(lib().wdg_read_raw(os.fsencode(fname), _size(out), p), "read_file")


def norm(x, system: Discretisation) -> float:
    return system.norm(x)


def error(x, y, system: Discretisation) -> float:
    return system.error(x, y)
