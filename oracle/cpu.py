"""CPU checkers for the tests -- TEST INFRASTRUCTURE ONLY.

Loads one of two shared libraries with the same C entry points:

* ``oracle``    -- ``oracle/_build/liboracle.so``, the plain C++ restatement of
  the reference algorithm (``oracle/wdg_oracle.cpp``); always buildable with g++.
* ``reference`` -- ``oracle/_ref/libwdgref.so``, the reference library itself
  compiled from its sources plus ``oracle/ref_harness.cpp``; built only where
  the reference sources are present, and shipped prebuilt otherwise.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module.  The product path (``wavedg_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {
    "oracle": (os.path.join(HERE, "_build", "liboracle.so"), "orc_"),
    "reference": (os.path.join(HERE, "_ref", "libwdgref.so"), "ref_"),
}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_v, _i, _d = C.c_void_p, C.c_int, C.c_double

_SIGS = {
    "mesh_create": ([_i, _dp, _i, _ip], _v),
    "mesh_from_file": ([C.c_char_p], _v),
    "mesh_destroy": ([_v], None),
    "mesh_n_elem": ([_v], _i),
    "mesh_n_edges": ([_v, _i], _i),
    "mesh_min_h": ([_v], _d),
    "mesh_edges": ([_v, _i, _ip], None),
    "mesh_boundary_midpoints": ([_v, _dp], None),
    "basis": ([_i, _dp, _dp, _dp], None),
    "op_create": ([_v, _i, _ip], _v),
    "op_destroy": ([_v], None),
    "node_coords": ([_v, _dp], None),
    "div": ([_v, _dp, _dp], None),
    "wave_action": ([_v, _dp, _dp], None),
    "bc_action": ([_v, _dp, _dp], None),
    "prolong": ([_v, _i, _dp, _dp], None),
    "prolong_t": ([_v, _i, _dp, _dp], None),
    "flux": ([_v, _i, _dp, _dp], None),
    "apply_bc": ([_v, _dp], None),
    "mass_inv": ([_v, _i, _dp], None),
    "mass_action": ([_v, _i, _dp, _dp], None),
    "rhs": ([_v, _dp, _dp], None),
    "rhs_forced": ([_v, _dp, _dp, _dp, _d], None),
    "rk4": ([_v, _d, _i, C.POINTER(C.c_double), _dp], None),
    "opa_create": ([_v, _i, _i, _dp], _v),
    "opa_destroy": ([_v], None),
    "opa_action": ([_v, _dp, _dp], None),
    "opa_bc_action": ([_v, _dp, _dp], None),
    "opa_rhs": ([_v, _dp, _dp], None),
    "opa_rk4": ([_v, _d, _i, C.POINTER(C.c_double), _dp], None),
    "mb_create": ([_v, _i, _i, _i], _v),
    "mb_destroy": ([_v], None),
    "mb_action": ([_v, _i, _dp, _dp], None),
    "mb_inv": ([_v, _i, _dp], None),
    "mb_points": ([_v, _dp], None),
    "mb_load": ([_v, _i, _dp, _dp], None),
    "opv_create": ([_v, _i, _i, _dp, _i, _i], _v),
    "opv_destroy": ([_v], None),
    "opv_action": ([_v, _dp, _dp], None),
    "opv_bc_action": ([_v, _dp, _dp], None),
    "opv_rhs": ([_v, _dp, _dp], None),
    "opv_steps": ([_v, _i, _d, _i, C.POINTER(C.c_double), _dp], None),
    "ope_create": ([_v, _i], _v),
    "ope_destroy": ([_v], None),
    "ope_div": ([_v, _dp, _dp], None),
    "ope_flux": ([_v, _i, _dp, _dp], None),
    "ope_prolong": ([_v, _i, _dp, _dp], None),
    "ope_rhs": ([_v, _dp, _dp], None),
    "ope_steps": ([_v, _i, _d, _i, C.POINTER(C.c_double), _dp], None),
    "opeq_create": ([_v, _i], _v),
    "opeq_destroy": ([_v], None),
    "opeq_div": ([_v, _dp, _dp], None),
    "opeq_flux": ([_v, _i, _dp, _dp], None),
    "opeq_rhs": ([_v, _dp, _dp], None),
    "opeq_steps": ([_v, _i, _d, _i, C.POINTER(C.c_double), _dp], None),
    "opq_create": ([_v, _i, _ip], _v),
    "opq_destroy": ([_v], None),
    "opq_div": ([_v, _dp, _dp], None),
    "opq_flux": ([_v, _i, _dp, _dp], None),
    "opq_wave_action": ([_v, _dp, _dp], None),
    "opq_bc_action": ([_v, _dp, _dp], None),
    "opq_mass_inv": ([_v, _i, _dp], None),
    "opq_mass_action": ([_v, _i, _dp, _dp], None),
    "opq_rhs": ([_v, _dp, _dp], None),
    "opq_rk4": ([_v, _d, _i, C.POINTER(C.c_double), _dp], None),
    "load_gaussians": ([_v, _i, _dp, _dp, _dp, _dp, _d, _i, _i, _dp], None),
    "norm": ([_i, _dp], _d),
    "error": ([_i, _dp, _dp], _d),
    "wh_create": ([_v, _d], _v),
    "whq_create": ([_v, _d], _v),
    "wh_destroy": ([_v], None),
    "wh_params": ([_v, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)], None),
    "wh_pi0": ([_v, _dp, _dp], None),
    "wh_S": ([_v, _dp], None),
    "wh_postprocess": ([_v, _dp, _dp], None),
    "wh_solve": ([_v, _dp, _d, _i, _dp, C.POINTER(C.c_double)], _i),
}

_loaded: dict[str, C.CDLL] = {}


def build_oracle() -> str:
    """Compile the C++ restatement (g++ only, a couple of seconds)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return LIBS["oracle"][0]


def available(kind: str) -> bool:
    return os.path.exists(LIBS[kind][0])


def lib(kind: str = "oracle"):
    if kind in _loaded:
        return _loaded[kind]
    path, prefix = LIBS[kind]
    if kind == "oracle" and not os.path.exists(path):
        build_oracle()
    if not os.path.exists(path):
        raise FileNotFoundError(f"{kind} checker library not built: {path}")
    L = C.CDLL(path)
    ns = type("CPUChecker", (), {})()
    for name, (args, res) in _SIGS.items():
        fn = getattr(L, prefix + name, None)
        if fn is None:
            if kind == "oracle" and name.startswith(("opeq_", "opv_", "mb_")):
                continue  # operators that only the reference harness carries
            raise AttributeError(f"{path}: missing {prefix + name}")
        fn.argtypes = args
        fn.restype = res
        setattr(ns, name, fn)
    ns._cdll = L
    _loaded[kind] = ns
    return ns


_REF_READER = r"""
import ctypes as C, struct, sys
L = C.CDLL(sys.argv[1])
L.ref_mesh_from_file.restype = C.c_void_p
L.ref_mesh_from_file.argtypes = [C.c_char_p]
L.ref_mesh_min_h.restype = C.c_double
for f in ("ref_mesh_n_elem", "ref_mesh_n_edges", "ref_mesh_min_h", "ref_mesh_edges", "ref_mesh_boundary_midpoints",
          "ref_mesh_destroy"):
    getattr(L, f).argtypes = None
h = L.ref_mesh_from_file(sys.argv[2].encode())
with open(sys.argv[3], "wb") as out:
    if not h:
        out.write(struct.pack("<i", -1))
        sys.exit(0)
    h = C.c_void_p(h)
    ne, ni, nb = L.ref_mesh_n_elem(h), L.ref_mesh_n_edges(h, 0), L.ref_mesh_n_edges(h, 1)
    ei, eb, mp = (C.c_int * (5 * ni))(), (C.c_int * (5 * nb))(), (C.c_double * (2 * nb))()
    L.ref_mesh_edges(h, 0, ei)
    L.ref_mesh_edges(h, 1, eb)
    L.ref_mesh_boundary_midpoints(h, mp)
    out.write(struct.pack("<iiid", ne, ni, nb, L.ref_mesh_min_h(h)))
    out.write(bytes(ei) + bytes(eb) + bytes(mp))
"""


def reference_mesh_from_file(directory):
    """The reference's own Mesh2D::from_file (source/Mesh2D.cpp:94-128) through the compiled
    reference, in a child process: its reader uses iostreams and the library carries its own
    C++ runtime, which must not meet another one in the same process.  Returns the mesh tables
    {n_elem, edges_interior, edges_boundary, min_h, midpoints}, or None on a reader error."""
    import sys
    import tempfile

    path = LIBS["reference"][0]
    with tempfile.TemporaryDirectory() as td:
        f = os.path.join(td, "tables.bin")
        subprocess.run([sys.executable, "-c", _REF_READER, path, str(directory), f], check=True, timeout=120)
        raw = open(f, "rb").read()
    ne = int(np.frombuffer(raw[:4], dtype="<i4")[0])
    if ne < 0:
        return None
    ni, nb = (int(x) for x in np.frombuffer(raw[4:12], dtype="<i4"))
    mh = float(np.frombuffer(raw[12:20], dtype="<f8")[0])
    o = 20
    ei = np.frombuffer(raw[o:o + 20 * ni], dtype=np.int32).reshape(ni, 5)
    o += 20 * ni
    eb = np.frombuffer(raw[o:o + 20 * nb], dtype=np.int32).reshape(nb, 5)
    o += 20 * nb
    mp = np.frombuffer(raw[o:o + 16 * nb], dtype=np.float64).reshape(nb, 2)
    return {"n_elem": ne, "edges_interior": ei, "edges_boundary": eb, "min_h": mh, "midpoints": mp}


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Mesh:
    """Mesh2D::from_vertices on the CPU checker (vertices (nv,2), quads (nel,4))."""

    def __init__(self, verts, quads, kind="oracle"):
        self.L = lib(kind)
        self.verts = _f64(verts).reshape(-1, 2)
        self.quads = np.ascontiguousarray(quads, dtype=np.int32).reshape(-1, 4)
        self.h = self.L.mesh_create(len(self.verts), self.verts.ravel(), len(self.quads), self.quads.ravel())

    @classmethod
    def from_file(cls, directory, kind="oracle"):
        """Mesh2D::from_file on the CPU checker; None if the checker reports an error."""
        self = cls.__new__(cls)
        self.L = lib(kind)
        self.verts = self.quads = None
        self.h = self.L.mesh_from_file(os.fsencode(directory))
        return self if self.h else None

    def __del__(self):
        if getattr(self, "h", None):
            self.L.mesh_destroy(self.h)
            self.h = None

    @property
    def n_elem(self):
        return self.L.mesh_n_elem(self.h)

    def n_edges(self, kind):
        return self.L.mesh_n_edges(self.h, kind)

    def edges(self, kind):
        out = np.zeros((self.n_edges(kind), 5), dtype=np.int32)
        self.L.mesh_edges(self.h, kind, out.ravel())
        return out

    def min_h(self):
        return self.L.mesh_min_h(self.h)

    def boundary_midpoints(self):
        out = np.zeros((self.n_edges(1), 2))
        self.L.mesh_boundary_midpoints(self.h, out.ravel())
        return out


def basis(n, kind="oracle"):
    L = lib(kind)
    x, w, D = np.zeros(n), np.zeros(n), np.zeros(n * n)
    L.basis(n, x, w, D)
    return x, w, D.reshape(n, n, order="F")


class Op:
    """WaveEquation + boundary operator + MassMatrix<true> on the CPU checker."""

    def __init__(self, mesh: Mesh, n: int, bc):
        self.L, self.mesh, self.n = mesh.L, mesh, n
        self.bc = np.ascontiguousarray(bc, dtype=np.int32)
        assert len(self.bc) == mesh.n_edges(1)
        self.h = self.L.op_create(mesh.h, n, self.bc)
        self.ndof = 3 * n * n * mesh.n_elem

    def __del__(self):
        if getattr(self, "h", None):
            self.L.op_destroy(self.h)
            self.h = None

    def zeros(self):
        return np.zeros(self.ndof)

    def node_coords(self):
        out = np.zeros(2 * self.ndof // 3)
        self.L.node_coords(self.h, out)
        return out

    def div(self, u, du):
        self.L.div(self.h, _f64(u), du)

    def wave_action(self, u, du):
        self.L.wave_action(self.h, _f64(u), du)

    def bc_action(self, u, du):
        self.L.bc_action(self.h, _f64(u), du)

    def prolong(self, kind, u):
        uf = np.zeros(self.n * 3 * 2 * self.mesh.n_edges(kind))
        self.L.prolong(self.h, kind, _f64(u), uf)
        return uf

    def prolong_t(self, kind, uf, u):
        self.L.prolong_t(self.h, kind, _f64(uf), u)

    def flux(self, kind, uf):
        fb = np.zeros_like(uf)
        self.L.flux(self.h, kind, _f64(uf), fb)
        return fb

    def apply_bc(self, uB):
        self.L.apply_bc(self.h, uB)

    def mass_inv(self, nv, x):
        self.L.mass_inv(self.h, nv, x)

    def mass_action(self, nv, x):
        y = np.zeros_like(x)
        self.L.mass_action(self.h, nv, _f64(x), y)
        return y

    def rhs(self, u, F=None, s=0.0):
        du = self.zeros()
        if F is None:
            self.L.rhs(self.h, _f64(u), du)
        else:
            self.L.rhs_forced(self.h, _f64(u), du, _f64(F), s)
        return du

    def rk4(self, u, dt, nsteps, t=0.0):
        u = _f64(u).copy()
        tt = C.c_double(t)
        self.L.rk4(self.h, dt, nsteps, C.byref(tt), u)
        return u, tt.value

    def load_gaussians(self, centers, sigmas, amps, scale=1.0, comp=0, mass_inv=False):
        c = _f64(centers).reshape(-1, 2)
        F = self.zeros()
        self.L.load_gaussians(self.h, len(c), _f64(c[:, 0]), _f64(c[:, 1]), _f64(sigmas), _f64(amps),
                              scale, comp, 1 if mass_inv else 0, F)
        return F


class WaveHoltz:
    def __init__(self, op: Op, omega: float):
        self.op, self.L = op, op.L
        self.h = (self.L.whq_create if isinstance(op, OpQ) else self.L.wh_create)(op.h, omega)
        T, dt, nt = C.c_double(), C.c_double(), C.c_int()
        self.L.wh_params(self.h, C.byref(T), C.byref(dt), C.byref(nt))
        self.T, self.dt, self.nt = T.value, dt.value, nt.value

    def __del__(self):
        if getattr(self, "h", None):
            self.L.wh_destroy(self.h)
            self.h = None

    def pi0(self, F):
        u = self.op.zeros()
        self.L.wh_pi0(self.h, u, _f64(F))
        return u

    def S(self, W):
        W = _f64(W).copy()
        self.L.wh_S(self.h, W)
        return W

    def postprocess(self, W):
        H = np.zeros(2 * self.op.ndof // 3)
        self.L.wh_postprocess(self.h, H, _f64(W))
        return H

    def solve(self, pi0, tol, maxit, W0=None):
        W = self.op.zeros() if W0 is None else _f64(W0).copy()
        err = C.c_double()
        it = self.L.wh_solve(self.h, _f64(pi0), tol, maxit, W, C.byref(err))
        return W, it, err.value


class OpE:
    """The compressible Euler system of examples/cl2d.cpp (gamma = 1.4, local Lax-Friedrichs
    flux) with DivF2D<true>, EdgeFluxF2D<true> (interior and boundary; exterior boundary state =
    interior state), the Lobatto prolongators and MassMatrix<true>, on the CPU checker.  State
    (4, n, n, n_elem): density, x- and y-momentum, energy."""

    nv = 4

    def __init__(self, mesh: Mesh, n: int):
        self.L, self.mesh, self.n = mesh.L, mesh, n
        self.h = self.L.ope_create(mesh.h, n)
        self.ndof = 4 * n * n * mesh.n_elem

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ope_destroy(self.h)
            self.h = None

    def div(self, u, du):
        self.L.ope_div(self.h, _f64(u), du)

    def prolong(self, kind, u):
        ub = np.zeros(self.n * 4 * 2 * self.mesh.n_edges(kind))
        self.L.ope_prolong(self.h, kind, _f64(u), ub)
        return ub

    def flux(self, kind, ub):
        fb = np.zeros_like(_f64(ub))
        self.L.ope_flux(self.h, kind, _f64(ub), fb)
        return fb

    def rhs(self, u):
        du = np.zeros(self.ndof)
        self.L.ope_rhs(self.h, _f64(u), du)
        return du

    def steps(self, u, dt, nsteps, method="rk4", t=0.0):
        """ode::RungeKutta4 ("rk4") or ode::SSPRK3 ("ssprk3") steps of the time derivative."""
        u = _f64(u).copy()
        tt = C.c_double(t)
        self.L.ope_steps(self.h, {"rk4": 0, "ssprk3": 1}[method], dt, nsteps, C.byref(tt), u)
        return u, tt.value


class OpEQ(OpE):
    """The Euler operators with approx_quad = false, as examples/cl2d.cpp ships them
    (DivF2D<false>, EdgeFluxF2D<false> with their default 2n-point rules, MassMatrix<false>);
    the reference harness only."""

    def __init__(self, mesh: Mesh, n: int):
        self.L, self.mesh, self.n = mesh.L, mesh, n
        self.h = self.L.opeq_create(mesh.h, n)
        self.ndof = 4 * n * n * mesh.n_elem

    def __del__(self):
        if getattr(self, "h", None):
            self.L.opeq_destroy(self.h)
            self.h = None

    def div(self, u, du):
        self.L.opeq_div(self.h, _f64(u), du)

    def flux(self, kind, ub):
        fb = np.zeros_like(_f64(ub))
        self.L.opeq_flux(self.h, kind, _f64(ub), fb)
        return fb

    def rhs(self, u):
        du = np.zeros(self.ndof)
        self.L.opeq_rhs(self.h, _f64(u), du)
        return du

    def steps(self, u, dt, nsteps, method="rk4", t=0.0):
        u = _f64(u).copy()
        tt = C.c_double(t)
        self.L.opeq_steps(self.h, {"rk4": 0, "ssprk3": 1}[method], dt, nsteps, C.byref(tt), u)
        return u, tt.value


class MassB:
    """MassMatrix<AQ> and LinearFunctional2D on a Gauss-Lobatto (basis_type 1) or
    Gauss-Legendre (0) basis; the reference harness only."""

    def __init__(self, mesh: Mesh, n: int, basis_type: int, approx_quad: bool):
        self.L, self.mesh, self.n = mesh.L, mesh, n
        self.h = self.L.mb_create(mesh.h, n, int(basis_type), int(bool(approx_quad)))
        self.npts = n * n * mesh.n_elem

    def __del__(self):
        if getattr(self, "h", None):
            self.L.mb_destroy(self.h)
            self.h = None

    def action(self, nv, x):
        y = np.zeros_like(_f64(x))
        self.L.mb_action(self.h, nv, _f64(x), y)
        return y

    def inv(self, nv, x):
        y = _f64(x).copy()
        self.L.mb_inv(self.h, nv, y)
        return y

    def points(self):
        xy = np.zeros(2 * self.npts)
        self.L.mb_points(self.h, xy)
        return xy

    def load(self, nv, fq):
        F = np.zeros(nv * self.npts)
        self.L.mb_load(self.h, nv, _f64(fq), F)
        return F


class OpV:
    """Advection<AQ> + AdvectionHomogeneousBC<AQ> + MassMatrix<AQ> with a spatially varying
    coefficient a(n_var, n_var, 2, n, n, n_elem) (constant_coefficient = false) on a Gauss-Lobatto
    (basis_type 1) or Gauss-Legendre (0) basis; the reference harness only."""

    def __init__(self, mesh: Mesh, n: int, nv: int, a, approx_quad: bool, basis_type: int = 1):
        self.L, self.mesh, self.n, self.nv = mesh.L, mesh, n, nv
        self.a = _f64(a).reshape(-1)
        assert self.a.size == 2 * nv * nv * n * n * mesh.n_elem
        self.h = self.L.opv_create(mesh.h, n, nv, self.a, int(bool(approx_quad)), int(basis_type))
        self.ndof = nv * n * n * mesh.n_elem

    def __del__(self):
        if getattr(self, "h", None):
            self.L.opv_destroy(self.h)
            self.h = None

    def action(self, u, du):
        self.L.opv_action(self.h, _f64(u), du)

    def bc_action(self, u, du):
        self.L.opv_bc_action(self.h, _f64(u), du)

    def rhs(self, u):
        du = np.zeros(self.ndof)
        self.L.opv_rhs(self.h, _f64(u), du)
        return du

    def steps(self, u, dt, nsteps, method="rk4", t=0.0):
        u = _f64(u).copy()
        tt = C.c_double(t)
        self.L.opv_steps(self.h, {"rk4": 0, "ssprk3": 1}[method], dt, nsteps, C.byref(tt), u)
        return u, tt.value


class OpQ:
    """The same system with approx_quad = false (Div<false>, EdgeFlux<false>, MassMatrix<false>;
    default quadrature rules) on the CPU checker."""

    def __init__(self, mesh: Mesh, n: int, bc):
        self.L, self.mesh, self.n = mesh.L, mesh, n
        self.bc = np.ascontiguousarray(bc, dtype=np.int32)
        assert len(self.bc) == mesh.n_edges(1)
        self.h = self.L.opq_create(mesh.h, n, self.bc)
        self.ndof = 3 * n * n * mesh.n_elem

    def __del__(self):
        if getattr(self, "h", None):
            self.L.opq_destroy(self.h)
            self.h = None

    def zeros(self):
        return np.zeros(self.ndof)

    def div(self, u, du):
        self.L.opq_div(self.h, _f64(u), du)

    def flux(self, kind, uf):
        fb = np.zeros_like(uf)
        self.L.opq_flux(self.h, kind, _f64(uf), fb)
        return fb

    def wave_action(self, u, du):
        self.L.opq_wave_action(self.h, _f64(u), du)

    def bc_action(self, u, du):
        self.L.opq_bc_action(self.h, _f64(u), du)

    def mass_inv(self, nv, x):
        self.L.opq_mass_inv(self.h, nv, x)

    def mass_action(self, nv, x):
        y = np.zeros_like(x)
        self.L.opq_mass_action(self.h, nv, _f64(x), y)
        return y

    def rhs(self, u):
        du = np.zeros(self.ndof)
        self.L.opq_rhs(self.h, _f64(u), du)
        return du

    def rk4(self, u, dt, nsteps, t=0.0):
        u = _f64(u).copy()
        tt = C.c_double(t)
        self.L.opq_rk4(self.h, dt, nsteps, C.byref(tt), u)
        return u, tt.value


class OpA:
    """Advection<true> + AdvectionHomogeneousBC<true> + MassMatrix<true> for n_var variables with
    constant coefficients a (n_var, n_var, 2) on the CPU checker."""

    def __init__(self, mesh: Mesh, n: int, nv: int, a):
        self.L, self.mesh, self.n, self.nv = mesh.L, mesh, n, nv
        self.a = _f64(a).reshape(-1)
        assert self.a.size == 2 * nv * nv
        self.h = self.L.opa_create(mesh.h, n, nv, self.a)
        self.ndof = nv * n * n * mesh.n_elem

    def __del__(self):
        if getattr(self, "h", None):
            self.L.opa_destroy(self.h)
            self.h = None

    def action(self, u, du):
        self.L.opa_action(self.h, _f64(u), du)

    def bc_action(self, u, du):
        self.L.opa_bc_action(self.h, _f64(u), du)

    def rhs(self, u):
        du = np.zeros(self.ndof)
        self.L.opa_rhs(self.h, _f64(u), du)
        return du

    def rk4(self, u, dt, nsteps, t=0.0):
        u = _f64(u).copy()
        tt = C.c_double(t)
        self.L.opa_rk4(self.h, dt, nsteps, C.byref(tt), u)
        return u, tt.value
