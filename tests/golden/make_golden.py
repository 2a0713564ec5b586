"""Generate the golden fixtures in tests/golden/ from the reference library.

    make -C oracle ref          # compiles the reference (needs its sources)
    python tests/golden/make_golden.py [--exact-quadrature-only | --advection-only | --reference-meshes | --euler | --vadvection]

Every output array is produced by the reference waveDG code compiled from its
own sources (oracle/_ref/libwdgref.so, driven through oracle/ref_harness.cpp).
Inputs are seeded (numpy PCG64) and stored beside the outputs, so the fixtures
are self-contained: the GPU box and the CPU tests read only these files.

The absorbing (code 0) and Dirichlet (code 2) boundary operators are the
harness's compositions of reference parts (see oracle/ref_harness.cpp); code 1
and all interior operators are the reference classes themselves.
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import cpu  # noqa: E402
from wavedg_b200 import meshgen as mg  # noqa: E402

KIND = "reference"
# the reference's own mesh files (meshes/<name>/{info,coordinates,elements}.txt)
REF_DIR = os.environ.get("WDG_REFERENCE_DIR", "/root/reference")
REF_MESHES = ("Square", "L", "skew")


def meshes():
    v, q = mg.uniform_rect(4, -1.0, 1.0, 3, 0.0, 2.0)
    yield "rect4x3", v, q
    v, q = mg.perturbed_rect(6, 0.2, seed=11)
    v, q = mg.scrambled(v, q, seed=12)
    yield "scrambled6", v, q
    v, q = mg.l_shape(3)
    v, q = mg.scrambled(v, q, seed=13)
    yield "lshape3", v, q


def mesh_fixture(name, v, q):
    m = cpu.Mesh(v, q, KIND)
    np.savez_compressed(os.path.join(HERE, f"mesh_{name}.npz"), verts=v, quads=q, edges_interior=m.edges(0),
                        edges_boundary=m.edges(1), min_h=m.min_h(), midpoints=m.boundary_midpoints())
    return m


def op_fixture(name, v, q, m, n, seed):
    rng = np.random.default_rng(seed)
    bc = rng.integers(0, 3, size=m.n_edges(1)).astype(np.int32)
    op = cpu.Op(m, n, bc)
    u = rng.standard_normal(op.ndof)
    out = dict(verts=v, quads=q, n=n, bc=bc, u=u)
    for nm in ("div", "wave_action", "bc_action"):
        r = rng.standard_normal(op.ndof)  # these accumulate: start from a nonzero du
        out[f"{nm}_in"] = r.copy()
        getattr(op, nm)(u, r)
        out[nm] = r
    out["rhs"] = op.rhs(u)
    F = rng.standard_normal(op.ndof)
    out["F"] = F
    out["rhs_forced"] = op.rhs(u, F, 0.37)
    for k in (0, 1):
        out[f"prolong{k}"] = op.prolong(k, u)
        uf = rng.standard_normal(out[f"prolong{k}"].size)
        out[f"flux{k}_in"] = uf
        out[f"flux{k}"] = op.flux(k, uf)
        r = rng.standard_normal(op.ndof)
        out[f"prolong_t{k}_in"] = r.copy()
        op.prolong_t(k, uf, r)
        out[f"prolong_t{k}"] = r
    uB = rng.standard_normal(n * 3 * 2 * m.n_edges(1))
    out["apply_bc_in"] = uB.copy()
    op.apply_bc(uB)
    out["apply_bc"] = uB
    x = u.copy()
    op.mass_inv(3, x)
    out["mass_inv"] = x
    out["mass_action"] = op.mass_action(3, u)
    out["rk4_dt"] = 1e-3
    out["rk4"], _ = op.rk4(u, 1e-3, 3)
    out["node_coords"] = op.node_coords()
    cen = np.array([[0.1, 0.2], [-0.3, 0.4]])
    out["load"] = op.load_gaussians(cen, [0.3, 0.2], [1.0, -0.5], 2.0, 0, False)
    out["load_minv"] = op.load_gaussians(cen, [0.3, 0.2], [1.0, -0.5], 2.0, 1, True)
    np.savez_compressed(os.path.join(HERE, f"op_{name}_n{n}.npz"), **out)


def config1():
    """32 x 32 uniform mesh on [-1,1]^2, P = 3, Dirichlet p = 0 on every boundary edge,
    p0 = exp(-(x^2 + y^2)/0.01) assembled as M^{-1}(f, phi), dt = 0.1 h / (P+1)^2, 200 RK4 steps."""
    v, q = mg.uniform_rect(32, -1.0, 1.0, 32, -1.0, 1.0)
    m = cpu.Mesh(v, q, KIND)
    bc = np.full(m.n_edges(1), 2, dtype=np.int32)
    op = cpu.Op(m, 4, bc)
    u0 = op.load_gaussians([[0.0, 0.0]], [np.sqrt(0.005)], [1.0], 1.0, 0, True)
    dt = 0.1 * m.min_h() / 16.0
    u1, _ = op.rk4(u0, dt, 1)
    u200, t = op.rk4(u0, dt, 200)
    np.savez_compressed(os.path.join(HERE, "config1_32x32_P3.npz"), verts=v, quads=q, bc=bc, n=4, dt=dt, u0=u0,
                        rhs0=op.rhs(u0), u1=u1, u200=u200, t200=t)


def waveholtz():
    """5 x 5 perturbed mesh, P = 3, omega = 2; reflecting left/bottom walls, absorbing elsewhere
    (the split examples/waveholtz2d.cpp uses), Gaussian forcing on p."""
    v, q = mg.perturbed_rect(5, 0.2, seed=21)
    m = cpu.Mesh(v, q, KIND)
    bc = mg.boundary_codes_by_wall(m.boundary_midpoints(), left=1, bottom=1, right=0, top=0)
    op = cpu.Op(m, 4, bc)
    F = op.load_gaussians([[0.1, 0.2]], [0.2], [1.0], 4.0, 0, False)
    wh = cpu.WaveHoltz(op, 2.0)
    pi0 = wh.pi0(F)
    S = wh.S(pi0)
    W, it, err = wh.solve(pi0, 1e-6, 200)
    H = wh.postprocess(W)
    np.savez_compressed(os.path.join(HERE, "waveholtz_5x5_P3.npz"), verts=v, quads=q, bc=bc, n=4, omega=2.0, F=F,
                        T=wh.T, dt=wh.dt, nt=wh.nt, pi0=pi0, S_pi0=S, W=W, iters=it, err=err, H=H)
    # all-reflecting walls: the reference's own WaveHoltz class (pi0 and S)
    bc1 = np.ones(m.n_edges(1), dtype=np.int32)
    op1 = cpu.Op(m, 4, bc1)
    wh1 = cpu.WaveHoltz(op1, 2.0)
    p1 = wh1.pi0(F)
    np.savez_compressed(os.path.join(HERE, "waveholtz_reflect_5x5_P3.npz"), verts=v, quads=q, bc=bc1, n=4,
                        omega=2.0, F=F, pi0=p1, S_pi0=wh1.S(p1))


def waveholtz_exact():
    """approx_quad = false WaveHoltz on the 5 x 5 perturbed mesh, P = 3, omega = 2: all-reflecting
    walls through the reference's own WaveHoltz class (pi0, S); reflecting left/bottom and
    absorbing elsewhere through the harness's restated loop over the exact operators (pi0, S,
    a solve to 1e-6)."""
    v, q = mg.perturbed_rect(5, 0.2, seed=21)
    m = cpu.Mesh(v, q, KIND)
    bc1 = np.ones(m.n_edges(1), dtype=np.int32)
    F = cpu.Op(m, 4, bc1).load_gaussians([[0.1, 0.2]], [0.2], [1.0], 4.0, 0, False)
    wh1 = cpu.WaveHoltz(cpu.OpQ(m, 4, bc1), 2.0)
    p1 = wh1.pi0(F)
    bc = mg.boundary_codes_by_wall(m.boundary_midpoints(), left=1, bottom=1, right=0, top=0)
    wh = cpu.WaveHoltz(cpu.OpQ(m, 4, bc), 2.0)
    p = wh.pi0(F)
    W, it, err = wh.solve(p, 1e-6, 200)
    np.savez_compressed(os.path.join(HERE, "waveholtz_exact_5x5_P3.npz"), verts=v, quads=q, n=4, omega=2.0, F=F,
                        bc_reflect=bc1, pi0_reflect=p1, S_pi0_reflect=wh1.S(p1), bc=bc, T=wh.T, dt=wh.dt, nt=wh.nt,
                        pi0=p, S_pi0=wh.S(p), W=W, iters=it, err=err)


def advection_fixture(name, v, q, m, n, nv, seed):
    """Advection<true> + AdvectionHomogeneousBC<true> with constant symmetric coefficients
    (n_var = 1: a velocity; n_var > 1: random symmetric A_0, A_1), MassMatrix<true>, RHS, RK4."""
    rng = np.random.default_rng(seed)
    if nv == 1:
        a = np.array([0.7, -0.4])
    else:
        A = rng.standard_normal((2, nv, nv))
        A = A + A.transpose(0, 2, 1)
        a = np.concatenate([A[0].reshape(-1, order="F"), A[1].reshape(-1, order="F")])  # a(d, c, k)
    op = cpu.OpA(m, n, nv, a)
    u = rng.standard_normal(op.ndof)
    out = dict(verts=v, quads=q, n=n, nv=nv, a=a, u=u)
    for nm in ("action", "bc_action"):
        r = rng.standard_normal(op.ndof)
        out[f"{nm}_in"] = r.copy()
        getattr(op, nm)(u, r)
        out[nm] = r
    out["rhs"] = op.rhs(u)
    dt = 0.1 * m.min_h() / n ** 2
    out["dt"] = dt
    out["rk4_5"], _ = op.rk4(u, dt, 5)
    np.savez_compressed(os.path.join(HERE, f"adv_{name}_n{n}_v{nv}.npz"), **out)


def node_coordinates(v, q, n, legendre=False):
    """Physical coordinates (x, y) of the basis nodes (GLL, or Gauss-Legendre), shape
    (n_elem, n, n) each, node (i, j) at [el, j, i]: the bilinear map of the corners
    (QuadElement::physical_coordinates)."""
    xs = np.polynomial.legendre.leggauss(n)[0] if legendre else np.asarray(cpu.basis(n, KIND)[0])
    c = np.asarray(v)[np.asarray(q)]  # (nel, 4, 2)
    xi, eta = xs[None, None, :], xs[None, :, None]
    out = []
    for k in range(2):
        out.append(0.25 * ((1 - xi) * (1 - eta) * c[:, 0, k][:, None, None] + (1 + xi) * (1 - eta) * c[:, 1, k][:, None, None]
                           + (1 + xi) * (1 + eta) * c[:, 2, k][:, None, None] + (1 - xi) * (1 + eta) * c[:, 3, k][:, None, None]))
    return out


def variable_coefficient(v, q, n, nv, legendre=False):
    """a(n_var, n_var, 2, n, n, n_elem) from a smooth field at the nodes: n_var = 1 the rotating
    velocity r (y, -x) of examples/advec2d.cpp's coefficient(); n_var > 1 symmetric matrices
    varying in space."""
    x, y = node_coordinates(v, q, n, legendre)  # (nel, n, n), [el, j, i]
    nel = x.shape[0]
    a = np.zeros((nel, n, n, 2, nv, nv))  # C order of the reverse of (k, l, comp, i, j, el)
    if nv == 1:
        r = np.hypot(x, y)
        a[..., 0, 0, 0] = r * y
        a[..., 1, 0, 0] = -r * x
    else:
        for k in range(nv):
            for l in range(k, nv):
                c0 = (1.0 + 0.3 * x + 0.1 * k) if k == l else 0.2 * np.sin(x + 2 * y + k + l)
                c1 = (-0.5 + 0.2 * y * x - 0.1 * l) if k == l else 0.3 * np.cos(2 * x - y + k * l)
                a[..., 0, l, k] = a[..., 0, k, l] = c0
                a[..., 1, l, k] = a[..., 1, k, l] = c1
    return a.reshape(-1)


def vadvection_fixture(name, v, q, m, n, nv, approx, seed, legendre=False):
    """Advection<AQ> + AdvectionHomogeneousBC<AQ> with a spatially varying coefficient
    (constant_coefficient = false), MassMatrix<AQ>, on a Gauss-Lobatto or (legendre) a
    Gauss-Legendre basis; actions, RHS, 3 steps of RK4 and SSPRK3."""
    rng = np.random.default_rng(seed)
    a = variable_coefficient(v, q, n, nv, legendre)
    op = cpu.OpV(m, n, nv, a, approx, 0 if legendre else 1)
    u = rng.standard_normal(op.ndof)
    out = dict(verts=v, quads=q, n=n, nv=nv, approx=int(approx), basis_type=0 if legendre else 1, a=a, u=u)
    for nm in ("action", "bc_action"):
        r = rng.standard_normal(op.ndof)
        out[f"{nm}_in"] = r.copy()
        getattr(op, nm)(u, r)
        out[nm] = r
    out["rhs"] = op.rhs(u)
    dt = 0.1 * m.min_h() / n ** 2
    out["dt"] = dt
    out["rk4_3"], _ = op.steps(u, dt, 3, "rk4")
    out["ssprk3_3"], _ = op.steps(u, dt, 3, "ssprk3")
    tag = ("aq" if approx else "ex") + ("_gl" if legendre else "")
    np.savez_compressed(os.path.join(HERE, f"vadv_{name}_n{n}_v{nv}_{tag}.npz"), **out)


def mass_basis_fixture(name, v, q, m, n, legendre, approx, seed):
    """MassMatrix<AQ> (action, inverse) and LinearFunctional2D on a Gauss-Legendre or
    Gauss-Lobatto basis: the load of examples/advec2d.cpp's coefficient r (y, -x) and its
    projection M^{-1} (f, phi), as that example forms it."""
    rng = np.random.default_rng(seed)
    bt = 0 if legendre else 1
    mb = cpu.MassB(m, n, bt, approx)
    x = rng.standard_normal(2 * mb.npts)
    pts = mb.points()
    px, py = pts[0::2], pts[1::2]
    r = np.hypot(px, py)
    fq = np.stack([r * py, -r * px], axis=1).reshape(-1)  # (d, point)
    F = mb.load(2, fq)
    out = dict(verts=v, quads=q, n=n, basis_type=bt, approx=int(approx), x=x, action=mb.action(2, x),
               inv=mb.inv(2, x), points=pts, fq=fq, load=F, projection=mb.inv(2, F))
    tag = ("gl" if legendre else "gll") + ("_aq" if approx else "_ex")
    np.savez_compressed(os.path.join(HERE, f"massb_{name}_n{n}_{tag}.npz"), **out)


def opq_fixture(name, v, q, m, n, seed):
    """approx_quad = false: Div<false>, EdgeFlux<false> (interior and boundary), WaveEquation,
    the composed boundary operator over EdgeFlux<false>, MassMatrix<false>, RHS, 5 RK4 steps."""
    rng = np.random.default_rng(seed)
    bc = rng.integers(0, 3, size=m.n_edges(1)).astype(np.int32)
    op = cpu.OpQ(m, n, bc)
    u = rng.standard_normal(op.ndof)
    out = dict(verts=v, quads=q, n=n, bc=bc, u=u)
    for nm in ("div", "wave_action", "bc_action"):
        r = rng.standard_normal(op.ndof)
        out[f"{nm}_in"] = r.copy()
        getattr(op, nm)(u, r)
        out[nm] = r
    for k, tag in ((0, "interior"), (1, "boundary")):
        uf = rng.standard_normal(n * 3 * 2 * m.n_edges(k))
        out[f"flux_{tag}_in"] = uf
        out[f"flux_{tag}"] = op.flux(k, uf)
    x = u.copy()
    op.mass_inv(3, x)
    out["mass_inv"] = x
    out["mass_action"] = op.mass_action(3, u)
    out["rhs"] = op.rhs(u)
    dt = 0.1 * m.min_h() / n ** 2
    out["dt"] = dt
    out["rk4_5"], _ = op.rk4(u, dt, 5)
    np.savez_compressed(os.path.join(HERE, f"opq_{name}_n{n}.npz"), **out)


def euler_state(ndof, rng):
    """A positive Euler state per node: density 1 + 0.2 U, velocities 0.3 N, pressure 1 + 0.2 U
    (total energy p / (gamma - 1) + rho |v|^2 / 2)."""
    nn = ndof // 4
    rho = 1.0 + 0.2 * rng.random(nn)
    u, v = 0.3 * rng.standard_normal(nn), 0.3 * rng.standard_normal(nn)
    p = 1.0 + 0.2 * rng.random(nn)
    return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], axis=1).ravel()


def euler_fixture(name, v, q, m, n, seed):
    """The compressible Euler operators of examples/cl2d.cpp with approx_quad = true:
    DivF2D<true> (accumulating), the prolongators, EdgeFluxF2D<true> with the local
    Lax-Friedrichs flux (interior traces; boundary traces with exterior = interior), the time
    derivative, 3 steps of ode::RungeKutta4 and of ode::SSPRK3."""
    rng = np.random.default_rng(seed)
    op = cpu.OpE(m, n)
    u = euler_state(op.ndof, rng)
    out = dict(verts=v, quads=q, n=n, u=u)
    r = rng.standard_normal(op.ndof)
    out["div_in"] = r.copy()
    op.div(u, r)
    out["div"] = r
    for k in (0, 1):
        ub = op.prolong(k, u)
        out[f"prolong{k}"] = ub.copy()
        if k == 1:  # exterior boundary state = interior state, as the example sets it
            ub = ub.reshape(-1, 2, 4 * n)
            ub[:, 1] = ub[:, 0]
            ub = ub.reshape(-1)
        out[f"flux{k}_in"] = ub
        out[f"flux{k}"] = op.flux(k, ub)
    out["rhs"] = op.rhs(u)
    dt = 0.1 * m.min_h() / (n * n)
    out["dt"] = dt
    out["rk4_3"], _ = op.steps(u, dt, 3, "rk4")
    out["ssprk3_3"], _ = op.steps(u, dt, 3, "ssprk3")
    np.savez_compressed(os.path.join(HERE, f"euler_{name}_n{n}.npz"), **out)


def euler_exact_fixture(name, v, q, m, n, seed):
    """The Euler operators with approx_quad = false (examples/cl2d.cpp as shipped): DivF2D<false>,
    EdgeFluxF2D<false> on the prolonged traces (boundary: exterior = interior), the time
    derivative with MassMatrix<false>, 3 RK4 and 3 SSPRK3 steps."""
    rng = np.random.default_rng(seed)
    op = cpu.OpEQ(m, n)
    prol = cpu.OpE(m, n)  # the Lobatto prolongators are the same for both rules
    u = euler_state(op.ndof, rng)
    out = dict(verts=v, quads=q, n=n, u=u)
    r = rng.standard_normal(op.ndof)
    out["div_in"] = r.copy()
    op.div(u, r)
    out["div"] = r
    for k in (0, 1):
        ub = prol.prolong(k, u)
        if k == 1:
            ub = ub.reshape(-1, 2, 4 * n)
            ub[:, 1] = ub[:, 0]
            ub = ub.reshape(-1)
        out[f"flux{k}_in"] = ub
        out[f"flux{k}"] = op.flux(k, ub)
    out["rhs"] = op.rhs(u)
    dt = 0.1 * m.min_h() / (n * n)
    out["dt"] = dt
    out["rk4_3"], _ = op.steps(u, dt, 3, "rk4")
    out["ssprk3_3"], _ = op.steps(u, dt, 3, "ssprk3")
    np.savez_compressed(os.path.join(HERE, f"eulerq_{name}_n{n}.npz"), **out)


def reference_meshes():
    """The reference's mesh files, copied unchanged into tests/golden/meshes/<name>/ (data, read
    by Mesh2D::from_file, source/Mesh2D.cpp:94-128); per mesh the connectivity the reference's
    own reader builds from them (mesh_file_<name>.npz), and operator fixtures on all three
    (their sides meet with every relative orientation, delta = -1 included)."""
    cases = {"Square": [6], "L": [5], "skew": [4]}
    for k, name in enumerate(REF_MESHES):
        src, dst = os.path.join(REF_DIR, "meshes", name), os.path.join(HERE, "meshes", name)
        os.makedirs(dst, exist_ok=True)
        for f in ("info.txt", "coordinates.txt", "elements.txt"):
            shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
        g = cpu.reference_mesh_from_file(dst)
        v = np.loadtxt(os.path.join(dst, "coordinates.txt"), dtype=np.float64).reshape(-1, 2)
        q = np.loadtxt(os.path.join(dst, "elements.txt"), dtype=np.int32).reshape(-1, 4)
        np.savez_compressed(os.path.join(HERE, f"mesh_file_{name}.npz"), verts=v, quads=q,
                            edges_interior=g["edges_interior"], edges_boundary=g["edges_boundary"], min_h=g["min_h"],
                            midpoints=g["midpoints"])
        m = cpu.Mesh(v, q, KIND)
        for n in cases[name]:
            op_fixture(f"file{name}", v, q, m, n, 3000 + 100 * k + n)


def main():
    if not cpu.available("reference"):
        raise SystemExit("build the reference first: make -C oracle ref")
    if "--euler" in sys.argv:
        ecases = {"scrambled6": [4], "lshape3": [5]}
        for seed, (name, v, q) in enumerate(meshes()):
            for n in ecases.get(name, []):
                euler_fixture(name, v, q, cpu.Mesh(v, q, KIND), n, 4000 + 100 * seed + n)
        g = os.path.join(HERE, "meshes", "Square")
        v = np.loadtxt(os.path.join(g, "coordinates.txt")).reshape(-1, 2)
        q = np.loadtxt(os.path.join(g, "elements.txt"), dtype=np.int32).reshape(-1, 4)
        euler_fixture("fileSquare", v, q, cpu.Mesh(v, q, KIND), 3, 4999)
        qcases = {"scrambled6": [4], "lshape3": [3]}
        for seed, (name, v, q) in enumerate(meshes()):
            for n in qcases.get(name, []):
                euler_exact_fixture(name, v, q, cpu.Mesh(v, q, KIND), n, 4500 + 100 * seed + n)
        print("Euler fixtures written to", HERE)
        return
    if "--vadvection" in sys.argv:
        vcases = {"scrambled6": [(4, 1), (5, 2)], "lshape3": [(3, 1), (4, 3)]}
        for seed, (name, v, q) in enumerate(meshes()):
            for n, nv in vcases.get(name, []):
                for approx in (True, False):
                    vadvection_fixture(name, v, q, cpu.Mesh(v, q, KIND), n, nv, approx,
                                       6000 + 100 * seed + 10 * n + nv + 5 * approx)
        # Gauss-Legendre bases (examples/advec2d.cpp: n = 5, n_var = 1, approx_quad = false)
        gcases = {"scrambled6": [(5, 1), (3, 2)], "lshape3": [(4, 1)]}
        for seed, (name, v, q) in enumerate(meshes()):
            for n, nv in gcases.get(name, []):
                for approx in (True, False):
                    vadvection_fixture(name, v, q, cpu.Mesh(v, q, KIND), n, nv, approx,
                                       6500 + 100 * seed + 10 * n + nv + 5 * approx, legendre=True)
        mcases = {"scrambled6": [5, 3], "lshape3": [4]}
        for seed, (name, v, q) in enumerate(meshes()):
            for n in mcases.get(name, []):
                for legendre in (True, False):
                    for approx in (True, False):
                        mass_basis_fixture(name, v, q, cpu.Mesh(v, q, KIND), n, legendre, approx,
                                           6800 + 100 * seed + 10 * n + 2 * legendre + approx)
        print("variable-coefficient advection and mass / load-vector fixtures written to", HERE)
        return
    if "--reference-meshes" in sys.argv:
        reference_meshes()
        print("reference-mesh fixtures written to", HERE)
        return
    qcases = {"scrambled6": [3, 5], "lshape3": [4]}
    acases = {"scrambled6": [(5, 1), (4, 2)], "lshape3": [(3, 4)]}
    if "--advection-only" in sys.argv:
        for seed, (name, v, q) in enumerate(meshes()):
            for n, nv in acases.get(name, []):
                advection_fixture(name, v, q, cpu.Mesh(v, q, KIND), n, nv, 2000 + 100 * seed + 10 * n + nv)
        print("advection fixtures written to", HERE)
        return
    if "--exact-quadrature-only" in sys.argv:
        for seed, (name, v, q) in enumerate(meshes()):
            for n in qcases.get(name, []):
                opq_fixture(name, v, q, cpu.Mesh(v, q, KIND), n, 1000 + 100 * seed + n)
        waveholtz_exact()
        print("exact-quadrature fixtures written to", HERE)
        return
    x = {}
    for n in range(2, 10):
        xs, ws, D = cpu.basis(n, KIND)
        x[f"x{n}"], x[f"w{n}"], x[f"D{n}"] = xs, ws, D
    np.savez_compressed(os.path.join(HERE, "basis.npz"), **x)
    cases = {"rect4x3": [6], "scrambled6": [3, 4, 5, 7], "lshape3": [5]}
    for seed, (name, v, q) in enumerate(meshes()):
        m = mesh_fixture(name, v, q)
        for n in cases[name]:
            op_fixture(name, v, q, m, n, 100 * seed + n)
        for n in qcases.get(name, []):
            opq_fixture(name, v, q, m, n, 1000 + 100 * seed + n)
        for n, nv in acases.get(name, []):
            advection_fixture(name, v, q, m, n, nv, 2000 + 100 * seed + 10 * n + nv)
    config1()
    waveholtz()
    waveholtz_exact()
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
