"""Domain decomposition of one mesh across ranks (one GPU per rank), RK4 stepping.

The reference distributes a mesh with MPI (Mesh2D::distribute, source/Mesh2D.cpp:384-592)
and exchanges the face traces of cut edges before each operator application
(FaceVector::send_recv, source/FEMVector.cpp:153-216).  Here each rank holds a discretisation
of its own elements (wdg_wave_create_halo) whose state buffers end in a halo: one n x 3 trace
per cut side, in the face-node order of that side.  Before every RK stage the ranks exchange
the traces of the stage's input buffer (gather on the sender, one message per neighbouring
rank, write into the receiver's halo); then the stage runs as on an undivided mesh, and every
element's arithmetic is the same as there.

The plan is computed from the global mesh and the element -> rank map on every rank, without
communication, and both sides of each exchange derive the same slot order from it: the
receiver's cut sides sorted by (sending rank, local element, side).

    part = decomp.partition(mesh.n_elem(), world)
    dom = decomp.Domain(mesh, basis, bc, part, rank)
    dom.upload(u_global)
    dom.rk4_steps(dt, nsteps, decomp.dist_exchange(dom))      # torch.distributed, NCCL
    dom.download(u_global)                                     # this rank's elements only

On one GPU, several Domains of the same mesh can step together (`step_all`: device copies
between them), which is how the tests check the decomposed result against
the undivided one.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import WdgError, check, lib

_STAGE_BUFFER = (0, 1, 2, 1, 2)  # the input buffer of RK stage st (rk4 rotation)


def partition(n_elem: int, world: int) -> np.ndarray:
    """Element -> rank: contiguous blocks of element ids, sizes within one of each other."""
    if world < 1:
        raise ValueError("world size must be positive")
    return (np.arange(n_elem, dtype=np.int64) * world // max(n_elem, 1)).astype(np.int32)


def partition_mesh(mesh, world: int, method: str = "rcb") -> np.ndarray:
    """Element -> rank by Mesh2D::distribute's methods (wdg_mesh_partition,
    source/Mesh2D.cpp:233-382): "rcb" recursive coordinate bisection, "rcm" reverse
    Cuthill-McKee blocks.  Deterministic, so every rank computes the same map."""
    e2p = np.zeros(mesh.n_elem(), dtype=np.int32)
    check(lib().wdg_mesh_partition(mesh._h, int(world), {"rcb": 0, "rcm": 1}[method], C.c_void_p(e2p.ctypes.data)),
          "partition_mesh")
    return e2p


def partner_table(mesh, n: int, bc=None):
    """(fbase (nel, 4), fcode (nel,)) of the fused kernels for `mesh` (wdg_mesh_partner_table)."""
    nel = mesh.n_elem()
    fb = np.zeros(4 * nel, dtype=np.int32)
    fc = np.zeros(nel, dtype=np.uint32)
    codes = None if bc is None else np.ascontiguousarray(bc, dtype=np.int32)
    check(lib().wdg_mesh_partner_table(mesh._h, int(n), None if codes is None else C.c_void_p(codes.ctypes.data),
                                       C.c_void_p(fb.ctypes.data), C.c_void_p(fc.ctypes.data)), "partner_table")
    return fb.reshape(nel, 4), fc


class Plan:
    """This rank's share of a decomposed mesh and its exchange lists (pure host arithmetic)."""

    def __init__(self, mesh, n: int, bc, part, rank: int):
        part = np.asarray(part, dtype=np.int32)
        nel = mesh.n_elem()
        if part.shape != (nel,):
            raise ValueError("one rank per element")
        self.n, self.rank, self.world = int(n), int(rank), int(part.max()) + 1
        nd = 3 * n * n
        self.nd = nd
        fb, fc = partner_table(mesh, n, bc)
        side = np.arange(4)
        byte = (fc[:, None] >> (8 * side[None, :]).astype(np.uint32)) & 0xFF
        boundary = (byte & 0x80) != 0
        nb = np.where(boundary, -1, fb // nd)
        cut = ~boundary & (part[np.maximum(nb, 0)] != part[:, None])
        stride = np.array([3, -3, 3 * n, -3 * n])[(byte & 3).astype(np.int64)]
        # every rank's local element order, the same on all ranks: the elements that read no
        # halo trace first, then those with a cut side (a stage can then run its first part
        # while the halo is in flight)
        g2l = np.full(nel, -1, dtype=np.int64)
        cut_any = cut.any(axis=1)
        for r in range(self.world):
            ids = np.nonzero(part == r)[0]
            order = np.concatenate([ids[~cut_any[ids]], ids[cut_any[ids]]])
            g2l[order] = np.arange(len(order))
            if r == rank:
                self.local = order.astype(np.int64)
                self.n_inner = int(np.count_nonzero(~cut_any[ids]))
        k = np.arange(n)

        def slots(r):
            """Rank r's cut sides in slot order: (src rank, global element, side), sorted."""
            el, f = np.nonzero(cut & (part[:, None] == r))
            src = part[nb[el, f]]
            order = np.lexsort((f, el, src))
            return el[order], f[order], src[order]

        # receive side: this rank's halo slots, grouped by the sending rank
        el, f, src = slots(rank)
        self.halo_elem = g2l[el].astype(np.int32)
        self.halo_side = f.astype(np.int32)
        self.recv = {}  # src rank -> (first slot, slot count)
        for s in np.unique(src):
            idx = np.nonzero(src == s)[0]
            self.recv[int(s)] = (int(idx[0]), len(idx))
        # send side: for every rank whose halo holds traces of this rank's elements, the node
        # offsets (this rank's numbering) in that rank's slot order
        self.send = {}
        for r in range(self.world):
            if r == rank:
                continue
            el, f, src = slots(r)
            m = src == rank
            if not m.any():
                continue
            el, f = el[m], f[m]
            off = fb[el, f][:, None] + k[None, :] * stride[el, f][:, None]  # global node offsets
            nbe = off // nd
            local_off = off - nbe * nd + g2l[nbe] * nd
            self.send[r] = local_off.reshape(-1).astype(np.int32)
        # the local mesh: this rank's elements (global vertex numbering), boundary codes of the
        # physical boundary, 0 on cut sides (overridden by the halo)
        self.quads = mesh.quads[self.local]
        self.verts = mesh.verts
        self._byte = byte
        self._boundary = boundary

    def local_bc(self, local_mesh):
        """Boundary codes of the local mesh's boundary edges (in its edge order)."""
        e = local_mesh.edges(1)
        g = self.local[e[:, 0]]
        s = e[:, 1]
        phys = self._boundary[g, s]
        return np.where(phys, (self._byte[g, s] >> 3) & 3, 0).astype(np.int32)


class Domain:
    """One rank's discretisation with its halo (wdg_wave_create_halo)."""

    def __init__(self, mesh, basis, bc, part, rank: int, precision="fp64", device: int = -1):
        import torch

        from . import dg

        if mesh.verts is None:
            raise WdgError(-1, "decomposition needs a mesh built from vertices")
        n = dg._gll_n(basis)
        self.plan = Plan(mesh, n, bc, part, rank)
        if len(self.plan.local) == 0:
            raise ValueError(f"rank {rank} owns no elements")
        self.rank, self.n = rank, n
        self.mesh = dg.Mesh2D.from_vertices(self.plan.verts, self.plan.quads)
        codes = self.plan.local_bc(self.mesh)
        self.precision = dg._precision(precision)
        h = C.c_void_p()
        p = self.plan
        check(lib().wdg_wave_create_halo(self.mesh._h, n, C.c_void_p(codes.ctypes.data), self.precision, device,
                                         len(p.halo_elem), C.c_void_p(p.halo_elem.ctypes.data),
                                         C.c_void_p(p.halo_side.ctypes.data), C.byref(h)), "wdg_wave_create_halo")
        self._h = h
        nd, hv = C.c_longlong(), C.c_longlong()
        check(lib().wdg_halo_info(h, C.byref(nd), C.byref(hv)))
        self.ndof, self.halo = nd.value, hv.value
        self.torch = torch
        self.dtype = torch.float32 if precision == "fp32" else torch.float64
        dev = torch.device("cuda", torch.cuda.current_device() if device < 0 else device)
        self.device = dev
        # every launch of this domain goes to torch's current stream, so collectives issued
        # through torch.distributed are ordered after the gathers and before the puts on the
        # device, with no host synchronisation
        self.stream = torch.cuda.current_stream(dev)
        check(lib().wdg_wave_set_stream(h, C.c_void_p(self.stream.cuda_stream)), "Domain stream")
        # the elements [0, split) read no halo trace (split: a multiple of 4, as the partial
        # stage launches need)
        self.split = (p.n_inner // 4) * 4
        self._send_idx = {r: torch.from_numpy(v).to(dev) for r, v in p.send.items()}
        self._send_buf = {r: torch.empty(3 * len(v), dtype=self.dtype, device=dev) for r, v in p.send.items()}
        self._recv_buf = {s: torch.empty(3 * n * cnt, dtype=self.dtype, device=dev) for s, (_, cnt) in p.recv.items()}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().wdg_wave_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------- state
    def upload(self, u_global) -> None:
        """The local elements' values of a global state (float64 numpy array)."""
        loc = np.ascontiguousarray(np.asarray(u_global, dtype=np.float64).reshape(-1, self.plan.nd)[self.plan.local])
        check(lib().wdg_state_upload(self._h, C.c_void_p(loc.ctypes.data)), "Domain.upload")

    def download(self, u_global) -> None:
        """Write the local elements' values into a global state (float64 numpy array)."""
        loc = np.zeros((len(self.plan.local), self.plan.nd))
        check(lib().wdg_state_download(self._h, C.c_void_p(loc.ctypes.data)), "Domain.download")
        u_global.reshape(-1, self.plan.nd)[self.plan.local] = loc

    # ------------------------------------------------------------- exchange pieces
    def gather(self, stage: int, dst: int):
        """The traces rank `dst` needs from the input buffer of RK stage `stage` (device tensor)."""
        idx, out = self._send_idx[dst], self._send_buf[dst]
        check(lib().wdg_halo_gather(self._h, _STAGE_BUFFER[stage], C.c_void_p(idx.data_ptr()), int(idx.numel()),
                                    C.c_void_p(out.data_ptr())), "halo gather")
        return out

    def put(self, stage: int, src: int, values) -> None:
        """Traces received from rank `src` into the halo of stage `stage`'s input buffer."""
        first, cnt = self.plan.recv[src]
        check(lib().wdg_halo_put(self._h, _STAGE_BUFFER[stage], 3 * self.n * first, C.c_void_p(values.data_ptr()),
                                 3 * self.n * cnt), "halo put")

    def stage(self, stage: int, dt: float, t: float = 0.0, F=None, omega: float = 0.0, acc=None,
              acc_c: float = 0.0, part=None) -> None:
        """RK stage `stage` of the step starting at t; optionally the WaveHoltz forcing F (device,
        the domain's precision) and, at stage 4, the filter acc += acc_c u (device FP64).
        part: None all elements; 0 those that read no halo trace (runs before the halo is
        filled); 1 the rest."""
        if part is None and F is None and acc is None:
            check(lib().wdg_rk4_stage(self._h, int(stage), float(dt)), "rk4 stage")
            return
        b, e = (0, self.ndof // self.plan.nd) if part is None else \
            ((0, self.split) if part == 0 else (self.split, self.ndof // self.plan.nd))
        check(lib().wdg_rk4_stage_elems(self._h, int(stage), float(dt), float(t),
                                        None if F is None else C.c_void_p(F.data_ptr()), float(omega),
                                        None if acc is None else C.c_void_p(acc.data_ptr()), float(acc_c), b, e),
              "rk4 stage")

    def set_state(self, u_local) -> None:
        """The resident state from this domain's own values (device FP64 tensor, local order)."""
        check(lib().wdg_state_upload(self._h, C.c_void_p(u_local.data_ptr())), "Domain.set_state")

    def local(self, u_global):
        """This domain's values of a global array (numpy), local element order."""
        return np.ascontiguousarray(np.asarray(u_global).reshape(-1, self.plan.nd)[self.plan.local]).reshape(-1)

    def sync(self) -> None:
        check(lib().wdg_wave_sync(self._h))

    def rk4_steps(self, dt: float, nsteps: int, exchange, overlap: bool = True) -> None:
        """nsteps of ode::RungeKutta4::step; exchange fills the stage's input halo (with
        overlap, its start / finish bracket the stage's halo-free part)."""
        for _ in range(nsteps):
            for st in range(5):
                stage_all([self], st, exchange, overlap, dt)


class Exchange:
    """A halo exchange in two halves: start(stage) sends and posts the receives, finish(stage)
    completes them and fills the halos; calling it does both."""

    def __init__(self, start, finish):
        self.start, self.finish = start, finish

    def __call__(self, stage):
        self.start(stage)
        self.finish(stage)


def local_exchange(domains):
    """Exchange among Domains of one process (one GPU): device copies.  Every Domain issues its
    work on torch's current stream, so gathers, copies and stages of all domains run in issue
    order without host synchronisation; a gather buffer is rewritten only by a later gather,
    issued after the copy that read it.  Everything happens in start()."""

    def start(stage):
        for d in domains:
            for r in d.plan.send:
                domains[r].put(stage, d.rank, d.gather(stage, r))

    return Exchange(start, lambda stage: None)


def stage_all(domains, st: int, exchange, overlap: bool = True, dt: float = 0.0, **kw) -> None:
    """RK stage st of every domain of this process with its halo exchange: with overlap, the
    elements that read no halo trace run between the exchange's start and finish."""
    if overlap and isinstance(exchange, Exchange):
        exchange.start(st)
        for d in domains:
            d.stage(st, dt, part=0, **kw)
        exchange.finish(st)
        for d in domains:
            d.stage(st, dt, part=1, **kw)
    else:
        exchange(st)
        for d in domains:
            d.stage(st, dt, **kw)


def step_all(domains, dt: float, nsteps: int, overlap: bool = True) -> None:
    """RK4 steps of Domains sharing one process: per stage, the exchange and every domain's stage."""
    ex = local_exchange(domains)
    for _ in range(nsteps):
        for st in range(5):
            stage_all(domains, st, ex, overlap, dt)


def dist_exchange(domain, group=None):
    """Exchange over torch.distributed: one send and one receive per neighbouring rank per stage,
    posted together.  With NCCL everything stays on the device and in stream order: the gathers
    run on torch's current stream, NCCL's sends wait for them there, req.wait() makes the
    current stream wait for the receives, and the puts and the stage follow; the host never
    waits.  Backends without CUDA tensors (gloo) move the traces through host buffers."""
    import torch
    import torch.distributed as dist

    on_device = dist.get_backend(group) == "nccl"
    host = {}
    if not on_device:
        host = {s: torch.empty(b.numel(), dtype=b.dtype) for s, b in domain._recv_buf.items()}

    pending = []

    def start(stage):
        ops = []
        for r in sorted(domain.plan.send):
            buf = domain.gather(stage, r)
            ops.append(dist.P2POp(dist.isend, buf if on_device else buf.cpu(), r, group))
        for s in sorted(domain.plan.recv):
            ops.append(dist.P2POp(dist.irecv, domain._recv_buf[s] if on_device else host[s], s, group))
        pending[:] = dist.batch_isend_irecv(ops) if ops else []

    def finish(stage):
        for req in pending:
            req.wait()
        pending.clear()
        for s in sorted(domain.plan.recv):
            domain.put(stage, s, domain._recv_buf[s] if on_device else host[s])

    return Exchange(start, finish)


def dist_allreduce(group=None, device=None):
    """Global sums over torch.distributed (the two FP64 sums of WaveHoltz's norm and error,
    source/linalg.cpp:102-131): a list of floats -> the list of their sums over all ranks."""
    import torch
    import torch.distributed as dist

    dev = device if dist.get_backend(group) == "nccl" else "cpu"

    def run(values):
        t = torch.tensor(values, dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().tolist()

    return run


class DomainWaveHoltz:
    """WaveHoltz (source/WaveHoltz.cpp:5-145) on one domain of a decomposed mesh.  T, dt and nt
    follow WaveHoltz::WaveHoltz (:5-30) with min_h of the whole mesh, so every rank steps alike.
    One forced period from W, with the filter started at 0.5 dt K(0) W, yields S W + pi0 by
    linearity (the first period from zero is pi0 itself); the filter's weights and the
    stage times are those of WaveHoltz::pi0 / S (:55-121)."""

    def __init__(self, domain: Domain, omega: float, mesh_min_h: float):
        import math

        self.d, self.omega = domain, float(omega)
        n = domain.n
        self.T = 2.0 * math.pi / self.omega
        dt0 = 0.5 * mesh_min_h / (n * n)
        self.nt = int(math.ceil(self.T / dt0))
        self.dt = self.T / self.nt
        self.ndof = domain.ndof

    def K(self, t: float) -> float:
        import math

        return self.omega / math.pi * (math.cos(self.omega * t) - 0.25)


def waveholtz_solve(whs, Fs, tol: float, maxit: int, exchange, allreduce, W=None):
    """The fixed-point loop of examples/waveholtz2d.cpp:165-185 on a decomposed mesh:
    W <- S W + pi0 until |W - W_prev| / |pi0| < tol (norms over the whole mesh, by `allreduce`).

    whs: this process's DomainWaveHoltz objects (one per rank under torch.distributed; every
    rank's when they share a process); Fs: their local load vectors (device, FP64); exchange(st)
    fills the input halo of RK stage st of all of them (dist_exchange, local_exchange);
    allreduce(list) -> global sums.  W: initial local iterates (default zero), overwritten.
    Returns (W list, iterations, residual)."""
    torch = whs[0].d.torch
    W = [torch.zeros(wh.ndof, dtype=torch.float64, device=wh.d.device) if W is None else W[i]
         for i, wh in enumerate(whs)]
    F = [f if wh.d.dtype == torch.float64 else f.to(wh.d.dtype) for f, wh in zip(Fs, whs)]
    acc = [torch.empty_like(w) for w in W]
    wh0 = whs[0]
    pz, res, it = None, float("inf"), 0
    zero = all(float(w.abs().max()) == 0.0 for w in W) if W else True
    for it in range(1, maxit + 1):
        for wh, w, a in zip(whs, W, acc):
            wh.d.set_state(w)
            torch.mul(w, 0.5 * wh0.dt * wh0.K(0.0), out=a)
        t = 0.0
        doms = [wh.d for wh in whs]
        for k in range(1, wh0.nt + 1):
            t1 = t + wh0.dt  # the step's end time, accumulated as ode::RungeKutta4::step does
            c = (0.5 if k == wh0.nt else 1.0) * wh0.dt * wh0.K(t1)
            for st in range(5):
                if isinstance(exchange, Exchange):
                    exchange.start(st)
                    for d, f, a in zip(doms, F, acc):
                        d.stage(st, wh0.dt, t, f, wh0.omega, a, c, part=0)
                    exchange.finish(st)
                    for d, f, a in zip(doms, F, acc):
                        d.stage(st, wh0.dt, t, f, wh0.omega, a, c, part=1)
                else:
                    exchange(st)
                    for d, f, a in zip(doms, F, acc):
                        d.stage(st, wh0.dt, t, f, wh0.omega, a, c)
            t = t1
        sums = [0.0, 0.0]
        for w, a in zip(W, acc):
            sums[0] += float(torch.sum((a - w) ** 2))
            sums[1] += float(torch.sum(a * a))
        dsum, nsum = allreduce(sums)
        if pz is None:
            # a zero start's first period is pi0; a warm start would need it separately
            if not zero:
                raise ValueError("waveholtz_solve starts from zero")
            pz = nsum ** 0.5
        for w, a in zip(W, acc):
            w.copy_(a)
        res = dsum ** 0.5 / pz
        if res < tol:
            break
    return W, it, res
