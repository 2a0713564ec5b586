"""Domain decomposition plans on the CPU: every halo slot receives exactly the neighbour trace
the undivided mesh's kernels would read, for contiguous and scattered partitions, in one
process and over two gloo ranks exchanging real messages."""
import os
import socket

import numpy as np
import pytest


@pytest.fixture(scope="module")
def W():
    from wavedg_b200 import build

    build.build()
    import wavedg_b200

    return wavedg_b200


def _mesh(W, nx=9, seed=3):
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(nx, 0.2, seed=seed)
    v, q = mg.scrambled(v, q, seed=seed + 1)
    m = W.Mesh2D.from_vertices(v, q)
    bc = np.random.default_rng(seed).integers(0, 3, size=m.n_edges(1)).astype(np.int32)
    return m, bc


def _check_halos(plans, U, fb, fc, n):
    """Build each rank's halo from the other ranks' send lists and compare with the trace the
    partner table of the undivided mesh points at."""
    nd = 3 * n * n
    stride = {0: 3, 1: -3, 2: 3 * n, 3: -3 * n}
    for r, p in plans.items():
        halo = np.zeros(3 * n * len(p.halo_elem))
        for s, (first, cnt) in p.recv.items():
            idx = plans[s].send[r]
            local = U[plans[s].local].ravel()
            vals = np.stack([local[idx + f] for f in range(3)], axis=1).ravel()
            assert len(vals) == 3 * n * cnt
            halo[3 * n * first: 3 * n * (first + cnt)] = vals
        for j, (le, f) in enumerate(zip(p.halo_elem, p.halo_side)):
            g = p.local[le]
            code = (int(fc[g]) >> (8 * int(f))) & 3
            for k in range(n):
                off = fb[g, f] + k * stride[code]
                np.testing.assert_array_equal(halo[3 * n * j + 3 * k: 3 * n * j + 3 * k + 3], U.ravel()[off: off + 3])
        assert (p.local >= 0).all()
    covered = np.sort(np.concatenate([p.local for p in plans.values()]))
    np.testing.assert_array_equal(covered, np.arange(len(U)))


@pytest.mark.parametrize("world,kind", [(2, "blocks"), (3, "blocks"), (4, "random")])
def test_plans_deliver_the_partner_traces(W, world, kind):
    from wavedg_b200 import decomp

    m, bc = _mesh(W)
    n = 4
    nel = m.n_elem()
    part = decomp.partition(nel, world) if kind == "blocks" else \
        np.random.default_rng(7).integers(0, world, size=nel).astype(np.int32)
    plans = {r: decomp.Plan(m, n, bc, part, r) for r in range(world)}
    fb, fc = decomp.partner_table(m, n, bc)
    U = np.random.default_rng(1).standard_normal((nel, 3 * n * n))
    _check_halos(plans, U, fb, fc, n)
    # every cut side is a halo slot on exactly one rank
    assert sum(len(p.halo_elem) for p in plans.values()) == sum(len(v) for p in plans.values() for v in p.send.values()) // n


def test_single_rank_and_uneven_partitions(W):
    from wavedg_b200 import decomp

    m, bc = _mesh(W)
    nel = m.n_elem()
    p = decomp.Plan(m, 3, bc, np.zeros(nel, dtype=np.int32), 0)
    assert len(p.halo_elem) == 0 and p.send == {} and p.recv == {}
    np.testing.assert_array_equal(p.local, np.arange(nel))
    # blocks differ in size by at most one element and cover every element once
    for world in (1, 2, 5, nel):
        part = decomp.partition(nel, world)
        counts = np.bincount(part, minlength=world)
        assert counts.sum() == nel and counts.max() - counts.min() <= 1
    # a rank that owns nothing sends and receives nothing
    part = np.where(np.arange(nel) < nel // 2, 0, 2).astype(np.int32)
    p1 = decomp.Plan(m, 3, bc, part, 1)
    assert len(p1.local) == 0 and p1.send == {} and p1.recv == {}


def test_local_boundary_codes(W):
    """Physical boundary sides keep their codes; cut sides become boundary sides of the local mesh."""
    from wavedg_b200 import decomp

    m, bc = _mesh(W)
    part = decomp.partition(m.n_elem(), 3)
    p = decomp.Plan(m, 3, bc, part, 1)
    lm = W.Mesh2D.from_vertices(p.verts, p.quads)
    codes = p.local_bc(lm)
    e = lm.edges(1)
    n_cut = len(p.halo_elem)
    assert len(codes) == len(e)
    phys = p._boundary[p.local[e[:, 0]], e[:, 1]]
    assert (~phys).sum() == n_cut
    # a halo side is a boundary side of the local mesh that is not a physical boundary side
    cut_sides = {(int(a), int(b)) for a, b in zip(p.halo_elem, p.halo_side)}
    assert cut_sides == {(int(a), int(b)) for (a, b), ph in zip(e[:, :2], phys) if not ph}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    import wavedg_b200 as W
    from wavedg_b200 import decomp

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m, bc = _mesh(W)
        n = 4
        part = decomp.partition(m.n_elem(), world)
        p = decomp.Plan(m, n, bc, part, rank)
        U = np.random.default_rng(1).standard_normal((m.n_elem(), 3 * n * n))
        local = torch.from_numpy(U[p.local].ravel().copy())
        halo = torch.zeros(3 * n * len(p.halo_elem), dtype=torch.float64)

        class HostDomain:
            """The exchange-facing side of decomp.Domain over host tensors (gloo)."""
            plan = p
            _recv_buf = {s: torch.zeros(3 * n * cnt, dtype=torch.float64) for s, (_, cnt) in p.recv.items()}

            def gather(self, stage, r):
                idx = torch.from_numpy(p.send[r].astype(np.int64))
                return torch.stack([local[idx + f] for f in range(3)], dim=1).reshape(-1).contiguous()

            def put(self, stage, s, values):
                first, cnt = p.recv[s]
                halo[3 * n * first: 3 * n * (first + cnt)] = values

            def sync(self):
                pass

        decomp.dist_exchange(HostDomain())(0)  # the exchange Domain.rk4_steps uses with NCCL
        fb, fc = decomp.partner_table(m, n, bc)
        stride = {0: 3, 1: -3, 2: 3 * n, 3: -3 * n}
        bad = 0
        for j, (le, f) in enumerate(zip(p.halo_elem, p.halo_side)):
            g = p.local[le]
            code = (int(fc[g]) >> (8 * int(f))) & 3
            for k in range(n):
                off = fb[g, f] + k * stride[code]
                bad += int(not np.array_equal(halo[3 * n * j + 3 * k: 3 * n * j + 3 * k + 3].numpy(), U.ravel()[off: off + 3]))
        q.put((rank, len(p.halo_elem), bad))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_halos(W):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=180) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, nhalo, bad in res:
        assert nhalo > 0 and bad == 0, (rank, nhalo, bad)


def _rcb_restated(centres, nparts):
    """Recursive coordinate bisection as source/Mesh2D.cpp:233-294 describes it (principal axis
    of the part's centres, smallest-prime-divisor equal-count cuts, new ranks in breadth-first
    order), with the y mean taken from y; for centres whose projections are all distinct."""
    e2p = np.zeros(len(centres), dtype=np.int32)
    queue = [np.arange(len(centres))]
    parts = [nparts]
    rank = 1
    while queue:
        ids, p = queue.pop(0), parts.pop(0)
        x = centres[ids]
        m = x.mean(axis=0)
        c = np.cov(x.T)
        vx, vy, cv = c[0, 0], c[1, 1], c[0, 1]
        if cv != 0.0:
            ex, ey = (np.sqrt((vx - vy) ** 2 + 4 * cv * cv) + vx - vy) / (2 * cv), 1.0
        else:
            ex, ey = (1.0, 0.0) if vx >= vy else (0.0, 1.0)
        pc = ex * (x[:, 0] - m[0]) + ey * (x[:, 1] - m[1])
        d = next(k for k in range(2, p + 1) if p % k == 0 and all(k % j for j in range(2, int(k ** 0.5) + 1)))
        order = ids[np.argsort(pc, kind="stable")]
        pos = [k * len(ids) // d for k in range(d + 1)]
        for k in range(1, d):  # the first piece keeps the part's rank
            e2p[order[pos[k]:pos[k + 1]]] = rank
            rank += 1
        if p // d > 1:
            for k in range(d):
                queue.append(order[pos[k]:pos[k + 1]])
                parts.append(p // d)
    return e2p


@pytest.mark.parametrize("world", [2, 3, 4, 6, 8, 9])
def test_rcb_partition_matches_its_restatement(W, world):
    from wavedg_b200 import decomp
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(12, 0.2, seed=world)
    v, q = mg.scrambled(v, q, seed=world + 1)
    m = W.Mesh2D.from_vertices(v, q)
    e2p = decomp.partition_mesh(m, world, "rcb")
    centres = v[q].mean(axis=1)
    want = _rcb_restated(centres, world)
    # ranks are equal as sets of elements (the restatement numbers them the same way)
    np.testing.assert_array_equal(e2p, want)
    sizes = np.bincount(e2p, minlength=world)
    assert sizes.min() > 0 and sizes.max() - sizes.min() <= 2
    np.testing.assert_array_equal(decomp.partition_mesh(m, world, "rcb"), e2p)


def test_rcb_cuts_a_square_into_quadrants_and_rcm_into_blocks(W):
    from wavedg_b200 import decomp

    m = W.Mesh2D.uniform_rect(16, -1.0, 1.0, 16, -1.0, 1.0)
    e2p = decomp.partition_mesh(m, 4, "rcb").reshape(16, 16)  # [row (y), column (x)]
    for r in range(4):
        rows, cols = np.nonzero(e2p == r)
        assert len(rows) == 64 and np.ptp(rows) == 7 and np.ptp(cols) == 7
    for world in (1, 3, 5, 16):
        e = decomp.partition_mesh(m, world, "rcm")
        sizes = np.bincount(e, minlength=world)
        assert sizes.min() > 0 and sizes.max() - sizes.min() <= 1


def test_partition_errors(W):
    from wavedg_b200 import decomp
    from wavedg_b200 import meshgen as mg

    m = W.Mesh2D.uniform_rect(4, -1.0, 1.0, 4, -1.0, 1.0)
    for bad in (0, 17):
        with pytest.raises(W.WdgError):
            decomp.partition_mesh(m, bad)
    # two squares with no shared edge: rcm cannot order a disconnected mesh
    v1, q1 = mg.uniform_rect(2, 0.0, 1.0, 2, 0.0, 1.0)
    v2, q2 = mg.uniform_rect(2, 2.0, 3.0, 2, 0.0, 1.0)
    m2 = W.Mesh2D.from_vertices(np.vstack([v1, v2]), np.vstack([q1, q2 + len(v1)]))
    with pytest.raises(W.WdgError, match="not connected"):
        decomp.partition_mesh(m2, 2, "rcm")
    assert len(np.unique(decomp.partition_mesh(m2, 2, "rcb"))) == 2


def _allreduce_worker(rank, world, port, q):
    import torch.distributed as dist

    from wavedg_b200 import decomp

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, decomp.dist_allreduce()([rank + 1.0, 0.5 * rank])))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_the_norms(W):
    """The WaveHoltz norm / error sums (source/linalg.cpp:102-131) over two gloo ranks."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_allreduce_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=180) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for _, sums in res:
        assert sums == [3.0, 0.5]
