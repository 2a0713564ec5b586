"""Learned warm start for batched WaveHoltz on the single-solve Helmholtz family.

The family: 128 x 128 uniform quads of [-1, 1]^2, P = 4, outflow boundary, omega = 20,
forcing f = omega^2 exp(-|x - x0|^2 / (2 0.05^2)) with x0 uniform in [-0.5, 0.5]^2.

Pipeline (all on one GPU, all through this library's kernels):
  data      batched WaveHoltz solves (FP32 stepping, FP64 filter/residual) of seeded x0 to a
            training tolerance, resampled from the DG nodes to the FNO grid (exact element
            polynomials), scaled to unit RMS;
  train     the FNO (fno.FNO, BF16 operands, FP32 accumulation, hand-written backward),
            Adam with a cosine learning-rate schedule, MSE on the grid, each sample moved by a
            random symmetry of the square (eight pairs per solve);
  evaluate  fresh seeded problems solved three ways, each to the same FP64 residual 1e-6:
            plain FP64 WaveHoltz one solve at a time (the baseline), batched FP32 +
            FP64 finish from zero, and the same from the network's prediction.  The plain
            fixed-point iteration decides convergence in every arm.

    python -m wavedg_b200.warmstart --train 256 --epochs 20 --eval 64 --weights W.npz --json out.json
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

OMEGA, SIGMA, NE, NCOLLOC = 20.0, 0.05, 128, 5


def centers(count: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-0.5, 0.5, size=(count, 2))


# The family is invariant under the eight symmetries of the square (uniform mesh of [-1, 1]^2,
# the same boundary code on every wall, source centres drawn from a symmetric box): the
# solution for the source at R c is (p, v)(x) -> (p(R^T x), R v(R^T x)).  Symmetry k applies,
# in this order, x -> -x (bit 0), y -> -y (bit 1), x <-> y (bit 2).  The discrete operator
# shares them, so one solve gives eight training pairs.
def sym_centers(cs, k: int) -> np.ndarray:
    c = np.array(cs, dtype=np.float64).reshape(-1, 2)
    if k & 1:
        c[:, 0] = -c[:, 0]
    if k & 2:
        c[:, 1] = -c[:, 1]
    if k & 4:
        c = c[:, ::-1].copy()
    return c


def sym_grid(g, k: int):
    """Symmetry k of grid fields g[..., d, iy, ix] (d: p, v_x, v_y; torch tensor)."""
    import torch

    if k & 1:
        g = torch.flip(g, dims=(-1,))
        g = torch.stack((g[..., 0, :, :], -g[..., 1, :, :], g[..., 2, :, :]), dim=-3)
    if k & 2:
        g = torch.flip(g, dims=(-2,))
        g = torch.stack((g[..., 0, :, :], g[..., 1, :, :], -g[..., 2, :, :]), dim=-3)
    if k & 4:
        g = g.transpose(-1, -2)
        g = torch.stack((g[..., 0, :, :], g[..., 2, :, :], g[..., 1, :, :]), dim=-3)
    return g.contiguous()


def sym_nodes(u, ne: int, n: int, k: int) -> np.ndarray:
    """Symmetry k of a DG state of the uniform ne x ne mesh (element ex + ne ey, node a + n b,
    fields p, v_x, v_y interleaved per node; numpy)."""
    q = np.asarray(u).reshape(ne, ne, n, n, 3).copy()  # [ey, ex, b, a, d]
    if k & 1:
        q = q[:, ::-1, :, ::-1, :].copy()
        q[..., 1] *= -1
    if k & 2:
        q = q[::-1, :, ::-1, :, :].copy()
        q[..., 2] *= -1
    if k & 4:
        q = q.transpose(1, 0, 3, 2, 4)[..., [0, 2, 1]].copy()
    return q.reshape(-1)


class Family:
    """`nb` discretisations of the family's mesh per precision, batched."""

    def __init__(self, nb: int = 64, device: int = 0):
        import torch

        from . import dg

        self.torch, self.nb, self.device = torch, nb, device
        self.mesh = dg.Mesh2D.uniform_rect(NE, -1.0, 1.0, NE, -1.0, 1.0)
        self.basis = dg.QuadratureRule.quadrature_rule(NCOLLOC, dg.QuadratureRule.GaussLobatto)
        self.bc = np.zeros(self.mesh.n_edges(1), dtype=np.int32)
        self.sys32 = [dg.WaveSystem(self.mesh, self.basis, self.bc, "fp32", device) for _ in range(nb)]
        self.sys64 = [dg.WaveSystem(self.mesh, self.basis, self.bc, "fp64", device) for _ in range(nb)]
        self.b32 = dg.WaveHoltzBatch(self.sys32, [OMEGA] * nb)
        self.b64 = dg.WaveHoltzBatch(self.sys64, [OMEGA] * nb)
        self.ndof = self.sys64[0].ndof

    def forcing(self, cs):
        t = self.torch
        out = []
        for i, (cx, cy) in enumerate(cs):
            F = t.zeros(self.ndof, dtype=t.float64, device="cuda")
            self.sys64[i % self.nb].load_gaussians([[cx, cy]], [SIGMA], [OMEGA ** 2], 1.0, 0, False, out=F)
            out.append(F)
        return out

    def solve(self, F, tol, W0=None, fp64_finish=True, maxit=1000, tol32=3e-6):
        """Batched FP32 solve to max(tol, tol32) (FP32 rounding puts a floor near 2e-6 under
        the residual; the stall rule ends a solve that reaches it) then, if asked, the FP64
        batch from its iterates to `tol`.
        Returns (W list, FP32 iterations, FP64 iterations, FP64 residuals, status)."""
        t = self.torch
        n = len(F)
        assert n == self.nb
        W = [t.zeros(self.ndof, dtype=t.float64, device="cuda") if W0 is None else W0[i].clone() for i in range(n)]
        warm = None if W0 is None else [1] * n
        W, it32, r32, s32 = self.b32.solve(F, max(tol, tol32), maxit, W=W, warm=warm, stall_limit=3)
        if not fp64_finish:
            return W, it32, np.zeros_like(it32), r32, s32
        # the FP32 batch measured |pi0| (FP64 sums): the FP64 finish starts from W at once
        W, it64, r64, s64 = self.b64.solve(F, tol, maxit, W=W, warm=[1] * n, pi0_norm=self.b32.pi0_norm)
        return W, it32, it64, r64, s64


def make_dataset(fam: Family, count: int, seed: int, tol: float, G: int, log=print):
    """Solutions of `count` seeded problems on the G x G grid, plus their centres."""
    from .fno import NodalGrid

    t = fam.torch
    rs = NodalGrid(NE, NCOLLOC, G)
    cs = centers(count, seed)
    grids = t.empty((count, 3, G, G), dtype=t.float32, device="cuda")
    for b0 in range(0, count, fam.nb):
        blk = cs[b0:b0 + fam.nb]
        pad = fam.nb - len(blk)
        blk_full = np.concatenate([blk, blk[:pad]]) if pad else blk
        t0 = time.perf_counter()
        W, it32, _, res, st = fam.solve(fam.forcing(blk_full), tol, fp64_finish=False)
        t.cuda.synchronize()
        log(f"  data {b0 + len(blk)}/{count}: FP32 iterations {int(it32.min())}-{int(it32.max())}, "
            f"{time.perf_counter() - t0:.1f} s")
        for i in range(len(blk)):
            grids[b0 + i] = rs.to_grid(W[i], 1.0)
    return cs, grids


def train(net, cs, grids, epochs: int, batch: int = 4, lr: float = 2e-3, seed: int = 0, symmetries: bool = True,
          log=print):
    """Adam with a cosine schedule on the MSE; with `symmetries`, every sample of a batch is
    moved by a random one of the square's eight symmetries (source and solution alike)."""
    from .fno import inputs

    t = net.torch
    n = len(cs)
    steps = epochs * ((n + batch - 1) // batch)
    rng = np.random.default_rng(seed)
    k, hist = 0, []
    t0 = time.perf_counter()
    for ep in range(epochs):
        order = rng.permutation(n)
        tot = 0.0
        for b0 in range(0, n, batch):
            idx = order[b0:b0 + batch]
            if symmetries:
                ks = rng.integers(0, 8, size=len(idx))
                inp = inputs(net.G, np.concatenate([sym_centers(cs[i], int(q)) for i, q in zip(idx, ks)]), SIGMA, 1.0)
                tgt = t.stack([sym_grid(grids[int(i)], int(q)) for i, q in zip(idx, ks)]).contiguous()
            else:
                inp = inputs(net.G, cs[idx], SIGMA, 1.0)
                tgt = grids[t.from_numpy(idx).to("cuda")].contiguous()
            y = net.forward(inp, keep=True)
            sse, dy = net.mse(y, tgt)
            net.backward(dy)
            k += 1
            net.adam_step(lr=lr * 0.5 * (1 + math.cos(math.pi * k / steps)))
            tot += sse.item()
        rel = math.sqrt(tot / grids.square().sum().item())
        hist.append(rel)
        log(f"  epoch {ep + 1}/{epochs}: relative RMS error {rel:.3e} ({time.perf_counter() - t0:.0f} s)")
    t.cuda.synchronize()
    return hist, time.perf_counter() - t0


def predict(net, fam: Family, cs, scale: float):
    """Warm starts at the DG nodes of the family's mesh for the problems centred at cs."""
    from .fno import NodalGrid, inputs

    rs = NodalGrid(NE, NCOLLOC, net.G)
    out = []
    for c in cs:
        y = net.forward(inputs(net.G, np.asarray([c]), SIGMA, 1.0))
        out.append(rs.to_nodes(y[0], scale))
    return out


def evaluate(net, fam: Family, count: int, seed: int, scale: float, n_plain: int = 4, log=print) -> dict:
    """Fresh problems to FP64 residual 1e-6: plain single FP64 solves (a sample of n_plain),
    batched cold, batched warm."""
    from . import dg

    t = fam.torch
    cs = centers(count, seed)
    res = {"problems": count, "tol": 1e-6}
    # plain FP64 WaveHoltz, one solve at a time (the reference's algorithm on the GPU)
    wh = dg.WaveHoltz(OMEGA, fam.mesh, fam.basis, fam.bc, True)
    Fp = fam.forcing(cs[:n_plain])
    t.cuda.synchronize()
    t0 = time.perf_counter()
    plain_W, plain_it = [], []
    for F in Fp:
        Wp = t.zeros(fam.ndof, dtype=t.float64, device="cuda")
        _, it, _ = wh.solve(F, 1e-6, 1000, W=Wp)
        plain_W.append(Wp)
        plain_it.append(it)
    t.cuda.synchronize()
    tp = time.perf_counter() - t0
    res["plain_fp64"] = {"solves": n_plain, "seconds": tp, "solves_per_s": n_plain / tp,
                         "iterations_mean": float(np.mean(plain_it))}
    log(f"  plain FP64: {n_plain} solves in {tp:.1f} s, iterations {plain_it}")
    for arm in ("cold", "warm"):
        secs, it32s, it64s, errs = 0.0, [], [], []
        for b0 in range(0, count, fam.nb):
            blk = cs[b0:b0 + fam.nb]
            if len(blk) < fam.nb:
                break
            F = fam.forcing(blk)
            t.cuda.synchronize()
            t0 = time.perf_counter()
            W0 = predict(net, fam, blk, scale) if arm == "warm" else None
            W, it32, it64, r64, st = fam.solve(F, 1e-6, W0=W0)
            t.cuda.synchronize()
            secs += time.perf_counter() - t0
            assert (st == 0).all() and (r64 < 1e-6).all(), (st, r64)
            it32s += it32.tolist()
            it64s += it64.tolist()
            if b0 == 0:
                for i in range(n_plain):
                    errs.append((W[i] - plain_W[i]).norm().item() / plain_W[i].norm().item())
        done = len(it32s)
        res[f"batched_{arm}"] = {"solves": done, "seconds": secs, "solves_per_s": done / secs,
                                 "fp32_iterations_mean": float(np.mean(it32s)),
                                 "fp64_iterations_mean": float(np.mean(it64s)),
                                 "rel_diff_vs_plain_fp64": float(max(errs)) if errs else None}
        log(f"  batched {arm}: {done} solves in {secs:.1f} s, FP32 iterations {np.mean(it32s):.1f}, "
            f"FP64 finish {np.mean(it64s):.1f}")
    base = res["plain_fp64"]["solves_per_s"]
    res["speedup_batched_cold_vs_plain"] = res["batched_cold"]["solves_per_s"] / base
    res["speedup_batched_warm_vs_plain"] = res["batched_warm"]["solves_per_s"] / base
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=256, help="training solutions")
    ap.add_argument("--train-tol", type=float, default=1e-4)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--eval", type=int, default=64, help="fresh problems (a multiple of --batch)")
    ap.add_argument("--plain", type=int, default=4, help="plain FP64 single solves timed")
    ap.add_argument("--batch", type=int, default=64, help="solves per batched launch")
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--weights", default=None, help="load (if present) / save the network here")
    ap.add_argument("--json", default=None)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-symmetries", action="store_true", help="train without the square's symmetries")
    a = ap.parse_args(argv)
    import os

    from .fno import FNO

    fam = Family(a.batch)
    net = FNO(grid=a.grid, width=32, modes=16, layers=4, hidden=64, seed=a.seed)
    out = {"family": "waveholtz_128x128_P4_omega20_outflow", "grid": a.grid,
           "fno": {"layers": 4, "width": 32, "modes": 16, "hidden": 64}}
    if a.weights and os.path.exists(a.weights):
        sd = dict(np.load(a.weights))
        scale = float(sd.pop("__scale__"))
        net.load_state_dict(sd)
        out["trained"] = "loaded"
    else:
        t0 = time.perf_counter()
        cs, grids = make_dataset(fam, a.train, 1000 + a.seed, a.train_tol, a.grid)
        scale = math.sqrt(grids.square().mean().item())
        grids /= scale
        gen = time.perf_counter() - t0
        hist, ttrain = train(net, cs, grids, a.epochs, seed=a.seed, symmetries=not a.no_symmetries)
        out["data"] = {"solutions": a.train, "tol": a.train_tol, "seconds": gen,
                       "symmetries": 1 if a.no_symmetries else 8}
        out["training"] = {"epochs": a.epochs, "seconds": ttrain, "rel_rms_error": hist}
        del grids
        if a.weights:
            sd = net.state_dict()
            sd["__scale__"] = np.array(scale)
            np.savez(a.weights, **sd)
    out["eval"] = evaluate(net, fam, a.eval, 5000 + a.seed, scale, a.plain)
    print(json.dumps(out), flush=True)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
