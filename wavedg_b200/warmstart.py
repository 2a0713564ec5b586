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

    python -m wavedg_b200.warmstart --train 256 --epochs 100 --eval 128 --weights A.npz
    python -m wavedg_b200.warmstart --weights A.npz --finetune --data-seed 3000 --train 256 \
        --epochs 150 --lr 1e-3 --save B.npz --eval 0
    python -m wavedg_b200.warmstart --weights B.npz --eval 256 --plain 8 --json out.json
    python -m wavedg_b200.warmstart --time-batch 64          # period timing of the batch alone
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

OMEGA, SIGMA, NE, NCOLLOC = 20.0, 0.05, 128, 5

# the trained network shipped with the package (FNO(grid=512, width=32, modes=16, layers=4,
# hidden=64)); written by `--save` in the compact format below
PACKAGED_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "fno_waveholtz_c5.npz")


def save_weights(path: str, net, scale: float, meta: dict | None = None) -> None:
    """Compact weight file: the spectral tensors R* as float16 times a per-tensor power-of-two
    scale (their entries span a few decades below 1; 11 significant bits are far below what a
    warm start can resolve), every other parameter as float32, plus the output scale and a
    JSON record of how the network was trained."""
    out = {"__scale__": np.array(scale, dtype=np.float64)}
    for k, v in net.state_dict().items():
        if k.startswith("R"):
            e = int(np.ceil(np.log2(max(float(np.abs(v).max()), 1e-30)))) - 14  # max |v| / 2^e < 2^14
            out[k] = (v / np.float32(2.0 ** e)).astype(np.float16)
            out[k + ".exp2"] = np.array(e, dtype=np.int32)
        else:
            out[k] = v.astype(np.float32)
    if meta is not None:
        out["__meta__"] = np.array(json.dumps(meta))
    np.savez(path, **out)


def load_weights(path: str, net) -> float:
    """Load a file written by save_weights (or a plain float32 state dict with __scale__) into
    `net`; returns the output scale."""
    sd = dict(np.load(path))
    scale = float(sd.pop("__scale__"))
    sd.pop("__meta__", None)
    exps = {k[:-5]: int(sd.pop(k)) for k in [k for k in sd if k.endswith(".exp2")]}
    for k, e in exps.items():
        sd[k] = sd[k].astype(np.float32) * np.float32(2.0 ** e)
    net.load_state_dict(sd)
    return scale


def weights_meta(path: str) -> dict:
    sd = np.load(path)
    return json.loads(str(sd["__meta__"])) if "__meta__" in sd.files else {}


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
    """`nb` discretisations of the family's mesh per precision, batched (ne x ne elements,
    frequency omega; the defaults are the family above)."""

    def __init__(self, nb: int = 64, device: int = 0, ne: int = NE, omega: float = OMEGA):
        import torch

        from . import dg

        self.torch, self.nb, self.device, self.ne, self.omega = torch, nb, device, ne, omega
        self.mesh = dg.Mesh2D.uniform_rect(ne, -1.0, 1.0, ne, -1.0, 1.0)
        self.basis = dg.QuadratureRule.quadrature_rule(NCOLLOC, dg.QuadratureRule.GaussLobatto)
        self.bc = np.zeros(self.mesh.n_edges(1), dtype=np.int32)
        self.sys32 = [dg.WaveSystem(self.mesh, self.basis, self.bc, "fp32", device) for _ in range(nb)]
        self.sys64 = [dg.WaveSystem(self.mesh, self.basis, self.bc, "fp64", device) for _ in range(nb)]
        self.b32 = dg.WaveHoltzBatch(self.sys32, [omega] * nb)
        self.b64 = dg.WaveHoltzBatch(self.sys64, [omega] * nb)
        self.ndof = self.sys64[0].ndof

    def forcing(self, cs):
        t = self.torch
        out = []
        for i, (cx, cy) in enumerate(cs):
            F = t.zeros(self.ndof, dtype=t.float64, device="cuda")
            self.sys64[i % self.nb].load_gaussians([[cx, cy]], [SIGMA], [self.omega ** 2], 1.0, 0, False, out=F)
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


def make_dataset(fam: Family, count: int, seed: int, tol: float, G: int, net=None, scale: float = 1.0, log=print):
    """Solutions of `count` seeded problems on the G x G grid, plus their centres.  With a
    network, each solve starts from its prediction (fewer iterations to the same tolerance)."""
    from .fno import NodalGrid

    t = fam.torch
    rs = NodalGrid(fam.ne, NCOLLOC, G)
    cs = centers(count, seed)
    grids = t.empty((count, 3, G, G), dtype=t.float32, device="cuda")
    for b0 in range(0, count, fam.nb):
        blk = cs[b0:b0 + fam.nb]
        # a short last block is filled up to the batch size by repeating its problems (their
        # solutions are not kept twice)
        blk_full = np.resize(blk, (fam.nb, 2)) if len(blk) < fam.nb else blk
        t0 = time.perf_counter()
        W0 = predict(net, fam, blk_full, scale) if net is not None else None
        W, it32, _, res, st = fam.solve(fam.forcing(blk_full), tol, W0=W0, fp64_finish=False)
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


def predict(net, fam: Family, cs, scale: float, batch: int = 8):
    """Warm starts at the DG nodes of the family's mesh for the problems centred at cs
    (forward passes of `batch` problems at a time)."""
    from .fno import NodalGrid, inputs

    rs = NodalGrid(fam.ne, NCOLLOC, net.G)
    cs = np.asarray(cs, dtype=np.float64).reshape(-1, 2)
    out = []
    for b0 in range(0, len(cs), batch):
        y = net.forward(inputs(net.G, cs[b0:b0 + batch], SIGMA, 1.0))
        out += [rs.to_nodes(y[i], scale) for i in range(y.shape[0])]
    return out


def evaluate(net, fam: Family, count: int, seed: int, scale: float, n_plain: int = 4, arms=("cold", "warm"),
             log=print) -> dict:
    """Fresh problems to FP64 residual 1e-6: plain single FP64 solves (a sample of n_plain),
    batched cold, batched warm."""
    from . import dg

    t = fam.torch
    cs = centers(count, seed)
    res = {"problems": count, "tol": 1e-6}
    # plain FP64 WaveHoltz, one solve at a time (the reference's algorithm on the GPU)
    wh = dg.WaveHoltz(fam.omega, fam.mesh, fam.basis, fam.bc, True)
    Fp = fam.forcing(cs[:n_plain])
    t.cuda.synchronize()
    t0 = time.perf_counter()
    plain_W, plain_it, plain_r = [], [], []
    for F in Fp:
        Wp = t.zeros(fam.ndof, dtype=t.float64, device="cuda")
        _, it, r = wh.solve(F, 1e-6, 1000, W=Wp)
        plain_W.append(Wp)
        plain_it.append(it)
        plain_r.append(float(r))
    t.cuda.synchronize()
    tp = time.perf_counter() - t0
    res["plain_fp64"] = {"solves": n_plain, "seconds": tp, "solves_per_s": n_plain / tp,
                         "iterations": [int(i) for i in plain_it], "iterations_mean": float(np.mean(plain_it)),
                         "residuals": plain_r}
    log(f"  plain FP64: {n_plain} solves in {tp:.1f} s, iterations {plain_it}")
    for arm in arms:
        secs, it32s, it64s, errs, r64s = 0.0, [], [], [], []
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
            r64s += [float(r) for r in r64]
            if b0 == 0:
                for i in range(n_plain):
                    errs.append((W[i] - plain_W[i]).norm().item() / plain_W[i].norm().item())
        done = len(it32s)
        res[f"batched_{arm}"] = {"solves": done, "seconds": secs, "solves_per_s": done / secs,
                                 "fp32_iterations_mean": float(np.mean(it32s)),
                                 "fp64_iterations_mean": float(np.mean(it64s)),
                                 "fp64_residual_max": float(max(r64s)), "fp64_residuals": r64s,
                                 "all_converged": bool(max(r64s) < 1e-6),
                                 "rel_diff_vs_plain_fp64": float(max(errs)) if errs else None}
        log(f"  batched {arm}: {done} solves in {secs:.1f} s, FP32 iterations {np.mean(it32s):.1f}, "
            f"FP64 finish {np.mean(it64s):.1f}")
    base = res["plain_fp64"]["solves_per_s"]
    for arm in arms:
        res[f"speedup_batched_{arm}_vs_plain"] = res[f"batched_{arm}"]["solves_per_s"] / base
    return res


def time_batch(nb: int, periods: int = 3, precisions=("fp32", "fp64"), autotune: bool = True, log=print) -> dict:
    """Wall time of whole forced periods of an nb-solve batch of the family (fresh seeded
    sources), per precision: seconds per period, per solve-period, and DOF-stage updates/s."""
    import torch

    from . import dg

    mesh = dg.Mesh2D.uniform_rect(NE, -1.0, 1.0, NE, -1.0, 1.0)
    basis = dg.QuadratureRule.quadrature_rule(NCOLLOC, dg.QuadratureRule.GaussLobatto)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
    out = {}
    for prec in precisions:
        ss = [dg.WaveSystem(mesh, basis, bc, prec) for _ in range(nb)]
        b = dg.WaveHoltzBatch(ss, [OMEGA] * nb)
        F = []
        for i, c in enumerate(centers(nb, 9)):
            f = torch.zeros(ss[0].ndof, dtype=torch.float64, device="cuda")
            ss[i].load_gaussians([c], [SIGMA], [OMEGA ** 2], 1.0, 0, False, out=f)
            F.append(f)
        ms = b.autotune(64) if autotune else None
        W = [torch.zeros_like(f) for f in F]
        b.solve(F, 1e-30, 1, W=W)  # warm-up: one period (graph capture included)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.solve(F, 1e-30, periods, W=W)
        torch.cuda.synchronize()
        per = (time.perf_counter() - t0) / periods
        _, _, nt = b.params(0)
        rec = {"solves": nb, "launch": b.launch_config(), "autotune_ms_per_step": ms, "seconds_per_period": per,
               "ms_per_solve_period": per / nb * 1e3, "dof_stage_per_s": nb * ss[0].ndof * 5 * nt / per}
        log(f"  {prec}: {nb} solves, {rec['launch']}, {per:.3f} s per period = {rec['ms_per_solve_period']:.1f} ms "
            f"per solve-period, {rec['dof_stage_per_s']:.3e} DOF-stage/s")
        out[prec] = rec
        del b, ss
    return out


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
    ap.add_argument("--finetune", action="store_true",
                    help="load --weights, train further on fresh solutions (warm-started by the network), save")
    ap.add_argument("--data-seed", type=int, default=None, help="seed of the training sources (default 1000 + seed)")
    ap.add_argument("--lr", type=float, default=2e-3, help="peak learning rate")
    ap.add_argument("--save", default=None, help="save the trained network here (default: --weights)")
    ap.add_argument("--data-net", default=None,
                    help="weights of a network whose predictions start the training-data solves")
    ap.add_argument("--arms", default="cold,warm", help="batched arms evaluated (cold, warm)")
    ap.add_argument("--time-batch", type=int, default=0, help="only time whole periods of a batch of this many solves")
    ap.add_argument("--periods", type=int, default=3, help="--time-batch: periods timed")
    ap.add_argument("--precision", choices=["fp32", "fp64", "both"], default="both", help="--time-batch precision")
    ap.add_argument("--no-autotune", action="store_true", help="--time-batch: default launch shape")
    a = ap.parse_args(argv)

    if a.time_batch:
        prec = ("fp32", "fp64") if a.precision == "both" else (a.precision,)
        out = time_batch(a.time_batch, a.periods, prec, not a.no_autotune)
        print(json.dumps(out), flush=True)
        return

    from .fno import FNO

    fam = Family(a.batch)
    net = FNO(grid=a.grid, width=32, modes=16, layers=4, hidden=64, seed=a.seed)
    out = {"family": "waveholtz_128x128_P4_omega20_outflow", "grid": a.grid,
           "fno": {"layers": 4, "width": 32, "modes": 16, "hidden": 64}}
    loaded = bool(a.weights and os.path.exists(a.weights))
    if loaded:
        scale = load_weights(a.weights, net)
        out["trained"] = "loaded"
    if not loaded or a.finetune:
        t0 = time.perf_counter()
        dseed = 1000 + a.seed if a.data_seed is None else a.data_seed
        # the network whose predictions start the data solves (they only save iterations:
        # every solve still runs to the training tolerance)
        dnet, dscale = (net, scale) if loaded else (None, 1.0)
        if a.data_net:
            dnet = FNO(grid=a.grid, width=32, modes=16, layers=4, hidden=64, seed=a.seed)
            dscale = load_weights(a.data_net, dnet)
        cs, grids = make_dataset(fam, a.train, dseed, a.train_tol, a.grid, dnet, dscale)
        del dnet
        if not loaded:
            scale = math.sqrt(grids.square().mean().item())
        grids /= scale
        gen = time.perf_counter() - t0
        hist, ttrain = train(net, cs, grids, a.epochs, lr=a.lr, seed=a.seed, symmetries=not a.no_symmetries)
        out["data"] = {"solutions": a.train, "seed": dseed, "tol": a.train_tol, "seconds": gen,
                       "symmetries": 1 if a.no_symmetries else 8, "warm_started": loaded or bool(a.data_net)}
        out["training"] = {"epochs": a.epochs, "lr": a.lr, "seconds": ttrain, "rel_rms_error": hist,
                           "finetune": loaded, "from_scratch": not loaded}
        del grids
        dst = a.save or a.weights
        if dst:
            meta = {"fno": out["fno"], "grid": a.grid, "family": out["family"], "data": out["data"],
                    "training": {k: v for k, v in out["training"].items() if k != "rel_rms_error"},
                    "final_rel_rms_error": hist[-1], "seed": a.seed}
            save_weights(dst, net, scale, meta)
    if a.eval:
        out["eval"] = evaluate(net, fam, a.eval, 5000 + a.seed, scale, a.plain, arms=tuple(a.arms.split(",")))
    print(json.dumps(out), flush=True)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
