#!/usr/bin/env python
"""Benchmark: DOF-stage updates/s of the fused RK4 stage kernel on the
512 x 512, P = 4 perturbed-quad workload (19.7M DOF), FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One timed step = one RK4 time step = 5 fused stage launches on the resident
state.  K steps are timed with CUDA events on the launching stream, bracketed
by barrier + synchronize; the maximum over ranks is reported.  Under torchrun
(N > 1) each rank runs an independent replica of the workload (weak scaling;
a single mesh is not partitioned).  Rank 0 prints one JSON line.

--impl reference times the reference's own CPU code (oracle/_ref, compiled from
its sources) on the same workload, rank 0 only, one thread.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-stage updates/s & HBM %; WaveHoltz solves/s at 1e-6, learned vs plain"
UNIT = "DOF-stage/s"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0  # GB/s, used only when MEASURED_PEAKS.json is absent
REF_TIME_BUDGET = 150.0  # seconds of reference CPU work in --impl reference
LEGS = ("waveholtz_c3", "learned_warm_start", "exact_quadrature", "advection", "euler", "decomposition",
        "waveholtz_config4")
T_START = time.perf_counter()


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=512, help="elements per direction")
    ap.add_argument("--P", type=int, default=4, help="polynomial degree (n_colloc = P + 1)")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the FP32 and WaveHoltz companion measurements")
    ap.add_argument("--no-waveholtz", action="store_true", help="skip the WaveHoltz solve measurement")
    ap.add_argument("--ref-procs", type=int, default=0, help="--impl reference: host processes (0: one per core)")
    ap.add_argument("--tile", type=int, default=0, help="elements per block (0: autotune)")
    ap.add_argument("--stages", type=int, default=0, help="pipeline depth with --tile (0: default)")
    ap.add_argument("--legs", default="", help=f"companion measurements to run (comma list of {','.join(LEGS)}; "
                    "default: all)")
    ap.add_argument("--budget", type=float, default=1200.0,
                    help="seconds the whole run should take; the batched-solve leg stops its FP32 phase in time "
                         "(0: no limit)")
    ap.add_argument("--kernel", choices=["auto", "warp", "tiled", "ws"], default="auto",
                    help="fused-kernel family (auto: the autotuner picks)")
    return ap.parse_args()


# --------------------------------------------------------------- workload
def workload(n: int, P: int, seed: int = 2024):
    """Config: n x n quads on [-1,1]^2, interior vertices perturbed by U(-0.2h, 0.2h), outflow
    boundaries, initial p = sum of 8 Gaussian pulses (centres U[-0.8,0.8]^2, widths U[0.03,0.1],
    amplitudes N(0,1)), u = v = 0; dt = 0.1 min_h / (P+1)^2."""
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(n, 0.2, seed=seed)
    rng = np.random.default_rng(seed + 1)
    centers = rng.uniform(-0.8, 0.8, size=(8, 2))
    sigmas = rng.uniform(0.03, 0.1, size=8)
    amps = rng.standard_normal(8)
    return v, q, centers, sigmas, amps


def algorithmic_bytes_per_step(ndof: int, nel: int, real: int) -> int:
    """Per RK4 step: stage 0 reads u, writes du and u'; stages 1-4 also read du.
    Plus the 64-byte corner block of every element per stage."""
    return ndof * real * (3 + 4 * 4) + 5 * 64 * nel


def peak_hbm():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of the GPU's clocks and throttle reasons during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
            # wait (at most 5 s) for the first sample so the timed region is covered
            t0 = time.time()
            while time.time() - t0 < 5 and os.path.getsize(self.file.name) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.file is None:
            return None
        try:
            self.file.flush()
            rows = [r.split(", ") for r in open(self.file.name).read().strip().splitlines()]
            os.unlink(self.file.name)
        except Exception:
            return None
        rows = [r for r in rows if len(r) >= 9 and (self.uuid is None or self.uuid in r[0])]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].strip().replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].strip().replace(".", "").isdigit())
                if any(r[3].strip().replace(".", "").isdigit() for r in rows) else None}


# ------------------------------------------------------------ our arm
def run_ours(args, rank, world, local_rank):
    import torch

    import wavedg_b200 as W

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local_rank])
        torch.cuda.synchronize()

    v, q, centers, sigmas, amps = workload(args.n, args.P)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(args.P + 1, W.QuadratureRule.GaussLobatto)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
    dt = 0.1 * mesh.min_h() / (args.P + 1) ** 2
    stream = torch.cuda.current_stream()

    def measure(precision, steps, warmup, tile=0):
        sys_ = W.WaveSystem(mesh, basis, bc, precision=precision, device=local_rank)
        sys_.set_stream(stream)
        u0 = torch.zeros(sys_.ndof, dtype=torch.float64, device="cuda")
        sys_.load_gaussians(centers, sigmas, amps, 1.0, 0, True, out=u0)
        sys_.upload(u0)
        if args.kernel == "warp":
            sys_.set_kernel(0)
        elif args.kernel in ("tiled", "ws") or tile:
            sys_.set_kernel(2 if args.kernel == "ws" else 1)
            if args.stages:
                sys_.set_stages(args.stages)
            if tile:
                sys_.tile = tile
        else:
            sys_.autotune(4)  # kernel family, elements per block and pipeline depth, timed on this GPU
        t = sys_.step_state(dt, 0.0, warmup)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t = sys_.step_state(dt, t, steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        sys_.sync()
        energy = sys_.energy()
        return sys_, ms, energy, t

    dev_props = torch.cuda.get_device_properties(local_rank)
    uuid = str(getattr(dev_props, "uuid", "")) or None
    with ClockSampler(uuid) as clk:
        sys_, ms, energy, t_end = measure(args.precision, args.steps, args.warmup, args.tile)
    clocks = clk.summary()
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    ndof, nel = sys_.ndof, mesh.n_elem()
    real = 8 if args.precision == "fp64" else 4
    ms_step = ms / args.steps
    value = world * ndof * 5 * args.steps / (ms / 1e3)

    # e2e: the reference-facing C-ABI call with pinned host buffers, one RK4 step per call
    e2e_steps = max(1, min(args.e2e_steps, args.steps))
    host = torch.empty(ndof, dtype=torch.float64, pin_memory=True)
    host.copy_(torch.from_numpy(sys_.download()))
    hn = host.numpy()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sys_.rk4_steps(hn, dt, 0.0, 1)  # warm the staging path
    barrier()
    e0.record(stream)
    tt = 0.0
    for _ in range(e2e_steps):
        tt = sys_.rk4_steps(hn, dt, tt, 1)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_ms = float(e2e_t.item())
    e2e_value = world * ndof * 5 * e2e_steps / (e2e_ms / 1e3)

    # roofline of the stage kernel (the only kernel in the timed region, 5 launches per step):
    # average algorithmic bytes per launch / average launch time, both from the timed steps
    peak, peak_kind = peak_hbm()
    bytes_step = algorithmic_bytes_per_step(ndof, nel, real)
    bytes_launch = bytes_step / 5
    launch_s = ms_step / 5 / 1e3
    achieved = bytes_launch / launch_s / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")
    if os.path.exists(prof) and args.n == 512 and args.P == 4:
        try:
            traffic = json.load(open(prof)).get(f"{args.precision}_bytes_per_launch_512")
        except Exception:
            traffic = None
    kernel_name = {"ws": "ws_stage_kernel", "tiled": "stage_kernel", "warp": "warp_stage_kernel"}.get(
        sys_.launch_config()["kernel"], "stage_kernel")

    extra = {"energy_final": energy, "t_final": t_end, "dt": dt, "launch": sys_.launch_config(), "peak_kind": peak_kind}
    if not args.no_extras and args.precision == "fp64":
        s32, ms32, _, _ = measure("fp32", args.steps, args.warmup)
        b32 = algorithmic_bytes_per_step(ndof, nel, 4)
        extra["fp32"] = {"value": world * ndof * 5 * args.steps / (ms32 / 1e3), "unit": UNIT,
                         "ms_per_step": ms32 / args.steps,
                         "hbm_gbs": b32 / (ms32 / args.steps / 1e3) / 1e9,
                         "frac": b32 / (ms32 / args.steps / 1e3) / 1e9 / peak}
        del s32

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(v, q, bc, args.P + 1, dt, sys_.download())

    # single-GPU companion measurements: skipped under torchrun so that a multi-GPU run holds
    # its GPUs only for the replicated RK4 measurement
    def companion(name, fn, *a, **kw):
        # a companion leg that fails is reported in its place; the main measurement stands
        try:
            extra[name] = fn(*a, **kw)
        except Exception as e:  # noqa: BLE001
            extra[name] = {"error": f"{type(e).__name__}: {e}"}

    legs = set(args.legs.split(",")) if args.legs else set(LEGS)
    want = lambda name: name in legs and not args.no_extras and args.precision == "fp64" and world == 1  # noqa: E731
    wh_ok = not args.no_waveholtz
    if want("waveholtz_c3") and wh_ok:
        companion("waveholtz_c3", waveholtz_c3, local_rank)
    if want("learned_warm_start") and wh_ok:
        companion("learned_warm_start", learned_warm_start, local_rank)
    if want("exact_quadrature"):
        companion("exact_quadrature", exact_quadrature, local_rank, cpu_leg=not args.no_cpu_baseline)
    if want("advection"):
        companion("advection", advection, local_rank, cpu_leg=not args.no_cpu_baseline)
    if want("euler"):
        companion("euler", euler, local_rank, cpu_leg=not args.no_cpu_baseline)
    if want("decomposition"):
        companion("decomposition", decomposition, local_rank)
    if want("waveholtz_config4") and wh_ok:
        # last: its FP32 phase gets what is left of the run's time budget (0: no limit), keeping
        # about three minutes for its FP64 finish and the plain-FP64 periods.  All 64 solves
        # take about 21 minutes on one B200, more than a default run's budget: with a budget the
        # leg solves the first 32 problems of the same seeded draw (about 7 minutes)
        left = args.budget - (time.perf_counter() - T_START) - 180.0 if args.budget > 0 else 1e9
        count = 64 if args.budget <= 0 or left > 1500.0 else 32
        companion("waveholtz_config4", waveholtz_config4, local_rank, deadline=max(60.0, left), count=count)


    if dist is not None:
        dist.barrier(device_ids=[local_rank])
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32",
        "data": "synthetic: seeded perturbed quad mesh and 8-Gaussian initial pressure (no dataset)",
        "config": {"workload": f"rk4_{args.precision}_{args.n}x{args.n}_P{args.P}_perturbed_outflow",
                   "elements": nel, "ndof": ndof, "P": args.P, "step": "1 RK4 step = 5 fused stage launches",
                   "l2": "inputs larger than L2 (three 157 MB state buffers rotate)",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": kernel_name, "bytes_per_launch": bytes_launch,
                     "launch_us": launch_s * 1e6, "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": ndof * 8, "d2h_bytes_per_step": ndof * 8,
                "steps": e2e_steps, "api": "wdg_rk4_steps(host pinned u, nsteps=1)"},
        "gpu_launches": 5 * args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "extra": extra,
    }
    print(json.dumps(out), flush=True)


def waveholtz_c3(device: int, seed: int = 3) -> dict:
    """One WaveHoltz Helmholtz solve on 128 x 128 uniform quads of [-1, 1]^2, P = 4, outflow
    boundary, omega = 20, f = omega^2 exp(-|x - x0|^2 / (2 0.05^2)) with x0 seeded in
    [-0.5, 0.5]^2, from a zero guess to 1e-6 relative residual.
      fp64        FP64 stepping throughout (the plain method);
      fp32_fp64   FP32 stepping (FP64 filter / residual) to 3e-6, where FP32 rounding starts to
                  floor the residual, then FP64 iterations from that iterate to 1e-6 -- the
                  plain iteration decides convergence.
    Wall time of the solve calls (host-synchronous: they read the residual every iteration)."""
    import torch

    import wavedg_b200 as W

    x0 = np.random.default_rng(seed).uniform(-0.5, 0.5, size=2)
    omega = 20.0
    mesh = W.Mesh2D.uniform_rect(128, -1.0, 1.0, 128, -1.0, 1.0)
    basis = W.QuadratureRule.quadrature_rule(5, W.QuadratureRule.GaussLobatto)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
    s64 = W.WaveSystem(mesh, basis, bc, precision="fp64", device=device)
    s32 = W.WaveSystem(mesh, basis, bc, precision="fp32", device=device)
    wh64 = W.WaveHoltz(omega, mesh, basis, bc, True, system=s64)
    wh32 = W.WaveHoltz(omega, mesh, basis, bc, True, precision="fp32", system=s32)
    F = torch.zeros(s64.ndof, dtype=torch.float64, device="cuda")
    s64.load_gaussians([x0], [0.05], [omega ** 2], 1.0, 0, False, out=F)
    out = {}
    W64 = torch.zeros_like(F)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, it, res = wh64.solve(F, 1e-6, 1000, W=W64)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    out["fp64"] = {"iterations": it, "residual": res, "seconds": el, "solves_per_s": 1.0 / el,
                   "steps_per_period": wh64.nt, "dt": wh64.dt,
                   "dof_stage_per_s": s64.ndof * 5 * wh64.nt * (it + 1) / el}
    Wm = torch.zeros_like(F)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, it32, res32 = wh32.solve(F, 3e-6, 1000, W=Wm)
    _, it64, res64 = wh64.solve(F, 1e-6, 1000, W=Wm)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    out["fp32_fp64"] = {"fp32_iterations": it32, "fp32_residual": res32, "fp64_iterations": it64,
                        "residual": res64, "seconds": el, "solves_per_s": 1.0 / el,
                        "rel_diff_vs_fp64": (Wm - W64).norm().item() / W64.norm().item()}
    out["workload"] = "waveholtz_128x128_P4_omega20_outflow_tol1e-6"
    out["x0"] = [float(x0[0]), float(x0[1])]
    ref = c3_reference_compare(x0, {"fp64": W64, "fp32_fp64": Wm})
    if ref is not None:
        out["vs_cpu_reference"] = ref
        ref["iterations_equal"] = out["fp64"]["iterations"] == ref["iterations"]
    return out


C3_FIXTURE = os.path.join(ROOT, "tests", "golden", "waveholtz_c3_128x128_P4.npz")


def c3_reference_compare(x0, arms) -> dict | None:
    """Errors of converged iterates against the reference library's own solve of the same
    problem (the CPU oracle: tests/golden/waveholtz_c3_128x128_P4.npz, written by
    make_c3_waveholtz.py).  The fixture holds 8192 seeded entries, the 2-norm and four seeded
    random projections of the reference's W; per arm: the relative 2-norm error over the
    sampled entries, the largest projection error relative to |W|, and the norm error."""
    if not os.path.exists(C3_FIXTURE):
        return None
    g = np.load(C3_FIXTURE)
    if not np.array_equal(g["x0"], np.asarray(x0)):
        return None
    idx, r, nr = g["sample_index"], g["W_samples"], float(g["W_norm"])
    out = {"source": "reference library's WaveHoltz solve at this size (compiled from its sources, CPU)",
           "iterations": int(g["iterations"]), "residual": float(g["residuals"][-1])}
    for name, W in arms.items():
        x = W.cpu().numpy()
        proj = max(abs(np.random.default_rng(int(g["proj_seed"]) + k).standard_normal(x.size) @ x - g["W_proj"][k])
                   for k in range(int(g["nproj"]))) / nr
        out[name] = {"rel_err_sampled": float(np.linalg.norm(x[idx] - r) / np.linalg.norm(r)),
                     "rel_err_projections": float(proj), "rel_err_norm": float(abs(np.linalg.norm(x) - nr) / nr)}
    return out


def learned_warm_start(device: int, count: int = 32, seed: int = 7000, n_plain: int = 4) -> dict:
    """Learned warm start on the single-solve Helmholtz family (128 x 128 uniform quads, P = 4,
    omega = 20, one Gaussian source with x0 ~ U[-0.5, 0.5]^2, outflow) with the network shipped
    in wavedg_b200/weights/ (trained on the family's own solutions; its training record is
    stored in the file).  `count` fresh seeded problems (seeds disjoint from the training
    data's) solved three ways to FP64 residual 1e-6: plain FP64 WaveHoltz one solve at a time
    (n_plain of them), batched FP32 + FP64 finish from zero, and the same from the network's
    prediction (prediction time included).  The plain iteration decides convergence in all."""
    from wavedg_b200 import warmstart as ws
    from wavedg_b200.fno import FNO

    path = ws.PACKAGED_WEIGHTS
    net = FNO(grid=512, width=32, modes=16, layers=4, hidden=64, device=device)
    scale = ws.load_weights(path, net)
    fam = ws.Family(count, device=device)
    res = ws.evaluate(net, fam, count, seed, scale, n_plain=n_plain, arms=("cold", "warm"), log=lambda *_: None)
    meta = ws.weights_meta(path)
    res["workload"] = f"waveholtz_128x128_P4_omega20_outflow_{count}_fresh_problems_tol1e-6"
    res["weights"] = {"file": os.path.relpath(path, ROOT), "training": meta}
    res["speedup"] = res["speedup_batched_warm_vs_plain"]
    return res


def config4_problems(count: int = 64, seed: int = 4):
    """The batched-solve distribution: per solve omega ~ U[10, 40], an n x n uniform quad mesh of
    [-1, 1]^2 with n ~ U{64, 96, 128, 192, 256}, P ~ U{3, 4, 6}, 1-4 Gaussian sources (sigma 0.05,
    centres ~ U[-0.8, 0.8]^2, amplitudes ~ N(0, 1)), outflow boundary."""
    rng = np.random.default_rng(seed)
    probs = []
    for _ in range(count):
        n = int(rng.choice([64, 96, 128, 192, 256]))
        P = int(rng.choice([3, 4, 6]))
        om = float(rng.uniform(10.0, 40.0))
        k = int(rng.integers(1, 5))
        probs.append((n, P, om, rng.uniform(-0.8, 0.8, size=(k, 2)), rng.standard_normal(k)))
    return probs


def waveholtz_config4(device: int, count: int = 64, seed: int = 4, deadline: float = 720.0,
                      chunk_iters: int = 30) -> dict:
    """Batched WaveHoltz on 64 solves of the batched-solve distribution (config4_problems), to
    relative residual 1e-6.

    batched   FP32 stepping with FP64 filter / residual in one batch until each solve reaches
              3e-6 (or stalls 3 iterations on the FP32 floor), then an FP64 batch from those
              iterates to 1e-6.  The FP32 phase runs in calls of at most `chunk_iters`
              iterations, each on a batch of the solves still running (every later call starts
              from the iterate with the |pi0| measured before, so nothing is repeated); it stops
              at `deadline` seconds, and the record then says which solves were unfinished.
    plain     plain FP64 WaveHoltz, one solve at a time, is timed as one period of every solve
              (the faster of two WaveHoltz::S calls after a warm-up period) times the periods a
              plain solve of it runs:
              its iterations + 1 (the pi0 period), the iterations being those the batch needed
              (FP32 + FP64 iterations; the same fixed-point map).  The rule is checked on the two
              solves with the fewest DOF-steps per period, solved in full.
    Wall times on the host around synchronous calls."""
    import torch

    import wavedg_b200 as W

    probs = config4_problems(count, seed)
    s64, s32, Fs, meshes, bases, bcs = [], [], [], [], [], []
    for (n, P, om, cs, amps) in probs:
        mesh = W.Mesh2D.uniform_rect(n, -1.0, 1.0, n, -1.0, 1.0)
        basis = W.QuadratureRule.quadrature_rule(P + 1, W.QuadratureRule.GaussLobatto)
        bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
        a = W.WaveSystem(mesh, basis, bc, precision="fp64", device=device)
        s64.append(a)
        s32.append(W.WaveSystem(mesh, basis, bc, precision="fp32", device=device))
        F = torch.zeros(a.ndof, dtype=torch.float64, device="cuda")
        a.load_gaussians(cs, [0.05] * len(amps), amps, 1.0, 0, False, out=F)
        Fs.append(F)
        meshes.append(mesh)
        bases.append(basis)
        bcs.append(bc)
    oms = [p[2] for p in probs]
    ndof = np.array([a.ndof for a in s64], dtype=np.int64)

    # ---- batched: FP32 phase in chunks, then the FP64 finish
    b32 = W.WaveHoltzBatch(s32, oms)
    tune_ms = b32.autotune(32)
    launch = b32.launch_config()
    nt = np.array([b32.params(i)[2] for i in range(count)], dtype=np.int64)
    Wb = [torch.zeros_like(F) for F in Fs]
    it32 = np.zeros(count, dtype=np.int64)
    pi0n = np.zeros(count)
    started = np.zeros(count, dtype=bool)
    st32 = np.full(count, -1)
    active = list(range(count))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    calls = 0
    while active and time.perf_counter() - t0 < deadline:
        b = b32 if calls == 0 else W.WaveHoltzBatch([s32[i] for i in active], [oms[i] for i in active])
        if calls > 0:
            b.set_launch(launch["rounds"], launch["ring"])
        Wl = [Wb[i] for i in active]
        _, it, _, st = b.solve([Fs[i] for i in active], 3e-6, chunk_iters, W=Wl, warm=started[active].astype(np.int32),
                               stall_limit=3, pi0_norm=pi0n[active])
        for k, i in enumerate(active):
            it32[i] += it[k]
            pi0n[i] = b.pi0_norm[k]
            st32[i] = st[k]
        started[active] = True
        active = [i for k, i in enumerate(active) if st[k] == 1]
        calls += 1
        del b
    torch.cuda.synchronize()
    t_fp32 = time.perf_counter() - t0
    finished = not active
    del b32
    b64 = W.WaveHoltzBatch(s64, oms)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    _, it64, r64, st64 = b64.solve(Fs, 1e-6, 200, W=Wb, warm=[1] * count, pi0_norm=pi0n)
    torch.cuda.synchronize()
    t_fp64 = time.perf_counter() - t1
    t_batch = t_fp32 + t_fp64
    del b64
    # DOF-stage updates the FP32 phase ran: every iteration is one forced period (a zero start's
    # first period yields pi0 and counts as iteration 1; later calls start from W with |pi0| known)
    dofstage32 = float(np.sum(ndof * 5 * nt * it32))
    # algorithmic bytes per DOF-stage of the FP32 batched stage kernel: u, k in and u', k' out
    # (4 B each; stage 1 reads no k), FP32 forcing in, FP64 filter in and out on the fifth stage:
    # (16 + 3 x 20 + 36) / 5 = 22.4 B
    peak, _ = peak_hbm()
    achieved = 22.4 * dofstage32 / t_fp32 / 1e9

    # ---- plain FP64: one period per solve, then the iteration rule
    per = np.zeros(count)
    for i in range(count):
        wh = W.WaveHoltz(oms[i], meshes[i], bases[i], bcs[i], True, system=s64[i])
        w = torch.zeros_like(Fs[i])
        wh.pi0(w, Fs[i])  # warm-up: records the period's graph
        best = float("inf")
        for _ in range(2):
            torch.cuda.synchronize()
            ts = time.perf_counter()
            wh.S(w)
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - ts)
        per[i] = best
        del wh, w
    plain_iters = it32 + it64
    t_plain_est = per * (plain_iters + 1)
    check = []
    for i in np.argsort(ndof * nt)[:2]:
        wh = W.WaveHoltz(oms[i], meshes[i], bases[i], bcs[i], True, system=s64[i])
        w = torch.zeros_like(Fs[i])
        torch.cuda.synchronize()
        ts = time.perf_counter()
        _, itp, _ = wh.solve(Fs[i], 1e-6, 2000, W=w)
        torch.cuda.synchronize()
        tm = time.perf_counter() - ts
        check.append({"solve": int(i), "iterations": int(itp), "batch_iterations": int(plain_iters[i]),
                      "seconds": tm, "estimated_seconds": float(t_plain_est[i]),
                      "rel_diff_vs_batched": (Wb[i] - w).norm().item() / w.norm().item()})
        del wh, w
    t_plain = float(np.sum(t_plain_est))
    done = int(np.sum((st64 == 0) & (r64 < 1e-6)))
    return {"workload": f"waveholtz_batch_{count}_solves_n64-256_P3-6_omega10-40_1-4src_tol1e-6",
            "solves": count, "total_dof": int(ndof.sum()), "seed": seed,
            "draw": f"the first {count} problems of the seeded draw (seed {seed}) whose first 64 are the stated batch",
            "per_solve": [{"n": p[0], "P": p[1], "omega": round(p[2], 4), "sources": len(p[4]), "ndof": int(ndof[i]),
                           "nt": int(nt[i]), "fp32_iterations": int(it32[i]), "fp64_iterations": int(it64[i]),
                           "residual": float(r64[i]), "plain_period_s": float(per[i])}
                          for i, p in enumerate(probs)],
            "batched_fp32_fp64": {"seconds": t_batch, "fp32_seconds": t_fp32, "fp64_seconds": t_fp64,
                                  "solves_per_s": count / t_batch, "fp32_calls": calls,
                                  "fp32_phase_finished": finished, "converged": done,
                                  "all_converged": bool(finished and done == count),
                                  "max_residual": float(np.max(r64)), "launch": launch,
                                  "autotune_ms_per_step": tune_ms,
                                  "fp32_dof_stage_per_s": dofstage32 / t_fp32,
                                  "fp32_stage_kernel_hbm": {"bytes_per_dof_stage": 22.4, "achieved_gbs": achieved,
                                                            "peak_gbs": peak, "frac": achieved / peak}},
            "plain_fp64": {"seconds_estimated": t_plain, "solves_per_s": count / t_plain,
                           "rule": "per solve: one timed period x (batch FP32 + FP64 iterations + 1)",
                           "period_seconds_total": float(per.sum()), "checked_in_full": check},
            "speedup": t_plain / t_batch}


# ----------------------------------------------------------- CPU side
def _ref_lib():
    from oracle import cpu

    if cpu.available("reference"):
        return "reference", cpu
    return "port", cpu


def exact_quadrature(device: int, n_el: int = 128, P: int = 4, reps: int = 20, cpu_leg: bool = True) -> dict:
    """The approx_quad = false operators (Div<false>, EdgeFlux<false>, MassMatrix<false>): time of
    one RHS M^{-1}(A + B) u on the GPU (device arrays, CUDA events over `reps` calls) on a
    perturbed n_el x n_el mesh, P = 4, outflow boundary; beside it the reference's own CPU
    RHS on the same mesh (compiled from its sources, 1 thread), when present."""
    import torch

    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(n_el, 0.2, seed=1)
    mesh = W.Mesh2D.from_vertices(v, q)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
    d = W.ExactDiscretisation(mesh, P + 1, bc, device=device)
    u = torch.from_numpy(np.random.default_rng(2).standard_normal(d.ndof)).cuda()
    du = torch.empty_like(u)
    for _ in range(3):
        d.rhs(u, du)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s0.record()
    for _ in range(reps):
        d.rhs(u, du)
    s1.record()
    torch.cuda.synchronize()
    ms = s0.elapsed_time(s1) / reps
    c2 = (P + 1) ** 2
    out = {"workload": f"rhs_exact_quadrature_{n_el}x{n_el}_P{P}_perturbed_outflow", "ndof": d.ndof,
           "rules_div_face_mass": list(d.rules()), "ms_per_rhs": ms, "dof_per_s": d.ndof / (ms / 1e3),
           # per element: state in/out (2 x 3 c2 doubles), M^{-1} factors (c2^2 doubles, read once per RHS)
           "factor_bytes_per_rhs": 8 * c2 * c2 * mesh.n_elem()}
    peak, _ = peak_hbm()
    out["bytes_per_rhs"] = (8 * (6 * c2 + c2 * c2) + 64) * mesh.n_elem()
    out["achieved_gbs"] = out["bytes_per_rhs"] / (ms / 1e3) / 1e9
    out["frac"] = out["achieved_gbs"] / peak
    out["kernel"] = "qfused_kernel (one fused launch per RHS)"
    if cpu_leg:
        kind, cpu = _ref_lib()
        if kind == "reference":
            m = cpu.Mesh(v, q, "reference")
            op = cpu.OpQ(m, P + 1, bc)
            uh = u.cpu().numpy()
            t0 = time.perf_counter()
            op.rhs(uh)
            out["cpu_reference_ms_per_rhs"] = (time.perf_counter() - t0) * 1e3
            out["cpu_reference"] = "the reference's WaveEquation / WaveBC / MassMatrix<false>, 1 thread, set-up excluded"
    return out


def advection(device: int, n_el: int = 256, P: int = 4, nv: int = 2, reps: int = 20, cpu_leg: bool = True) -> dict:
    """Linear advection with constant symmetric coefficients (Advection<true>,
    AdvectionHomogeneousBC<true>, MassMatrix<true>), n_var = 2: time of one RHS on the GPU
    (device arrays, CUDA events over `reps` calls) on a perturbed n_el x n_el mesh; beside it
    the reference's own CPU RHS on the same mesh (1 thread), when present."""
    import torch

    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(n_el, 0.2, seed=1)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(P + 1, W.QuadratureRule.GaussLobatto)
    a = np.array([1.0, 0.5, 0.5, -0.3, 0.2, 0.0, 0.0, 0.8])  # symmetric A_0, A_1 (a(d, c, k))
    s = W.AdvectionSystem(nv, mesh, basis, a, device=device)
    u = torch.from_numpy(np.random.default_rng(2).standard_normal(s.ndof)).cuda()
    du = torch.empty_like(u)
    for _ in range(3):
        s.rhs(u, du)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        s.rhs(u, du)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nel = mesh.n_elem()
    # algorithmic bytes of the fused RHS: u in, dudt out, the per-side |n.A| tables (4 nv^2
    # doubles per element) and the 64-byte corner block of every element
    byts = 16 * s.ndof + 8 * 4 * nv * nv * nel + 64 * nel
    peak, _ = peak_hbm()
    out = {"workload": f"rhs_advection_nvar{nv}_{n_el}x{n_el}_P{P}_perturbed", "values": s.ndof,
           "ms_per_rhs": ms, "values_per_s": s.ndof / (ms / 1e3), "bytes_per_rhs": byts,
           "achieved_gbs": byts / (ms / 1e3) / 1e9, "frac": byts / (ms / 1e3) / 1e9 / peak,
           "kernel": "claw_kernel (one fused launch per RHS)"}
    if cpu_leg:
        kind, cpu = _ref_lib()
        if kind == "reference":
            op = cpu.OpA(cpu.Mesh(v, q, "reference"), P + 1, nv, a)
            uh = u.cpu().numpy()
            t0 = time.perf_counter()
            op.rhs(uh)
            out["cpu_reference_ms_per_rhs"] = (time.perf_counter() - t0) * 1e3
            out["cpu_reference"] = "the reference's Advection / AdvectionHomogeneousBC / MassMatrix<true>, 1 thread"
    out["advec2d"] = advection_variable(device, n_el, P, reps, cpu_leg)
    return out


def _rhs_ms(s, u, du, reps):
    import torch

    for _ in range(3):
        s.rhs(u, du)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        s.rhs(u, du)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def advection_variable(device: int, n_el: int, P: int, reps: int, cpu_leg: bool) -> dict:
    """examples/advec2d.cpp's operators: one variable, the rotating coefficient r (y, -x) at the
    nodes of a Gauss-Legendre basis, approx_quad = false (Div<false>, EdgeFlux<false>,
    MassMatrix<false>): one fused RHS on a perturbed n_el x n_el mesh.  Algorithmic bytes: u in,
    dudt out, the volume and face tables and the dense inverse mass matrix per element."""
    import torch

    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(n_el, 0.2, seed=1)
    mesh = W.Mesh2D.from_vertices(v, q)
    n = P + 1
    basis = W.QuadratureRule.quadrature_rule(n, W.QuadratureRule.GaussLegendre)
    xg = np.polynomial.legendre.leggauss(n)[0]
    c = np.asarray(v)[np.asarray(q)]
    xi, eta = xg[None, None, :], xg[None, :, None]
    xy = [0.25 * ((1 - xi) * (1 - eta) * c[:, 0, k][:, None, None] + (1 + xi) * (1 - eta) * c[:, 1, k][:, None, None]
                  + (1 + xi) * (1 + eta) * c[:, 2, k][:, None, None] + (1 - xi) * (1 + eta) * c[:, 3, k][:, None, None])
          for k in range(2)]
    r = np.hypot(xy[0], xy[1])
    a = np.stack([r * xy[1], -r * xy[0]], axis=-1).reshape(-1)  # a(0, 0, comp, i, j, el)
    s = W.VariableAdvectionSystem(1, mesh, basis, a, approx_quad=False, device=device)
    u = torch.from_numpy(np.random.default_rng(2).standard_normal(s.ndof)).cuda()
    du = torch.empty_like(u)
    ms = _rhs_ms(s, u, du, reps)
    nel = mesh.n_elem()
    Q, Qf = 1 + (3 * n - 3) // 2, 1 + (3 * n - 1) // 2
    byts = 16 * s.ndof + 8 * nel * (2 * Q * Q + 8 * Qf + n ** 4) + 64 * nel
    peak, _ = peak_hbm()
    out = {"workload": f"rhs_advec2d_nvar1_gauss_legendre_exact_{n_el}x{n_el}_P{P}_perturbed", "values": s.ndof,
           "ms_per_rhs": ms, "values_per_s": s.ndof / (ms / 1e3), "bytes_per_rhs": byts,
           "achieved_gbs": byts / (ms / 1e3) / 1e9, "frac": byts / (ms / 1e3) / 1e9 / peak,
           "kernel": "vadv_kernel (one fused launch per RHS)"}
    if cpu_leg:
        kind, cpu = _ref_lib()
        if kind == "reference":
            op = cpu.OpV(cpu.Mesh(v, q, "reference"), n, 1, a, False, 0)
            uh = u.cpu().numpy()
            t0 = time.perf_counter()
            op.rhs(uh)
            out["cpu_reference_ms_per_rhs"] = (time.perf_counter() - t0) * 1e3
            out["cpu_reference"] = "the reference's Advection<false> / AdvectionHomogeneousBC<false> / MassMatrix<false>, 1 thread"
    return out


def euler(device: int, n_el: int = 256, P: int = 4, reps: int = 20, cpu_leg: bool = True) -> dict:
    """The compressible Euler system of the reference's nonlinear example (DivF2D<true>,
    EdgeFluxF2D<true> with the local Lax-Friedrichs flux, MassMatrix<true>) on a perturbed
    n_el x n_el mesh, P = 4, a smooth positive state: one fused RHS launch and one SSPRK3 step
    on device arrays (CUDA events over `reps`), with the HBM fraction of the RHS; beside it the
    reference's own CPU time derivative on the same mesh (1 thread), when present."""
    import torch

    import wavedg_b200 as W
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(n_el, 0.2, seed=1, lo=0.0, hi=10.0)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(P + 1, W.QuadratureRule.GaussLobatto)
    s = W.EulerSystem(mesh, basis, device=device)
    n = P + 1
    rng = np.random.default_rng(2)
    nn = s.ndof // 4
    rho, p = 1.0 + 0.2 * rng.random(nn), 1.0 + 0.2 * rng.random(nn)
    uu, vv = 0.3 * rng.standard_normal(nn), 0.3 * rng.standard_normal(nn)
    U = np.stack([rho, rho * uu, rho * vv, p / 0.4 + 0.5 * rho * (uu * uu + vv * vv)], axis=1).ravel()
    u = torch.from_numpy(U).cuda()
    du = torch.empty_like(u)
    for _ in range(3):
        s.rhs(u, du)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        s.rhs(u, du)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    dt = 0.2 * mesh.min_h() / (6.0 * n * n)
    w = u.clone()
    s.steps(w, dt, 0.0, 2, "ssprk3")
    torch.cuda.synchronize()
    e0.record()
    s.steps(w, dt, 0.0, reps, "ssprk3")
    e1.record()
    torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / reps
    nel = mesh.n_elem()
    byts = 16 * s.ndof + 64 * nel  # u in, dudt out, corners
    peak, _ = peak_hbm()
    out = {"workload": f"rhs_euler_{n_el}x{n_el}_P{P}_perturbed", "values": s.ndof, "ms_per_rhs": ms,
           "values_per_s": s.ndof / (ms / 1e3), "bytes_per_rhs": byts, "achieved_gbs": byts / (ms / 1e3) / 1e9,
           "frac": byts / (ms / 1e3) / 1e9 / peak, "ms_per_ssprk3_step": ms_step,
           "kernel": "claw_kernel (one fused launch per RHS / stage)"}
    if cpu_leg:
        kind, cpu = _ref_lib()
        if kind == "reference":
            op = cpu.OpE(cpu.Mesh(v, q, "reference"), n)
            t0 = time.perf_counter()
            op.rhs(U)
            out["cpu_reference_ms_per_rhs"] = (time.perf_counter() - t0) * 1e3
            out["cpu_reference"] = "the reference's DivF2D / EdgeFluxF2D / MassMatrix<true> with the example's fluxes, 1 thread"
    # approx_quad = false, as the example ships: 2n-point rules and the dense inverse mass matrix
    sq = W.EulerSystem(mesh, basis, device=device, approx_quad=False)
    msq = _rhs_ms(sq, u, du, reps)
    byq = byts + 8 * nel * n ** 4
    out["exact"] = {"workload": f"rhs_euler_exact_{n_el}x{n_el}_P{P}_perturbed", "ms_per_rhs": msq,
                    "values_per_s": s.ndof / (msq / 1e3), "bytes_per_rhs": byq,
                    "achieved_gbs": byq / (msq / 1e3) / 1e9, "frac": byq / (msq / 1e3) / 1e9 / peak,
                    "kernel": "qeuler_kernel (one fused launch per RHS / stage)"}
    if cpu_leg:
        kind, cpu = _ref_lib()
        if kind == "reference":
            opq = cpu.OpEQ(cpu.Mesh(v, q, "reference"), n)
            t0 = time.perf_counter()
            opq.rhs(U)
            out["exact"]["cpu_reference_ms_per_rhs"] = (time.perf_counter() - t0) * 1e3
    return out


def decomposition(device: int, n_el: int = 512, P: int = 4, ranks: int = 2, steps: int = 10) -> dict:
    """One mesh split into `ranks` domains (contiguous element blocks), emulated on one GPU: the
    domains step one after another with their halo exchanged by device copies before every
    RK stage.  Against the undivided mesh on the same GPU this measures what the
    decomposition itself adds (halo gather, copies, the extra launches and host syncs), not
    multi-GPU speed; the states must agree bit for bit."""
    import torch

    import wavedg_b200 as W
    from wavedg_b200 import decomp
    from wavedg_b200 import meshgen as mg

    v, q = mg.perturbed_rect(n_el, 0.2, seed=1)
    mesh = W.Mesh2D.from_vertices(v, q)
    basis = W.QuadratureRule.quadrature_rule(P + 1, W.QuadratureRule.GaussLobatto)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
    whole = W.WaveSystem(mesh, basis, bc, device=device)
    u0 = np.random.default_rng(3).standard_normal(whole.ndof)
    dt = 0.1 * mesh.min_h() / (P + 1) ** 2
    part = decomp.partition(mesh.n_elem(), ranks)
    doms = [decomp.Domain(mesh, basis, bc, part, r, device=device) for r in range(ranks)]
    t_dd = {}
    for overlap in (False, True):
        for d in doms:
            d.upload(u0)
        decomp.step_all(doms, dt, 1, overlap=overlap)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        decomp.step_all(doms, dt, steps, overlap=overlap)
        for d in doms:
            d.sync()
        t_dd[overlap] = (time.perf_counter() - t0) / steps
    ud = np.zeros_like(u0)
    for d in doms:
        d.download(ud)
    uw = torch.from_numpy(u0.copy()).cuda()  # device array: no transfers in the timed loop
    whole.rk4_steps(uw, dt, 0.0, 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    whole.rk4_steps(uw, dt, 0.0, steps)
    torch.cuda.synchronize()
    t_whole = (time.perf_counter() - t0) / steps
    uw = uw.cpu().numpy()
    halo = sum(d.halo for d in doms)
    return {"workload": f"rk4_fp64_{n_el}x{n_el}_P{P}_{ranks}_domains_one_gpu",
            "ms_per_step_domains": t_dd[True] * 1e3, "ms_per_step_domains_unsplit": t_dd[False] * 1e3,
            "split": "each stage in a halo-free part and a halo part (the exchange runs between them)",
            "ms_per_step_undivided": t_whole * 1e3, "halo_values": halo,
            "halo_bytes_per_stage": 8 * halo, "identical_to_undivided": bool(np.array_equal(ud, uw)),
            "note": "domains run one after another on one GPU: the difference is the decomposition's own cost"}


def cpu_baseline(v, q, bc, n, dt, u0, budget=15.0):
    """Reference CPU code on the same workload, 1 thread: set-up excluded, then RK4 steps until
    the time budget (at least one full step)."""
    kind, cpu = _ref_lib()
    libkind = "reference" if kind == "reference" else "oracle"
    mesh = cpu.Mesh(v, q, libkind)
    op = cpu.Op(mesh, n, bc)
    u = np.ascontiguousarray(u0, dtype=np.float64)
    steps, t0 = 0, time.perf_counter()
    while True:
        u, _ = op.rk4(u, dt, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el > budget or steps >= 50:
            break
    value = op.ndof * 5 * steps / el
    return {"value": value, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{steps} RK4 step(s) of the same {mesh.n_elem} element P={n - 1} workload, "
                      f"operator set-up excluded, single thread ({os.cpu_count()} host cores present)"}


def _ref_worker(n_el, P, steps, budget, start_evt, out_q):
    """One serial reference process: builds the operator on the full workload, waits for the
    others, then times RK4 steps until `budget` seconds (at least one step)."""
    kind, cpu = _ref_lib()
    libkind = "reference" if kind == "reference" else "oracle"
    v, q, centers, sigmas, amps = workload(n_el, P)
    n = P + 1
    mesh = cpu.Mesh(v, q, libkind)
    bc = np.zeros(mesh.n_edges(1), dtype=np.int32)
    t_setup = time.perf_counter()
    op = cpu.Op(mesh, n, bc)
    u = op.load_gaussians(centers, sigmas, amps, 1.0, 0, True)
    t_setup = time.perf_counter() - t_setup
    dt = 0.1 * mesh.min_h() / n ** 2
    out_q.put(("ready", t_setup))
    start_evt.wait()
    runs, t0 = 0, time.perf_counter()
    while runs < steps:
        u, _ = op.rk4(u, dt, 1)
        runs += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    out_q.put(("done", kind, op.ndof, runs, el))


def run_reference(args, rank, world):
    """The reference's own CPU code (oracle/_ref, compiled from its sources) on the same
    workload.  The reference is serial (its MPI build needs a toolchain absent here), so all
    host cores are used by running one independent replica per core, concurrently; the
    throughput is the sum over the replicas.  Rank 0 only."""
    if rank != 0:
        return
    import multiprocessing as mp

    procs_n = max(1, min(os.cpu_count() or 1, args.ref_procs if args.ref_procs > 0 else 64))
    ctx = mp.get_context("spawn")
    start_evt, out_q = ctx.Event(), ctx.Queue()
    # each timed step of a replica is one RK4 step; the budget keeps the run to a few minutes
    budget = max(5.0, REF_TIME_BUDGET / 2)
    procs = [ctx.Process(target=_ref_worker, args=(args.n, args.P, args.steps, budget, start_evt, out_q))
             for _ in range(procs_n)]
    for p in procs:
        p.start()
    setups = [out_q.get()[1] for _ in procs]
    start_evt.set()
    results = [out_q.get() for _ in procs]
    for p in procs:
        p.join()
    kind = results[0][1]
    ndof = results[0][2]
    rates = [r[2] * 5 * r[3] / r[4] for r in results]
    value = float(sum(rates))
    runs = [r[3] for r in results]
    el = max(r[4] for r in results)
    sample = (f"{procs_n} concurrent serial replicas x {min(runs)}-{max(runs)} RK4 steps each (of {args.steps} "
              f"requested) on the full {args.n}x{args.n} P={args.P} mesh; set-up ({max(setups):.1f} s) excluded")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": el / max(1, min(runs)) * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (same workload as ours)",
           "config": {"workload": f"rk4_fp64_{args.n}x{args.n}_P{args.P}_perturbed_outflow",
                      "elements": args.n * args.n, "ndof": ndof, "P": args.P, "step": "1 RK4 step",
                      "parallelism": f"{procs_n} host processes (one serial replica per core)"},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs_n, "kind": kind, "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
