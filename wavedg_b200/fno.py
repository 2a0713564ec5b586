"""Learned warm start for WaveHoltz: a Fourier neural operator (FNO) on a uniform grid.

The network maps the forcing of a WaveHoltz problem (its normalised Gaussian, omega, and
the grid coordinates) on a G x G cell-centred grid of [-1, 1]^2 to the solution's (p, u, v)
on the same grid, which is interpolated to the DG nodes as the initial iterate W0.  The
WaveHoltz iteration still decides convergence: a warm-started solve stops at the same
residual tolerance as a cold one, only the iteration count changes.

Architecture: lift (4 -> width, pointwise), `layers` Fourier layers
v <- act(K v + W v + b) with K the spectral convolution on the retained modes
(kx in [0, modes), ky in [-modes, modes)), projection (width -> hidden -> 3, GELU between).

Every operation runs in the library's own kernels (wdg_fno_*, csrc/fno.cu): BF16
operands with FP32 accumulation on the tensor cores for the GEMMs (truncated DFT along x
and its inverse, channel mixes, weight gradients), FP32 for the small spectral steps;
the backward pass is written out by hand.  torch only allocates device memory.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, lib

def _fn(name):
    """The entry point with its signature (wavedg_b200._lib.SIGNATURES)."""
    return getattr(lib(), name)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class FNO:
    """Parameters (FP32 masters, BF16 copies for the GEMMs) and workspaces on one GPU."""

    def __init__(self, grid: int = 512, width: int = 32, modes: int = 16, layers: int = 4, hidden: int = 64,
                 in_ch: int = 4, out_ch: int = 3, seed: int = 0, device: int = 0):
        import torch

        self.torch = torch
        self.G, self.Cw, self.KX, self.KY = grid, width, modes, 2 * modes
        self.L, self.H, self.Cin, self.Cout = layers, hidden, in_ch, out_ch
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.dev)
        g = torch.Generator().manual_seed(seed)
        f32 = dict(dtype=torch.float32)

        def U(shape, scale):
            return ((torch.rand(shape, generator=g, **f32) * 2 - 1) * scale).to(self.dev)

        Cw, H, M = self.Cw, self.H, self.KY * self.KX
        self.params = {
            "P_w": U((Cw, in_ch), 1.0 / math.sqrt(in_ch)), "P_b": U((Cw,), 1.0 / math.sqrt(in_ch)),
            "Q1_w": U((H, Cw), 1.0 / math.sqrt(Cw)), "Q1_b": U((H,), 1.0 / math.sqrt(Cw)),
            "Q2_w": U((out_ch, H), 1.0 / math.sqrt(H)), "Q2_b": U((out_ch,), 1.0 / math.sqrt(H)),
        }
        for l in range(layers):
            self.params[f"R{l}"] = U((Cw, Cw, M, 2), 1.0 / (Cw * Cw))
            self.params[f"W{l}"] = U((Cw, Cw), 1.0 / math.sqrt(Cw))
            self.params[f"b{l}"] = U((Cw,), 1.0 / math.sqrt(Cw))
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.adam_m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.adam_v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.step_count = 0
        self._bf = {}
        self.refresh_bf16()
        # truncated DFT matrices along x (BF16) and the twiddle table along y (FP32)
        G, KX = self.G, self.KX
        x = np.arange(G)
        k = np.arange(KX)
        ang = 2 * np.pi * np.outer(x, k) / G  # (G, KX)
        ex = np.zeros((G, 2 * KX))
        ex[:, 0::2] = np.cos(ang)
        ex[:, 1::2] = -np.sin(ang)
        wk = np.where(k == 0, 1.0, 2.0)[:, None]
        ix = np.zeros((2 * KX, G))
        ix[0::2, :] = wk * np.cos(ang.T) / (G * G)
        ix[1::2, :] = -wk * np.sin(ang.T) / (G * G)
        self.Ex = torch.from_numpy(ex).to(self.dev, torch.bfloat16).contiguous()
        self.Ix = torch.from_numpy(ix).to(self.dev, torch.bfloat16).contiguous()
        m = np.arange(G)
        self.cos_t = torch.from_numpy(np.cos(2 * np.pi * m / G)).to(self.dev, torch.float32)
        self.sin_t = torch.from_numpy(np.sin(2 * np.pi * m / G)).to(self.dev, torch.float32)

    # --------------------------------------------------------------- helpers
    def refresh_bf16(self):
        for k in ("P_w", "Q1_w", "Q2_w") + tuple(f"W{l}" for l in range(self.L)):
            self._bf[k] = self.params[k].to(self.torch.bfloat16).contiguous()

    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def _gemm(self, A, B, Cm, M, N, K, lda, ldb, ldc, sA=0, sB=0, sC=0, batch=1, tA=0, tB=0, alpha=1.0, beta=0.0,
              ksplit=0):
        check(_fn("wdg_fno_gemm")(_p(A), _p(B), _p(Cm), M, N, K, lda, ldb, ldc, sA, sB, sC, batch, tA, tB,
                                  float(alpha), float(beta), int(ksplit), self._s()), "fno gemm")

    def _bf16(self, x):
        y = self.torch.empty(x.shape, dtype=self.torch.bfloat16, device=self.dev)
        check(_fn("wdg_fno_to_bf16")(_p(x), _p(y), x.numel(), self._s()))
        return y

    def _ksplit(self, K):
        # weight-gradient GEMMs reduce over every grid point: split K so the grid fills the GPU
        return max(1024, ((K + 255) // 256 + 31) // 32 * 32)

    # --------------------------------------------------------------- forward
    def forward(self, inp, keep: bool = False):
        """inp: (B, in_ch, G, G) FP32 CUDA tensor -> (B, out_ch, G, G) FP32."""
        t = self.torch
        B, G, Cw, KX, KY, H = inp.shape[0], self.G, self.Cw, self.KX, self.KY, self.H
        P = G * G
        tape = {"B": B}
        inb = self._bf16(inp)
        z = t.empty((B, Cw, P), dtype=t.float32, device=self.dev)
        self._gemm(self._bf["P_w"], inb, z, Cw, P, self.Cin, self.Cin, P, P, 0, self.Cin * P, Cw * P, B)
        v = t.empty((B, Cw, P), dtype=t.bfloat16, device=self.dev)
        check(_fn("wdg_fno_bias_act")(_p(z), _p(self.params["P_b"]), _p(v), None, B, Cw, P, 0, self._s()))
        if keep:
            tape["in"] = inb
        for l in range(self.L):
            act = 1 if l < self.L - 1 else 0
            vx = t.empty((B * Cw * G, 2 * KX), dtype=t.float32, device=self.dev)
            self._gemm(v, self.Ex, vx, B * Cw * G, 2 * KX, G, G, 2 * KX, 2 * KX)
            vh = t.empty((B * Cw, KY, KX, 2), dtype=t.float32, device=self.dev)
            check(_fn("wdg_fno_dft_y")(_p(vx), _p(vh), None, _p(self.cos_t), _p(self.sin_t), B * Cw, G, KY, KX, 0,
                                       -1.0, self._s()))
            wh = t.empty_like(vh)
            check(_fn("wdg_fno_mix")(_p(self.params[f"R{l}"]), _p(vh), _p(wh), B, Cw, Cw, KY * KX, self._s()))
            uy = t.empty((B * Cw * G, 2 * KX), dtype=t.bfloat16, device=self.dev)
            check(_fn("wdg_fno_dft_y")(_p(wh), None, _p(uy), _p(self.cos_t), _p(self.sin_t), B * Cw, G, KY, KX, 1,
                                       1.0, self._s()))
            zl = t.empty((B, Cw, P), dtype=t.float32, device=self.dev)
            self._gemm(uy, self.Ix, zl, B * Cw * G, G, 2 * KX, 2 * KX, G, G)
            self._gemm(self._bf[f"W{l}"], v, zl, Cw, P, Cw, Cw, P, P, 0, Cw * P, Cw * P, B, beta=1.0)
            vn = t.empty((B, Cw, P), dtype=t.bfloat16, device=self.dev)
            check(_fn("wdg_fno_bias_act")(_p(zl), _p(self.params[f"b{l}"]), _p(vn), None, B, Cw, P, act, self._s()))
            if keep:
                tape[f"v{l}"], tape[f"z{l}"], tape[f"vh{l}"] = v, zl, vh
            v = vn
        zq = t.empty((B, H, P), dtype=t.float32, device=self.dev)
        self._gemm(self._bf["Q1_w"], v, zq, H, P, Cw, Cw, P, P, 0, Cw * P, H * P, B)
        hb = t.empty((B, H, P), dtype=t.bfloat16, device=self.dev)
        check(_fn("wdg_fno_bias_act")(_p(zq), _p(self.params["Q1_b"]), _p(hb), None, B, H, P, 1, self._s()))
        y = t.empty((B, self.Cout, P), dtype=t.float32, device=self.dev)
        self._gemm(self._bf["Q2_w"], hb, y, self.Cout, P, H, H, P, P, 0, H * P, self.Cout * P, B)
        check(_fn("wdg_fno_bias_act")(_p(y), _p(self.params["Q2_b"]), None, None, B, self.Cout, P, 0, self._s()))
        if keep:
            tape["v_last"], tape["zq"], tape["hb"] = v, zq, hb
            self.tape = tape
        return y.view(B, self.Cout, G, G)

    # -------------------------------------------------------------- backward
    def backward(self, dy):
        """dy: dL/dy of the last forward(keep=True); fills self.grads (overwrites)."""
        t = self.torch
        tp = self.tape
        B, G, Cw, KX, KY, H = tp["B"], self.G, self.Cw, self.KX, self.KY, self.H
        P = G * G
        ks = self._ksplit(P)
        gr = self.grads
        dy = dy.reshape(B, self.Cout, P).contiguous()
        dyb = self._bf16(dy)
        check(_fn("wdg_fno_bias_grad")(_p(dy), _p(gr["Q2_b"]), B, self.Cout, P, 0, self._s()))
        # dQ2 = sum_b dy[b] hb[b]^T
        self._gemm(dyb, tp["hb"], gr["Q2_w"], self.Cout, H, P, P, P, H, self.Cout * P, H * P, 0, B, 0, 1,
                   beta=0.0, ksplit=ks)
        dh = t.empty((B, H, P), dtype=t.float32, device=self.dev)
        self._gemm(self._bf["Q2_w"], dyb, dh, H, P, self.Cout, H, P, P, 0, self.Cout * P, H * P, B, tA=1)
        dzq = t.empty_like(dh)
        dzqb = t.empty((B, H, P), dtype=t.bfloat16, device=self.dev)
        check(_fn("wdg_fno_act_bwd")(_p(dh), _p(tp["zq"]), _p(dzq), _p(dzqb), dh.numel(), 1, self._s()))
        check(_fn("wdg_fno_bias_grad")(_p(dzq), _p(gr["Q1_b"]), B, H, P, 0, self._s()))
        self._gemm(dzqb, tp["v_last"], gr["Q1_w"], H, Cw, P, P, P, Cw, H * P, Cw * P, 0, B, 0, 1, ksplit=ks)
        dv = t.empty((B, Cw, P), dtype=t.float32, device=self.dev)
        self._gemm(self._bf["Q1_w"], dzqb, dv, Cw, P, H, Cw, P, P, 0, H * P, Cw * P, B, tA=1)
        for l in reversed(range(self.L)):
            act = 1 if l < self.L - 1 else 0
            v, zl, vh = tp[f"v{l}"], tp[f"z{l}"], tp[f"vh{l}"]
            dz = t.empty_like(dv)
            dzb = t.empty((B, Cw, P), dtype=t.bfloat16, device=self.dev)
            check(_fn("wdg_fno_act_bwd")(_p(dv), _p(zl), _p(dz), _p(dzb), dv.numel(), act, self._s()))
            check(_fn("wdg_fno_bias_grad")(_p(dz), _p(gr[f"b{l}"]), B, Cw, P, 0, self._s()))
            self._gemm(dzb, v, gr[f"W{l}"], Cw, Cw, P, P, P, Cw, Cw * P, Cw * P, 0, B, 0, 1, ksplit=ks)
            dvp = t.empty((B, Cw, P), dtype=t.float32, device=self.dev)
            self._gemm(self._bf[f"W{l}"], dzb, dvp, Cw, P, Cw, Cw, P, P, 0, Cw * P, Cw * P, B, tA=1)
            # spectral branch, adjoints in reverse order
            duy = t.empty((B * Cw * G, 2 * KX), dtype=t.float32, device=self.dev)
            self._gemm(dzb, self.Ix, duy, B * Cw * G, 2 * KX, G, G, G, 2 * KX, tB=1)
            dwh = t.empty((B * Cw, KY, KX, 2), dtype=t.float32, device=self.dev)
            check(_fn("wdg_fno_dft_y")(_p(duy), _p(dwh), None, _p(self.cos_t), _p(self.sin_t), B * Cw, G, KY, KX, 0,
                                       -1.0, self._s()))
            dvh = t.empty_like(dwh)
            check(_fn("wdg_fno_mix_bwd")(_p(self.params[f"R{l}"]), _p(vh), _p(dwh), _p(dvh), _p(gr[f"R{l}"]), B, Cw,
                                         Cw, KY * KX, 0, self._s()))
            dvxb = t.empty((B * Cw * G, 2 * KX), dtype=t.bfloat16, device=self.dev)
            check(_fn("wdg_fno_dft_y")(_p(dvh), None, _p(dvxb), _p(self.cos_t), _p(self.sin_t), B * Cw, G, KY, KX, 1,
                                       1.0, self._s()))
            self._gemm(dvxb, self.Ex, dvp, B * Cw * G, G, 2 * KX, 2 * KX, 2 * KX, G, tB=1, beta=1.0)
            dv = dvp
        # lift: v0 = P_w in + P_b (no activation)
        check(_fn("wdg_fno_bias_grad")(_p(dv), _p(gr["P_b"]), B, Cw, P, 0, self._s()))
        dvb = self._bf16(dv)
        self._gemm(dvb, tp["in"], gr["P_w"], Cw, self.Cin, P, P, P, self.Cin, Cw * P, self.Cin * P, 0, B, 0, 1,
                   ksplit=ks)

    def mse(self, y, target):
        """Mean squared error (FP64 sum) and dL/dy."""
        t = self.torch
        dy = t.empty_like(y)
        sse = t.zeros(1, dtype=t.float64, device=self.dev)
        n = y.numel()
        check(_fn("wdg_fno_mse")(_p(y), _p(target), _p(dy), _p(sse), n, 1.0 / n, self._s()))
        return sse, dy

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.step_count += 1
        for k, p in self.params.items():
            check(_fn("wdg_fno_adam")(_p(p), _p(self.grads[k]), _p(self.adam_m[k]), _p(self.adam_v[k]), p.numel(),
                                      float(lr), beta1, beta2, eps, self.step_count, weight_decay, self._s()))
        self.refresh_bf16()

    def state_dict(self):
        return {k: v.detach().cpu().numpy() for k, v in self.params.items()}

    def load_state_dict(self, sd):
        for k, v in sd.items():
            self.params[k].copy_(self.torch.from_numpy(np.asarray(v, dtype=np.float32)))
        self.refresh_bf16()


# ------------------------------------------------------------ problem <-> grid
def inputs(G, centers, sigma, omega_scaled, device=0):
    """(B, 4, G, G) network inputs for Gaussian sources at `centers` (one per sample)."""
    import torch

    B = len(centers)
    x = torch.empty((B, 4, G, G), dtype=torch.float32, device=torch.device("cuda", device))
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for b, (cx, cy) in enumerate(centers):
        check(_fn("wdg_fno_inputs")(C.c_void_p(x[b].data_ptr()), G, float(cx), float(cy), float(sigma),
                                    float(omega_scaled), s))
    return x


class NodalGrid:
    """Resampling between the DG nodes of a uniform ne x ne mesh of [-1, 1]^2 (n GLL nodes per
    direction, reference element order) and the G x G cell-centred grid."""

    def __init__(self, ne: int, n: int, G: int, device: int = 0):
        import torch

        from .dg import QuadratureRule

        self.ne, self.n, self.G = ne, n, G
        xq = np.asarray(QuadratureRule.quadrature_rule(n, QuadratureRule.GaussLobatto).x, dtype=np.float64)
        bw = np.array([1.0 / np.prod([xq[j] - xq[k] for k in range(n) if k != j]) for j in range(n)])
        dev = torch.device("cuda", device)
        self.x = torch.from_numpy(xq).to(dev)
        self.bw = torch.from_numpy(bw).to(dev)
        self.torch = torch

    def to_grid(self, u, scale=1.0):
        t = self.torch
        out = t.empty((3, self.G, self.G), dtype=t.float32, device=u.device)
        check(_fn("wdg_fno_nodes_to_grid")(_p(u), _p(out), self.ne, self.n, _p(self.x), _p(self.bw), self.G,
                                           float(scale), C.c_void_p(t.cuda.current_stream().cuda_stream)))
        return out

    def to_nodes(self, g, scale=1.0):
        t = self.torch
        u = t.empty(3 * self.ne * self.ne * self.n * self.n, dtype=t.float64, device=g.device)
        check(_fn("wdg_fno_grid_to_nodes")(_p(g.contiguous()), _p(u), self.ne, self.n, _p(self.x), self.G,
                                           float(scale), C.c_void_p(t.cuda.current_stream().cuda_stream)))
        return u


def step_profile(grid: int = 512, width: int = 32, modes: int = 16, layers: int = 4, hidden: int = 64,
                 train_batch: int = 4, predict_batch: int = 8, warmup: int = 3) -> dict:
    """Time one training step (forward, MSE, backward, Adam) and one prediction after `warmup`
    rounds of both, on seeded inputs, and list every GEMM of the timed pair in launch order with
    its shape and algorithmic bytes (BF16 operands read once; the FP32 result written, and read
    again where beta = 1 or split-K accumulates).  The command to run under a launch-list
    profiler: python -m wavedg_b200.fno --step-profile."""
    import torch

    net = FNO(grid=grid, width=width, modes=modes, layers=layers, hidden=hidden, seed=0)
    rng = np.random.default_rng(0)
    tgt = torch.from_numpy(rng.standard_normal((train_batch, 3, grid, grid))).to("cuda", torch.float32)
    log = []
    gemm = net._gemm

    def logged(A, B, Cm, M, N, K, lda, ldb, ldc, sA=0, sB=0, sC=0, batch=1, tA=0, tB=0, alpha=1.0, beta=0.0,
               ksplit=0):
        rw = 2 if (beta != 0.0 or ksplit) else 1
        log.append(dict(M=M, N=N, K=K, batch=batch, tA=tA, tB=tB, beta=beta, ksplit=ksplit,
                        bytes=2 * batch * (M * K + K * N) + 4 * (batch if sC else 1) * M * N * rw,
                        flops=2.0 * M * N * K * batch))
        return gemm(A, B, Cm, M, N, K, lda, ldb, ldc, sA, sB, sC, batch, tA, tB, alpha, beta, ksplit)

    net._gemm = logged

    def train_step():
        x = inputs(grid, rng.uniform(-0.5, 0.5, (train_batch, 2)), 0.05, 1.0)
        y = net.forward(x, keep=True)
        _, dy = net.mse(y, tgt)
        net.backward(dy)
        net.adam_step(lr=1e-3)

    def predict():
        return net.forward(inputs(grid, rng.uniform(-0.5, 0.5, (predict_batch, 2)), 0.05, 1.0))

    for _ in range(warmup):
        train_step()
        predict()
    torch.cuda.synchronize()
    log.clear()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    train_step()
    e1.record()
    n_train = len(log)
    predict()
    e2.record()
    torch.cuda.synchronize()
    return {"train_step_ms": e0.elapsed_time(e1), "predict_ms": e1.elapsed_time(e2),
            "train_gemms": log[:n_train], "predict_gemms": log[n_train:]}


if __name__ == "__main__":
    import json
    import sys

    if "--step-profile" not in sys.argv:
        raise SystemExit("usage: python -m wavedg_b200.fno --step-profile")
    print(json.dumps(step_profile()), flush=True)
