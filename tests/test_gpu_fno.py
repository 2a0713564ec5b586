"""The learned warm start's FNO kernels (wdg_fno_*) against FP64 CPU references.

* the BF16 tensor-core GEMM, every transpose / batch / split-K form the network uses,
  against an FP64 product of the same BF16-rounded operands (FP32 accumulation: 1e-5);
* forward pass and every parameter gradient of a small FNO (grid 32, width 8, 4 modes,
  4 layers) and of one with the learned warm start's channel and mode counts (grid 64,
  width 32, 16 modes, hidden 64) against torch FP64 autograd on the CPU with torch.fft,
  from the same FP32 parameters.  BF16 activations and weights bound the agreement: 2e-2 on the output, 4e-2
  on each gradient tensor (relative 2-norm);
* resampling between DG nodes and the grid: exact for a bilinear field both ways.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("tA,tB,batch,ksplit", [(0, 0, 1, 0), (1, 0, 2, 0), (0, 1, 3, 0), (1, 1, 1, 64),
                                                (0, 1, 2, 96)])
def test_gemm(gpu_lib, tA, tB, batch, ksplit):
    import torch

    from wavedg_b200.fno import _fn

    rng = np.random.default_rng(tA + 2 * tB + 4 * batch)
    M, N, K = 70, 45, 300
    A = torch.from_numpy(rng.standard_normal((batch, K, M) if tA else (batch, M, K))).to("cuda", torch.bfloat16)
    B = torch.from_numpy(rng.standard_normal((batch, N, K) if tB else (batch, K, N))).to("cuda", torch.bfloat16)
    shared = ksplit > 0 and batch > 1  # batches summing into one C
    Cm = torch.full((1 if shared else batch, M, N), 7.0, dtype=torch.float32, device="cuda")
    import ctypes as C

    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _fn("wdg_fno_gemm")(C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), C.c_void_p(Cm.data_ptr()), M, N, K,
                             M if tA else K, K if tB else N, N, A[0].numel(), B[0].numel(), 0 if shared else M * N,
                             batch, tA, tB, 1.5, 0.0, ksplit, st)
    assert rc == 0
    torch.cuda.synchronize()
    a = A.to(torch.float64).cpu().numpy()
    b = B.to(torch.float64).cpu().numpy()
    a = np.transpose(a, (0, 2, 1)) if tA else a
    b = np.transpose(b, (0, 2, 1)) if tB else b
    ref = 1.5 * np.einsum("bmk,bkn->bmn", a, b)
    if shared:
        ref = ref.sum(axis=0, keepdims=True)
    assert _rel(Cm.cpu().numpy(), ref) < 1e-5


def _torch_reference(params, inp, L, modes):
    import torch
    import torch.nn.functional as Fn

    P = {k: torch.tensor(v, dtype=torch.float64, requires_grad=True) for k, v in params.items()}
    x = torch.tensor(inp, dtype=torch.float64)
    B, _, G, _ = x.shape
    v = torch.einsum("ci,bipq->bcpq", P["P_w"], x) + P["P_b"][None, :, None, None]
    for l in range(L):
        vf = torch.fft.rfft2(v)
        R = torch.complex(P[f"R{l}"][..., 0], P[f"R{l}"][..., 1]).reshape(v.shape[1], v.shape[1], 2 * modes, modes)
        out = torch.zeros(B, v.shape[1], G, G // 2 + 1, dtype=torch.complex128)
        out[:, :, :modes, :modes] = torch.einsum("bimk,iomk->bomk", vf[:, :, :modes, :modes], R[:, :, :modes])
        out[:, :, -modes:, :modes] = torch.einsum("bimk,iomk->bomk", vf[:, :, -modes:, :modes], R[:, :, modes:])
        z = torch.fft.irfft2(out, s=(G, G)) + torch.einsum("oc,bcpq->bopq", P[f"W{l}"], v) \
            + P[f"b{l}"][None, :, None, None]
        v = Fn.gelu(z) if l < L - 1 else z
    h = Fn.gelu(torch.einsum("hc,bcpq->bhpq", P["Q1_w"], v) + P["Q1_b"][None, :, None, None])
    y = torch.einsum("oh,bhpq->bopq", P["Q2_w"], h) + P["Q2_b"][None, :, None, None]
    return P, y


@pytest.mark.parametrize("G,width,modes,H", [(32, 8, 4, 16), (64, 32, 16, 64)])
def test_fno_forward_and_gradients(gpu_lib, G, width, modes, H):
    """A toy network, and the shipped network's channel, mode and hidden counts (32, 16, 64)
    on a 64 x 64 grid."""
    import torch

    from wavedg_b200 import fno

    L, B = 4, 2
    net = fno.FNO(grid=G, width=width, modes=modes, layers=L, hidden=H, seed=3)
    # larger spectral weights than the default initialisation so the Fourier branch matters
    for l in range(L):
        net.params[f"R{l}"].mul_(width * width / 4.0)
    net.refresh_bf16()
    inp = fno.inputs(G, [(0.1, -0.2), (-0.3, 0.25)], 0.15, 1.0)
    target = torch.from_numpy(np.random.default_rng(0).standard_normal((B, 3, G, G))).to("cuda", torch.float32)
    y = net.forward(inp, keep=True)
    sse, dy = net.mse(y, target.contiguous())
    net.backward(dy)
    torch.cuda.synchronize()
    params = {k: v.cpu().numpy().astype(np.float64) for k, v in net.params.items()}
    P, yr = _torch_reference(params, inp.cpu().numpy().astype(np.float64), L, modes)
    assert _rel(y.cpu().numpy(), yr.detach().numpy()) < 2e-2
    loss = ((yr - torch.tensor(target.cpu().numpy(), dtype=torch.float64)) ** 2).mean()
    assert abs(sse.item() / y.numel() - loss.item()) / loss.item() < 2e-2
    loss.backward()
    worst = {}
    for k in net.params:
        worst[k] = _rel(net.grads[k].cpu().numpy(), P[k].grad.numpy())
    print(f"G {G} width {width} modes {modes}: output {_rel(y.cpu().numpy(), yr.detach().numpy()):.1e}, gradients",
          {k: f"{v:.1e}" for k, v in worst.items()})
    assert max(worst.values()) < 4e-2, worst


def test_fno_training_reduces_loss(gpu_lib):
    """A few Adam steps on a fixed small batch bring the loss down."""
    import torch

    from wavedg_b200 import fno

    G = 32
    net = fno.FNO(grid=G, width=8, modes=4, layers=4, hidden=16, seed=1)
    inp = fno.inputs(G, [(0.1, -0.2), (-0.3, 0.25)], 0.15, 1.0)
    tgt = inp[:, :3].clone().contiguous()
    losses = []
    for _ in range(60):
        y = net.forward(inp, keep=True)
        sse, dy = net.mse(y, tgt)
        net.backward(dy)
        net.adam_step(lr=3e-3)
        losses.append(sse.item())
    assert losses[-1] < 0.2 * losses[0], losses[::10]


def test_resampling_bilinear_exact(gpu_lib):
    import torch

    from wavedg_b200 import fno
    from wavedg_b200.dg import QuadratureRule

    ne, n, G = 6, 5, 48
    xq = QuadratureRule.quadrature_rule(n, QuadratureRule.GaussLobatto).x
    h = 2.0 / ne
    u = np.zeros((ne * ne, n, n, 3))
    for el in range(ne * ne):
        ex, ey = el % ne, el // ne
        for b in range(n):
            for a in range(n):
                x = -1 + ex * h + 0.5 * h * (xq[a] + 1)
                y = -1 + ey * h + 0.5 * h * (xq[b] + 1)
                u[el, b, a] = (1 + 2 * x - y, x * y, 3 * y - 0.5)
    # layout u(d, i, j, el): d fastest, then i (x), then j (y)
    ud = torch.from_numpy(u.reshape(-1).copy()).to("cuda")
    rs = fno.NodalGrid(ne, n, G)
    g = rs.to_grid(ud, 2.0)
    xc = -1 + (np.arange(G) + 0.5) * 2 / G
    X, Y = np.meshgrid(xc, xc)
    ref = np.stack([1 + 2 * X - Y, X * Y, 3 * Y - 0.5]) * 2.0
    assert _rel(g.cpu().numpy(), ref) < 1e-6
    back = rs.to_nodes(g, 0.5)
    # bilinear reproduces bilinear fields inside the grid's cell-centre hull
    um = u.reshape(-1, 3)
    xs = np.array([[-1 + (el % ne) * h + 0.5 * h * (xq[a] + 1) for a in range(n)] for b in range(n)
                   for el in range(ne * ne)])
    bk = back.cpu().numpy().reshape(-1, 3)
    inside = []
    for el in range(ne * ne):
        ex, ey = el % ne, el // ne
        for b in range(n):
            for a in range(n):
                x = -1 + ex * h + 0.5 * h * (xq[a] + 1)
                y = -1 + ey * h + 0.5 * h * (xq[b] + 1)
                inside.append(abs(x) <= 1 - 1.0 / G and abs(y) <= 1 - 1.0 / G)
    inside = np.array(inside)
    assert _rel(bk[inside], um[inside]) < 1e-5
    del xs
