"""What the trained network gains over the method without it, on a small copy of the family.
(Collected after the other GPU tests: it is the slowest of them.)

32 x 32 elements of [-1, 1]^2, P = 4, omega = 20, one Gaussian source (sigma 0.05) centred in
[-0.5, 0.5]^2, outflow boundary.  The batch generates 48 training solutions, a small FNO is
trained on them (BF16 GEMMs, hand-written backward, the square's symmetries), and 16 fresh
problems are solved from zero and from the network's prediction.  Both arms end with the
plain FP64 iteration at residual < 1e-6; the warm start must need clearly fewer iterations.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_warm_start_needs_fewer_iterations(gpu_lib):
    import torch

    from wavedg_b200 import warmstart as ws
    from wavedg_b200.fno import FNO

    fam = ws.Family(16, ne=32)
    G = 64
    cs, grids = ws.make_dataset(fam, 48, 11, 1e-4, G, log=lambda *_: None)
    scale = math.sqrt(grids.square().mean().item())
    grids /= scale
    net = FNO(grid=G, width=16, modes=8, layers=4, hidden=32, seed=3)
    hist, _ = ws.train(net, cs, grids, epochs=200, batch=4, lr=3e-3, seed=5, log=lambda *_: None)
    assert hist[-1] < 0.25 * hist[0], hist[::20]

    probs = ws.centers(16, 23)
    F = fam.forcing(probs)
    Wc, it32c, it64c, r64c, stc = fam.solve(F, 1e-6)
    W0 = ws.predict(net, fam, probs, scale)
    # the prediction alone is already close: relative error against the converged answer
    pred_err = max((W0[i] - Wc[i]).norm().item() / Wc[i].norm().item() for i in range(16))
    Ww, it32w, it64w, r64w, stw = fam.solve(F, 1e-6, W0=W0)
    print(f"training error {hist[-1]:.3e}, prediction error {pred_err:.3e}; FP32 iterations cold "
          f"{it32c.mean():.1f} warm {it32w.mean():.1f}; FP64 finish cold {it64c.mean():.1f} warm {it64w.mean():.1f}")
    assert (stc == 0).all() and (stw == 0).all()
    assert (r64c < 1e-6).all() and (r64w < 1e-6).all()
    assert pred_err < 0.15
    assert it32w.mean() + it64w.mean() < 0.9 * (it32c.mean() + it64c.mean())
    for i in range(16):
        # the same fixed point to within what the tolerance allows
        assert (Ww[i] - Wc[i]).norm().item() < 2e-5 * Wc[i].norm().item()
    torch.cuda.synchronize()
