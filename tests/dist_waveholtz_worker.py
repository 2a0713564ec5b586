"""One rank of a decomposed WaveHoltz solve over torch.distributed (run by
tests/test_gpu_decomp.py as separate processes; not a test module itself).

    python tests/dist_waveholtz_worker.py OUT.npz     # RANK, WORLD_SIZE, MASTER_ADDR/PORT set

Solves the WaveHoltz problem of tests/golden/waveholtz_5x5_P3.npz (the reference's own
solve) on this rank's share of an RCB partition, exchanging halo traces and norm sums through
the process group (gloo: through host buffers), and writes its local iterate, its element
ids, the iteration count and the residual to OUT.npz.
"""
import os
import sys
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main(out):
    import torch
    import torch.distributed as dist

    import wavedg_b200 as W
    from wavedg_b200 import decomp

    backend = os.environ.get("WDG_DIST_BACKEND", "gloo")
    dist.init_process_group(backend, timeout=timedelta(seconds=120))
    try:
        rank, world = dist.get_rank(), dist.get_world_size()
        torch.cuda.set_device(0)
        g = np.load(os.path.join(ROOT, "tests", "golden", "waveholtz_5x5_P3.npz"))
        mesh = W.Mesh2D.from_vertices(g["verts"], g["quads"])
        basis = W.QuadratureRule.quadrature_rule(int(g["n"]), W.QuadratureRule.GaussLobatto)
        part = decomp.partition_mesh(mesh, world, "rcb")
        d = decomp.Domain(mesh, basis, g["bc"], part, rank)
        wh = decomp.DomainWaveHoltz(d, float(g["omega"]), mesh.min_h())
        F = torch.from_numpy(d.local(g["F"])).cuda()
        Wl, it, res = decomp.waveholtz_solve([wh], [F], 1e-6, 200, decomp.dist_exchange(d),
                                            decomp.dist_allreduce(device=d.device))
        np.savez(out, W=Wl[0].cpu().numpy(), elems=d.plan.local, iters=it, res=res, nt=wh.nt, dt=wh.dt)
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
