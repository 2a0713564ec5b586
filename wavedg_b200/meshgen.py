"""Quad-mesh generators: vertex arrays (nv, 2) and quads (nel, 4), corners CCW.

``uniform_rect`` numbers vertices and elements exactly as the reference's
``Mesh2D::uniform_rect`` (source/Mesh2D.cpp:130-163), so bc-code arrays and
state vectors line up element for element with a reference run on the same
mesh.  The others build the workloads and parity cases: seeded vertex
perturbation (bilinear, non-affine elements), scrambled connectivity (random
element order and corner rotation, which exercises every side pairing and
both edge orientations), and an L-shaped domain.
"""
from __future__ import annotations

import numpy as np


def uniform_rect(nx: int, ax: float, bx: float, ny: int, ay: float, by: float):
    dx = (bx - ax) / nx
    dy = (by - ay) / ny
    j, i = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    verts = np.stack([ax + dx * i, ay + dy * j], axis=-1).reshape(-1, 2)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    v = lambda a, b: a + (nx + 1) * b  # noqa: E731
    quads = np.stack([v(ii, jj), v(ii + 1, jj), v(ii + 1, jj + 1), v(ii, jj + 1)], axis=-1).reshape(-1, 4)
    return verts.astype(np.float64), quads.astype(np.int32)


def perturbed_rect(n: int, frac: float = 0.2, seed: int = 0, lo: float = -1.0, hi: float = 1.0):
    """n x n elements on [lo, hi]^2; interior vertices moved by U(-frac h, frac h) in x and y."""
    verts, quads = uniform_rect(n, lo, hi, n, lo, hi)
    h = (hi - lo) / n
    rng = np.random.default_rng(seed)
    g = verts.reshape(n + 1, n + 1, 2)
    d = rng.uniform(-frac * h, frac * h, size=(n - 1, n - 1, 2))
    g[1:-1, 1:-1, :] += d
    return g.reshape(-1, 2).copy(), quads


def scrambled(verts, quads, seed: int = 0):
    """Random element order and random cyclic rotation of each quad's corners."""
    rng = np.random.default_rng(seed)
    q = np.asarray(quads)[rng.permutation(len(quads))]
    rot = rng.integers(0, 4, size=len(q))
    idx = (np.arange(4)[None, :] + rot[:, None]) % 4
    q = np.take_along_axis(q, idx, axis=1)
    return np.asarray(verts, dtype=np.float64), q.astype(np.int32)


def l_shape(n: int):
    """[-1,1]^2 without the open quadrant (0,1]x(0,1], n x n cells per unit square."""
    verts, quads = uniform_rect(2 * n, -1.0, 1.0, 2 * n, -1.0, 1.0)
    c = verts[quads].mean(axis=1)
    keep = ~((c[:, 0] > 0) & (c[:, 1] > 0))
    q = quads[keep]
    used = np.unique(q)
    remap = -np.ones(len(verts), dtype=np.int64)
    remap[used] = np.arange(len(used))
    return verts[used].copy(), remap[q].astype(np.int32)


def boundary_codes_by_wall(midpoints, left=1, right=0, bottom=1, top=0, other=0, tol=1e-12):
    """Per-boundary-edge codes chosen by which wall of [-1,1]^2 the edge lies on."""
    x, y = midpoints[:, 0], midpoints[:, 1]
    codes = np.full(len(midpoints), other, dtype=np.int32)
    codes[np.abs(y - 1.0) < tol] = top
    codes[np.abs(x - 1.0) < tol] = right
    codes[np.abs(y + 1.0) < tol] = bottom
    codes[np.abs(x + 1.0) < tol] = left
    return codes
