"""Mesh generators and the node -> corner CSR, in numpy only.

Vectorised restatements of the reference's generators, so that workloads of millions
of elements are built in milliseconds; tests pin them to the reference's own.  This
module loads no native library, so code that only builds inputs (the CPU baselines,
the workload generators) can use it without bringing up the GPU library.
"""
from __future__ import annotations

import numpy as np

_KUHN = np.array([[0, 1, 3, 7], [0, 1, 7, 5], [0, 5, 7, 4], [0, 3, 2, 7], [0, 2, 6, 7], [0, 4, 6, 7]])


def box_tet_mesh(lx, ly, lz, nx, ny, nz):
    """fem::makeBoxTetMesh (engine/sim/fem.cpp:217-263): node (k*sy+j)*sx+i, six Kuhn
    tets per cell about the 0-7 diagonal, orientation fixed by swapping corners 1, 2."""
    sx, sy, sz = nx + 1, ny + 1, nz + 1
    k, j, i = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx), indexing="ij")
    pos = np.empty((sz, sy, sx, 3), np.float32)
    pos[..., 0] = np.float32(lx) * i.astype(np.float32) / np.float32(nx)
    pos[..., 1] = np.float32(ly) * j.astype(np.float32) / np.float32(ny)
    pos[..., 2] = np.float32(lz) * k.astype(np.float32) / np.float32(nz)
    pos = pos.reshape(-1)
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ci, cj, ck = ci.reshape(-1), cj.reshape(-1), ck.reshape(-1)
    corner = np.empty((ci.size, 8), np.uint32)
    for c in range(8):
        corner[:, c] = ((ck + ((c >> 2) & 1)) * sy + (cj + ((c >> 1) & 1))) * sx + (ci + (c & 1))
    tets = corner[:, _KUHN].reshape(-1, 4)  # cell-major, six per cell
    p = pos.reshape(-1, 3)
    d = p[tets[:, 1:]] - p[tets[:, :1]]          # (T, 3 edges, 3 axes)
    # determinant in float with fem.cpp's cofactor order (columns = edges)
    a = np.transpose(d, (0, 2, 1))              # a[t, row(axis), col(edge)]
    det = (a[:, 0, 0] * (a[:, 1, 1] * a[:, 2, 2] - a[:, 1, 2] * a[:, 2, 1])
           - a[:, 0, 1] * (a[:, 1, 0] * a[:, 2, 2] - a[:, 1, 2] * a[:, 2, 0])
           + a[:, 0, 2] * (a[:, 1, 0] * a[:, 2, 1] - a[:, 1, 1] * a[:, 2, 0]))
    flip = det < 0
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    return pos, tets.reshape(-1).astype(np.uint32)


def csr(nodes, index, corners):
    """Node -> corner CSR by counting sort (fem.cpp:147-157, zone.cpp:739-754)."""
    index = np.asarray(index, np.int64).reshape(-1)
    counts = np.bincount(index, minlength=nodes)
    offset = np.zeros(nodes + 1, np.uint32)
    offset[1:] = np.cumsum(counts)
    entry = np.argsort(index, kind="stable").astype(np.uint32)
    return offset, entry


def plate_mesh(lx, ly, thickness, nx, ny, nz=1):
    """solidshell::makePlateMesh (engine/sim/solid_shell.cpp:1152-1185): node
    (i*sy + j)*sz + k, thickness index fastest, mid-surface at z = 0."""
    sy, sz = ny + 1, nz + 1
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    pos = np.empty(i.shape + (3,))
    pos[..., 0] = lx * i.astype(np.float64) / nx
    pos[..., 1] = ly * j.astype(np.float64) / ny
    pos[..., 2] = -0.5 * thickness + thickness * k.astype(np.float64) / nz
    ei, ej, ek = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ei, ej, ek = ei.reshape(-1), ej.reshape(-1), ek.reshape(-1)

    def at(a, b, c):
        return ((a * sy + b) * sz + c).astype(np.uint32)

    idx = np.stack([at(ei, ej, ek), at(ei + 1, ej, ek), at(ei + 1, ej + 1, ek), at(ei, ej + 1, ek),
                    at(ei, ej, ek + 1), at(ei + 1, ej, ek + 1), at(ei + 1, ej + 1, ek + 1), at(ei, ej + 1, ek + 1)],
                   axis=1)
    return pos.reshape(-1), idx.reshape(-1)


def plate_pressure_load(position, index, pressure=1.0):
    """Consistent nodal loads of a pressure on the +zeta face of every element
    (solidshell::uniformPressureLoad, solid_shell.cpp:1505-1553, for one element
    through the thickness, where every top face is a boundary face), vectorised."""
    pos = np.asarray(position, np.float64).reshape(-1, 3)
    top = np.asarray(index, np.int64).reshape(-1, 8)[:, 4:8]
    load = np.zeros_like(pos)
    q = 1.0 / np.sqrt(3.0)
    corner = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], np.float64)
    x = pos[top]  # (E, 4, 3)
    for gs in (-q, q):
        for gt in (-q, q):
            shape = 0.25 * (1 + gs * corner[:, 0]) * (1 + gt * corner[:, 1])
            ds = 0.25 * corner[:, 0] * (1 + gt * corner[:, 1])
            dt = 0.25 * corner[:, 1] * (1 + gs * corner[:, 0])
            xs = np.einsum("c,eci->ei", ds, x)
            xt = np.einsum("c,eci->ei", dt, x)
            area = np.cross(xs, xt)
            contrib = -pressure * shape[None, :, None] * area[:, None, :]
            np.add.at(load, top, contrib)
    return load.reshape(-1)


def stiffened_panel(nx=2000, ny=1000, lx=20.0, ly=10.0, thickness=0.012, stiffeners=6, imperfection=1e-3,
                    peak_pressure=0.5e6, radius=1.5, seed=20261203):
    """The stiffened plate panel of the single-large-mesh workload: lx x ly plate of
    `thickness`, one solid-shell element through the thickness, edges clamped, the
    plating nodes on `stiffeners` evenly spaced longitudinal lines pinned (the
    reference's Stiffeners::RigidSupport, zone.hpp:380-390, zone.cpp:583-592), a seeded
    Gaussian out-of-plane imperfection applied identically to both faces of each
    through-thickness node pair, and a Gaussian pressure of `peak_pressure` and 1/e^0.5
    radius `radius` centred on the plate.  Returns (rest, index, pinned, load_at_peak)."""
    rest, index = plate_mesh(lx, ly, thickness, nx, ny, 1)
    p = rest.reshape(-1, 3)
    rng = np.random.default_rng(seed)
    bump = rng.normal(0.0, imperfection, (nx + 1) * (ny + 1))
    p[:, 2] += np.repeat(bump, 2)  # thickness index fastest: pairs (k = 0, 1) share it
    i = np.arange(p.shape[0]) // (2 * (ny + 1))
    j = (np.arange(p.shape[0]) // 2) % (ny + 1)
    edge = (i == 0) | (i == nx) | (j == 0) | (j == ny)
    lines = {int(round(ny * s / (stiffeners + 1))) for s in range(1, stiffeners + 1)}
    stiff = np.isin(j, list(lines))
    pinned = np.repeat(edge | stiff, 3).astype(np.uint8)
    unit = plate_pressure_load(rest, index, 1.0).reshape(-1, 3)
    r2 = (p[:, 0] - lx / 2) ** 2 + (p[:, 1] - ly / 2) ** 2
    load = unit * (peak_pressure * np.exp(-r2 / (2 * radius ** 2)))[:, None]
    return rest, index, pinned, load.reshape(-1)
