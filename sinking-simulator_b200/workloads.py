"""Seeded synthetic tet meshes for the batched and the served step.

This module loads no native library (numpy only), so the CPU baselines can build the
workload without the GPU library.

No dataset is involved: every mesh is a Kuhn-split box (fem::makeBoxTetMesh,
engine/sim/fem.cpp:217-263, restated in meshes.box_tet_mesh) of steel, shaped as a
beam or a plate, with a seeded size, material, clamped face and load.

  batch_meshes     many meshes with tet counts log-uniform in [lo, hi], yield uniform
                   in [235, 355] MPa, hardening modulus uniform in [0.5, 2] GPa; each
                   clamped on one random side face and loaded either at the opposite
                   (tip) face or by a pressure on its top face, with a magnitude scaled
                   to the load that first yields the clamped section, times U[0.5, 2].
  request_trace    Poisson arrivals of such meshes, each with its own step count.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

import meshes as M

DENSITY = 7850.0
YOUNGS = 210e9
POISSON = 0.3
# The Kuhn tet meshes here first yield at about 2.5 times the load that yields a beam
# of the same section (FP64 oracle, 1,000-step ramp plus 1,000 steps: plates at 2x the
# beam's load stay elastic or nearly so, at 4x a fifth to a half of their tets yield;
# beams yield from about 1.5x).  Scaled by U[0.5, 2], the batch then runs from
# elastic meshes to meshes with most of their tets yielded.
LOCKING = 2.5


@dataclass
class MeshSpec:
    """Everything needed to build one mesh and admit it."""
    seed: int
    cells: tuple            # (nx, ny, nz)
    size: tuple             # (lx, ly, lz) metres
    clamp: str              # "x0", "x1", "y0", "y1"
    load_kind: str          # "tip" or "pressure"
    load_factor: float      # times the first-yield load
    yield_strength: float
    hardening: float
    steps: int = 0
    ramp_steps: int = 0
    arrival: float = 0.0    # seconds (served requests)

    @property
    def tets(self) -> int:
        nx, ny, nz = self.cells
        return 6 * nx * ny * nz

    @property
    def nodes(self) -> int:
        nx, ny, nz = self.cells
        return (nx + 1) * (ny + 1) * (nz + 1)


@dataclass
class BuiltMesh:
    spec: MeshSpec
    position: np.ndarray
    index: np.ndarray
    fixed: np.ndarray
    external_force: np.ndarray

    def admit_kwargs(self):
        return dict(position=self.position, index=self.index, fixed=self.fixed, external_force=self.external_force,
                    density=DENSITY, youngs=YOUNGS, poisson=POISSON, yield_strength=self.spec.yield_strength,
                    hardening=self.spec.hardening, ramp_steps=self.spec.ramp_steps)


def _shape_for(n_target: int, rng: np.random.Generator):
    """Cells and size of a beam or a plate of about n_target tets (6 per cell)."""
    cells_total = max(1.0, n_target / 6.0)
    if rng.random() < 0.5:  # beam: ny = nz = k, nx = a k
        a = rng.uniform(4.0, 12.0)
        k = max(1, int(round((cells_total / a) ** (1.0 / 3.0))))
        nx = max(2, int(round(cells_total / (k * k))))
        ny = nz = k
        length = rng.uniform(0.5, 2.0)
        h = length * k / nx
        return (nx, ny, nz), (length, h, h)
    nz = 1 if cells_total < 4000 else 2  # plate: thin in z
    r = rng.uniform(1.0, 3.0)
    ny = max(2, int(round(math.sqrt(cells_total / (nz * r)))))
    nx = max(2, int(round(cells_total / (nz * ny))))
    lx = rng.uniform(0.5, 2.0)
    cell = lx / nx
    return (nx, ny, nz), (lx, cell * ny, cell * nz * 2.0)


def random_spec(rng: np.random.Generator, lo: float, hi: float, seed: int) -> MeshSpec:
    n = math.exp(rng.uniform(math.log(lo), math.log(hi)))
    cells, size = _shape_for(int(n), rng)
    if cells[1] > cells[2]:  # a plate: any side face
        clamp = ["x0", "x1", "y0", "y1"][int(rng.integers(0, 4))]
    else:                    # a beam: one end
        clamp = ["x0", "x1"][int(rng.integers(0, 2))]
    return MeshSpec(seed=seed, cells=cells, size=size, clamp=clamp,
                    load_kind="tip" if rng.random() < 0.5 else "pressure", load_factor=float(rng.uniform(0.5, 2.0)),
                    yield_strength=float(rng.uniform(235e6, 355e6)), hardening=float(rng.uniform(0.5e9, 2e9)))


def build(spec: MeshSpec) -> BuiltMesh:
    nx, ny, nz = spec.cells
    lx, ly, lz = spec.size
    pos, idx = M.box_tet_mesh(lx, ly, lz, nx, ny, nz)
    p = pos.reshape(-1, 3).astype(np.float64)
    axis = 0 if spec.clamp[0] == "x" else 1
    at_max = spec.clamp[1] == "1"
    extent = (lx, ly)[axis]
    eps = 1e-6 * extent
    clamped = (p[:, axis] > extent - eps) if at_max else (p[:, axis] < eps)
    fixed = clamped.astype(np.uint32)
    # first-yield load of the clamped section, as a cantilever of span `extent`, times
    # the mesh's stiffening: linear tets one to a few cells deep are several times
    # stiffer in bending than the beam, so their clamped section yields later
    width = (ly, lx)[axis]
    m_yield = LOCKING * spec.yield_strength * width * lz * lz / 6.0  # yield x elastic section modulus
    fext = np.zeros_like(p)
    if spec.load_kind == "tip":
        tip = (p[:, axis] < eps) if at_max else (p[:, axis] > extent - eps)
        total = spec.load_factor * m_yield / extent
        fext[tip, 2] = -total / tip.sum()
    else:
        top = p[:, 2] > lz - 1e-6 * lz
        total = spec.load_factor * 2.0 * m_yield / extent  # a uniform load: M = w L^2 / 2
        fext[top, 2] = -total / top.sum()
    return BuiltMesh(spec, pos, idx, fixed, fext.reshape(-1))


def batch_meshes(count=256, lo=2e3, hi=2e5, seed=20261203, steps=0, ramp_steps=1000):
    """Specs of the batched workload: `count` meshes of log-uniform size in [lo, hi]."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        s = random_spec(rng, lo, hi, seed=seed * 1000 + i)
        s.steps, s.ramp_steps = steps, ramp_steps
        specs.append(s)
    return specs


def drift_sample(specs):
    """Indices of eight meshes of a batch that between them cover its variety: the
    largest, and the smallest plate of each clamped face and load kind (x0, x1, y0, y1;
    tip and pressure) whose load factor is above 1.2, so that most of them yield.  The
    precision checks of the batched step run these."""
    def plate(s):
        return s.cells[1] > s.cells[2]

    picks = [max(range(len(specs)), key=lambda i: specs[i].tets)]
    for clamp, kind in (("x0", "tip"), ("x0", "pressure"), ("x1", "tip"), ("y0", "tip"), ("y0", "pressure"),
                        ("y1", "tip"), ("y1", "pressure")):
        c = [i for i, s in enumerate(specs) if plate(s) and s.clamp == clamp and s.load_kind == kind
             and s.load_factor > 1.2 and i not in picks]
        if c:
            picks.append(min(c, key=lambda i: specs[i].tets))
    return picks


def request_trace(rate=40.0, duration=120.0, lo=1e3, hi=5e5, steps=(500, 5000), seed=20261204):
    """Poisson arrivals at `rate` per second over `duration` seconds; each request is a
    mesh of log-uniform size in [lo, hi] with a step count uniform in `steps`."""
    rng = np.random.default_rng(seed)
    t, out, i = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        s = random_spec(rng, lo, hi, seed=seed * 100000 + i)
        s.steps = int(rng.integers(steps[0], steps[1] + 1))
        s.ramp_steps = max(1, s.steps // 2)
        s.arrival = t
        out.append(s)
        i += 1
    return out
