#!/usr/bin/env python3
"""Drift of the GPU step against the FP64 oracle over whole runs (test infrastructure).

    python tests/drift_study.py [tet-precision] [shell-bay] [tet-batch]
                                [--oracle-cache DIR] [--oracle-only] [--threads N]

Each study prints one JSON line: the errors of the GPU results against the FP64 CPU
oracle (oracle/femoracle.c, pinned bit for bit to the reference), over
  tet-precision  the precision-study beam: 200 x 20 x 20 cells x 6 Kuhn tets (480,000
                 tets), 165 kN tip load ramped over 10,000 steps, 20,000 steps at 0.9 x
                 the FP64 element bound; GPU FP32, FP32-compensated and FP64;
  shell-bay      a bay of the single-large-mesh panel (its 10 mm cells, 12 mm plating,
                 1 mm seeded imperfection, 0.5 MPa Gaussian pulse of 1.5 m with a 5 ms
                 rise; 200 x 143 cells between two stiffener lines, clamped edges) for
                 5,000 steps, through the rise; GPU FP32-compensated;
  tet-batch      the batched workload's drift sample (workloads.drift_sample: the
                 largest mesh and the smallest plate of each clamped face and load kind)
                 in one pool for the 1,000-step ramp plus 1,000 steps; GPU FP32-compensated.
Errors: max |a - a64| / max |a64| of the displacement (over nodes), of the von Mises
stress (from the final state, through one routine for every variant) and of the
equivalent plastic strain; the energy terms (external work, dissipation, strain,
kinetic) against the oracle's, over the external work; each variant's own energy
balance |W - (D + U + K)| / W.

The oracle's side of a study depends only on its inputs.  --oracle-only computes it on
this machine's cores and stores it under --oracle-cache; a later run with the same
cache (on a GPU machine) loads it instead of recomputing, after checking that the
inputs match.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (os.path.join(ROOT, "sinking-simulator_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

import meshes as M  # noqa: E402
import oracle as O  # noqa: E402

SHELL_MAT = dict(youngs=206e9, poisson=0.3, yield_strength=355e6, hardening=1e9)


def tet_von_mises(position, rest, index, plastic, mu, kappa):
    """Von Mises stress per tet in FP64 from a state (positions, plastic strain): the
    co-rotated strain of fem.cpp's tet (four Higham iterations), sigma = 2 mu dev(e -
    ep) + kappa tr(e - ep) I.  The same routine for every variant."""
    x = np.asarray(position, np.float64).reshape(-1, 3)
    X = np.asarray(rest, np.float64).reshape(-1, 3)
    idx = np.asarray(index).reshape(-1, 4).astype(np.int64)
    dm = np.stack([X[idx[:, c]] - X[idx[:, 0]] for c in (1, 2, 3)], axis=2)
    ds = np.stack([x[idx[:, c]] - x[idx[:, 0]] for c in (1, 2, 3)], axis=2)
    f = ds @ np.linalg.inv(dm)
    r = f.copy()
    for _ in range(4):
        r = 0.5 * (r + np.transpose(np.linalg.inv(r), (0, 2, 1)))
    sm = np.transpose(r, (0, 2, 1)) @ f
    e = 0.5 * (sm + np.transpose(sm, (0, 2, 1))) - np.eye(3)
    ep = np.asarray(plastic).reshape(-1, 7)
    el = np.empty((len(idx), 6))
    el[:, 0], el[:, 1], el[:, 2] = e[:, 0, 0] - ep[:, 0], e[:, 1, 1] - ep[:, 1], e[:, 2, 2] - ep[:, 2]
    el[:, 3], el[:, 4], el[:, 5] = 2 * e[:, 0, 1] - ep[:, 3], 2 * e[:, 1, 2] - ep[:, 4], 2 * e[:, 2, 0] - ep[:, 5]
    tr = el[:, 0] + el[:, 1] + el[:, 2]
    s = 2 * mu * (el[:, :3] - tr[:, None] / 3)
    t = mu * el[:, 3:]
    return np.sqrt(1.5 * ((s ** 2).sum(1) + 2 * (t ** 2).sum(1)))


def errors(u, u64, vm, vm64, ep, ep64, e, e64):
    def balance(x):
        w = x[0] + (x[4] if len(x) > 4 else 0.0)
        return float(abs(w - (x[1] + x[2] + x[3])) / abs(w))

    e, e64 = np.asarray(e, np.float64), np.asarray(e64, np.float64)
    return {"max_rel_displacement_error": float(np.abs(u - u64).max() / np.abs(u64).max()),
            "max_rel_von_mises_error": float(np.abs(vm - vm64).max() / vm64.max()),
            "max_rel_plastic_strain_error": float(np.abs(ep - ep64).max() / ep64.max()) if ep64.max() > 0 else 0.0,
            "energy_terms_vs_work": float(np.abs(e[:4] - e64[:4]).max() / abs(e64[0])),
            "energy_balance": balance(e), "energy_balance_fp64_oracle": balance(e64)}


class Cache:
    """Oracle results stored by study name, with a digest of the inputs."""

    def __init__(self, path):
        self.path = path

    def _file(self, name):
        return os.path.join(self.path, name + ".npz") if self.path else None

    def load(self, name, digest):
        f = self._file(name)
        if not f or not os.path.exists(f):
            return None
        z = np.load(f)
        if str(z["digest"]) != digest:
            raise SystemExit(f"{f}: cached oracle results are for other inputs")
        return {k: z[k] for k in z.files if k != "digest"}

    def save(self, name, digest, **arrays):
        if self.path:
            os.makedirs(self.path, exist_ok=True)
            np.savez_compressed(self._file(name), digest=np.array(digest), **arrays)


def digest(*arrays, **scalars):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(json.dumps(scalars, sort_keys=True).encode())
    return h.hexdigest()[:32]


# ---------------------------------------------------------------------------------

def tet_precision(args, cache):
    cells, load, ramp, steps = (200, 20, 20), 165e3, 10000, 20000
    pos, idx = M.box_tet_mesh(1.0, 0.1, 0.1, *cells)
    fixed = (pos[0::3] < 1e-6).astype(np.uint32)
    tip = pos[0::3] > 1.0 - 1e-6
    fext = np.zeros(pos.size)
    fext[2::3][tip] = -load / tip.sum()
    port = O.Oracle("port")
    ref = O.TetMesh64(port, pos, idx, fixed, fext)
    dt = port.tet64_critical_dt(C.byref(ref._s), 210e9, 0.3, 7850.0, 0.9)
    mu, kappa = 210e9 / 2.6, 210e9 / (3 * 0.4)
    rest = pos.astype(np.float64)
    key = digest(pos, idx, fixed, fext, dt=dt, steps=steps, ramp=ramp)
    got = cache.load("tet-precision", key)
    if got is None:
        t0 = time.perf_counter()
        ref.step(O.tet64_params(dt=dt, ramp_steps=ramp), steps, threads=args.threads)
        pl = ref.plastic.reshape(-1, 7)
        got = dict(position=ref.position.copy(), ep=pl[:, 6].copy(),
                   vm=tet_von_mises(ref.position, rest, idx, pl, mu, kappa), energy=ref.energy.copy(),
                   seconds=np.array(time.perf_counter() - t0))
        cache.save("tet-precision", key, **got)
    out = {"study": "tet-precision", "tets": idx.size // 4, "nodes": pos.size // 3, "steps": steps, "dt": dt,
           "tip_load_n": load, "ramp_steps": ramp, "oracle_seconds": float(got["seconds"]),
           "yielded_fraction_fp64": float((got["ep"] > 0).mean())}
    if args.oracle_only:
        return out
    import femstep as F

    for mode in ("f64", "f32k", "f32"):
        s = F.TetSolver(pos, idx, mode=mode, fixed=fixed, external_force=fext, density=7850.0)
        assert s.critical_dt(210e9, 0.3, 7850.0, 0.9) == dt
        ms = s.run(steps, dt=dt, ramp_steps=ramp)
        p, _ = s.readback64()
        pl = s.plastic()
        e = s.energy()
        s.close()
        r = errors(p - rest, got["position"] - rest, tet_von_mises(p, rest, idx, pl, mu, kappa), got["vm"],
                   pl[:, 6], got["ep"], e, got["energy"])
        r["bit_identical_to_oracle"] = bool(np.array_equal(p, got["position"]) and np.array_equal(pl[:, 6], got["ep"]))
        r["elem_upd_per_s"] = (idx.size // 4) * steps / (ms / 1e3)
        out[mode] = r
    return out


def shell_bay(args, cache, steps=5000, nx=200, ny=143):
    rest, index, pinned, load = M.stiffened_panel(nx=nx, ny=ny, lx=0.01 * nx, ly=0.01 * ny, thickness=0.012,
                                                  stiffeners=0, imperfection=1e-3, peak_pressure=0.5e6, radius=1.5)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    port = O.Oracle("port")
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    # the element bound in FP64, the same number the device forms (bit-identical)
    corners = rest.reshape(-1, 3)[index.reshape(-1, 8).astype(np.int64)].reshape(-1, 24)
    per = [port.shell_critical_dt(np.ascontiguousarray(c), 206e9, 0.3, 7850.0, 2, 0.9) for c in corners]
    dt = min(x for x in per if x > 0)
    key = digest(rest, index, pinned, load, dt=dt, steps=steps)
    got = cache.load("shell-bay", key)
    if got is None:
        t0 = time.perf_counter()
        ref.step(dt, steps, rise_time=5e-3, threads=args.threads)
        st = ref.state.reshape(-1, 129)
        got = dict(position=ref.position.copy(), ep=st[:, 12:120:15].copy(), vm=ref.von_mises(ref.position, st),
                   energy=ref.compute_energy().copy(), seconds=np.array(time.perf_counter() - t0))
        cache.save("shell-bay", key, **got)
    out = {"study": "shell-bay", "elements": index.size // 8, "nodes": rest.size // 3, "steps": steps, "dt": dt,
           "simulated_ms": steps * dt * 1e3, "rise_ms": 5.0, "oracle_seconds": float(got["seconds"]),
           "yielded_gauss_points_fp64": int((got["ep"] > 0).sum())}
    if args.oracle_only:
        return out
    import femstep as F

    s = F.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0)
    assert s.critical_dt(206e9, 0.3, 7850.0, 0.9) == dt
    ms = s.run(steps, dt=dt, rise_time=5e-3, compensated=True, max_iterations=12, **SHELL_MAT)
    p, _ = s.readback()
    st = s.state()
    e = s.energy()
    stats = s.stats()
    s.close()
    r = errors(p - rest, got["position"] - rest, ref.von_mises(p, st), got["vm"], st[:, 12:120:15], got["ep"],
               e, got["energy"])
    r["elem_upd_per_s"] = (index.size // 8) * steps / (ms / 1e3)
    r["newton"] = stats
    out["f32k"] = r
    return out


def tet_batch(args, cache, steps=2000):
    import workloads as W

    specs = W.batch_meshes(256)
    picks = W.drift_sample(specs)
    built = [W.build(specs[i]) for i in picks]
    port = O.Oracle("port")
    mu, kappa = W.YOUNGS / (2 * (1 + W.POISSON)), W.YOUNGS / (3 * (1 - 2 * W.POISSON))
    refs = []
    for i, b in zip(picks, built):
        m = O.TetMesh64(port, b.position, b.index, b.fixed, b.external_force)
        dt = port.tet64_critical_dt(C.byref(m._s), W.YOUNGS, W.POISSON, W.DENSITY, 0.9)
        key = digest(b.position, b.index, b.fixed, b.external_force, dt=dt, steps=steps,
                     y=b.spec.yield_strength, h=b.spec.hardening, ramp=b.spec.ramp_steps)
        got = cache.load(f"tet-batch-{i}", key)
        if got is None:
            m.step(O.tet64_params(dt=dt, ramp_steps=b.spec.ramp_steps, yield_=b.spec.yield_strength,
                                  hardening=b.spec.hardening), steps, threads=args.threads)
            pl = m.plastic.reshape(-1, 7)
            got = dict(position=m.position.copy(), ep=pl[:, 6].copy(),
                       vm=tet_von_mises(m.position, b.position, b.index, pl, mu, kappa), energy=m.energy.copy())
            cache.save(f"tet-batch-{i}", key, **got)
        refs.append((dt, got))
    out = {"study": "tet-batch", "meshes": picks, "steps": steps}
    if args.oracle_only:
        return out
    import femstep as F

    T = sum(b.spec.tets for b in built)
    N = sum(b.spec.nodes for b in built)
    pool = F.TetPool(T, N + len(built) + 1, max_meshes=len(built) + 1)
    ids = [pool.admit(steps=steps, dt=dt, **b.admit_kwargs()) for b, (dt, _) in zip(built, refs)]
    pool.run(steps)
    rows = []
    for b, i, (dt, got) in zip(built, ids, refs):
        p, _ = pool.readback(i)
        pl = pool.plastic(i)
        rest = b.position.astype(np.float64)
        r = errors(p - rest, got["position"] - rest, tet_von_mises(p, rest, b.index, pl, mu, kappa), got["vm"],
                   pl[:, 6], got["ep"], pool.energy(i), got["energy"])
        r.update(tets=b.spec.tets, clamp=b.spec.clamp, load=b.spec.load_kind,
                 yielded_fraction_fp64=float((got["ep"] > 0).mean()))
        rows.append(r)
    pool.close()
    for k in ("max_rel_displacement_error", "max_rel_von_mises_error", "max_rel_plastic_strain_error",
              "energy_terms_vs_work"):
        out[k] = max(r[k] for r in rows)
    out["per_mesh"] = rows
    return out


STUDIES = {"tet-precision": tet_precision, "shell-bay": shell_bay, "tet-batch": tet_batch}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("studies", nargs="*", default=list(STUDIES))
    ap.add_argument("--oracle-cache", default=None)
    ap.add_argument("--oracle-only", action="store_true")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    cache = Cache(args.oracle_cache)
    for name in args.studies:
        t0 = time.perf_counter()
        out = STUDIES[name](args, cache)
        out["wall_seconds"] = time.perf_counter() - t0
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
