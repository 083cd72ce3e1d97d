#!/usr/bin/env python3
"""Benchmark of the B200 explicit FEM step: element-updates/s on one or more GPUs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One JSON line from rank 0.  `value` is element-updates/s over all ranks (each rank
steps its own replica: the meshes are independent, so there is no data-path
collective and the scaling is weak).  Inputs are resident in HBM when the timed region
starts; the device time is taken with CUDA events on the library's own stream around
exactly K steps, after W untimed warm-up steps, with a barrier and a device
synchronize on both sides, and the maximum over ranks is reported.  `e2e` is the same
metric through the C ABI from host buffers: upload (femstep_*_create), K steps,
readback, all inside the timed region.

Workloads (synthetic, seeded; no dataset is involved):
  tet-precision   the 200x20x20-cell Kuhn beam of the precision study (480,000 tets,
                  88,641 nodes), J2 FP32 with Kahan-compensated state
  tet-cantilever  the 40x4x4 config-0 cantilever (3,840 tets), J2 FP32-compensated
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sinking-simulator_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "element-updates/s @1 B200 (batched vs plain, % HBM peak); p50/p99 step latency"
UNIT = "element-updates/s"


# ---------------------------------------------------------------------------------
# workloads

def tet_beam(nx, ny, nz, length=1.0, width=0.1, depth=0.1, load=20e3):
    import femstep as F

    pos, idx = F.box_tet_mesh(length, width, depth, nx, ny, nz)
    fixed = (pos[0::3] < 1e-6).astype(np.uint32)
    tip = pos[0::3] > length - 1e-6
    fext = np.zeros(pos.size)
    fext[2::3][tip] = -load / tip.sum()
    return pos, idx, fixed, fext


WORKLOADS = {
    # precision-study beam, load scaled with the cross-section (20 kN on 0.1 x 0.1
    # grows with the grid as 1:1 here; the mesh is what sizes the workload)
    "tet-precision": dict(kind="tet", cells=(200, 20, 20), load=60e3, mode="f32k"),
    "tet-cantilever": dict(kind="tet", cells=(40, 4, 4), load=20e3, mode="f32k"),
}


def tet_bytes(T, N, mode):
    """Algorithmic bytes of one element-kernel launch and one node-kernel launch
    (each array counted once per launch; 4-byte ints)."""
    if mode == "f64":
        elem = T * (16 + 16 + 72 + 8 + 2 * 56 + 4 * 3 * 8) + N * 24
        node = N * (4 + 2 * 24 + 2 * 24 + 8 + 1 + 24) + T * 4 * 24
    else:
        comp = 2 if mode == "f32k" else 1
        elem = T * (16 + 16 + 36 + 4 + comp * 2 * 28 + 4 * 12) + N * 12
        node = N * (4 + comp * 2 * 12 + 2 * 12 + 4 + 4 + 1 + 12) + T * 4 * 12
    return elem, node


# ---------------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device = device_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------------

def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get(workload)
    return None


def cpu_baseline(wl, seconds=15.0):
    """The reference's CPU path on this box's host cores, on a bounded sample of the
    same workload: the compiled reference (oracle/_ref) when present, else the C
    restatement.  O-tet64: fem.cpp kinematics + plasticity::update in double, element
    loop over all host cores with core::JobSystem, serial CSR gather."""
    import oracle as O

    kind = "reference" if O.have_ref() else "port"
    o = O.Oracle("ref" if kind == "reference" else "port")
    pos, idx, fixed, fext = tet_beam(*wl["cells"], load=wl["load"])
    m = O.TetMesh64(o, pos, idx, fixed, fext)
    p = O.tet64_params(dt=1e-7, ramp_steps=2000)
    workers = os.cpu_count() or 1
    T = idx.size // 4
    if kind == "reference":
        rate = o.tet64_time_parallel(C.byref(m._s), C.byref(p), 1, workers)  # warm
        steps = max(1, int(seconds * rate / T))
        rate = o.tet64_time_parallel(C.byref(m._s), C.byref(p), steps, workers)
        cores = workers
    else:
        t0 = time.perf_counter()
        m.step(p, 1)
        rate = T / (time.perf_counter() - t0)
        steps = max(1, int(seconds * rate / T))
        t0 = time.perf_counter()
        m.step(p, steps)
        rate = T * steps / (time.perf_counter() - t0)
        cores = 1
    return {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{steps} steps of the {T}-tet workload mesh, FP64 J2 (O-tet64)"}


def run_reference(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t_all = []
    base = None
    for _ in range(args.warmup):
        cpu_baseline(wl, seconds=2.0)
    for _ in range(args.steps):
        base = cpu_baseline(wl, seconds=max(2.0, 30.0 / max(args.steps, 1)))
        t_all.append(base["value"])
    value = float(np.median(t_all))
    base["value"] = value
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": args.workload, "tets": int(np.prod(wl["cells"]) * 6)},
           "cpu_baseline": base, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                         "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tet-precision", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, wl)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        os.environ.setdefault("CUDA_VISIBLE_DEVICES", str(local))
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        os.environ.setdefault("CUDA_VISIBLE_DEVICES", "0")

    import femstep as F

    pos, idx, fixed, fext = tet_beam(*wl["cells"], load=wl["load"])
    T, N = idx.size // 4, pos.size // 3
    s = F.TetSolver(pos, idx, mode=wl["mode"], fixed=fixed, external_force=fext, density=7850.0)
    dt = s.critical_dt(210e9, 0.3, 7850.0, 0.9)
    kw = dict(dt=dt, ramp_steps=2000)

    s.run(args.warmup, **kw)

    def barrier():
        if dist is not None:
            import torch

            torch.cuda.synchronize()
            dist.barrier()

    barrier()
    with ClockSampler(local) as clocks:
        ms = s.run(args.steps, **kw)
    launches = s.launches
    barrier()
    if dist is not None:
        import torch

        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = T * args.steps * world / (ms / 1e3)

    # per-kernel device time for the roofline (separate, untimed for `value`)
    elem_ms, node_ms = s.profile(20, **kw)
    elem_b, node_b = tet_bytes(T, N, wl["mode"])
    peak, peak_kind = measured_peak()
    achieved = elem_b / (elem_ms / 1e3) / 1e9
    traffic = ncu_traffic(args.workload)
    s.close()

    # end to end through the C ABI from host buffers
    t0 = time.perf_counter()
    e = F.TetSolver(pos, idx, mode=wl["mode"], fixed=fixed, external_force=fext, density=7850.0)
    e.run(args.steps, **kw)
    p_host, v_host = e.readback()
    e.close()
    wall = time.perf_counter() - t0
    h2d = pos.nbytes + idx.nbytes + fixed.nbytes + fext.nbytes
    d2h = p_host.nbytes + v_host.nbytes

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "tets": T, "nodes": N, "mode": wl["mode"], "dt": dt,
                   "element_kernel_ms": elem_ms, "node_kernel_ms": node_ms,
                   "step_effective_gbs": (elem_b + node_b) / (ms / args.steps / 1e3) / 1e9,
                   "l2": "inputs larger than L2 (%.0f MB per step)" % ((elem_b + node_b) / 1e6),
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": T * args.steps / wall, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": "element (f32_forces)",
                     "peak_source": peak_kind},
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(wl)
    print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
