#!/usr/bin/env python3
"""Benchmark of the B200 explicit FEM step: element-updates/s on one or more GPUs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One JSON line from rank 0.  `value` is element-updates/s over all ranks: each rank
steps its own replica (the meshes are independent, so there is no data-path
collective and the scaling is weak).  Inputs are resident in HBM when the timed region
starts; device time is taken with CUDA events on the library's stream around exactly
K steps, after W untimed warm-up steps, with a barrier and a device synchronize on
both sides; the maximum over ranks is reported.  Every workload moves more bytes per
step than the 126 MB L2 holds, so no flush is needed between steps.  `e2e` is the same
metric through the C ABI from host buffers: upload (femstep_*_create), K steps and the
readback of positions and velocities, all inside one wall-clock region.

Workloads (synthetic and seeded; no dataset is involved):
  shell-panel     the single-large-mesh case: a 20 x 10 m, 12 mm stiffened panel as
                  2000 x 1000 solid-shell hexes (2.0 M elements, 4.0 M nodes), six
                  longitudinal stiffener lines pinned, edges clamped, 1 mm seeded
                  imperfection, 0.5 MPa Gaussian pulse (1.5 m, 5 ms rise); FP32 with
                  Kahan-compensated state.
  tet-precision   the precision-study beam, 200 x 20 x 20 cells x 6 Kuhn tets (480,000
                  tets), J2 FP32-compensated, 200 kN tip load ramped over 10,000 steps
  tet-cantilever  the 40 x 4 x 4 cantilever (3,840 tets), same element
  tet-precision-study
                  the precision study: the 480,000-tet beam with a 165 kN tip load
                  ramped over 10,000 steps (about 40 % of the tets yield), 20,000 steps
                  in FP32, FP32-compensated and FP64 on the GPU; errors of displacement,
                  von Mises stress, equivalent plastic strain and energy balance against
                  the FP64 GPU step (bit-identical to the FP64 oracle; the same study
                  against the CPU oracle itself is tests/drift_study.py tet-precision)
  tet-batched     256 independent tet beams and plates, tet counts log-uniform in
                  [2e3, 2e5] (11.0 M tets), yield U[235, 355] MPa, hardening U[0.5, 2]
                  GPa, a random clamped face, a tip or pressure load of seeded size;
                  all stepped together in one pool (FP32-compensated), schedule and
                  tile picked by the autotuner.  Beside it the same meshes one at a
                  time through the plain single-mesh step (FP64 and FP32-compensated).
                  The default: the metric is batched against plain.
  tet-serving     Poisson arrivals (40/s) of tet meshes of log-uniform size in
                  [1e3, 5e5] and U[500, 5000] steps, admitted into a pool sized to a
                  150 GB budget as room frees up, with p50/p99 step latency; the trace
                  lasts --serve-seconds (default 120 s, the configuration's) of arrivals.
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

WORKLOADS = {
    # the configuration's whole run: 5,000 steps, through the pressure pulse's 5 ms rise
    # (the plating yields as the load comes on); --steps times fewer
    "shell-panel": dict(kind="shell", cells=(2000, 1000), sample_cells=(100, 50), run_steps=5000),
    # a 2 x 1 m corner of the same panel (20,000 elements, 0.14 GB per step): the size
    # the ncu captures are taken on
    "shell-sample": dict(kind="shell", cells=(200, 100), sample_cells=(100, 50)),
    "tet-precision": dict(kind="tet", cells=(200, 20, 20), load=200e3, ramp=10000, mode="f32k"),
    "tet-cantilever": dict(kind="tet", cells=(40, 4, 4), load=200e3, ramp=1000, mode="f32k"),
    "tet-precision-study": dict(kind="precision", cells=(200, 20, 20), load=165e3, ramp=10000, steps=20000),
    "tet-batched": dict(kind="pool", count=256, lo=2e3, hi=2e5),
    # the first 16 meshes of the batch (1.1 M tets): the size ncu captures are taken on
    "tet-batched-sample": dict(kind="pool", count=16, lo=2e3, hi=2e5),
    "tet-serving": dict(kind="serve", rate=40.0, lo=1e3, hi=5e5, budget=150e9),
}
SHELL_MATERIAL = dict(youngs=206e9, poisson=0.3, yield_strength=355e6, hardening=1e9)


# ---------------------------------------------------------------------------------
# inputs

def tet_beam(nx, ny, nz, length=1.0, width=0.1, depth=0.1, load=20e3):
    import meshes as M

    pos, idx = M.box_tet_mesh(length, width, depth, nx, ny, nz)
    fixed = (pos[0::3] < 1e-6).astype(np.uint32)
    tip = pos[0::3] > length - 1e-6
    fext = np.zeros(pos.size)
    fext[2::3][tip] = -load / tip.sum()
    return pos, idx, fixed, fext


def shell_panel(nx, ny):
    import meshes as M

    # the full panel is 2000 x 1000 cells of 10 mm; a sample keeps the cell size
    return M.stiffened_panel(nx=nx, ny=ny, lx=20.0 * nx / 2000, ly=10.0 * ny / 1000)


# ---------------------------------------------------------------------------------
# algorithmic bytes (each array counted once per launch; 4-byte ints)

def tet_bytes(T, N, mode):
    """Element pass: index 16, slot map 16, Dm^-1 36, volume 4, plastic state R/W 2 x 28
    (and its compensation), four corner forces 4 x 12; per node the displacement (and
    its compensation) read once.  Node pass: offsets 4, displacement (+ compensation)
    R/W, velocity R/W 24, mass 4, 1/mass 4, flag 1, load 12; the corner forces read."""
    comp = 2 if mode == "f32k" else 1
    elem = T * (16 + 16 + 36 + 4 + comp * 2 * 28 + 4 * 12) + N * 12 * comp
    node = N * (4 + comp * 2 * 12 + 2 * 12 + 4 + 4 + 1 + 12) + T * 4 * 12
    return elem, node


def shell_bytes(E, N):
    """Element kernel: the element row (J0^-1 and the enhanced-mode scales) 64 + state
    R/W 2 x 8 x 14 floats + alpha R/W 2 x 32 + index 32 + slot map 32 + corner forces 96,
    and the node reads (rest 24 + displacement 12) once per node; B and G are formed in
    the kernel from the rest corners.  Node kernel: offsets 4, forces 12 per slot,
    displacement and compensation R/W 48, velocity R/W 24, mass 8, pins 1, load 12."""
    elem = E * (64 + 2 * 8 * 14 * 4 + 2 * 32 + 32 + 32 + 96) + N * (24 + 12)
    node = N * (4 + 48 + 24 + 8 + 1 + 12) + E * 8 * 12
    return elem, node


# FP32 operations per solid-shell element update, counted by ncu on the shell-sample
# workload (SASS thread instructions: 2 x FFMA + FADD + FMUL, 16,707 per element with B
# and G formed in the kernel; the 473 FP64 operations -- rest-corner differences and
# the energy account -- are left out).  The second roofline of the shell element,
# against the FP32 SIMT peak: SMs x 128 lanes x 2 x the SM clock.
SHELL_FP32_FLOP_PER_ELEMENT = 16707


def simt_roofline(flop_per_unit, units, kernel_ms, max_mhz):
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    peak = sms * 128 * 2 * max_mhz * 1e6 / 1e12
    achieved = flop_per_unit * units / (kernel_ms / 1e3) / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "flop_per_unit": flop_per_unit,
            "peak_source": f"nominal: {sms} SMs x 128 FP32 lanes x 2 x {max_mhz:.0f} MHz (max SM clock)"}


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
        self.mark = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def wait_first(self, limit=3.0):
        """Block until the sampler has produced a line, so the timed region is covered."""
        t0 = time.perf_counter()
        while self.proc and not self.rows and time.perf_counter() - t0 < limit:
            time.sleep(0.01)

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

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in self.rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in self.rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def max_over_ranks(value, dist):
    """The largest `value` over all ranks: a multi-GPU step takes as long as its slowest
    rank.  The collective runs on the process group's own device (CUDA under NCCL, the
    host under gloo)."""
    if dist is None:
        return value
    import torch

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, steps, world, ms):
    """Whole-job element-updates/s: every rank steps its own replica (weak scaling)."""
    return units_per_rank * steps * world / (ms / 1e3)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload):
    """DRAM bytes per launch of the dominant kernel, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get(workload)
    return None


# ---------------------------------------------------------------------------------
# the reference's CPU path on this box's host cores (bounded samples)

def cpu_baseline(wl, seconds=15.0):
    """The compiled reference (oracle/_ref) when present, else the C restatement.

    tet:   O-tet64 -- fem.cpp kinematics + plasticity::update in double, element loop
           over all host cores with core::JobSystem, serial CSR gather.
    shell: zone::Solver's element loop (elementPlasticUpdate with cached RestForms,
           zone.cpp:967) over all host cores with core::JobSystem, serial CSR gather and
           node update, on a sub-panel with the full panel's 10 mm cells."""
    import oracle as O

    workers = os.cpu_count() or 1
    if wl["kind"] in ("pool", "serve"):
        batch = RefBatch(wl)
        per_step = batch.time(1, workers)  # warm-up step, and the size of a step
        steps = max(1, min(20, int(seconds / max(per_step, 1e-9))))
        spent = batch.time(steps, workers)
        return {"value": batch.tets * steps / spent, "unit": UNIT, "cores": workers, "kind": batch.kind,
                "sample": batch.sample(1, steps, workers)}
    kind = "reference" if O.have_ref() else "port"
    o = O.Oracle("ref" if kind == "reference" else "port")
    if wl["kind"] == "tet":
        pos, idx, fixed, fext = tet_beam(*wl["cells"], load=wl["load"])
        m = O.TetMesh64(o, pos, idx, fixed, fext)
        p = O.tet64_params(dt=1e-7, ramp_steps=wl["ramp"])
        T = idx.size // 4
        if kind == "reference":
            rate = o.tet64_time_parallel(C.byref(m._s), C.byref(p), 1, workers)
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
        sample = f"{steps} steps of the {T}-tet workload mesh, FP64 J2 (O-tet64)"
    else:
        nx, ny = wl["sample_cells"]
        rest, index, pinned, load = shell_panel(nx, ny)
        mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
        m = O.ShellModel(o, rest, index, pinned, mat, fext=load)
        E = index.size // 8
        if kind == "reference":
            rate = m.time_parallel(1e-6, 1, workers, rise_time=5e-3)
            steps = max(1, int(seconds * rate / E))
            rate = m.time_parallel(1e-6, steps, workers, rise_time=5e-3)
            cores = workers
        else:
            t0 = time.perf_counter()
            m.step(1e-6, 1, rise_time=5e-3)
            rate = E / (time.perf_counter() - t0)
            steps = max(1, int(seconds * rate / E))
            t0 = time.perf_counter()
            m.step(1e-6, steps, rise_time=5e-3)
            rate = E * steps / (time.perf_counter() - t0)
            cores = 1
        sample = (f"{steps} steps of a {nx}x{ny}-cell sub-panel ({E} elements, the full panel's 10 mm cells), "
                  "FP64 elastoplastic solid-shell")
    return {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}


class RefBatch:
    """The batched workload's meshes as O-tet64 states for the reference's CPU step:
    the compiled reference (oracle/_ref) when present, else the C restatement.  Each
    mesh has its own material, load ramp and time step (0.9 x its FP64 element bound,
    as on the GPU).  A step is one time step of every mesh, one mesh after another
    (the reference steps one mesh per solver, fem.cpp:187), each mesh's element loop
    over the host threads.  Imports neither the product library nor anything that
    loads it."""

    def __init__(self, wl):
        import oracle as O
        import workloads as W

        self.O = O
        self.kind = "reference" if O.have_ref() else "port"
        self.o = O.Oracle("ref" if self.kind == "reference" else "port")
        port = self.o if self.kind == "port" else O.Oracle("port")
        self.specs = batch_specs(wl)
        self.meshes, self.params = [], []
        for sp in self.specs:
            b = W.build(sp)
            m = O.TetMesh64(self.o, b.position, b.index, b.fixed, b.external_force)
            dt = port.tet64_critical_dt(C.byref(m._s), W.YOUNGS, W.POISSON, W.DENSITY, 0.9)
            self.meshes.append(m)
            self.params.append(O.tet64_params(dt=dt, ramp_steps=sp.ramp_steps, yield_=sp.yield_strength,
                                              hardening=sp.hardening))
        self.tets = sum(sp.tets for sp in self.specs)

    def time(self, steps, workers):
        """Seconds of `steps` steps of the whole batch (the step loop's own clock)."""
        O = self.O
        if self.kind == "reference":
            arr = (C.POINTER(O.Tet64) * len(self.meshes))(*[C.pointer(m._s) for m in self.meshes])
            ps = (O.Tet64Params * len(self.params))(*self.params)
            return self.o.tet64_time_batch(arr, ps, len(self.meshes), steps, workers)
        t0 = time.perf_counter()
        for _ in range(steps):
            for m, p in zip(self.meshes, self.params):
                m.step(p, 1, threads=workers)
        return time.perf_counter() - t0

    def sample(self, warmup, steps, workers):
        what = "the compiled reference" if self.kind == "reference" else "the C restatement"
        return (f"all {len(self.specs)} meshes of the workload ({self.tets:,} tets), {warmup} warm-up + {steps} "
                f"timed steps, each step one mesh after another; O-tet64 (fem.cpp kinematics with "
                f"plasticity::update in FP64) from {what}, element loop on {workers} host threads")


def run_reference(args, wl):
    """The reference's CPU step on the same workload, W warm-up and K timed steps; rank
    0 only (the other ranks exit without work)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    workers = os.cpu_count() or 1
    if wl["kind"] in ("pool", "serve"):
        batch = RefBatch(wl)
        batch.time(args.warmup, workers)
        spent = batch.time(args.steps, workers)
        value = batch.tets * args.steps / spent
        base = {"value": value, "unit": UNIT, "cores": workers, "kind": batch.kind,
                "sample": batch.sample(args.warmup, args.steps, workers)}
        config = pool_config(args, wl, batch.specs, args.gpus)
        ms = spent / args.steps * 1e3
    else:
        cpu_baseline(wl, seconds=2.0)
        rates = [cpu_baseline(wl, seconds=max(2.0, 60.0 / max(args.steps, 1)))["value"]
                 for _ in range(min(args.steps, 10))]
        base = cpu_baseline(wl, seconds=2.0)
        value = base["value"] = float(np.median(rates))
        config = {"workload": args.workload}
        ms = None
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": config, "cpu_baseline": base,
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------------
# the batched and served workloads (a pool of many meshes)

def batch_specs(wl):
    import workloads as W

    if wl["kind"] == "serve":
        return W.request_trace(rate=wl["rate"], duration=4.0, lo=wl["lo"], hi=wl["hi"])
    return W.batch_meshes(count=wl["count"], lo=wl["lo"], hi=wl["hi"], steps=0, ramp_steps=1000)


def pool_config(args, wl, specs, world):
    """The batched workload's description, the same in both arms' lines."""
    T = sum(sp.tets for sp in specs)
    N = sum(sp.nodes for sp in specs)
    per_step = sum(sum(tet_bytes(sp.tets, sp.nodes, "f32k")) for sp in specs)
    return {"workload": args.workload, "meshes": len(specs), "elements": T, "nodes": N,
            "mesh_seed": "workloads.batch_meshes defaults", "load_ramp_steps": 1000,
            "l2": "no flush: %.2f GB move per step, above the 126 MB L2" % (per_step / 1e9),
            "parallelism": f"replicas x{world}"}


def tet_von_mises(position, rest, index, plastic, mu, kappa):
    """Von Mises stress per tet in FP64 from a state (positions, plastic strain): the
    co-rotated strain of fem.cpp's tet (four Higham iterations), sigma = 2 mu dev(e - ep)
    + kappa tr(e - ep) I.  The same host routine for every variant, so the comparison
    sees only the state."""
    x = position.reshape(-1, 3)
    X = rest.reshape(-1, 3).astype(np.float64)
    idx = index.reshape(-1, 4).astype(np.int64)
    dm = np.stack([X[idx[:, c]] - X[idx[:, 0]] for c in (1, 2, 3)], axis=2)
    ds = np.stack([x[idx[:, c]] - x[idx[:, 0]] for c in (1, 2, 3)], axis=2)
    f = ds @ np.linalg.inv(dm)
    r = f.copy()
    for _ in range(4):
        r = 0.5 * (r + np.transpose(np.linalg.inv(r), (0, 2, 1)))
    sm = np.transpose(r, (0, 2, 1)) @ f
    e = 0.5 * (sm + np.transpose(sm, (0, 2, 1))) - np.eye(3)
    ep = plastic
    el = np.empty((len(idx), 6))
    el[:, 0], el[:, 1], el[:, 2] = e[:, 0, 0] - ep[:, 0], e[:, 1, 1] - ep[:, 1], e[:, 2, 2] - ep[:, 2]
    el[:, 3], el[:, 4], el[:, 5] = 2 * e[:, 0, 1] - ep[:, 3], 2 * e[:, 1, 2] - ep[:, 4], 2 * e[:, 2, 0] - ep[:, 5]
    tr = el[:, 0] + el[:, 1] + el[:, 2]
    s = 2 * mu * (el[:, :3] - tr[:, None] / 3)
    t = mu * el[:, 3:]
    return np.sqrt(1.5 * ((s ** 2).sum(1) + 2 * (t ** 2).sum(1)))


def run_precision(args, wl, rank):
    """The precision study on one GPU (rank 0 only): FP32, FP32-compensated and FP64 on
    the GPU, the errors of the first two against FP64.  The FP64 GPU step is
    bit-identical to the FP64 oracle (tests/test_tet_gpu.py); the same study against
    the oracle itself is tests/drift_study.py tet-precision."""
    import femstep as F

    if rank != 0:
        return
    pos, idx, fixed, fext = tet_beam(*wl["cells"], load=wl["load"])
    T = idx.size // 4
    mu, kappa = 210e9 / 2.6, 210e9 / (3 * 0.4)
    solvers = {m: F.TetSolver(pos, idx, mode=m, fixed=fixed, external_force=fext, density=7850.0)
               for m in ("f64", "f32k", "f32")}
    dt = solvers["f64"].critical_dt(210e9, 0.3, 7850.0, 0.9)
    kw = dict(dt=dt, ramp_steps=wl["ramp"])
    ms = {}
    with ClockSampler(0) as clocks:
        clocks.wait_first()
        for m, s in solvers.items():
            ms[m] = s.run(wl["steps"], **kw)
    rest = pos.astype(np.float64)
    state = {}
    for m, s in solvers.items():
        p, _ = s.readback64()
        pl = s.plastic()
        e = s.energy()
        state[m] = dict(u=p - rest, vm=tet_von_mises(p, rest, idx, pl, mu, kappa), ep=pl[:, 6], energy=e)
    r = state["f64"]
    yielded = float((r["ep"] > 0).mean())

    def drift(e):
        w = e[0] + e[4]  # external work incl. gravity
        return float(abs(w - (e[1] + e[2] + e[3])) / abs(w))

    out = {}
    for m in ("f32", "f32k", "f64"):
        v = state[m]
        out[m] = {
            "max_rel_displacement_error": float(np.abs(v["u"] - r["u"]).max() / np.abs(r["u"]).max()),
            "max_rel_von_mises_error": float(np.abs(v["vm"] - r["vm"]).max() / r["vm"].max()),
            "max_rel_plastic_strain_error": float(np.abs(v["ep"] - r["ep"]).max() / max(r["ep"].max(), 1e-300)),
            "energy_balance_drift": drift(v["energy"]),
            "energy_drift_vs_fp64": abs(drift(v["energy"]) - drift(r["energy"])),
            "elem_upd_per_s": T * wl["steps"] / (ms[m] / 1e3),
        }
    for s in solvers.values():
        s.close()
    line = {"metric": METRIC, "value": out["f32k"]["elem_upd_per_s"], "unit": UNIT, "n_gpus": 1,
            "steps": wl["steps"], "warmup": 0, "ms_per_step": ms["f32k"] / wl["steps"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "elements": T, "nodes": pos.size // 3, "dt": dt,
                       "tip_load_n": wl["load"], "ramp_steps": wl["ramp"], "yielded_fraction_fp64": yielded,
                       "reference": "GPU FP64 step (bit-identical to the FP64 oracle)",
                       "errors": "max |a - a64| / max |a64| over nodes (displacement) or tets (von Mises from the "
                                 "final state, equivalent plastic strain); energy drift |W - (U + D + K)| / W"},
            "precision": out, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def fixed_schedule(F, pool, spec):
    """`TILE:graph|persistent|graph-staged|graph-tiled` set by hand (None: the autotuner)."""
    if not spec:
        return None
    tile, mode = spec.split(":")
    code = {v: k for k, v in F.POOL_MODE_NAMES.items()}[mode]
    pool.set_schedule(int(tile), code)
    return {"tile": int(tile), "mode": mode, "ms_per_step": None, "set_by": "--schedule"}


def plain_sequential(F, W, built, steps, mode):
    """The plain single-mesh step (gpu::FemGpuSolver's shape): one mesh at a time, each
    in its own handle for `steps` steps.  Device ms summed over the meshes."""
    total_ms, units = 0.0, 0
    for b in built:
        s = F.TetSolver(b.position, b.index, mode=mode, fixed=b.fixed, external_force=b.external_force,
                        density=W.DENSITY)
        dt = s.critical_dt(W.YOUNGS, W.POISSON, W.DENSITY, 0.9)
        kw = dict(dt=dt, ramp_steps=b.spec.ramp_steps, yield_strength=b.spec.yield_strength,
                  hardening=b.spec.hardening)
        s.run(3, **kw)  # warm (graph capture)
        total_ms += s.run(steps, **kw)
        units += b.spec.tets * steps
        s.close()
    return units / (total_ms / 1e3), total_ms


def pool_drift(F, W, specs, tune, steps=2000):
    """Drift of the batched FP32-compensated step against FP64 on a sample of the
    batch (workloads.drift_sample: the largest mesh and the smallest plate of each
    clamped face and load kind), over the 1,000-step load ramp plus 1,000 steps, in the
    schedule and tile the line reports (`tune`).  The FP64 side is the plain single-mesh
    FP64 GPU step, which is bit-identical to the FP64 oracle (tests/test_tet_gpu.py,
    tests/test_pool_gpu.py)."""
    picks = W.drift_sample(specs)
    built = [W.build(specs[i]) for i in picks]
    T = sum(b.spec.tets for b in built)
    N = sum(b.spec.nodes for b in built)
    pool = F.TetPool(T, N + len(built) + 1, max_meshes=len(built) + 1, tile=tune["tile"])
    pool.set_schedule(tune["tile"], {v: k for k, v in F.POOL_MODE_NAMES.items()}[tune["mode"]])
    mu, kappa = W.YOUNGS / (2 * (1 + W.POISSON)), W.YOUNGS / (3 * (1 - 2 * W.POISSON))
    ids, refs = [], []
    for b in built:
        s = F.TetSolver(b.position, b.index, mode="f64", fixed=b.fixed, external_force=b.external_force,
                        density=W.DENSITY)
        dt = s.critical_dt(W.YOUNGS, W.POISSON, W.DENSITY, 0.9)
        s.run(steps, dt=dt, ramp_steps=b.spec.ramp_steps, yield_strength=b.spec.yield_strength,
              hardening=b.spec.hardening)
        p64, _ = s.readback64()
        refs.append((p64, s.plastic(), s.energy()))
        s.close()
        ids.append(pool.admit(steps=steps, dt=dt, **b.admit_kwargs()))
    pool.run(steps)

    def balance(e):
        w = e[0] + (e[4] if len(e) > 4 else 0.0)  # external work, and gravity's where it is kept
        return abs(w - (e[1] + e[2] + e[3])) / abs(w)

    rows = []
    for b, i, (p64, pl64, e64) in zip(built, ids, refs):
        p, _ = pool.readback(i)
        pl = pool.plastic(i)
        e = pool.energy(i)
        rest = b.position.astype(np.float64)
        u, u64 = p - rest, p64 - rest
        vm = tet_von_mises(p, rest, b.index, pl, mu, kappa)
        vm64 = tet_von_mises(p64, rest, b.index, pl64, mu, kappa)
        ep, ep64 = pl[:, 6], pl64[:, 6]
        rows.append({"tets": b.spec.tets, "clamp": b.spec.clamp, "load": b.spec.load_kind,
                     "yielded_fraction_fp64": float((ep64 > 0).mean()),
                     "displacement": float(np.abs(u - u64).max() / np.abs(u64).max()),
                     "von_mises": float(np.abs(vm - vm64).max() / vm64.max()),
                     "plastic_strain": float(np.abs(ep - ep64).max() / ep64.max()) if ep64.max() > 0 else 0.0,
                     "energy_balance_fp32k": float(balance(e)), "energy_balance_fp64": float(balance(e64)),
                     "energy_terms_vs_work": float(np.abs(np.asarray(e[:4]) - np.asarray(e64[:4])).max()
                                                   / abs(e64[0]))})
    pool.close()
    return {"meshes": picks, "steps": steps, "schedule": f"{tune['tile']}:{tune['mode']}",
            "reference": "FP64 GPU step, bit-identical to the FP64 oracle",
            "max_rel_displacement_error": max(r["displacement"] for r in rows),
            "max_rel_von_mises_error": max(r["von_mises"] for r in rows),
            "max_rel_plastic_strain_error": max(r["plastic_strain"] for r in rows),
            "max_energy_term_error_over_work": max(r["energy_terms_vs_work"] for r in rows),
            "errors": "max |a - a64| / max |a64| per mesh (displacement over nodes; von Mises from the final "
                      "state and equivalent plastic strain over tets); energy terms (work, dissipation, strain, "
                      "kinetic) against FP64, over the external work",
            "per_mesh": rows}


def run_pool(args, wl, rank, world, barrier, dist, local):
    import femstep as F
    import workloads as W

    specs = batch_specs(wl)
    built = [W.build(sp) for sp in specs]
    T = sum(sp.tets for sp in specs)
    N = sum(sp.nodes for sp in specs)
    pool = F.TetPool(T, N + len(specs) + 1, max_meshes=len(specs) + 1)
    t_admit = time.perf_counter()
    ids = pool.admit_many([b.admit_kwargs() for b in built], [10 ** 12] * len(built))
    assert len(ids) == len(built)
    pool.run(0)
    admit_s = time.perf_counter() - t_admit
    tune = fixed_schedule(F, pool, args.schedule) or pool.autotune(steps=48)
    # the work list and the schedule's captured graph are built before the warm-up, so
    # the timed chunk does no set-up whatever W is
    pool.prepare()
    warm = args.warmup
    pool.run(warm)
    barrier()
    with ClockSampler(local) as clocks:
        clocks.wait_first()
        ms = pool.run(args.steps)
        launches = pool.info()["launches"]
        barrier()
        time.sleep(0.25)
    ms = max_over_ranks(ms, dist)
    value = job_rate(T, args.steps, world, ms)
    elem_ms, node_ms = pool.profile(5)
    eb = sum(tet_bytes(sp.tets, sp.nodes, "f32k")[0] for sp in specs)
    nb = sum(tet_bytes(sp.tets, sp.nodes, "f32k")[1] for sp in specs)
    info = pool.info()
    pool.close()

    # the plain single-mesh step over the same meshes, one at a time
    plain_steps = max(10, min(args.steps, 50))
    plain = None
    if not args.no_plain:
        plain64, _ = plain_sequential(F, W, built, plain_steps, "f64")
        plain32, _ = plain_sequential(F, W, built, plain_steps, "f32k")
        plain = {"f64_elem_upd_per_s": plain64, "f32k_elem_upd_per_s": plain32, "steps": plain_steps,
                 "batched_over_plain_f64": value / world / plain64,
                 "batched_over_plain_f32k": value / world / plain32,
                 "note": "the same meshes one at a time, each through its own single-mesh handle "
                         "(femstep_tet_run, graph-captured), device time summed"}

    e2e = None
    if not args.no_e2e:
        def job():
            """One whole job through the C ABI from host arrays, wall clock."""
            t0 = time.perf_counter()
            p2 = F.TetPool(T, N + len(specs) + 1, max_meshes=len(specs) + 1)
            p2.set_schedule(tune["tile"], {v: k for k, v in F.POOL_MODE_NAMES.items()}[tune["mode"]])
            t1 = time.perf_counter()
            ids2 = p2.admit_many([b.admit_kwargs() for b in built], [args.steps] * len(built))
            t2 = time.perf_counter()
            p2.run(args.steps)
            t3 = time.perf_counter()
            d2h = 0
            for pp, vv in p2.readback_many(ids2):
                d2h += pp.nbytes + vv.nbytes
            t4 = time.perf_counter()
            p2.close()
            wall = time.perf_counter() - t0
            phases = {"create_s": t1 - t0, "admit_s": t2 - t1, "steps_s": t3 - t2, "readback_s": t4 - t3,
                      "destroy_s": wall - (t4 - t0)}
            return T * args.steps / wall, phases, d2h

        cold_rate, cold_phases, _ = job()
        warm_rate, phases, d2h = job()
        h2d = sum(b.position.nbytes + b.index.nbytes + b.fixed.nbytes + b.external_force.nbytes for b in built)
        e2e = {"value": warm_rate, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
               "d2h_bytes_per_step": d2h / args.steps, "phases": phases,
               "cold_value": cold_rate, "cold_phases": cold_phases,
               "note": "one whole job through the C ABI, wall clock: create the pool, admit every mesh from host "
                       "arrays (femstep_pool_admit_many: node ids, positions, pins and loads staged on all host "
                       "cores and uploaded; CSR, slot map and the FP64 rest state on the device), K steps, read back "
                       "every mesh's positions and velocities (femstep_pool_readback_many), destroy.  `value` is "
                       "the second such job in the process, with the pinned staging and device memory the first "
                       "one left in the library's caches, as in a serving process; `cold_value` is the first"}
    drift = None if args.no_drift else pool_drift(F, W, specs, tune)
    element_kernel = {"graph": "pool_elements", "graph-staged": "pool_elements_ring",
                      "persistent": "pool_persistent", "graph-tiled": "pool_elements_tiled_ring"}[tune["mode"]]
    peak, peak_kind = measured_peak()
    if tune["mode"] == "graph-tiled":
        # the tiled schedule moves fewer bytes than the formula counts (per-(tile, node)
        # partials instead of per-corner slots): the step's formula bytes over the step's
        # time, an effective bandwidth that can exceed the copy peak
        achieved = (eb + nb) / (ms / args.steps / 1e3) / 1e9
        kernel_label = ("pool_elements_tiled_ring + pool_nodes (the whole step of the tiled schedule; effective "
                        "bandwidth: the formula's bytes, slot exchange included, over the step's time)")
    else:
        achieved = eb / (elem_ms / 1e3) / 1e9
        kernel_label = f"{element_kernel} (tet element pass, the {tune['mode']} schedule's)"
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": pool_config(args, wl, specs, world),
            "detail": {"schedule": tune, "element_kernel_ms": elem_ms, "node_kernel_ms": node_ms,
                       "step_effective_gbs": (eb + nb) / (ms / args.steps / 1e3) / 1e9,
                       "admit_seconds": admit_s, "device_bytes": info["device_bytes"],
                       "warmup_note": "the work list and the 16-step graph are built (femstep_pool_prepare) "
                                      "before the W warm-up steps"},
            "plain": plain,
            "drift": drift,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": ncu_traffic(f"{args.workload}:{element_kernel}"),
                         "kernel": kernel_label,
                         "peak_source": peak_kind},
        }
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(wl)
        print(json.dumps(out), flush=True)


def run_serving(args, wl, rank, world, barrier, dist, local):
    import femstep as F
    import serving as S
    import workloads as W

    trace = W.request_trace(rate=wl["rate"], duration=args.serve_seconds, lo=wl["lo"], hi=wl["hi"])
    pool = F.TetPool.for_budget(wl["budget"], nodes_per_tet=0.25, max_meshes=4096)
    # the schedule, tuned once on a representative mix
    warm = pool.admit_many([W.build(sp).admit_kwargs() for sp in trace[:48]], [10 ** 6] * 48)
    tune = fixed_schedule(F, pool, args.schedule) or pool.autotune(steps=48)
    if not args.schedule and tune["mode"] == "graph-tiled":
        # the tiled schedule rebuilds its tables whenever the mix changes, which a serving
        # loop does at every chunk: serve with the staged pass at the same tile instead
        pool.set_schedule(tune["tile"], F.POOL_GRAPH_STAGED)
        tune = dict(tune, mode="graph-staged", note="the autotuner's graph-tiled replaced for serving")
    for i in warm:
        pool.release(i)
    reqs = [S.Request(key=k, arrival=sp.arrival, tets=sp.tets, steps=sp.steps,
                      build=(lambda sp=sp: W.build(sp).admit_kwargs())) for k, sp in enumerate(trace)]
    barrier()
    with ClockSampler(local) as clocks:
        clocks.wait_first()
        rep = S.Server(pool, chunk=args.serve_chunk, full_error=F.PoolFull).serve(reqs)
        barrier()
        time.sleep(0.25)
    summ = rep.summary()
    value = summ["elem_upd_per_s"] * world
    info = pool.info()
    pool.close()
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": rep.chunks,
            "warmup": args.warmup, "ms_per_step": summ["p50_step_ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "arrival_rate": wl["rate"], "seconds": args.serve_seconds,
                       "budget_bytes": wl["budget"], "pool_device_bytes": info["device_bytes"],
                       "chunk_steps": args.serve_chunk, "schedule": tune,
                       "offered_elem_upd_per_s": sum(r.tets * r.steps for r in reqs) / args.serve_seconds,
                       "l2": "no flush: the resident solves move GBs per step, above the 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            "serving": summ,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "the serving loop is end to end: arrivals admitted from host arrays, results read "
                            "back; value is completed element-updates over the wall clock of the trace"},
            "gpu_launches": summ["launches"],
            "clocks": clocks.summary(),
        }
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(wl)
        print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------------

class Solver:
    """One workload's solver behind a common face."""

    def __init__(self, wl):
        import femstep as F

        self.wl = wl
        if wl["kind"] == "tet":
            pos, idx, fixed, fext = tet_beam(*wl["cells"], load=wl["load"])
            self.inputs = dict(position=pos, index=idx, fixed=fixed, external_force=fext)
            self.units = idx.size // 4
            self.nodes = pos.size // 3
            self.make = lambda: F.TetSolver(pos, idx, mode=wl["mode"], fixed=fixed, external_force=fext,
                                            density=7850.0)
            s = self.make()
            self.kw = dict(dt=s.critical_dt(210e9, 0.3, 7850.0, 0.9), ramp_steps=wl["ramp"])
            self.bytes = tet_bytes(self.units, self.nodes, wl["mode"])
            self.kernel = "f32_forces (tet element)"
        else:
            rest, index, pinned, load = shell_panel(*wl["cells"])
            self.inputs = dict(rest=rest, index=index, pinned=pinned, load=load)
            self.units = index.size // 8
            self.nodes = rest.size // 3
            self.make = lambda: F.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0)
            s = self.make()
            dt = s.critical_dt(206e9, 0.3, 7850.0, 0.9)
            self.kw = dict(dt=dt, rise_time=5e-3, compensated=True, **SHELL_MATERIAL)
            self.bytes = shell_bytes(self.units, self.nodes)
            self.kernel = "shell_forces (solid-shell element)"
        self.s = s

    def readback(self, s):
        return s.readback()

    def h2d_bytes(self):
        return sum(v.nbytes for v in self.inputs.values())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 100; shell-panel 5000)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tet-batched", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="tet-batched: skip the one-mesh-at-a-time comparison")
    ap.add_argument("--schedule", default=None,
                    help="pool workloads: TILE:graph|persistent|graph-staged|graph-tiled instead of the autotuner")
    ap.add_argument("--no-drift", action="store_true", help="tet-batched: skip the drift sample against FP64")
    ap.add_argument("--serve-seconds", type=float, default=120.0)
    ap.add_argument("--serve-chunk", type=int, default=64)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    wl = WORKLOADS[args.workload]
    if args.steps is None:
        args.steps = wl.get("run_steps", 100)
    if args.impl == "reference":
        return run_reference(args, wl)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    import femstep as F

    F.set_device(local)  # one process per GPU

    def barrier():
        if dist is not None:
            import torch

            torch.cuda.synchronize()
            dist.barrier()

    if wl["kind"] == "precision":
        run_precision(args, wl, rank)
        if dist is not None:
            dist.destroy_process_group()
        return
    if wl["kind"] in ("pool", "serve"):
        (run_pool if wl["kind"] == "pool" else run_serving)(args, wl, rank, world, barrier, dist, local)
        if dist is not None:
            dist.destroy_process_group()
        return
    w = Solver(wl)
    s = w.s
    # W warm-up steps, at least one captured graph's worth (32 steps), so the graph the
    # timed run replays is built before the timed region
    warm = max(args.warmup, 32)
    s.run(warm, **w.kw)
    barrier()
    with ClockSampler(local) as clocks:
        clocks.wait_first()
        ms = s.run(args.steps, **w.kw)
        launches = s.launches
        barrier()
        time.sleep(0.25)
    ms = max_over_ranks(ms, dist)
    value = job_rate(w.units, args.steps, world, ms)

    # per-kernel device time for the roofline (outside the timed region)
    elem_ms, node_ms = s.profile(5, **w.kw)
    elem_b, node_b = w.bytes
    peak, peak_kind = measured_peak()
    achieved = elem_b / (elem_ms / 1e3) / 1e9
    stats = s.stats() if hasattr(s, "stats") else None
    s.close()

    e2e = None
    if not args.no_e2e:
        t0 = time.perf_counter()
        e = w.make()
        t1 = time.perf_counter()
        e.run(args.steps, **w.kw)
        t2 = time.perf_counter()
        p_host, v_host = w.readback(e)
        t3 = time.perf_counter()
        e.close()
        t4 = time.perf_counter()
        wall = t4 - t0
        e2e = {"value": w.units * args.steps / wall, "unit": UNIT,
               "h2d_bytes_per_step": w.h2d_bytes() / args.steps,
               "d2h_bytes_per_step": (p_host.nbytes + v_host.nbytes) / args.steps,
               "phases": {"create_s": t1 - t0, "steps_s": t2 - t1, "readback_s": t3 - t2, "destroy_s": t4 - t3},
               "note": "upload + K steps + readback through the C ABI, wall clock"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": warm, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "elements": w.units, "nodes": w.nodes,
                       "dt": w.kw["dt"], "element_kernel_ms": elem_ms, "node_kernel_ms": node_ms,
                       "step_effective_gbs": (elem_b + node_b) / (ms / args.steps / 1e3) / 1e9,
                       "l2": "no flush: %.1f GB move per step, above the 126 MB L2" % ((elem_b + node_b) / 1e9),
                       "parallelism": f"replicas x{world}", "newton": stats},
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": ncu_traffic(args.workload), "kernel": w.kernel,
                         "peak_source": peak_kind},
        }
        if wl["kind"] == "shell":
            out["roofline_simt"] = simt_roofline(SHELL_FP32_FLOP_PER_ELEMENT, w.units, elem_ms,
                                                 out["clocks"].get("sm_max_mhz") or 1965.0)
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(wl)
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
