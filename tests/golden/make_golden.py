"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own C++ (compiled from its sources by `make -C oracle ref`, into
oracle/_ref/libshipsim_ref.so) on seeded inputs and stores inputs and outputs as small
.npz fixtures.  The reference ships no golden files of its own -- its tests assert
closed forms computed in code -- so these vectors are the pin for the CPU restatement
(oracle/femoracle.c) on machines where the reference source is not present.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def plasticity(ref):
    rng = np.random.default_rng(20261203)
    mats = [O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9),
            O.material(E=210e9, nu=0.3, yield_=235e6, hardening=0.0),
            O.material(E=206e9, nu=0.3, yield_=355e6, hardening=2e9, kinematic=5e9),
            O.material(E=206e9, nu=0.3, yield_=355e6, swift=(355e6 / 0.01 ** 0.2, 0.01, 0.2),
                       failure=(0.18, 0.8))]
    rows = []
    for mi, m in enumerate(mats):
        for _ in range(40):
            strain = rng.normal(0, 3e-3, 6)
            state = np.zeros(O.POINT_LEN)
            state[:6] = rng.normal(0, 1e-3, 6)
            state[:3] -= state[:3].mean()
            state[12] = abs(rng.normal(0, 2e-2))
            if mats[mi][4] > 0:
                state[6:12] = rng.normal(0, 2e7, 6)
            s_in = state.copy()
            stress, tangent, inc = np.zeros(6), np.zeros(36), np.zeros(O.INCR_LEN)
            ref.plastic_update(m, 0.3 if mi == 3 else np.inf, strain, state, stress, tangent.ctypes.data, inc)
            rows.append(np.concatenate([[mi], strain, s_in, state, stress, tangent, inc]))
    np.savez_compressed(os.path.join(HERE, "plasticity.npz"), materials=np.array(mats), rows=np.array(rows))


def tet32(ref):
    # tools/fem_spike/main.cpp:143-205: the GPU-vs-CPU mesh, deformed and twisted.
    pos, idx = O.box_tet_mesh(ref, 0.4, 0.1, 0.02, 16, 4, 2)
    m = O.TetMesh32(ref, pos, idx)
    m.fixed[:] = (m.position[0::3] < 1e-6).astype(np.uint32)
    m.rest_state(210e9, 0.3, 7850.0)
    x = m.position[0::3].copy()
    m.position[2::3] += np.float32(0.02) * x * x
    m.position[1::3] += np.float32(0.01) * x
    start = m.position.copy()
    import ctypes as C
    dt = ref.tet32_critical_dt(C.byref(m.struct()), 210e9, 0.3, 7850.0, 0.5)
    out = {}
    done = 0
    for target in (1, 10, 100):
        m.step(210e9, 0.3, 7850.0, dt, 9.80665, 1.0, target - done)
        done = target
        out[f"position_{target}"] = m.position.copy()
        out[f"velocity_{target}"] = m.velocity.copy()
    np.savez_compressed(os.path.join(HERE, "tet32_spike.npz"), start=start, index=idx, fixed=m.fixed,
                        mass=m.mass, rest_inv=m.rest_inv, rest_volume=m.rest_volume, adj_offset=m.adj_offset,
                        adj_entry=m.adj_entry, dt=np.float32(dt), **out)


def tet64(ref, port):
    # The CPU-runnable cantilever: 40x4x4 cells, 3840 tets; clamped at x = 0, a 20 kN tip
    # load spread over the x = 1 face, ramped over 2000 steps.  The FP64 J2 tet is a
    # composition (fem.cpp kinematics + plasticity::update), run here with the
    # reference's compiled point law.
    import ctypes as C
    pos, idx = O.box_tet_mesh(ref, 1.0, 0.1, 0.1, 40, 4, 4)
    fixed = (pos[0::3] < 1e-6).astype(np.uint32)
    tip = pos[0::3] > 1.0 - 1e-6
    fext = np.zeros(pos.size)
    fext[2::3][tip] = -20e3 / tip.sum()
    m = O.TetMesh64(ref, pos, idx, fixed, fext)
    dt = port.tet64_critical_dt(C.byref(O.TetMesh64(port, pos, idx, fixed, fext)._s), 210e9, 0.3, 7850.0, 0.9)
    p = O.tet64_params(dt=dt, ramp_steps=2000)
    m.step(p, 150)
    np.savez_compressed(os.path.join(HERE, "tet64_cantilever.npz"), dt=dt, steps=150,
                        position=m.position, velocity=m.velocity, plastic=m.plastic, energy=m.energy)


def shell(ref):
    rng = np.random.default_rng(7)
    base = np.array([[0, 0, -.006], [.01, 0, -.006], [.01, .01, -.006], [0, .01, -.006],
                     [0, 0, .006], [.01, 0, .006], [.01, .01, .006], [0, .01, .006]], float).reshape(-1)
    rest = base + rng.normal(0, 5e-4, 24)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    forms = np.zeros(O.FORMS_LEN)
    ref.shell_forms(rest, 2, forms)
    state = np.zeros(O.SHELL_STATE_LEN)
    ref.shell_init_state(rest, mat, state)
    currents, forces, stresses, states, infos = [], [], [], [], []
    for k in range(12):
        cur = rest + rng.normal(0, 2e-4, 24) * (1 + k / 4)
        f, st, info = np.zeros(24), np.zeros(48), np.zeros(7)
        ref.shell_plastic_update(forms, rest, cur, mat, state, f, st, info)
        currents.append(cur)
        forces.append(f)
        stresses.append(st)
        states.append(state.copy())
        infos.append(info)
    k = np.zeros(576)
    ref.shell_stiffness(rest, 206e9, 0.3, 2, k)
    mass = np.zeros(8)
    ref.shell_mass(rest, 7850.0, mass)
    dtc = ref.shell_critical_dt(rest, 206e9, 0.3, 7850.0, 2, 0.9)
    np.savez_compressed(os.path.join(HERE, "shell_element.npz"), rest=rest, material=mat, forms=forms,
                        currents=np.array(currents), forces=np.array(forces), stresses=np.array(stresses),
                        states=np.array(states), infos=np.array(infos), stiffness=k, mass=mass, dt=dtc)


def shell_plate(ref):
    # A 6x4-element clamped plate, 12 mm, Gaussian pressure pulse: the composed step
    # of zone::Solver (zone.cpp:928-989, 1094-1111, 1200) with an external load.
    pos, idx = O.plate_mesh(ref, 0.06, 0.04, 0.012, 6, 4, 1)
    n = pos.size // 3
    x, y = pos[0::3], pos[1::3]
    edge = (x < 1e-9) | (x > 0.06 - 1e-9) | (y < 1e-9) | (y > 0.04 - 1e-9)
    pinned = np.repeat(edge, 3).astype(np.uint8)
    unit = np.zeros(pos.size)
    ref.plate_pressure_load(pos, idx, n, idx.size // 8, 1.0, unit)
    r2 = (x - 0.03) ** 2 + (y - 0.02) ** 2
    fext = unit * np.repeat(5e7 * np.exp(-r2 / (2 * 0.01 ** 2)), 3)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    m = O.ShellModel(ref, pos, idx, pinned, mat, fext=fext)
    dts = [ref.shell_critical_dt(pos[np.repeat(idx[e * 8:e * 8 + 8], 3) * 3 + np.tile([0, 1, 2], 8)],
                                 206e9, 0.3, 7850.0, 2, 0.9) for e in range(idx.size // 8)]
    dt = min(dts)
    m.step(dt, 60, rise_time=30 * dt)
    energy = m.compute_energy()
    np.savez_compressed(os.path.join(HERE, "shell_plate.npz"), rest=pos, index=idx, pinned=pinned, fext=fext,
                        material=mat, dt=dt, steps=60, rise=30 * dt, position=m.position, velocity=m.velocity,
                        state=m.state, energy=energy, mass=m.mass)


ZONE_CASES = {
    # name: (zone_plate keyword arguments); the plate of the reference's zone GPU tests
    "prescribed": dict(steps=300),
    "inertial_damped_edge": dict(steps=300, mass=40.0, speed=20.0, damping=0.999, edge_drive=(2e-3, 1e-3, 3e-3),
                                 edge_ramp=2e-4),
    "arrest": dict(steps=3000, mass=0.6, speed=6.0),
    "tearing": dict(steps=3000, edge_drive=(1e-3, 0.0, 2e-3), edge_ramp=1e-3),
    # flat-bar stiffeners as constraint fibres (constraint::addStiffener), yielding and tearing
    "stiffened": dict(steps=300, stiffeners=1),
    "stiffened_tearing": dict(steps=3000, stiffeners=2, web_height=0.03, web_thickness=0.006),
}


def zone_plate(ref):
    # zone::Solver itself (engine/sim/zone.cpp) on the flat plate of the reference's zone
    # GPU tests: the arrays it was built from and, per case, where it ended.
    out = {}
    for name, case in ZONE_CASES.items():
        r = ref.zone_plate(**case)
        assert r["problems"] == 0, name
        if not out:
            out.update(rest=r["rest"], index=r["index"], pinned=r["pinned"], driven=r["driven"], mass=r["mass"],
                       state0=r["state0"], material=r["mat"], density=r["density"], dt=r["dt"])
        assert np.array_equal(out["state0"], r["state0"]) and out["dt"] == r["dt"]
        out[f"{name}_prescribed"] = r["prescribed"]
        out[f"{name}_mass"] = r["mass"]  # with the fibres' lumped mass when there are stiffeners
        for k in ("fiber_tie", "fiber_weight", "fiber_area", "fiber_length", "fiber_fail", "fiber_state"):
            out[f"{name}_{k}"] = r[k]
        out[f"{name}_position"] = r["position"]
        out[f"{name}_velocity"] = r["velocity"]
        out[f"{name}_state"] = r["state"]
        out[f"{name}_account"] = np.array([r["account"][k] for k in O.ZONE_ACCOUNT])
    np.savez_compressed(os.path.join(HERE, "zone_plate.npz"), **out)


if __name__ == "__main__":
    ref = O.Oracle("ref")
    port = O.Oracle("port")
    plasticity(ref)
    tet32(ref)
    tet64(ref, port)
    shell(ref)
    shell_plate(ref)
    zone_plate(ref)
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))
