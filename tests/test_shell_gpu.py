"""Solid-shell zone on the GPU, through the C ABI, against the oracle.

The FP64 forms, lumped masses and element critical steps formed on the device are
bit-identical to the reference's (solidshell::computeRestForms, elementMass,
criticalTimestep).  The FP32 step (Kahan-compensated) is held against the FP64 CPU
composition of elementPlasticUpdate + CSR gather + node update."""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
BASE = np.array([[0, 0, -.006], [.01, 0, -.006], [.01, .01, -.006], [0, .01, -.006],
                 [0, 0, .006], [.01, 0, .006], [.01, .01, .006], [0, .01, .006]], float).reshape(-1)


def test_device_forms_bit_identical(fem, port):
    rng = np.random.default_rng(5)
    nodes = np.array([BASE * s + rng.normal(0, 6e-4, 24) for s in (1, 1, 2, 0.5, 3, 1)])
    for form in (0, 1, 2):
        forms, mass, dt = fem.shell_forms(nodes, form, 206e9, 0.3, 7850.0, 0.9)
        for e in range(nodes.shape[0]):
            f = np.zeros(O.FORMS_LEN)
            port.shell_forms(nodes[e], form, f)
            assert np.array_equal(forms[e], f), (form, e, np.abs(forms[e] - f).max())
            m = np.zeros(8)
            port.shell_mass(nodes[e], 7850.0, m)
            assert np.array_equal(mass[e], m)
            assert dt[e] == port.shell_critical_dt(nodes[e], 206e9, 0.3, 7850.0, form, 0.9)


def small_plate(fem, nx=12, ny=8, peak=6e7):
    """A 120 x 80 mm, 4 mm panel, one stiffener line, clamped edges, 0.2 mm seeded
    imperfection, a Gaussian pulse that yields ~20 % of the Gauss points in 400 steps."""
    rest, index, pinned, load = fem.stiffened_panel(nx=nx, ny=ny, lx=0.12, ly=0.08, thickness=0.004, stiffeners=1,
                                                    imperfection=2e-4, peak_pressure=peak, radius=0.02)
    return rest, index, pinned, load


@pytest.mark.parametrize("compensated,tol", [(True, 2e-5), (False, 2e-4)])
def test_shell_step_against_fp64_oracle(fem, port, compensated, tol):
    rest, index, pinned, load = small_plate(fem)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    s = fem.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0)
    dt = s.critical_dt(206e9, 0.3, 7850.0, 0.9)
    steps, rise = 400, 200 * dt
    ref.step(dt, steps, rise_time=rise)
    s.run(steps, dt=dt, rise_time=rise, compensated=compensated, max_iterations=12)
    p, v = s.readback()
    u, ur = p - rest, ref.position - rest
    err = np.abs(u - ur).max() / np.abs(ur).max()
    st = s.state()
    ep_gpu = st[:, 12:120:15].max()
    ep_ref = ref.state.reshape(-1, 129)[:, 12:120:15].max()
    assert ep_ref > 0.0, "the case must yield"
    assert err < tol, err
    assert abs(ep_gpu - ep_ref) <= 1e-3 * ep_ref + 1e-9
    e = s.energy()
    er = ref.compute_energy()
    assert abs(e[0] - er[0]) < 1e-3 * abs(er[0])
    assert abs(e[1] - er[1]) < 5e-3 * abs(er[1]) + 1e-12


def panel_bay(fem, nx=200, ny=143):
    """A bay of the single-large-mesh panel: its 10 mm cells, 12 mm plating, 1 mm seeded
    imperfection and 0.5 MPa Gaussian pulse (1.5 m, 5 ms rise), nx x ny cells with
    clamped edges.  At 200 x 143 it is the plating between two of the panel's stiffener
    lines (1.43 m apart), whose pins are its long edges."""
    return fem.stiffened_panel(nx=nx, ny=ny, lx=0.01 * nx, ly=0.01 * ny, thickness=0.012, stiffeners=0,
                               imperfection=1e-3, peak_pressure=0.5e6, radius=1.5)


def shell_drift(fem, port, steps, nx=200, ny=143, threads=None):
    """The bay stepped `steps` times on the GPU (FP32, Kahan-compensated) and by the
    FP64 oracle; errors of displacement, von Mises stress, equivalent plastic strain and
    the energy terms against the oracle."""
    rest, index, pinned, load = panel_bay(fem, nx, ny)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    s = fem.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0)
    dt = s.critical_dt(206e9, 0.3, 7850.0, 0.9)
    ref.step(dt, steps, rise_time=5e-3, threads=threads or os.cpu_count() or 1)
    s.run(steps, dt=dt, rise_time=5e-3, compensated=True, max_iterations=12)
    p, _ = s.readback()
    st = s.state()
    u, ur = p - rest, ref.position - rest
    ep, epr = st[:, 12:120:15], ref.state.reshape(-1, 129)[:, 12:120:15]
    vm, vmr = ref.von_mises(p, st), ref.von_mises(ref.position, ref.state)
    e, er = s.energy(), ref.compute_energy()
    s.close()
    return {"elements": index.size // 8, "steps": steps, "dt": dt, "simulated_s": steps * dt,
            "max_rel_displacement_error": float(np.abs(u - ur).max() / np.abs(ur).max()),
            "max_rel_von_mises_error": float(np.abs(vm - vmr).max() / vmr.max()),
            "max_rel_plastic_strain_error": float(np.abs(ep - epr).max() / epr.max()) if epr.max() > 0 else 0.0,
            "yielded_gauss_points_fp64": int((epr > 0).sum()),
            "energy_gpu": [float(x) for x in e[:4]], "energy_fp64": [float(x) for x in er[:4]],
            "max_energy_term_error_over_work": float(np.abs(np.asarray(e[:4]) - np.asarray(er[:4])).max() / abs(er[0]))}


def test_panel_bay_against_fp64_oracle(fem, port):
    """The single-large-mesh panel's bay (28,600 elements of its cells, plating, seeded
    imperfection and pressure pulse) for 500 steps, the first 0.7 ms of the pulse's
    rise, against the FP64 oracle: 2e-5 relative displacement, von Mises within 1e-3 of
    its peak, energy terms within 0.5 % of the external work."""
    r = shell_drift(fem, port, 500)
    assert r["max_rel_displacement_error"] < 2e-5, r
    assert r["max_rel_von_mises_error"] < 1e-3, r
    assert r["max_energy_term_error_over_work"] < 5e-3, r


def test_wide_launch_form_against_fp64_oracle(fem, port):
    """A zone of more warps than one wave at the narrow register budget (7,296 elements,
    1,824 warp groups against 148 SMs x 12 warps): the element pass takes its wide launch
    form (five blocks per SM), the one the full-size panel runs.  Against the FP64
    oracle, yielding, 120 steps."""
    nx, ny = 96, 76
    rest, index, pinned, load = fem.stiffened_panel(nx=nx, ny=ny, lx=0.01 * nx, ly=0.01 * ny, thickness=0.004,
                                                    stiffeners=1, imperfection=2e-4, peak_pressure=2e7, radius=0.1)
    assert index.size // 8 // 4 > 148 * 12
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    s = fem.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0)
    dt = s.critical_dt(206e9, 0.3, 7850.0, 0.9)
    steps, rise = 120, 40 * dt
    ref.step(dt, steps, rise_time=rise)
    s.run(steps, dt=dt, rise_time=rise, compensated=True, max_iterations=12)
    p, _ = s.readback()
    u, ur = p - rest, ref.position - rest
    ep_ref = ref.state.reshape(-1, 129)[:, 12:120:15]
    assert (ep_ref > 0).sum() > 100, "the case must yield"
    err = np.abs(u - ur).max() / np.abs(ur).max()
    assert err < 2e-5, err
    ep = s.state()[:, 12:120:15]
    assert abs(ep.max() - ep_ref.max()) <= 1e-3 * ep_ref.max()


@pytest.mark.parametrize("nx,ny", [(1, 1), (3, 1), (5, 1), (5, 3), (7, 2)])
def test_ragged_element_counts_against_fp64_oracle(fem, port, nx, ny):
    """Element counts that do not fill the last warp group of four (1, 3, 5, 15, 14):
    the tail lanes shadow the last element and write nothing, in the step and in the
    set-up.  A cantilever strip, clamped at x = 0, bent by a tip load into yield."""
    rest, index = fem.plate_mesh(0.01 * nx, 0.01 * ny, 0.004, nx, ny, 1)
    p0 = rest.reshape(-1, 3)
    pinned = np.repeat(p0[:, 0] < 1e-9, 3).astype(np.uint8)
    tip = p0[:, 0] > 0.01 * nx - 1e-9
    load = np.zeros_like(p0)
    load[tip, 2] = 600.0 * ny / tip.sum()
    load = load.reshape(-1)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    s = fem.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0)
    dt = s.critical_dt(206e9, 0.3, 7850.0, 0.9)
    steps, rise = 300, 100 * dt
    ref.step(dt, steps, rise_time=rise)
    s.run(steps, dt=dt, rise_time=rise, compensated=True, max_iterations=40, tol_residual=1e-6, tol_work=1e-16)
    p, _ = s.readback()
    u, ur = p - rest, ref.position - rest
    assert np.abs(ur).max() > 1e-6, "the strip must bend"
    err = np.abs(u - ur).max() / np.abs(ur).max()
    assert err < 1e-4, err
    st, sr = s.state(), ref.state.reshape(-1, 129)
    assert st.shape == sr.shape
    assert np.abs(st[:, 12:120:15] - sr[:, 12:120:15]).max() <= 1e-3 * max(sr[:, 12:120:15].max(), 1e-12) + 1e-9


def test_caller_forms_match_device_forms(fem, port):
    """Forms handed over from the CPU solver (ZoneGpuSolver::initialise's path) give the
    same step as forms built on the device: the same doubles narrowed the same way."""
    rest, index, pinned, load = small_plate(fem, nx=6, ny=4)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    forms = ref.forms.reshape(-1, O.FORMS_LEN)[:, :1505]
    a = fem.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0)
    b = fem.ShellSolver(rest, index, pinned=pinned, load=load, forms=forms, mass=ref.mass)
    dt = a.critical_dt()
    a.run(50, dt=dt, rise_time=20 * dt)
    b.run(50, dt=dt, rise_time=20 * dt)
    pa, va = a.readback()
    pb, vb = b.readback()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)


def test_caller_forms_of_another_geometry_are_refused(fem, port):
    """The step forms B and G from the rest positions, so forms a caller hands over are
    only checked: a Gauss weight, or a B entry of one of the first 64 elements, that is
    not the solid-shell's of those positions is refused at create."""
    rest, index, pinned, load = small_plate(fem, nx=6, ny=4)
    mat = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9)
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    forms = ref.forms.reshape(-1, O.FORMS_LEN)[:, :1505].copy()
    fem.ShellSolver(rest, index, pinned=pinned, load=load, forms=forms, mass=ref.mass).close()
    bad = forms.copy()
    bad[-1, 1488 + 5] *= 1.0 + 1e-6  # the last element's sixth Gauss weight
    with pytest.raises(fem.FemStepError, match="Gauss weights"):
        fem.ShellSolver(rest, index, pinned=pinned, load=load, forms=bad, mass=ref.mass)
    bad = forms.copy()
    bad[2, 7] += 1e-6 * np.abs(bad[2, :1152]).max()  # one B entry of element 2
    with pytest.raises(fem.FemStepError, match="solid-shell forms"):
        fem.ShellSolver(rest, index, pinned=pinned, load=load, forms=bad, mass=ref.mass)


def test_device_adjacency_is_the_counting_sort(fem):
    """Without a caller's adjacency the solver builds the node -> corner CSR on the
    device (atomic scatter, then each node's run sorted); with zone::Solver's
    (element-order counting sort, zone.cpp:739-755) handed over it checks and uploads
    that one.  The gather order is the CSR order, so the two runs agree bit for bit --
    on a plate and on a mesh whose elements are shuffled."""
    rest, index, pinned, load = small_plate(fem)
    rng = np.random.default_rng(7)
    shuffled = index.reshape(-1, 8)[rng.permutation(index.size // 8)].reshape(-1)
    for idx in (index, shuffled):
        offset, entry = fem.csr(rest.size // 3, idx, 8)
        a = fem.ShellSolver(rest, idx, pinned=pinned, load=load, density=7850.0)
        b = fem.ShellSolver(rest, idx, pinned=pinned, load=load, density=7850.0, adjacency_offset=offset,
                            adjacency_entry=entry)
        dt = a.critical_dt(206e9, 0.3, 7850.0, 0.9)
        a.run(60, dt=dt, rise_time=20 * dt)
        b.run(60, dt=dt, rise_time=20 * dt)
        pa, va = a.readback()
        pb, vb = b.readback()
        assert np.abs(pa - rest).max() > 0
        assert np.array_equal(pa, pb) and np.array_equal(va, vb)
        a.close()
        b.close()


def test_rigid_translation_carries_no_force(fem):
    """tests/test_zone.cpp:529: a uniform velocity moves the patch rigidly."""
    rest, index = fem.plate_mesh(0.06, 0.04, 0.012, 6, 4, 1)
    v0 = np.tile([0.3, -0.2, 0.1], rest.size // 3)
    s = fem.ShellSolver(rest, index, velocity=v0, density=7850.0)
    dt = s.critical_dt()
    s.run(100, dt=dt)
    p, v = s.readback()
    assert np.abs(v - v0).max() < 1e-6
    assert np.abs((p - rest) - v0 * 100 * dt).max() < 1e-9


def test_frame_indifference(fem):
    """tests/test_solid_shell.cpp:1493: the co-rotational element is objective.  The
    same plate, clamped round its edge and set moving in a bending bump, run once as
    meshed and once rigidly rotated by 40 degrees about an oblique axis (positions and
    velocities rotated alike): the rotated run ends at the rotated positions."""
    rest, index = fem.plate_mesh(0.06, 0.04, 0.012, 6, 4, 1)
    p0 = rest.reshape(-1, 3)
    edge = (p0[:, 0] < 1e-9) | (p0[:, 0] > 0.06 - 1e-9) | (p0[:, 1] < 1e-9) | (p0[:, 1] > 0.04 - 1e-9)
    pinned = np.repeat(edge, 3).astype(np.uint8)
    bump = np.sin(np.pi * p0[:, 0] / 0.06) * np.sin(np.pi * p0[:, 1] / 0.04)
    v0 = np.zeros_like(p0)
    v0[:, 2] = 3.0 * bump * ~edge
    axis = np.array([1.0, 2.0, 2.0]) / 3.0
    a = np.deg2rad(40.0)
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    R = np.eye(3) + np.sin(a) * k + (1 - np.cos(a)) * k @ k
    runs, dt = [], None
    for rot in (np.eye(3), R):
        r = (p0 @ rot.T).reshape(-1)
        s = fem.ShellSolver(r, index, pinned=pinned, velocity=(v0 @ rot.T).reshape(-1), density=7850.0)
        dt = dt or s.critical_dt()  # one step size for both runs
        s.run(300, dt=dt, yield_strength=355e6, hardening=1e9, compensated=True)
        runs.append(s.readback()[0].reshape(-1, 3))
    u = runs[0] - p0
    assert np.abs(u).max() > 1e-5, "the plate must move"
    err = np.abs(runs[1] - runs[0] @ R.T).max() / np.abs(u).max()
    assert err < 1e-4, err


def test_rest_stays_at_rest(fem):
    rest, index, pinned, _ = small_plate(fem, nx=6, ny=4)
    s = fem.ShellSolver(rest, index, pinned=pinned, density=7850.0)
    s.run(64, dt=s.critical_dt())
    p, v = s.readback()
    assert np.abs(p - rest).max() == 0.0 and np.abs(v).max() == 0.0


# The general point law: the benchmark workloads use the linear curve with failure off, but
# the reference's zone step (and its GPU shader) carries Swift hardening, kinematic
# hardening, ductile damage and the element failure rules.
SWIFT = (600e6, 0.02, 0.18)   # K, eps0, n: sigma_y(0) = 600e6 * 0.02^0.18 ~ 296 MPa


def general(kinematic, failure):
    mat = O.material(E=206e9, nu=0.3, yield_=SWIFT[0] * SWIFT[1] ** SWIFT[2], hardening=0.0, kinematic=kinematic,
                     swift=SWIFT, failure=failure)
    dev = dict(hardening=1, strength_coefficient=SWIFT[0], reference_strain=SWIFT[1], hardening_exponent=SWIFT[2],
               kinematic_modulus=kinematic, triaxiality_sensitivity=1.5, reference_triaxiality=1.0 / 3.0,
               cutoff_triaxiality=-1.0 / 3.0)
    return mat, dev


def run_general(fem, port, mat, dev, steps, peak):
    rest, index, pinned, load = small_plate(fem, peak=peak)
    ref = O.ShellModel(port, rest, index, pinned, mat, fext=load)
    state0 = ref.state.copy()  # the oracle's initial state: per-element failure strains
    s = fem.ShellSolver(rest, index, pinned=pinned, load=load, density=7850.0, state=state0.reshape(-1, 129))
    dt = s.critical_dt(206e9, 0.3, 7850.0, 0.9)
    rise = 200 * dt
    ref.step(dt, steps, rise_time=rise)
    s.run(steps, dt=dt, rise_time=rise, compensated=True, max_iterations=40, material=dev)
    p, _ = s.readback()
    u, ur = p - rest, ref.position - rest
    return np.abs(u - ur).max() / np.abs(ur).max(), s.state(), ref.state.reshape(-1, 129)


def test_swift_and_kinematic_hardening_against_fp64_oracle(fem, port):
    mat, dev = general(kinematic=2e9, failure=None)
    err, st, sr = run_general(fem, port, mat, dev, 400, 6e7)
    ep, epr = st[:, 12:120:15], sr[:, 12:120:15]
    assert epr.max() > 1e-3, "the case must yield"
    assert err < 5e-5, err
    assert np.abs(ep - epr).max() <= 2e-3 * epr.max()
    back, backr = st[:, [g * 15 + 6 + k for g in range(8) for k in range(6)]], sr[:, [g * 15 + 6 + k for g in range(8)
                                                                                      for k in range(6)]]
    assert np.abs(backr).max() > 0 and np.abs(back - backr).max() <= 5e-3 * np.abs(backr).max()


def test_damage_failure_and_degraded_elements_against_fp64_oracle(fem, port):
    """A short failure strain: points fail, their elements lose the enhanced modes and
    retry, some tear.  Failure is a threshold, so the comparison is on the failed set
    and the damage field rather than bit for bit."""
    mat, dev = general(kinematic=0.0, failure=(0.004, 0.008))
    err, st, sr = run_general(fem, port, mat, dev, 400, 6e7)
    failed = st[:, 14:120:15] != 0
    failed_r = sr[:, 14:120:15] != 0
    assert failed_r.sum() > 8, "the case must fail points"
    # the same points fail, up to the few at the threshold
    assert (failed != failed_r).sum() <= max(2, 0.05 * failed_r.sum()), ((failed != failed_r).sum(), failed_r.sum())
    dmg, dmg_r = st[:, 13:120:15], sr[:, 13:120:15]
    assert np.abs(dmg - dmg_r)[~(failed | failed_r)].max() <= 2e-2
    # an element with a failed point carries no enhanced modes
    assert np.all(st[failed.any(axis=1)][:, 120:127] == 0.0)
    assert (st[:, 128] != 0).sum() == (sr[:, 128] != 0).sum()
    assert err < 5e-3, err


@pytest.mark.parametrize("law", ["linear", "swift"])
def test_punch_against_fp64_oracle(fem, port, law):
    """The prescribed punch of zone::Solver::step (zone.cpp:1150-1198): the nodes under a
    small footprint in the middle of the plate's top face are driven down at a ramped
    speed; positions and the punch's work against the FP64 oracle."""
    rest, index, pinned, load = small_plate(fem, peak=0.0)
    p = rest.reshape(-1, 3)
    top = p[:, 2] > 0.0
    centre = (np.abs(p[:, 0] - 0.06) < 0.011) & (np.abs(p[:, 1] - 0.04) < 0.011)
    pinned3 = pinned.reshape(-1, 3).any(axis=1)
    driven = np.nonzero(top & centre & ~pinned3)[0]
    assert driven.size >= 4
    if law == "linear":
        mat, dev = O.material(E=206e9, nu=0.3, yield_=355e6, hardening=1e9), None
    else:
        mat, dev = general(kinematic=0.0, failure=None)
    ref = O.ShellModel(port, rest, index, pinned, mat)
    ref.set_punch(driven, (0.0, 0.0, 1.0))
    s = fem.ShellSolver(rest, index, pinned=pinned, density=7850.0, state=ref.state.copy().reshape(-1, 129))
    dt = s.critical_dt(206e9, 0.3, 7850.0, 0.9)
    s.set_punch(driven, (0.0, 0.0, 1.0), speed=4.0, ramp_time=100 * dt)
    steps = 400
    ref.step(dt, steps, punch_speed=4.0, punch_ramp=100 * dt)
    kw = dict(dt=dt, compensated=True, max_iterations=40, yield_strength=355e6, hardening=1e9)
    if dev is not None:
        kw["material"] = dev
    s.run(steps, **kw)
    pos, _ = s.readback()
    u, ur = pos - rest, ref.position - rest
    err = np.abs(u - ur).max() / np.abs(ur).max()
    st = s.punch_state()
    assert st["steps"] == steps
    assert st["penetration"] == pytest.approx(sum(4.0 * min(k * dt / (100 * dt), 1.0) * dt for k in range(steps)),
                                              rel=1e-12)
    assert ref.punch_work > 0 and abs(st["work"] - ref.punch_work) <= 2e-3 * ref.punch_work
    assert err < 1e-4, err
    # the driven nodes went down with the punch
    assert np.all(u.reshape(-1, 3)[driven, 2] < 0)


def zone_fixture():
    import importlib.util

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(here, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.ZONE_CASES, np.load(os.path.join(here, "zone_plate.npz"))


def device_material(mat):
    """plasticity::Material as the flat oracle array -> femstep_shell_material fields."""
    return dict(hardening=1 if mat[5] != 0 else 0, strength_coefficient=mat[6], reference_strain=mat[7],
                hardening_exponent=mat[8], kinematic_modulus=mat[4], triaxiality_sensitivity=mat[11],
                reference_triaxiality=mat[12], cutoff_triaxiality=mat[13])


# (position error of the run's travel, relative punch work, relative damping loss and
# boundary work) for FP32-K against zone::Solver in double.  Measured on a B200: 1.4e-7,
# 2.1e-7, 1.2e-7 and 1.4e-6 (3,000 steps, 18 elements torn) of the travel; work within
# 2.6e-6; damping loss and boundary work within 1.7e-7.  A point failing a step apart
# from the reference would move its neighbours, so the tearing case keeps more margin.
ZONE_TOL = {"prescribed": (2e-5, 1e-5, 1e-5), "inertial_damped_edge": (2e-5, 1e-5, 1e-5),
            "arrest": (2e-5, 1e-4, 1e-5), "tearing": (1e-4, 1e-4, 1e-4), "stiffened": (2e-5, 1e-5, 1e-5),
            "stiffened_tearing": (1e-3, 1e-3, 1e-3)}


@pytest.mark.parametrize("name", ["prescribed", "inertial_damped_edge", "arrest", "tearing", "stiffened",
                                  "stiffened_tearing"])
def test_zone_step_against_reference_solver(fem, name):
    """The full zone step (zone.cpp:1088-1230) on the device -- the general point law with
    failure and tearing, damping and its loss, the driven edge and its work, the punch
    prescribed or inertial with its arrest -- against the end state the reference's own
    zone::Solver wrote into tests/golden/zone_plate.npz for the same plate and case."""
    cases, g = zone_fixture()
    case = cases[name]
    rest = g["rest"]
    mass = case.get("mass", 0.0)
    s = zone_solver(fem, g, name, case)
    zone_run(s, g, case, case["steps"])
    acc = dict(zip(O.ZONE_ACCOUNT, g[f"{name}_account"]))
    pos, _ = s.readback()
    ref_pos = g[f"{name}_position"]
    travel = np.abs(ref_pos - rest).max()
    err = np.abs(pos - ref_pos).max() / travel
    ps, a = s.punch_state(), s.account()
    tol_pos, tol_work, tol_acc = ZONE_TOL[name]
    print(name, "pos", err, "work", ps["work"], acc["work"], "pen", ps["penetration"], acc["penetration"], "steps",
          ps["steps"], acc["steps"], "dloss", a["damping_loss"], acc["damping_loss"], "bwork", a["boundary_work"],
          acc["boundary_work"], "speed", a["punch_speed"], acc["punch_speed"], "arrested", a["arrested"])
    assert err < tol_pos, err
    assert abs(ps["work"] - acc["work"]) <= tol_work * abs(acc["work"])
    if mass == 0.0:
        assert ps["penetration"] == acc["penetration"]  # host double arithmetic, as the reference's
        assert ps["steps"] == acc["steps"]
    else:
        assert abs(ps["steps"] - acc["steps"]) <= 1
        assert abs(ps["penetration"] - acc["penetration"]) <= 1e-5 * acc["penetration"]
        assert a["arrested"] == bool(acc["arrested"])
    if acc["damping_loss"]:
        assert abs(a["damping_loss"] - acc["damping_loss"]) <= tol_acc * acc["damping_loss"]
    if acc["boundary_work"]:
        assert a["edge_dof"] == acc["edge_dof"]
        assert abs(a["boundary_work"] - acc["boundary_work"]) <= tol_acc * abs(acc["boundary_work"])
    st, sr = s.state(), g[f"{name}_state"].reshape(-1, 129)
    if name in ("tearing", "stiffened_tearing"):
        torn, torn_r = (st[:, 128] != 0).sum(), (sr[:, 128] != 0).sum()
        assert torn_r > 0 and abs(int(torn) - int(torn_r)) <= max(1, torn_r // 10), (torn, torn_r)
    if case.get("stiffeners", 0):
        fs, fr = s.fiber_state(), g[f"{name}_fiber_state"].reshape(-1, 4)
        print(name, "fibres: eps_p", np.abs(fs[:, 1] - fr[:, 1]).max(), "of", fr[:, 1].max(), "failed",
              int((fs[:, 3] != 0).sum()), int((fr[:, 3] != 0).sum()))
        assert (fr[:, 1] > 0).any()
        assert np.abs(fs[:, 1] - fr[:, 1]).max() <= tol_pos * 10 * fr[:, 1].max()
        assert np.array_equal(fs[:, 3] != 0, fr[:, 3] != 0)


def zone_solver(fem, g, name, case, **extra):
    # the solver's lumped mass, which holds the fibres' when the case has stiffeners
    s = fem.ShellSolver(g["rest"], g["index"], pinned=g["pinned"], mass=g[f"{name}_mass"],
                        state=extra.get("state", g["state0"].reshape(-1, 129)), position=extra.get("position"),
                        velocity=extra.get("velocity"))
    if case.get("stiffeners", 0):
        s.set_fibers(g[f"{name}_fiber_tie"], g[f"{name}_fiber_weight"], g[f"{name}_fiber_area"],
                     rest_length=g[f"{name}_fiber_length"], failure_strain=g[f"{name}_fiber_fail"])
    mass = case.get("mass", 0.0)
    s.set_punch(np.nonzero(g["driven"])[0], (0.0, 0.0, 1.0), speed=case.get("speed", 20.0),
                ramp_time=0.0 if mass > 0 else 1e-4, mass=mass)
    if any(case.get("edge_drive", (0.0, 0.0, 0.0))):
        s.set_edge(g[f"{name}_prescribed"], ramp=case.get("edge_ramp", 0.0))
    return s


def zone_run(s, g, case, steps):
    mat = g["material"]
    s.run(steps, dt=float(g["dt"]), damping=case.get("damping", 1.0), youngs=mat[0], poisson=mat[1],
          compensated=True, max_iterations=40, tol_residual=1e-6, tol_work=1e-16, material=device_material(mat))


def everything(s):
    p, v = s.readback()
    return dict(position=p, velocity=v, state=s.state(), energy=s.energy(), account=s.account(),
                punch=s.punch_state(), fibers=s.fiber_state())


def same(a, b):
    for k in a:
        if isinstance(a[k], dict):
            assert a[k] == b[k], k
        else:
            assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("name", ["inertial_damped_edge", "tearing", "stiffened_tearing"])
def test_checkpoint_resume_is_bit_identical(fem, name):
    """Checkpoint, then run on: the same bits as restoring the checkpoint into the same
    solver, or into a fresh one built from the same mesh (evict and bring back)."""
    cases, g = zone_fixture()
    case = cases[name]
    first, rest_steps = (120, 180) if "tearing" not in name else (1500, 1500)
    s = zone_solver(fem, g, name, case)
    zone_run(s, g, case, first)
    ck = s.checkpoint()
    zone_run(s, g, case, rest_steps)
    straight = everything(s)
    s.restore(ck)
    zone_run(s, g, case, rest_steps)
    same(straight, everything(s))
    del s
    t = zone_solver(fem, g, name, case)
    t.restore(ck)
    zone_run(t, g, case, rest_steps)
    same(straight, everything(t))
    if name == "tearing":
        assert (straight["state"][:, 128] != 0).sum() > 0
    # the configuration is not in the checkpoint: a solver without the punch refuses it
    u = fem.ShellSolver(g["rest"], g["index"], pinned=g["pinned"], mass=g["mass"])
    with pytest.raises(fem.FemStepError):
        u.restore(ck)


def test_readback_round_trip_is_exact(fem):
    """Positions and plastic state read back in double and handed to a new solver come
    back unchanged: the compensated float pair re-splits exactly."""
    cases, g = zone_fixture()
    case = cases["tearing"]
    s = zone_solver(fem, g, "tearing", case)
    zone_run(s, g, case, 800)
    p, v = s.readback()
    st = s.state()
    assert np.abs(p - g["rest"]).max() > 1e-3 and np.abs(st[:, 12:120:15]).max() > 1e-3
    t = zone_solver(fem, g, "tearing", case, state=st, position=p, velocity=v)
    p2, v2 = t.readback()
    assert np.array_equal(p2, p) and np.array_equal(v2, v)
    assert np.array_equal(t.state(), st)


def test_zone_inputs_are_checked(fem):
    """Bad zone inputs are refused with a reason, before any device work, and leave the
    solver usable."""
    cases, g = zone_fixture()
    s = fem.ShellSolver(g["rest"], g["index"], pinned=g["pinned"], mass=g["prescribed_mass"])
    n = s.nodes
    driven = np.nonzero(g["driven"])[0]
    with pytest.raises(fem.FemStepError, match="out of range"):
        s.set_punch(np.array([n]), (0.0, 0.0, 1.0), speed=1.0)
    with pytest.raises(fem.FemStepError, match="approach speed"):
        s.set_punch(driven, (0.0, 0.0, 1.0), speed=0.0, mass=10.0)  # zone.cpp:779-801
    with pytest.raises(fem.FemStepError, match="mass"):
        s.set_punch(driven, (0.0, 0.0, 1.0), speed=1.0, mass=-1.0)
    bad = np.zeros(3 * n)
    bad[np.nonzero(g["pinned"])[0][0]] = np.nan
    with pytest.raises(fem.FemStepError, match="not finite"):
        s.set_edge(bad)
    with pytest.raises(fem.FemStepError, match="ramp"):
        s.set_edge(np.zeros(3 * n), ramp=-1.0)
    with pytest.raises(fem.FemStepError, match="out of range"):
        s.set_fibers(np.array([[0, 1, 2, n]]), np.array([[0.5, 0.5]]), np.array([1e-4]))
    with pytest.raises(fem.FemStepError, match="not a shell checkpoint"):
        s.restore(np.zeros(64, np.uint8))
    with pytest.raises(fem.FemStepError, match="dt"):
        s.run(1, dt=0.0)
    # still usable: a clean run from rest stays at rest
    s.run(16, dt=float(g["dt"]))
    p, v = s.readback()
    assert np.array_equal(p, g["rest"]) and not np.abs(v).any()
