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


def test_rest_stays_at_rest(fem):
    rest, index, pinned, _ = small_plate(fem, nx=6, ny=4)
    s = fem.ShellSolver(rest, index, pinned=pinned, density=7850.0)
    s.run(64, dt=s.critical_dt())
    p, v = s.readback()
    assert np.abs(p - rest).max() == 0.0 and np.abs(v).max() == 0.0
