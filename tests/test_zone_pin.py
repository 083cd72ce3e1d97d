"""The oracle's zone step against the reference's own zone::Solver (CPU, no GPU).

`ref.zone_plate` builds a flat plate as the reference's zone GPU tests build theirs
(tests/test_zone_gpu.cpp:163-197 in the reference), constructs zone::Solver on it
(engine/sim/zone.cpp) and calls step(); the oracle's or_shell_step then runs from the
same arrays.  The two must agree bit for bit: the element update, the CSR gather, the
velocity update, the damping and its loss, the driven edge and its work, the punch
(prescribed and inertial) and its work, the penetration, the arrest of an inertial
punch, and element failure and tearing.  This pins the oracle's composition of
zone::Solver::step (zone.cpp:1088-1230) that the GPU tests compare against.
"""
import numpy as np
import pytest

import oracle as O

CASES = {
    "prescribed": dict(steps=300),
    "damping": dict(steps=300, damping=0.999),
    "inertial": dict(steps=300, mass=40.0, speed=20.0),
    "edge-ramped": dict(steps=300, edge_drive=(2e-3, 1e-3, 3e-3), edge_ramp=2e-4),
    "edge-at-once": dict(steps=300, edge_drive=(2e-3, 0.0, 1e-3)),
    "arrest": dict(steps=3000, mass=0.6, speed=6.0),
    "tearing": dict(steps=3000),
    "everything": dict(steps=3000, mass=400.0, speed=20.0, damping=0.9995, edge_drive=(1e-3, 0.0, 2e-3),
                       edge_ramp=1e-3),
    "stiffened": dict(steps=300, stiffeners=1),
    "stiffened-tearing": dict(steps=3000, stiffeners=2, web_height=0.03, web_thickness=0.006),
    "stiffened-no-fibre-failure": dict(steps=3000, stiffeners=1, fiber_failure=False),
}


def port_zone(port, r, case):
    m = O.ShellModel(port, r["rest"], r["index"], r["pinned"], r["mat"], density=r["density"])
    m.set_punch(np.nonzero(r["driven"])[0], (0.0, 0.0, 1.0), mass=case.get("mass", 0.0),
                speed=case.get("speed", 20.0))
    if any(case.get("edge_drive", (0.0, 0.0, 0.0))):
        m.set_edge(r["prescribed"], ramp=case.get("edge_ramp", 0.0))
    if case.get("stiffeners", 0):
        m.set_fibers(r["fiber_tie"], r["fiber_weight"], r["fiber_area"], r["fiber_length"], r["fiber_fail"],
                     density=r["density"])
    m.step(r["dt"], case["steps"], damping=case.get("damping", 1.0), punch_speed=case.get("speed", 20.0),
           punch_ramp=1e-4)
    return m


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_zone_step_is_the_reference_solver(ref, port, name):
    case = CASES[name]
    r = ref.zone_plate(**case)
    assert r["problems"] == 0
    m = port_zone(port, r, case)
    # the set-up: lumped mass and the initial plastic state with its failure strains
    assert np.array_equal(m.mass, r["mass"])
    a, ra = m.account, r["account"]
    assert m.steps == ra["steps"]
    assert np.array_equal(m.position, r["position"])
    assert np.array_equal(m.velocity, r["velocity"])
    assert np.array_equal(m.state, r["state"])
    assert m.punch_work == ra["work"]
    assert a["penetration"] == ra["penetration"]
    assert a["time"] == ra["time"]
    assert a["damping_loss"] == ra["damping_loss"]
    assert a["boundary_work"] == ra["boundary_work"]
    assert a["arrested"] == bool(ra["arrested"])
    if case.get("mass", 0.0) > 0:
        assert a["punch_speed"] == ra["punch_speed"]
    st = r["state"].reshape(-1, O.SHELL_STATE_LEN)
    # what each case must have exercised, so that agreement is not agreement on nothing
    assert ra["work"] > 0 and ra["penetration"] > (0.0 if name == "arrest" else 1e-3)
    if case.get("damping", 1.0) != 1.0:
        assert ra["damping_loss"] > 0
    if any(case.get("edge_drive", (0.0, 0.0, 0.0))):
        assert ra["edge_dof"] > 0 and ra["boundary_work"] != 0
    if name == "arrest":
        assert ra["arrested"] and ra["steps"] < case["steps"]
    if name in ("tearing", "everything"):
        assert (st[:, 128] != 0).sum() > 0 and (st[:, 14:120:15] != 0).sum() > 0
    if case.get("stiffeners", 0):
        # the stiffeners: lumped mass (checked above), and the fibres' own state
        fs = r["fiber_state"].reshape(-1, 4)
        assert np.array_equal(m.fiber_state, r["fiber_state"])
        assert fs.shape[0] > 0 and (fs[:, 1] > 0).any(), "the fibres must yield"
        if name == "stiffened-tearing":
            assert (fs[:, 3] != 0).any(), "and some must tear"
        if not case.get("fiber_failure", True):
            assert not (fs[:, 3] != 0).any()


def golden_zone():
    """The zone fixture and the cases it was made with (tests/golden/make_golden.py)."""
    import importlib.util
    import os

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(here, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.ZONE_CASES, np.load(os.path.join(here, "zone_plate.npz"))


@pytest.mark.parametrize("name", ["prescribed", "inertial_damped_edge", "arrest", "tearing", "stiffened",
                                  "stiffened_tearing"])
def test_oracle_zone_step_golden(port, name):
    """The same pin without the compiled reference: the restatement reproduces the
    fixture zone::Solver wrote, bit for bit."""
    cases, g = golden_zone()
    case = cases[name]
    r = dict(rest=g["rest"], index=g["index"], pinned=g["pinned"], mat=g["material"], density=float(g["density"]),
             driven=g["driven"], prescribed=g[f"{name}_prescribed"], dt=float(g["dt"]))
    for k in ("fiber_tie", "fiber_weight", "fiber_area", "fiber_length", "fiber_fail"):
        r[k] = g[f"{name}_{k}"]
    m = port_zone(port, r, case)
    assert np.array_equal(m.mass, g[f"{name}_mass"])
    if case.get("stiffeners", 0):
        assert np.array_equal(m.fiber_state, g[f"{name}_fiber_state"])
    assert np.array_equal(m.position, g[f"{name}_position"])
    assert np.array_equal(m.velocity, g[f"{name}_velocity"])
    assert np.array_equal(m.state, g[f"{name}_state"])
    acc = dict(zip(O.ZONE_ACCOUNT, g[f"{name}_account"]))
    a = m.account
    assert (m.punch_work, a["penetration"], a["damping_loss"], a["boundary_work"]) == (
        acc["work"], acc["penetration"], acc["damping_loss"], acc["boundary_work"])
    assert m.steps == acc["steps"] and a["arrested"] == bool(acc["arrested"])
