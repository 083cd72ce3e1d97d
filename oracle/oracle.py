"""ctypes view of the CPU oracle (test infrastructure only).

Loads oracle/liboracle.so (the plain-C restatement, femoracle.c) and, when it has
been built, oracle/_ref/libshipsim_ref.so (the reference's own sources compiled by
oracle/Makefile, behind ref_shim.cpp).  Both expose the C interface of femoracle.h,
under the prefixes ``or_`` and ``ref_``.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module; the
product path (sinking-simulator_b200/) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libshipsim_ref.so")

MAT_LEN = 14
POINT_LEN = 15
INCR_LEN = 9
FORMS_LEN = 1507
SHELL_STATE_LEN = 129

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


class Tet32(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("tets", C.c_size_t),
                ("position", C.POINTER(C.c_float)), ("velocity", C.POINTER(C.c_float)),
                ("mass", C.POINTER(C.c_float)), ("fixed", C.POINTER(C.c_uint32)),
                ("index", C.POINTER(C.c_uint32)), ("rest_inv", C.POINTER(C.c_float)),
                ("rest_volume", C.POINTER(C.c_float)), ("tet_force", C.POINTER(C.c_float)),
                ("adj_offset", C.POINTER(C.c_uint32)), ("adj_entry", C.POINTER(C.c_uint32))]


class Tet64(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("tets", C.c_size_t),
                ("position", C.POINTER(C.c_double)), ("velocity", C.POINTER(C.c_double)),
                ("mass", C.POINTER(C.c_double)), ("fixed", C.POINTER(C.c_uint32)),
                ("index", C.POINTER(C.c_uint32)), ("rest_inv", C.POINTER(C.c_double)),
                ("rest_volume", C.POINTER(C.c_double)), ("tet_force", C.POINTER(C.c_double)),
                ("adj_offset", C.POINTER(C.c_uint32)), ("adj_entry", C.POINTER(C.c_uint32)),
                ("plastic", C.POINTER(C.c_double)), ("stress", C.POINTER(C.c_double)),
                ("fext", C.POINTER(C.c_double)), ("energy", C.c_double * 5), ("step", C.c_long)]


class Tet64Params(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double),
                ("yield_", C.c_double), ("hardening", C.c_double), ("dt", C.c_double),
                ("gravity", C.c_double), ("damping", C.c_double), ("ramp_steps", C.c_int),
                ("polar_fixed", C.c_int)]


class Shell(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("elements", C.c_size_t),
                ("rest", C.POINTER(C.c_double)), ("position", C.POINTER(C.c_double)),
                ("velocity", C.POINTER(C.c_double)), ("mass", C.POINTER(C.c_double)),
                ("pinned", C.POINTER(C.c_uint8)), ("index", C.POINTER(C.c_uint32)),
                ("forms", C.POINTER(C.c_double)), ("state", C.POINTER(C.c_double)),
                ("element_force", C.POINTER(C.c_double)), ("stress", C.POINTER(C.c_double)),
                ("gauss_volume", C.POINTER(C.c_double)), ("adj_offset", C.POINTER(C.c_uint32)),
                ("adj_entry", C.POINTER(C.c_uint32)), ("fext", C.POINTER(C.c_double)),
                ("energy", C.c_double * 5), ("step", C.c_long), ("driven", C.POINTER(C.c_uint8)),
                ("axis", C.c_double * 3), ("prescribed", C.POINTER(C.c_double)),
                ("meshed", C.POINTER(C.c_double)), ("edge_ramp", C.c_double), ("punch_mass", C.c_double),
                ("punch_velocity", C.c_double), ("arrested", C.c_int), ("account", C.c_double * 4),
                ("fibers", C.c_size_t), ("fiber_tie", C.POINTER(C.c_uint32)), ("fiber_weight", C.POINTER(C.c_double)),
                ("fiber_area", C.POINTER(C.c_double)), ("fiber_length", C.POINTER(C.c_double)),
                ("fiber_fail", C.POINTER(C.c_double)), ("fiber_state", C.POINTER(C.c_double)),
                ("fiber_energy", C.c_double)]


class ShellParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("damping", C.c_double), ("rise_time", C.c_double),
                ("punch_speed", C.c_double), ("punch_ramp", C.c_double)]


class ZoneCase(C.Structure):
    _fields_ = [("lx", C.c_double), ("ly", C.c_double), ("thickness", C.c_double), ("nx", C.c_int),
                ("ny", C.c_int), ("nz", C.c_int), ("half_length", C.c_double), ("half_width", C.c_double),
                ("speed", C.c_double), ("ramp_time", C.c_double), ("mass", C.c_double), ("damping", C.c_double),
                ("edge_ramp", C.c_double), ("edge_drive", C.c_double * 3), ("steps", C.c_int),
                ("stiffeners", C.c_int), ("web_height", C.c_double), ("web_thickness", C.c_double),
                ("fiber_failure", C.c_int)]


class ZoneOut(C.Structure):
    _fields_ = [("rest", C.POINTER(C.c_double)), ("index", C.POINTER(C.c_uint32)),
                ("pinned", C.POINTER(C.c_uint8)), ("prescribed", C.POINTER(C.c_double)),
                ("driven", C.POINTER(C.c_uint8)), ("mass", C.POINTER(C.c_double)),
                ("state0", C.POINTER(C.c_double)), ("position", C.POINTER(C.c_double)),
                ("velocity", C.POINTER(C.c_double)), ("state", C.POINTER(C.c_double)),
                ("mat", C.c_double * MAT_LEN), ("density", C.c_double), ("dt", C.c_double),
                ("account", C.c_double * 10), ("fiber_tie", C.POINTER(C.c_uint32)),
                ("fiber_weight", C.POINTER(C.c_double)), ("fiber_area", C.POINTER(C.c_double)),
                ("fiber_length", C.POINTER(C.c_double)), ("fiber_fail", C.POINTER(C.c_double)),
                ("fiber_state", C.POINTER(C.c_double))]


ZONE_ACCOUNT = ("work", "dissipation", "penetration", "time", "damping_loss", "boundary_work", "punch_speed",
                "steps", "arrested", "edge_dof")


def build_port() -> str:
    """Compile liboracle.so with oracle/Makefile if it is missing (gcc is in the image)."""
    if not os.path.exists(PORT_SO):
        subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
    return PORT_SO


def have_ref() -> bool:
    return os.path.exists(REF_SO)


class Oracle:
    """One implementation of femoracle.h: prefix 'or_' (restatement) or 'ref_'."""

    def __init__(self, which: str = "port"):
        if which == "port":
            self.lib = C.CDLL(build_port())
            self.p = "or_"
        elif which == "ref":
            if not have_ref():
                raise FileNotFoundError(REF_SO)
            self.lib = C.CDLL(REF_SO)
            self.p = "ref_"
        else:
            raise ValueError(which)
        self.which = which
        L = self.lib
        g = self._fn
        g("plastic_update", C.c_int, [f64p, C.c_double, f64p, f64p, f64p, C.c_void_p, f64p])
        g("box_tet_sizes", None, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)])
        g("box_tet_mesh", None, [C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, f32p, u32p])
        g("tet32_rest_state", None, [C.POINTER(Tet32), C.c_float, C.c_float, C.c_float])
        g("tet32_forces", None, [C.POINTER(Tet32), C.c_size_t, C.c_float, C.c_float, f32p])
        g("tet32_step", None, [C.POINTER(Tet32), C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                               C.c_float, C.c_int])
        g("tet32_critical_dt", C.c_float, [C.POINTER(Tet32), C.c_float, C.c_float, C.c_float, C.c_float])
        g("tet64_rest_state", None, [C.POINTER(Tet64), C.c_double])
        g("tet64_step", None, [C.POINTER(Tet64), C.POINTER(Tet64Params), C.c_int])
        g("shell_forms", C.c_int, [f64p, C.c_int, f64p])
        g("shell_mass", None, [f64p, C.c_double, f64p])
        g("shell_gauss_volumes", None, [f64p, f64p])
        g("shell_init_state", None, [f64p, f64p, f64p])
        g("shell_plastic_update", C.c_int, [f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p])
        g("shell_rotation", None, [f64p, f64p, f64p])
        g("shell_stiffness", None, [f64p, C.c_double, C.c_double, C.c_int, f64p])
        g("shell_critical_dt", C.c_double, [f64p, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double])
        g("plate_sizes", None, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)])
        g("plate_mesh", None, [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, f64p, u32p])
        g("plate_pressure_load", None, [f64p, u32p, C.c_size_t, C.c_size_t, C.c_double, f64p])
        g("shell_setup", None, [C.POINTER(Shell), f64p, C.c_double])
        g("shell_step", None, [C.POINTER(Shell), f64p, C.POINTER(ShellParams), C.c_int])
        g("shell_energy", None, [C.POINTER(Shell), f64p])
        if which == "port":
            g("tet64_critical_dt", C.c_double, [C.POINTER(Tet64), C.c_double, C.c_double, C.c_double,
                                                C.c_double])
            g("tet64_step_threads", None, [C.POINTER(Tet64), C.POINTER(Tet64Params), C.c_int, C.c_int])
            g("shell_step_threads", None, [C.POINTER(Shell), f64p, C.POINTER(ShellParams), C.c_int, C.c_int])
        else:
            g("shell_time_parallel", C.c_double, [C.POINTER(Shell), f64p, C.POINTER(ShellParams), C.c_int,
                                                  C.c_int])
            g("default_workers", C.c_uint, [])
            g("tet64_time_parallel", C.c_double, [C.POINTER(Tet64), C.POINTER(Tet64Params), C.c_int, C.c_int])
            g("tet64_time_batch", C.c_double, [C.POINTER(C.POINTER(Tet64)), C.POINTER(Tet64Params), C.c_size_t,
                                               C.c_int, C.c_int])
            g("tet32_time", C.c_double, [C.POINTER(Tet32), C.c_float, C.c_float, C.c_float, C.c_float, C.c_int])
            g("zone_sizes", C.c_int, [C.POINTER(ZoneCase), C.POINTER(C.c_size_t)])
            g("zone_run", C.c_int, [C.POINTER(ZoneCase), C.POINTER(ZoneOut)])

    def zone_plate(self, lx=0.4, ly=0.2, thickness=0.01, nx=8, ny=4, nz=1, half_length=0.05, half_width=0.05,
                   speed=20.0, ramp_time=1e-4, mass=0.0, damping=1.0, edge_ramp=0.0, edge_drive=(0.0, 0.0, 0.0),
                   steps=100, stiffeners=0, web_height=0.05, web_thickness=0.008, fiber_failure=True) -> dict:
        """The reference's zone::Solver stepped `steps` times on a flat plate (ref only):
        the arrays it was built from, where it ended and its account."""
        c = ZoneCase(lx, ly, thickness, nx, ny, nz, half_length, half_width, speed, ramp_time, mass, damping,
                     edge_ramp, (C.c_double * 3)(*edge_drive), steps, stiffeners, web_height, web_thickness,
                     int(bool(fiber_failure)))
        sizes = (C.c_size_t * 3)()
        self.zone_sizes(C.byref(c), sizes)
        n, e, f = sizes[0], sizes[1], sizes[2]
        r = dict(rest=np.zeros(3 * n), index=np.zeros(8 * e, np.uint32), pinned=np.zeros(3 * n, np.uint8),
                 prescribed=np.zeros(3 * n), driven=np.zeros(n, np.uint8), mass=np.zeros(n),
                 state0=np.zeros(SHELL_STATE_LEN * e), position=np.zeros(3 * n), velocity=np.zeros(3 * n),
                 state=np.zeros(SHELL_STATE_LEN * e), fiber_tie=np.zeros(4 * f, np.uint32),
                 fiber_weight=np.zeros(2 * f), fiber_area=np.zeros(f), fiber_length=np.zeros(f),
                 fiber_fail=np.zeros(f), fiber_state=np.zeros(4 * f))
        o = ZoneOut()
        for name, ct in (("rest", C.c_double), ("index", C.c_uint32), ("pinned", C.c_uint8),
                         ("prescribed", C.c_double), ("driven", C.c_uint8), ("mass", C.c_double),
                         ("state0", C.c_double), ("position", C.c_double), ("velocity", C.c_double),
                         ("state", C.c_double), ("fiber_tie", C.c_uint32), ("fiber_weight", C.c_double),
                         ("fiber_area", C.c_double), ("fiber_length", C.c_double), ("fiber_fail", C.c_double),
                         ("fiber_state", C.c_double)):
            setattr(o, name, _ptr(r[name], ct))
        r["problems"] = self.zone_run(C.byref(c), C.byref(o))
        r["mat"] = np.array(list(o.mat))
        r["density"], r["dt"] = o.density, o.dt
        r["account"] = dict(zip(ZONE_ACCOUNT, list(o.account)))
        return r

    def _fn(self, name, res, args):
        f = getattr(self.lib, self.p + name)
        f.restype = res
        f.argtypes = args
        setattr(self, name, f)


def material(E=210e9, nu=0.3, yield_=235e6, hardening=1e9, kinematic=0.0, swift=None,
             failure=None) -> np.ndarray:
    """Flat point-law material (femoracle.h).  failure: (uniform, fracture) or None = never."""
    m = np.zeros(MAT_LEN)
    m[0], m[1], m[2], m[3], m[4] = E, nu, yield_, hardening, kinematic
    if swift is not None:
        m[5] = 1.0
        m[6], m[7], m[8] = swift
    if failure is None:
        m[9], m[10] = np.inf, np.inf
    else:
        m[9], m[10] = failure
    m[11], m[12], m[13] = 1.5, 1.0 / 3.0, -1.0 / 3.0
    return m


class TetMesh32:
    """A fem::TetMesh in numpy arrays, bound to an or_tet32 struct."""

    def __init__(self, o: Oracle, position, index):
        self.o = o
        self.position = np.array(position, np.float32).reshape(-1)
        self.index = np.array(index, np.uint32).reshape(-1)
        n = self.position.size // 3
        t = self.index.size // 4
        self.nodes, self.tets = n, t
        self.velocity = np.zeros(3 * n, np.float32)
        self.mass = np.zeros(n, np.float32)
        self.fixed = np.zeros(n, np.uint32)
        self.rest_inv = np.zeros(9 * t, np.float32)
        self.rest_volume = np.zeros(t, np.float32)
        self.tet_force = np.zeros(12 * t, np.float32)
        self.adj_offset = np.zeros(n + 1, np.uint32)
        self.adj_entry = np.zeros(4 * t, np.uint32)

    def struct(self) -> Tet32:
        s = Tet32()
        s.nodes, s.tets = self.nodes, self.tets
        for name, ct in (("position", C.c_float), ("velocity", C.c_float), ("mass", C.c_float),
                         ("fixed", C.c_uint32), ("index", C.c_uint32), ("rest_inv", C.c_float),
                         ("rest_volume", C.c_float), ("tet_force", C.c_float),
                         ("adj_offset", C.c_uint32), ("adj_entry", C.c_uint32)):
            setattr(s, name, _ptr(getattr(self, name), ct))
        return s

    def rest_state(self, E, nu, rho):
        s = self.struct()
        fixed = self.fixed.copy()
        self.o.tet32_rest_state(C.byref(s), E, nu, rho)
        self.fixed[:] = fixed

    def step(self, E, nu, rho, dt, gravity, damping, steps):
        s = self.struct()
        self.o.tet32_step(C.byref(s), E, nu, rho, dt, gravity, damping, steps)

    def copy(self):
        c = TetMesh32.__new__(TetMesh32)
        c.__dict__.update({k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
        return c


def box_tet_mesh(o: Oracle, lx, ly, lz, nx, ny, nz):
    n, t = C.c_size_t(), C.c_size_t()
    o.box_tet_sizes(nx, ny, nz, C.byref(n), C.byref(t))
    pos = np.zeros(3 * n.value, np.float32)
    idx = np.zeros(4 * t.value, np.uint32)
    o.box_tet_mesh(lx, ly, lz, nx, ny, nz, pos, idx)
    return pos, idx


class TetMesh64:
    """O-tet64 state (double, J2) bound to an or_tet64 struct."""

    def __init__(self, o: Oracle, position32, index, fixed, fext=None, rho=7850.0):
        self.o = o
        self.position = np.ascontiguousarray(position32, np.float32).astype(np.float64).reshape(-1)
        self.index = np.array(index, np.uint32).reshape(-1)
        n = self.position.size // 3
        t = self.index.size // 4
        self.nodes, self.tets = n, t
        self.velocity = np.zeros(3 * n)
        self.mass = np.zeros(n)
        self.fixed = np.ascontiguousarray(fixed, np.uint32)
        self.rest_inv = np.zeros(9 * t)
        self.rest_volume = np.zeros(t)
        self.tet_force = np.zeros(12 * t)
        self.adj_offset = np.zeros(n + 1, np.uint32)
        self.adj_entry = np.zeros(4 * t, np.uint32)
        self.plastic = np.zeros(7 * t)
        self.stress = np.zeros(6 * t)
        self.fext = None if fext is None else np.ascontiguousarray(fext, np.float64).reshape(-1)
        self.energy = np.zeros(5)
        self.steps = 0
        self._s = self._make()
        o.tet64_rest_state(C.byref(self._s), rho)

    def _make(self) -> Tet64:
        s = Tet64()
        s.nodes, s.tets = self.nodes, self.tets
        for name, ct in (("position", C.c_double), ("velocity", C.c_double), ("mass", C.c_double),
                         ("fixed", C.c_uint32), ("index", C.c_uint32), ("rest_inv", C.c_double),
                         ("rest_volume", C.c_double), ("tet_force", C.c_double),
                         ("adj_offset", C.c_uint32), ("adj_entry", C.c_uint32),
                         ("plastic", C.c_double), ("stress", C.c_double), ("fext", C.c_double)):
            setattr(s, name, _ptr(getattr(self, name), ct))
        s.step = 0
        return s

    def step(self, params: Tet64Params, steps: int, threads: int = 1):
        """`steps` steps; with threads > 1 the element loop runs on that many host
        threads (restatement only), bit-identical to the serial step."""
        if threads > 1:
            self.o.tet64_step_threads(C.byref(self._s), C.byref(params), steps, threads)
        else:
            self.o.tet64_step(C.byref(self._s), C.byref(params), steps)
        self.energy[:] = list(self._s.energy)
        self.steps = self._s.step


def tet64_params(E=210e9, nu=0.3, rho=7850.0, yield_=235e6, hardening=1e9, dt=1e-7, gravity=0.0,
                 damping=1.0, ramp_steps=0, polar_fixed=0) -> Tet64Params:
    return Tet64Params(E, nu, rho, yield_, hardening, dt, gravity, damping, ramp_steps, polar_fixed)


def plate_mesh(o: Oracle, lx, ly, t, nx, ny, nz=1):
    n, e = C.c_size_t(), C.c_size_t()
    o.plate_sizes(nx, ny, nz, C.byref(n), C.byref(e))
    pos = np.zeros(3 * n.value)
    idx = np.zeros(8 * e.value, np.uint32)
    o.plate_mesh(lx, ly, t, nx, ny, nz, pos, idx)
    return pos, idx


class ShellModel:
    """The composed explicit shell step (or_shell)."""

    def __init__(self, o: Oracle, rest, index, pinned, mat, density=7850.0, fext=None, position=None):
        self.o = o
        self.mat = np.ascontiguousarray(mat, np.float64)
        self.rest = np.ascontiguousarray(rest, np.float64).reshape(-1)
        self.position = self.rest.copy() if position is None else np.ascontiguousarray(position, np.float64).reshape(-1).copy()
        self.index = np.array(index, np.uint32).reshape(-1)
        n = self.rest.size // 3
        e = self.index.size // 8
        self.nodes, self.elements = n, e
        self.velocity = np.zeros(3 * n)
        self.mass = np.zeros(n)
        self.pinned = np.ascontiguousarray(pinned, np.uint8).reshape(-1)
        self.forms = np.zeros(FORMS_LEN * e)
        self.state = np.zeros(SHELL_STATE_LEN * e)
        self.element_force = np.zeros(24 * e)
        self.stress = np.zeros(48 * e)
        self.gauss_volume = np.zeros(8 * e)
        self.adj_offset = np.zeros(n + 1, np.uint32)
        self.adj_entry = np.zeros(8 * e, np.uint32)
        self.fext = None if fext is None else np.ascontiguousarray(fext, np.float64).reshape(-1)
        self._s = Shell()
        s = self._s
        s.nodes, s.elements = n, e
        for name, ct in (("rest", C.c_double), ("position", C.c_double), ("velocity", C.c_double),
                         ("mass", C.c_double), ("pinned", C.c_uint8), ("index", C.c_uint32),
                         ("forms", C.c_double), ("state", C.c_double), ("element_force", C.c_double),
                         ("stress", C.c_double), ("gauss_volume", C.c_double),
                         ("adj_offset", C.c_uint32), ("adj_entry", C.c_uint32), ("fext", C.c_double)):
            setattr(s, name, _ptr(getattr(self, name), ct))
        s.step = 0
        o.shell_setup(C.byref(s), self.mat, density)

    @property
    def energy(self):
        return np.array(list(self._s.energy))

    @property
    def steps(self):
        return self._s.step

    def set_punch(self, driven_nodes, axis, mass=0.0, speed=0.0):
        """The punch (zone.cpp:1147-1198) grips these nodes and travels along -axis.  With
        mass > 0 it is a striking body of that mass arriving at `speed` (the inertial
        punch); otherwise the speed is prescribed per step (ShellModel.step)."""
        self.driven = np.zeros(self.nodes, np.uint8)
        self.driven[np.asarray(driven_nodes, np.int64)] = 1
        self._s.driven = _ptr(self.driven, C.c_uint8)
        for k in range(3):
            self._s.axis[k] = float(axis[k])
        self._s.punch_mass = float(mass)
        self._s.punch_velocity = float(speed) if mass > 0 else 0.0

    def set_edge(self, prescribed, meshed=None, ramp=0.0):
        """The driven edge (zone.cpp:833-842, 1123-1145): each pinned DOF with a non-zero
        prescribed value follows meshed + prescribed * smoothstep(t / ramp)."""
        self.prescribed = np.ascontiguousarray(prescribed, np.float64).reshape(-1).copy()
        self._s.prescribed = _ptr(self.prescribed, C.c_double)
        if meshed is not None:
            self.meshed = np.ascontiguousarray(meshed, np.float64).reshape(-1).copy()
            self._s.meshed = _ptr(self.meshed, C.c_double)
        self._s.edge_ramp = float(ramp)

    def set_fibers(self, tie, weight, area, length, fail, density=None):
        """Constraint fibres (constraint.hpp): tie [F][4] node ids (end 0 bottom, top; end 1
        bottom, top), weight [F][2], area, rest length and failure strain [F].  With a
        density, each fibre's mass is lumped a quarter to each of its four nodes, in fibre
        order (lumpFiberMass, constraint.cpp:260-276)."""
        f = int(np.asarray(area).size)
        if density is not None:
            t = np.asarray(tie, np.int64).reshape(-1, 4)
            for i in range(f):
                if not (length[i] > 0 and area[i] > 0):
                    continue
                quarter = 0.25 * density * float(area[i]) * float(length[i])
                for k in range(4):
                    self.mass[t[i, k]] += quarter
        self.fiber_tie = np.ascontiguousarray(tie, np.uint32).reshape(-1).copy()
        self.fiber_weight = np.ascontiguousarray(weight, np.float64).reshape(-1).copy()
        self.fiber_area = np.ascontiguousarray(area, np.float64).reshape(-1).copy()
        self.fiber_length = np.ascontiguousarray(length, np.float64).reshape(-1).copy()
        self.fiber_fail = np.ascontiguousarray(fail, np.float64).reshape(-1).copy()
        self.fiber_state = np.zeros(4 * f)
        s = self._s
        s.fibers = f
        for name, ct in (("fiber_tie", C.c_uint32), ("fiber_weight", C.c_double), ("fiber_area", C.c_double),
                         ("fiber_length", C.c_double), ("fiber_fail", C.c_double), ("fiber_state", C.c_double)):
            setattr(s, name, _ptr(getattr(self, name), ct))

    @property
    def account(self):
        """dict: damping loss, boundary work, penetration, time, punch speed, arrested."""
        a = self._s.account
        return dict(damping_loss=a[0], boundary_work=a[1], penetration=a[2], time=a[3],
                    punch_speed=self._s.punch_velocity, arrested=bool(self._s.arrested))

    @property
    def punch_work(self):
        return self._s.energy[4]

    def step(self, dt, steps, damping=1.0, rise_time=0.0, punch_speed=0.0, punch_ramp=0.0, threads=1):
        """`steps` steps; with threads > 1 the element loop runs on that many host
        threads (restatement only), bit-identical to the serial step."""
        p = ShellParams(dt, damping, rise_time, punch_speed, punch_ramp)
        if threads > 1:
            self.o.shell_step_threads(C.byref(self._s), self.mat, C.byref(p), steps, threads)
        else:
            self.o.shell_step(C.byref(self._s), self.mat, C.byref(p), steps)

    def compute_energy(self):
        self.o.shell_energy(C.byref(self._s), self.mat)
        return self.energy

    def von_mises(self, position, state):
        """Von Mises stress at each Gauss point, (elements, 8), of a state (positions and
        the 129-double ElementPlasticState per element) of this model's mesh: the element
        update (elementPlasticUpdate) run on a copy of each element's state at those
        positions, so any two states go through the same routine."""
        pos = np.ascontiguousarray(position, np.float64).reshape(-1, 3)
        st = np.ascontiguousarray(state, np.float64).reshape(self.elements, -1)
        idx = self.index.reshape(-1, 8).astype(np.int64)
        rest = self.rest.reshape(-1, 3)
        out = np.empty((self.elements, 8))
        force, stress, info = np.zeros(24), np.zeros(48), np.zeros(7)
        for e in range(self.elements):
            cur = np.ascontiguousarray(pos[idx[e]].reshape(-1))
            r = np.ascontiguousarray(rest[idx[e]].reshape(-1))
            copy = st[e].copy()
            self.o.shell_plastic_update(self.forms[e * FORMS_LEN:(e + 1) * FORMS_LEN], r, cur, self.mat, copy, force,
                                        stress, info)
            sv = stress.reshape(8, 6)
            out[e] = np.sqrt(0.5 * ((sv[:, 0] - sv[:, 1]) ** 2 + (sv[:, 1] - sv[:, 2]) ** 2 +
                                    (sv[:, 2] - sv[:, 0]) ** 2) + 3.0 * (sv[:, 3:] ** 2).sum(1))
        return out

    def time_parallel(self, dt, steps, workers=0, rise_time=0.0):
        p = ShellParams(dt, 1.0, rise_time, 0.0, 0.0)
        return self.o.shell_time_parallel(C.byref(self._s), self.mat, C.byref(p), steps, workers)
