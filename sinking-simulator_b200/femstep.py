"""Python host binding of libfemstep.so (the C ABI in include/femstep.h).

The classes here mirror the reference's step interfaces so that code written against
them reads the same:

  TetSolver    gpu::FemGpuSolver (engine/gpu/fem_gpu.hpp:17-45): initialise / run /
               readback / deviceName, extended with the J2 tet modes, the FP64 energy
               account and the FP64 critical time step.

Failure convention, as the reference's: no CUDA device raises ``NoDevice`` (the
"skip, not fail" of fem_gpu.hpp:21-22); every other failure raises ``FemStepError``
with the library's text.  There is no CPU fallback: if libfemstep.so is missing the
import fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfemstep.so")

OK, SKIP, EINVAL, ENOMEM, ECUDA, ESTATE, ETIMEOUT = range(7)
TET_REF32, TET_J2_F32, TET_J2_F32K, TET_J2_F64 = range(4)
MODES = {"ref32": TET_REF32, "f32": TET_J2_F32, "f32k": TET_J2_F32K, "f64": TET_J2_F64}


class FemStepError(RuntimeError):
    def __init__(self, code: int, text: str):
        super().__init__(f"femstep error {code}: {text}")
        self.code = code


class NoDevice(FemStepError):
    pass


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libfemstep.so is not built ({LIB_PATH}); run `make -C {HERE}`")
    return C.CDLL(LIB_PATH)


lib = _load()


class TetMeshC(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("tets", C.c_size_t),
                ("position", C.c_void_p), ("velocity", C.c_void_p), ("mass", C.c_void_p),
                ("fixed", C.c_void_p), ("index", C.c_void_p), ("rest_inv", C.c_void_p),
                ("rest_volume", C.c_void_p), ("adjacency_offset", C.c_void_p),
                ("adjacency_entry", C.c_void_p), ("external_force", C.c_void_p),
                ("density", C.c_double)]


class TetParamsC(C.Structure):
    _fields_ = [("youngs_modulus", C.c_double), ("poisson_ratio", C.c_double),
                ("yield_strength", C.c_double), ("hardening_modulus", C.c_double),
                ("dt", C.c_double), ("gravity", C.c_double), ("damping", C.c_double),
                ("ramp_steps", C.c_int)]


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


_last_error = _sig("femstep_last_error", C.c_char_p, [])
_device_name = _sig("femstep_device_name", C.c_int, [C.c_char_p, C.c_size_t])
_tet_create = _sig("femstep_tet_create", C.c_int, [C.POINTER(TetMeshC), C.c_int, C.POINTER(C.c_void_p)])
_tet_run = _sig("femstep_tet_run", C.c_int, [C.c_void_p, C.c_int, C.POINTER(TetParamsC), C.POINTER(C.c_double)])
_tet_readback = _sig("femstep_tet_readback", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p])
_tet_readback64 = _sig("femstep_tet_readback_f64", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p])
_tet_plastic = _sig("femstep_tet_plastic", C.c_int, [C.c_void_p, C.c_void_p])
_tet_energy = _sig("femstep_tet_energy", C.c_int, [C.c_void_p, C.c_void_p])
_tet_dt = _sig("femstep_tet_critical_dt", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                                      C.c_double, C.POINTER(C.c_double)])
_tet_profile = _sig("femstep_tet_profile", C.c_int, [C.c_void_p, C.c_int, C.POINTER(TetParamsC), C.c_void_p])
_tet_launches = _sig("femstep_tet_launches", C.c_longlong, [C.c_void_p])
_tet_error = _sig("femstep_tet_error", C.c_char_p, [C.c_void_p])
_tet_destroy = _sig("femstep_tet_destroy", None, [C.c_void_p])


def _raise(code: int, text: bytes | None):
    msg = (text or b"").decode(errors="replace")
    if code == SKIP:
        raise NoDevice(code, msg)
    raise FemStepError(code, msg)


_set_device = _sig("femstep_set_device", C.c_int, [C.c_int])


def set_device(device: int) -> None:
    """Select the GPU this process's solvers live on (one process per GPU)."""
    rc = _set_device(int(device))
    if rc:
        _raise(rc, _last_error())


def device_name() -> str:
    buf = C.create_string_buffer(256)
    rc = _device_name(buf, 256)
    if rc:
        _raise(rc, _last_error())
    return buf.value.decode()


def _p(a):
    return None if a is None else a.ctypes.data


class TetSolver:
    """A tet mesh resident on the GPU; the reference's gpu::FemGpuSolver.

    mode: "ref32" (fem::stepCpu arithmetic, bit-exact), "f32", "f32k" (Kahan), "f64".
    Arrays use the reference's TetMesh layout (fem.hpp:38-68).
    """

    def __init__(self, position, index, mode="ref32", velocity=None, mass=None, fixed=None, rest_inv=None,
                 rest_volume=None, adjacency_offset=None, adjacency_entry=None, external_force=None,
                 density=0.0):
        self.mode = MODES[mode] if isinstance(mode, str) else int(mode)
        keep = {}

        def arr(name, a, dt):
            if a is None:
                return None
            keep[name] = np.ascontiguousarray(a, dt).reshape(-1)
            return keep[name]

        pos = arr("position", position, np.float32)
        idx = arr("index", index, np.uint32)
        self.nodes = pos.size // 3
        self.tets = idx.size // 4
        m = TetMeshC()
        m.nodes, m.tets = self.nodes, self.tets
        m.position = _p(pos)
        m.velocity = _p(arr("velocity", velocity, np.float32))
        m.mass = _p(arr("mass", mass, np.float32))
        m.fixed = _p(arr("fixed", fixed, np.uint32))
        m.index = _p(idx)
        m.rest_inv = _p(arr("rest_inv", rest_inv, np.float32))
        m.rest_volume = _p(arr("rest_volume", rest_volume, np.float32))
        m.adjacency_offset = _p(arr("adjacency_offset", adjacency_offset, np.uint32))
        m.adjacency_entry = _p(arr("adjacency_entry", adjacency_entry, np.uint32))
        m.external_force = _p(arr("external_force", external_force, np.float64))
        m.density = float(density)
        h = C.c_void_p()
        rc = _tet_create(C.byref(m), self.mode, C.byref(h))
        if rc:
            _raise(rc, _last_error())
        self._h = h

    def _check(self, rc):
        if rc:
            _raise(rc, _tet_error(self._h))

    def run(self, substeps, youngs=210e9, poisson=0.3, dt=1e-7, gravity=0.0, damping=1.0, yield_strength=235e6,
            hardening=1e9, ramp_steps=0) -> float:
        """gpu::FemGpuSolver::run: `substeps` steps; returns device milliseconds."""
        p = TetParamsC(youngs, poisson, yield_strength, hardening, dt, gravity, damping, int(ramp_steps))
        ms = C.c_double()
        self._check(_tet_run(self._h, int(substeps), C.byref(p), C.byref(ms)))
        return ms.value

    def readback(self):
        """Positions and velocities, 3N float each (gpu::FemGpuSolver::readback)."""
        p = np.zeros(3 * self.nodes, np.float32)
        v = np.zeros(3 * self.nodes, np.float32)
        self._check(_tet_readback(self._h, _p(p), _p(v)))
        return p, v

    def readback64(self):
        p = np.zeros(3 * self.nodes)
        v = np.zeros(3 * self.nodes)
        self._check(_tet_readback64(self._h, _p(p), _p(v)))
        return p, v

    def plastic(self):
        out = np.zeros(7 * self.tets)
        self._check(_tet_plastic(self._h, _p(out)))
        return out.reshape(self.tets, 7)

    def energy(self):
        """[external work, dissipation, strain energy, kinetic, gravity work], FP64 on device."""
        out = np.zeros(5)
        self._check(_tet_energy(self._h, _p(out)))
        return out

    def critical_dt(self, youngs=210e9, poisson=0.3, density=7850.0, safety=0.9) -> float:
        dt = C.c_double()
        self._check(_tet_dt(self._h, youngs, poisson, density, safety, C.byref(dt)))
        return dt.value

    def profile(self, steps, youngs=210e9, poisson=0.3, dt=1e-7, gravity=0.0, damping=1.0,
                yield_strength=235e6, hardening=1e9, ramp_steps=0):
        """Mean device milliseconds per launch of (element kernel, node kernel)."""
        p = TetParamsC(youngs, poisson, yield_strength, hardening, dt, gravity, damping, int(ramp_steps))
        out = np.zeros(2)
        self._check(_tet_profile(self._h, int(steps), C.byref(p), _p(out)))
        return float(out[0]), float(out[1])

    @property
    def launches(self) -> int:
        return int(_tet_launches(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _tet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------
# Meshes: the numpy generators of meshes.py (which loads no native library),
# re-exported so callers of this binding find them here too.

from meshes import box_tet_mesh, csr, plate_mesh, plate_pressure_load, stiffened_panel  # noqa: E402,F401


# ---------------------------------------------------------------------------------
# Solid-shell zone: gpu::ZoneGpuSolver (engine/gpu/zone_gpu.hpp:179-234).

class ShellMeshC(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("elements", C.c_size_t), ("rest", C.c_void_p), ("position", C.c_void_p),
                ("velocity", C.c_void_p), ("index", C.c_void_p), ("pinned", C.c_void_p), ("load", C.c_void_p),
                ("forms", C.c_void_p), ("mass", C.c_void_p), ("state", C.c_void_p),
                ("adjacency_offset", C.c_void_p), ("adjacency_entry", C.c_void_p), ("density", C.c_double)]


class ShellMaterialC(C.Structure):
    """femstep_shell_material: the general point law (Swift or linear flow, kinematic
    hardening, ductile damage)."""
    _fields_ = [("hardening", C.c_int), ("strength_coefficient", C.c_double), ("reference_strain", C.c_double),
                ("hardening_exponent", C.c_double), ("kinematic_modulus", C.c_double),
                ("triaxiality_sensitivity", C.c_double), ("reference_triaxiality", C.c_double),
                ("cutoff_triaxiality", C.c_double)]


SHELL_LINEAR, SHELL_SWIFT = 0, 1


class ShellParamsC(C.Structure):
    _fields_ = [("youngs_modulus", C.c_double), ("poisson_ratio", C.c_double), ("yield_strength", C.c_double),
                ("hardening_modulus", C.c_double), ("dt", C.c_double), ("damping", C.c_double),
                ("rise_time", C.c_double), ("max_iterations", C.c_int), ("tol_residual", C.c_double),
                ("tol_work", C.c_double), ("compensated", C.c_int), ("material", C.c_void_p),
                ("eas_fp64", C.c_int)]


_sh_create = _sig("femstep_shell_create", C.c_int, [C.POINTER(ShellMeshC), C.POINTER(C.c_void_p)])
_sh_run = _sig("femstep_shell_run", C.c_int, [C.c_void_p, C.c_int, C.POINTER(ShellParamsC), C.POINTER(C.c_double)])
_sh_readback = _sig("femstep_shell_readback", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p])
_sh_state = _sig("femstep_shell_state", C.c_int, [C.c_void_p, C.c_void_p])
_sh_energy = _sig("femstep_shell_energy", C.c_int, [C.c_void_p, C.c_void_p])
_sh_stats = _sig("femstep_shell_stats", C.c_int, [C.c_void_p, C.c_void_p])
_sh_dt = _sig("femstep_shell_critical_dt", C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double,
                                                       C.POINTER(C.c_double)])
_sh_profile = _sig("femstep_shell_profile", C.c_int, [C.c_void_p, C.c_int, C.POINTER(ShellParamsC), C.c_void_p])
_sh_launches = _sig("femstep_shell_launches", C.c_longlong, [C.c_void_p])
_sh_bytes = _sig("femstep_shell_device_bytes", C.c_size_t, [C.c_void_p])
_sh_error = _sig("femstep_shell_error", C.c_char_p, [C.c_void_p])
_sh_destroy = _sig("femstep_shell_destroy", None, [C.c_void_p])
_sh_set_punch = _sig("femstep_shell_set_punch", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                                           C.c_double, C.c_double, C.c_double])
_sh_punch_state = _sig("femstep_shell_punch_state", C.c_int, [C.c_void_p, C.c_void_p])
_sh_set_edge = _sig("femstep_shell_set_edge", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double])
_sh_account = _sig("femstep_shell_account", C.c_int, [C.c_void_p, C.c_void_p])
class ShellFibersC(C.Structure):
    _fields_ = [("count", C.c_size_t), ("tie", C.c_void_p), ("weight", C.c_void_p), ("area", C.c_void_p),
                ("rest_length", C.c_void_p), ("failure_strain", C.c_void_p), ("density", C.c_double)]


_sh_set_fibers = _sig("femstep_shell_set_fibers", C.c_int, [C.c_void_p, C.POINTER(ShellFibersC)])
_sh_fiber_state = _sig("femstep_shell_fiber_state", C.c_int, [C.c_void_p, C.c_void_p])
_sh_ck_size = _sig("femstep_shell_checkpoint_size", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)])
_sh_ck = _sig("femstep_shell_checkpoint", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t])
_sh_restore = _sig("femstep_shell_restore", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t])
_sh_forms = _sig("femstep_shell_forms", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_double, C.c_double,
                                                    C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p])


class ShellSolver:
    """A solid-shell zone resident on the GPU; the reference's gpu::ZoneGpuSolver.

    rest/index are the HexMesh arrays (solid_shell.hpp:464-477); pinned is 3 flags per
    node; load is the full-amplitude external nodal force.  forms/mass/state may be
    handed over from a CPU zone::Solver, as ZoneGpuSolver::initialise does; otherwise
    the forms and the lumped mass are built on the device in FP64.
    """

    def __init__(self, rest, index, pinned=None, load=None, position=None, velocity=None, forms=None, mass=None,
                 state=None, adjacency_offset=None, adjacency_entry=None, density=7850.0):
        keep = {}

        def arr(name, a, dt):
            if a is None:
                return None
            keep[name] = np.ascontiguousarray(a, dt).reshape(-1)
            return keep[name]

        r = arr("rest", rest, np.float64)
        idx = arr("index", index, np.uint32)
        self.nodes = r.size // 3
        self.elements = idx.size // 8
        m = ShellMeshC()
        m.nodes, m.elements = self.nodes, self.elements
        m.rest = _p(r)
        m.position = _p(arr("position", position, np.float64))
        m.velocity = _p(arr("velocity", velocity, np.float64))
        m.index = _p(idx)
        m.pinned = _p(arr("pinned", pinned, np.uint8))
        m.load = _p(arr("load", load, np.float64))
        m.forms = _p(arr("forms", forms, np.float64))
        m.mass = _p(arr("mass", mass, np.float64))
        m.state = _p(arr("state", state, np.float64))
        m.adjacency_offset = _p(arr("adjacency_offset", adjacency_offset, np.uint32))
        m.adjacency_entry = _p(arr("adjacency_entry", adjacency_entry, np.uint32))
        m.density = float(density)
        h = C.c_void_p()
        rc = _sh_create(C.byref(m), C.byref(h))
        if rc:
            _raise(rc, _last_error())
        self._h = h

    def _check(self, rc):
        if rc:
            _raise(rc, _sh_error(self._h))

    def params(self, youngs=206e9, poisson=0.3, yield_strength=355e6, hardening=1e9, dt=1e-7, damping=1.0,
               rise_time=0.0, max_iterations=12, tol_residual=1e-12, tol_work=1e-16, compensated=True, material=None,
               eas_fp64=0):
        """eas_fp64: how much of the enhanced-strain block runs in FP64 (0-3, needs a material).
        material: None (the linear law) or a dict of femstep_shell_material fields
        (hardening=SHELL_SWIFT|SHELL_LINEAR, strength_coefficient, reference_strain,
        hardening_exponent, kinematic_modulus, triaxiality_sensitivity,
        reference_triaxiality, cutoff_triaxiality)."""
        p = ShellParamsC(youngs, poisson, yield_strength, hardening, dt, damping, rise_time, int(max_iterations),
                         tol_residual, tol_work, int(bool(compensated)), None, int(eas_fp64))
        if material is not None:
            m = dict(hardening=SHELL_LINEAR, strength_coefficient=0.0, reference_strain=0.0, hardening_exponent=1.0,
                     kinematic_modulus=0.0, triaxiality_sensitivity=1.5, reference_triaxiality=1.0 / 3.0,
                     cutoff_triaxiality=-1.0 / 3.0)
            m.update(material)
            self._material = ShellMaterialC(**m)  # kept alive while the handle may read it
            p.material = C.addressof(self._material)
        return p

    def run(self, substeps, **kw) -> float:
        p = self.params(**kw)
        ms = C.c_double()
        self._check(_sh_run(self._h, int(substeps), C.byref(p), C.byref(ms)))
        return ms.value

    def readback(self):
        p = np.zeros(3 * self.nodes)
        v = np.zeros(3 * self.nodes)
        self._check(_sh_readback(self._h, _p(p), _p(v)))
        return p, v

    def state(self):
        out = np.zeros(129 * self.elements)
        self._check(_sh_state(self._h, _p(out)))
        return out.reshape(self.elements, 129)

    def energy(self):
        """[external work, dissipation, strain energy, kinetic], FP64 on device."""
        out = np.zeros(4)
        self._check(_sh_energy(self._h, _p(out)))
        return out

    def set_punch(self, driven_nodes, axis, speed, ramp_time=0.0, mass=0.0):
        """The punch (zone.cpp:1147-1198).  mass 0: prescribed, each step the driven nodes
        move at -speed along `axis` (speed ramped over ramp_time seconds).  mass > 0: a
        striking body of that mass arriving at `speed`, which the plating decelerates."""
        dn = np.ascontiguousarray(driven_nodes, np.uint32)
        ax = np.ascontiguousarray(axis, np.float64)
        self._check(_sh_set_punch(self._h, _p(dn), dn.size, _p(ax), float(speed), float(ramp_time), float(mass)))

    def punch_state(self):
        """{work, penetration, time, steps} of the punch (ZoneGpuState)."""
        out = np.zeros(4)
        self._check(_sh_punch_state(self._h, _p(out)))
        return {"work": out[0], "penetration": out[1], "time": out[2], "steps": int(out[3])}

    def set_edge(self, prescribed, meshed=None, ramp=0.0):
        """The driven edge (zone.cpp:833-842, 1123-1145): every pinned DOF with a non-zero
        prescribed value follows meshed + prescribed * smoothstep(t / ramp)."""
        pr = np.ascontiguousarray(prescribed, np.float64).reshape(-1)
        me = None if meshed is None else np.ascontiguousarray(meshed, np.float64).reshape(-1)
        if pr.size != 3 * self.nodes or (me is not None and me.size != 3 * self.nodes):
            raise ValueError("prescribed and meshed are 3 values per node")
        self._check(_sh_set_edge(self._h, _p(pr), None if me is None else _p(me), float(ramp)))

    def set_fibers(self, tie, weight, area, rest_length=None, failure_strain=None, density=0.0):
        """Constraint fibres (constraint.hpp): tie [F][4] (end 0 bottom, top; end 1 bottom,
        top), weight [F][2], area [F]; rest length (None: from the rest positions) and
        failure strain (None: never) per fibre; density > 0 adds their lumped mass."""
        t = np.ascontiguousarray(tie, np.uint32).reshape(-1)
        w = np.ascontiguousarray(weight, np.float64).reshape(-1)
        a = np.ascontiguousarray(area, np.float64).reshape(-1)
        n = a.size
        if t.size != 4 * n or w.size != 2 * n:
            raise ValueError("tie is 4 and weight 2 values per fibre")
        ln = None if rest_length is None else np.ascontiguousarray(rest_length, np.float64).reshape(-1)
        fs = None if failure_strain is None else np.ascontiguousarray(failure_strain, np.float64).reshape(-1)
        self._fibers = (t, w, a, ln, fs)  # kept alive for the call
        f = ShellFibersC(n, _p(t), _p(w), _p(a), _p(ln), _p(fs), float(density))
        self._check(_sh_set_fibers(self._h, C.byref(f)))
        self.fibers = n

    def fiber_state(self) -> np.ndarray:
        """[F][4]: plastic strain, eq. plastic strain, damage, failed."""
        out = np.zeros(4 * getattr(self, "fibers", 0))
        if out.size:
            self._check(_sh_fiber_state(self._h, _p(out)))
        return out.reshape(-1, 4)

    def checkpoint(self) -> np.ndarray:
        """The whole mutable state as a host byte array (femstep_shell_checkpoint)."""
        n = C.c_size_t()
        self._check(_sh_ck_size(self._h, C.byref(n)))
        buf = np.zeros(n.value, np.uint8)
        self._check(_sh_ck(self._h, _p(buf), buf.size))
        return buf

    def restore(self, buf):
        """Continue from a checkpoint of a solver of the same mesh, punch and edge."""
        b = np.ascontiguousarray(buf, np.uint8)
        self._check(_sh_restore(self._h, _p(b), b.size))

    def account(self):
        """{damping_loss, boundary_work, punch_speed, striker_kinetic, arrested, edge_dof}."""
        out = np.zeros(6)
        self._check(_sh_account(self._h, _p(out)))
        return {"damping_loss": out[0], "boundary_work": out[1], "punch_speed": out[2], "striker_kinetic": out[3],
                "arrested": bool(out[4]), "edge_dof": int(out[5])}

    def stats(self):
        out = np.zeros(2, np.int64)
        self._check(_sh_stats(self._h, _p(out)))
        return {"nonconverged_element_steps": int(out[0]), "yielded_points": int(out[1])}

    def critical_dt(self, youngs=206e9, poisson=0.3, density=7850.0, safety=0.9) -> float:
        dt = C.c_double()
        self._check(_sh_dt(self._h, youngs, poisson, density, safety, C.byref(dt)))
        return dt.value

    def profile(self, steps, **kw):
        p = self.params(**kw)
        out = np.zeros(2)
        self._check(_sh_profile(self._h, int(steps), C.byref(p), _p(out)))
        return float(out[0]), float(out[1])

    @property
    def launches(self) -> int:
        return int(_sh_launches(self._h))

    @property
    def device_bytes(self) -> int:
        return int(_sh_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _sh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shell_forms(nodes, formulation=2, youngs=206e9, poisson=0.3, density=7850.0, safety=0.9):
    """Rest forms, lumped masses and element critical steps of standalone elements,
    formed on the device in FP64.  nodes: (E, 24)."""
    nodes = np.ascontiguousarray(nodes, np.float64).reshape(-1, 24)
    E = nodes.shape[0]
    forms = np.zeros((E, 1507))
    mass = np.zeros((E, 8))
    dt = np.zeros(E)
    rc = _sh_forms(_p(nodes), E, int(formulation), youngs, poisson, density, safety, _p(forms), _p(mass), _p(dt))
    if rc:
        _raise(rc, _last_error())
    return forms, mass, dt


# ---------------------------------------------------------------------------------
# Pool of many tet meshes: the batched and the served step (no reference counterpart:
# the reference steps one mesh at a time, fem.cpp:187).

POOL_AUTO, POOL_GRAPH, POOL_PERSISTENT, POOL_GRAPH_STAGED, POOL_GRAPH_TILED = 0, 1, 2, 3, 4
POOL_MODE_NAMES = {POOL_GRAPH: "graph", POOL_PERSISTENT: "persistent", POOL_GRAPH_STAGED: "graph-staged",
                   POOL_GRAPH_TILED: "graph-tiled"}


class PoolMeshC(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("tets", C.c_size_t), ("position", C.c_void_p), ("index", C.c_void_p),
                ("fixed", C.c_void_p), ("external_force", C.c_void_p), ("density", C.c_double),
                ("youngs_modulus", C.c_double), ("poisson_ratio", C.c_double), ("yield_strength", C.c_double),
                ("hardening_modulus", C.c_double), ("dt", C.c_double), ("gravity", C.c_double),
                ("damping", C.c_double), ("ramp_steps", C.c_int)]


_pl_create = _sig("femstep_pool_create", C.c_int, [C.c_size_t, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_void_p)])
_pl_bpt = _sig("femstep_pool_bytes_per_tet", C.c_size_t, [])
_pl_bpn = _sig("femstep_pool_bytes_per_node", C.c_size_t, [])
_pl_admit = _sig("femstep_pool_admit", C.c_int, [C.c_void_p, C.POINTER(PoolMeshC), C.c_longlong, C.POINTER(C.c_int)])
_pl_admit_many = _sig("femstep_pool_admit_many", C.c_int, [C.c_void_p, C.POINTER(PoolMeshC), C.c_void_p, C.c_int,
                                                           C.c_void_p, C.POINTER(C.c_int)])
_pl_release = _sig("femstep_pool_release", C.c_int, [C.c_void_p, C.c_int])
_pl_ck_size = _sig("femstep_pool_checkpoint_size", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)])
_pl_ck = _sig("femstep_pool_checkpoint", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t])
_pl_resume = _sig("femstep_pool_admit_resume", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p,
                                                          C.c_size_t, C.POINTER(C.c_int)])
_pl_run_async = _sig("femstep_pool_run_async", C.c_int, [C.c_void_p, C.c_int, C.c_int])
_pl_wait = _sig("femstep_pool_wait", C.c_int, [C.c_void_p, C.POINTER(C.c_double)])
_pl_prepare = _sig("femstep_pool_prepare", C.c_int, [C.c_void_p])
_pl_run = _sig("femstep_pool_run", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)])
_pl_finished = _sig("femstep_pool_finished", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)])
_pl_status = _sig("femstep_pool_status", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_longlong),
                                                     C.POINTER(C.c_longlong)])
_pl_readback = _sig("femstep_pool_readback", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p])
_pl_plastic = _sig("femstep_pool_plastic", C.c_int, [C.c_void_p, C.c_int, C.c_void_p])
_pl_readback_many = _sig("femstep_pool_readback_many", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                                                  C.c_void_p])
_pl_energy = _sig("femstep_pool_energy", C.c_int, [C.c_void_p, C.c_int, C.c_void_p])
_pl_dt = _sig("femstep_pool_dt", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)])
_pl_autotune = _sig("femstep_pool_autotune", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                                         C.POINTER(C.c_double)])
_pl_schedule = _sig("femstep_pool_set_schedule", C.c_int, [C.c_void_p, C.c_int, C.c_int])
_pl_profile = _sig("femstep_pool_profile", C.c_int, [C.c_void_p, C.c_int, C.c_void_p])
_pl_info = _sig("femstep_pool_info", C.c_int, [C.c_void_p, C.c_void_p])
_pl_error = _sig("femstep_pool_error", C.c_char_p, [C.c_void_p])
_pl_destroy = _sig("femstep_pool_destroy", None, [C.c_void_p])


def pool_bytes(tets: int, nodes: int) -> int:
    """Device bytes a pool of this capacity holds (without the small per-mesh tables)."""
    return int(_pl_bpt()) * int(tets) + int(_pl_bpn()) * int(nodes)


class PoolFull(FemStepError):
    """The mesh does not fit in the pool's free space now (FEMSTEP_ENOMEM on admit)."""


class TetPool:
    """Many J2 tet meshes resident on one GPU, stepped together (FP32, Kahan-compensated).

    Every mesh has its own material, load, time step and step count.  A mesh's
    displacement, velocity and plastic state are those of ``TetSolver(mode="f32k")``
    with the same dt, bit for bit, and do not depend on what else is in the pool.
    """

    def __init__(self, tet_capacity, node_capacity, max_meshes=1024, tile=256):
        h = C.c_void_p()
        rc = _pl_create(int(tet_capacity), int(node_capacity), int(max_meshes), int(tile), C.byref(h))
        if rc:
            _raise(rc, _last_error())
        self._h = h
        self.max_meshes = int(max_meshes)
        self.sizes = {}  # id -> (nodes, tets)

    @classmethod
    def for_budget(cls, budget_bytes, nodes_per_tet=0.25, max_meshes=1024, tile=256):
        """A pool whose arrays fill `budget_bytes` of device memory, with node capacity
        `nodes_per_tet` per tet (Kuhn box meshes have fewer than 1/4)."""
        per = int(_pl_bpt()) + nodes_per_tet * int(_pl_bpn())
        tets = min(int(budget_bytes // per), 1_000_000_000)
        return cls(tets, int(tets * nodes_per_tet) + max_meshes + 1, max_meshes=max_meshes, tile=tile)

    def _check(self, rc):
        if rc:
            text = _pl_error(self._h)
            if rc == ENOMEM:
                raise PoolFull(rc, (text or b"").decode(errors="replace"))
            _raise(rc, text)

    @staticmethod
    def _mesh(keep, position, index, fixed=None, external_force=None, density=7850.0, youngs=210e9, poisson=0.3,
              yield_strength=235e6, hardening=1e9, dt=0.0, gravity=0.0, damping=1.0, ramp_steps=0):
        pos = np.ascontiguousarray(position, np.float32).reshape(-1)
        idx = np.ascontiguousarray(index, np.uint32).reshape(-1)
        fx = None if fixed is None else np.ascontiguousarray(fixed, np.uint32).reshape(-1)
        fe = None if external_force is None else np.ascontiguousarray(external_force, np.float64).reshape(-1)
        keep.extend([pos, idx, fx, fe])
        return PoolMeshC(pos.size // 3, idx.size // 4, _p(pos), _p(idx), _p(fx), _p(fe), density, youngs, poisson,
                         yield_strength, hardening, dt, gravity, damping, int(ramp_steps))

    def admit(self, steps, **mesh) -> int:
        """Admit a mesh for `steps` steps; raises PoolFull when it does not fit now.
        mesh: position, index, fixed, external_force, density, youngs, poisson,
        yield_strength, hardening, dt (0: the device bound), gravity, damping, ramp_steps."""
        keep = []
        m = self._mesh(keep, **mesh)
        out = C.c_int()
        self._check(_pl_admit(self._h, C.byref(m), int(steps), C.byref(out)))
        self.sizes[out.value] = (m.nodes, m.tets)
        return out.value

    def admit_many(self, meshes, steps):
        """Admit meshes (keyword dicts as for admit) in order while they fit; their host
        work runs on all host cores.  Returns the ids of the admitted prefix."""
        keep = []
        arr = (PoolMeshC * max(1, len(meshes)))(*[self._mesh(keep, **m) for m in meshes])
        st = np.ascontiguousarray(steps, np.int64)
        ids = np.zeros(max(1, len(meshes)), np.int32)
        n = C.c_int()
        rc = _pl_admit_many(self._h, arr, _p(st), len(meshes), _p(ids), C.byref(n))
        if rc and rc != ENOMEM:
            self._check(rc)
        out = [int(i) for i in ids[: n.value]]
        for k, i in enumerate(out):
            self.sizes[i] = (arr[k].nodes, arr[k].tets)
        return out

    def release(self, mesh_id):
        self._check(_pl_release(self._h, int(mesh_id)))
        self.sizes.pop(mesh_id, None)

    def checkpoint(self, mesh_id) -> np.ndarray:
        """One mesh's whole mutable state as a host byte array (for eviction)."""
        n = C.c_size_t()
        self._check(_pl_ck_size(self._h, int(mesh_id), C.byref(n)))
        buf = np.zeros(n.value, np.uint8)
        self._check(_pl_ck(self._h, int(mesh_id), _p(buf), buf.size))
        return buf

    def admit_resume(self, checkpoint, steps, **mesh) -> int:
        """Admit the mesh of `checkpoint` again and continue from it, up to `steps` in
        total; raises PoolFull when it does not fit now."""
        keep = []
        m = self._mesh(keep, **mesh)
        b = np.ascontiguousarray(checkpoint, np.uint8)
        out = C.c_int()
        self._check(_pl_resume(self._h, C.byref(m), int(steps), _p(b), b.size, C.byref(out)))
        self.sizes[out.value] = (m.nodes, m.tets)
        return out.value

    def run(self, steps, mode=POOL_AUTO) -> float:
        ms = C.c_double()
        self._check(_pl_run(self._h, int(steps), int(mode), C.byref(ms)))
        return ms.value

    def run_async(self, steps, mode=POOL_AUTO):
        self._check(_pl_run_async(self._h, int(steps), int(mode)))

    def prepare(self):
        """Upload the work list and capture the schedule's graph without stepping."""
        self._check(_pl_prepare(self._h))

    def wait(self) -> float:
        ms = C.c_double()
        self._check(_pl_wait(self._h, C.byref(ms)))
        return ms.value

    def finished(self):
        ids = np.zeros(self.max_meshes, np.int32)
        n = C.c_int()
        self._check(_pl_finished(self._h, _p(ids), self.max_meshes, C.byref(n)))
        return [int(i) for i in ids[: min(n.value, self.max_meshes)]]

    def status(self, mesh_id):
        done, target = C.c_longlong(), C.c_longlong()
        self._check(_pl_status(self._h, int(mesh_id), C.byref(done), C.byref(target)))
        return done.value, target.value

    def readback(self, mesh_id):
        n = self.sizes[mesh_id][0]
        p = np.zeros(3 * n)
        v = np.zeros(3 * n)
        self._check(_pl_readback(self._h, int(mesh_id), _p(p), _p(v)))
        return p, v

    def readback_many(self, mesh_ids):
        """[(positions, velocities)] of several meshes in one call (3N doubles each)."""
        ids = np.ascontiguousarray(mesh_ids, np.int32)
        outs = [(np.zeros(3 * self.sizes[int(i)][0]), np.zeros(3 * self.sizes[int(i)][0])) for i in ids]
        pp = (C.c_void_p * max(len(outs), 1))(*[o[0].ctypes.data for o in outs])
        vp = (C.c_void_p * max(len(outs), 1))(*[o[1].ctypes.data for o in outs])
        self._check(_pl_readback_many(self._h, ids.size, _p(ids), C.cast(pp, C.c_void_p), C.cast(vp, C.c_void_p)))
        return outs

    def plastic(self, mesh_id):
        t = self.sizes[mesh_id][1]
        out = np.zeros(7 * t)
        self._check(_pl_plastic(self._h, int(mesh_id), _p(out)))
        return out.reshape(t, 7)

    def energy(self, mesh_id):
        """[external work (load + gravity), dissipation, strain energy, kinetic] (FP64)."""
        out = np.zeros(4)
        self._check(_pl_energy(self._h, int(mesh_id), _p(out)))
        return out

    def dt(self, mesh_id) -> float:
        v = C.c_double()
        self._check(_pl_dt(self._h, int(mesh_id), C.byref(v)))
        return v.value

    def autotune(self, steps=32):
        tile, mode, ms = C.c_int(), C.c_int(), C.c_double()
        self._check(_pl_autotune(self._h, int(steps), C.byref(tile), C.byref(mode), C.byref(ms)))
        return {"tile": tile.value, "mode": POOL_MODE_NAMES[mode.value], "ms_per_step": ms.value}

    def set_schedule(self, tile, mode):
        self._check(_pl_schedule(self._h, int(tile), int(mode)))

    def profile(self, steps=5):
        """Mean device milliseconds per launch of (element pass, node pass)."""
        out = np.zeros(2)
        self._check(_pl_profile(self._h, int(steps), _p(out)))
        return float(out[0]), float(out[1])

    def info(self):
        out = np.zeros(8, np.int64)
        self._check(_pl_info(self._h, _p(out)))
        keys = ("tets", "nodes", "meshes", "tile", "mode", "launches", "device_bytes", "staging_buffers")
        return dict(zip(keys, (int(x) for x in out)))

    def close(self):
        if getattr(self, "_h", None):
            _pl_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
