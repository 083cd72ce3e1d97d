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
# Meshes.  Vectorised restatements of the reference generators, so workloads of
# millions of elements are built in milliseconds; tests pin them to the reference's.

_KUHN = np.array([[0, 1, 3, 7], [0, 1, 7, 5], [0, 5, 7, 4], [0, 3, 2, 7], [0, 2, 6, 7], [0, 4, 6, 7]])


def box_tet_mesh(lx, ly, lz, nx, ny, nz):
    """fem::makeBoxTetMesh (engine/sim/fem.cpp:217-263): node (k*sy+j)*sx+i, six Kuhn
    tets per cell about the 0-7 diagonal, orientation fixed by swapping corners 1, 2."""
    sx, sy, sz = nx + 1, ny + 1, nz + 1
    k, j, i = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx), indexing="ij")
    pos = np.empty((sz, sy, sx, 3), np.float32)
    pos[..., 0] = np.float32(lx) * i.astype(np.float32) / np.float32(nx)
    pos[..., 1] = np.float32(ly) * j.astype(np.float32) / np.float32(ny)
    pos[..., 2] = np.float32(lz) * k.astype(np.float32) / np.float32(nz)
    pos = pos.reshape(-1)
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ci, cj, ck = ci.reshape(-1), cj.reshape(-1), ck.reshape(-1)
    corner = np.empty((ci.size, 8), np.uint32)
    for c in range(8):
        corner[:, c] = ((ck + ((c >> 2) & 1)) * sy + (cj + ((c >> 1) & 1))) * sx + (ci + (c & 1))
    tets = corner[:, _KUHN].reshape(-1, 4)  # cell-major, six per cell
    p = pos.reshape(-1, 3)
    d = p[tets[:, 1:]] - p[tets[:, :1]]          # (T, 3 edges, 3 axes)
    # determinant in float with fem.cpp's cofactor order (columns = edges)
    a = np.transpose(d, (0, 2, 1))              # a[t, row(axis), col(edge)]
    det = (a[:, 0, 0] * (a[:, 1, 1] * a[:, 2, 2] - a[:, 1, 2] * a[:, 2, 1])
           - a[:, 0, 1] * (a[:, 1, 0] * a[:, 2, 2] - a[:, 1, 2] * a[:, 2, 0])
           + a[:, 0, 2] * (a[:, 1, 0] * a[:, 2, 1] - a[:, 1, 1] * a[:, 2, 0]))
    flip = det < 0
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    return pos, tets.reshape(-1).astype(np.uint32)


def csr(nodes, index, corners):
    """Node -> corner CSR by counting sort (fem.cpp:147-157, zone.cpp:739-754)."""
    index = np.asarray(index, np.int64).reshape(-1)
    counts = np.bincount(index, minlength=nodes)
    offset = np.zeros(nodes + 1, np.uint32)
    offset[1:] = np.cumsum(counts)
    entry = np.argsort(index, kind="stable").astype(np.uint32)
    return offset, entry
