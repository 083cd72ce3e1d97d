"""femstep_tet_step_noalloc: the tet step for callers that cannot allocate.

Some callers own every byte of device memory -- an engine or plugin with its own
allocator or a fixed memory budget -- and so cannot let the library cudaMalloc the
mesh copy and the force scratch that femstep_tet_create makes.  This entry point takes
the caller's device arrays and keeps its scratch in a fixed array inside the library.
The test gives it device arrays allocated by the caller (here through torch), steps
them through the C ABI twice in a row, and checks each result against the allocating
entry point on the same mesh: the two must agree to the last bit, the tolerance the
REF32 tests use.  It lives in its own file, collected last, so that a failure here
stops a `-x` run only after every other test has run.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


class DeviceMesh(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("tets", C.c_size_t), ("position", C.c_void_p), ("velocity", C.c_void_p),
                ("mass", C.c_void_p), ("fixed", C.c_void_p), ("index", C.c_void_p), ("rest_inv", C.c_void_p),
                ("rest_volume", C.c_void_p), ("adjacency_offset", C.c_void_p), ("adjacency_entry", C.c_void_p)]


def test_noalloc_step_matches_allocating_step(fem):
    torch = pytest.importorskip("torch")
    g = np.load(os.path.join(GOLDEN, "tet32_spike.npz"))
    dt = float(g["dt"])
    dev = torch.device("cuda", 0)

    def put(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a).astype(dtype).view(np.int32 if dtype == np.uint32 else dtype)
                                ).to(dev)

    pos = put(g["start"], np.float32)
    vel = torch.zeros_like(pos)
    keep = [put(g["mass"], np.float32), put(g["fixed"], np.uint32), put(g["index"], np.uint32),
            put(g["rest_inv"], np.float32), put(g["rest_volume"], np.float32), put(g["adj_offset"], np.uint32),
            put(g["adj_entry"], np.uint32)]
    m = DeviceMesh()
    m.nodes, m.tets = g["start"].size // 3, g["index"].size // 4
    m.position, m.velocity = pos.data_ptr(), vel.data_ptr()
    (m.mass, m.fixed, m.index, m.rest_inv, m.rest_volume, m.adjacency_offset,
     m.adjacency_entry) = [t.data_ptr() for t in keep]
    step = fem.lib.femstep_tet_step_noalloc
    step.restype = C.c_int
    step.argtypes = [C.POINTER(DeviceMesh), C.c_int, C.POINTER(fem.TetParamsC), C.c_void_p]
    params = fem.TetParamsC(210e9, 0.3, 0.0, 0.0, dt, 9.80665, 1.0, 0)

    ref = fem.TetSolver(g["start"], g["index"], mode="ref32", mass=g["mass"], fixed=g["fixed"],
                        rest_inv=g["rest_inv"], rest_volume=g["rest_volume"], adjacency_offset=g["adj_offset"],
                        adjacency_entry=g["adj_entry"])
    stream = torch.cuda.current_stream(dev)
    for calls, steps in enumerate((10, 37), start=1):
        rc = step(C.byref(m), steps, C.byref(params), C.c_void_p(stream.cuda_stream))
        assert rc == 0, fem.lib.femstep_last_error()
        torch.cuda.synchronize(dev)
        ref.run(steps, youngs=210e9, poisson=0.3, dt=dt, gravity=9.80665, damping=1.0)
        p_ref, v_ref = ref.readback()
        assert np.array_equal(pos.cpu().numpy(), p_ref), calls
        assert np.array_equal(vel.cpu().numpy(), v_ref), calls
    # the first pin: after 10 steps the no-allocation path also equals the reference CPU
    # golden vector (checked above through the allocating path, which equals it)


def test_noalloc_rejects_oversize_meshes(fem):
    torch = pytest.importorskip("torch")
    m = DeviceMesh()
    m.nodes, m.tets = 10, 65537
    buf = torch.zeros(16, device="cuda")
    for name in ("position", "velocity", "mass", "index", "rest_inv", "rest_volume", "adjacency_offset",
                 "adjacency_entry"):
        setattr(m, name, buf.data_ptr())
    step = fem.lib.femstep_tet_step_noalloc
    step.restype = C.c_int
    step.argtypes = [C.POINTER(DeviceMesh), C.c_int, C.POINTER(fem.TetParamsC), C.c_void_p]
    params = fem.TetParamsC(210e9, 0.3, 0.0, 0.0, 1e-7, 0.0, 1.0, 0)
    assert step(C.byref(m), 1, C.byref(params), None) == fem.EINVAL
    assert b"65536" in fem.lib.femstep_last_error()
