"""femstep_tet_step_noalloc: the tet step for callers that cannot allocate.

Some callers own every byte of device memory -- an engine or plugin with its own
allocator or a fixed memory budget -- and so cannot let the library cudaMalloc the
mesh copy and the force scratch that femstep_tet_create makes.  This entry point takes
the caller's device arrays and keeps its scratch in a fixed array inside the library.
The test gives it device arrays allocated by the caller (here through torch), steps
them through the C ABI twice in a row, and checks each result against the allocating
entry point on the same mesh: the two must agree to the last bit, the tolerance the
REF32 tests use.  Further cases: a mesh at the size limit (65,536 tets, many blocks)
followed by a second, smaller mesh on the same stream; sizes and parameters the entry
point must refuse; and a caller that runs under its own CUDA context, which needs the
scratch's address in that context rather than the one the library saw first.  It
lives in its own file, collected last, so that a failure here stops a `-x` run only
after every other test has run.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


class DeviceMesh(C.Structure):
    _fields_ = [("nodes", C.c_size_t), ("tets", C.c_size_t), ("position", C.c_void_p), ("velocity", C.c_void_p),
                ("mass", C.c_void_p), ("fixed", C.c_void_p), ("index", C.c_void_p), ("rest_inv", C.c_void_p),
                ("rest_volume", C.c_void_p), ("adjacency_offset", C.c_void_p), ("adjacency_entry", C.c_void_p)]


def bind(fem):
    step = fem.lib.femstep_tet_step_noalloc
    step.restype = C.c_int
    step.argtypes = [C.POINTER(DeviceMesh), C.c_int, C.POINTER(fem.TetParamsC), C.c_void_p]
    return step


def limit_mesh():
    """A box mesh cut to exactly 65,536 tets (the entry point's limit).  Nodes the cut
    leaves without a tet have no mass and are held fixed."""
    import meshes as M
    import oracle as O

    pos, idx = M.box_tet_mesh(0.43, 0.16, 0.16, 43, 16, 16)
    idx = idx[:65536 * 4]
    m = O.TetMesh32(O.Oracle("port"), pos, idx)
    used = np.zeros(m.nodes, bool)
    used[idx] = True
    m.fixed[:] = ((pos[0::3] < 1e-6) | ~used).astype(np.uint32)
    m.rest_state(210e9, 0.3, 7850.0)
    # a bent start, so the step has forces to gather
    x = pos[0::3].astype(np.float64)
    start = pos.copy()
    start[2::3] += (1e-3 * (x / 0.43) ** 2).astype(np.float32)
    return dict(start=start, index=idx, mass=m.mass, fixed=m.fixed, rest_inv=m.rest_inv,
                rest_volume=m.rest_volume, adj_offset=m.adj_offset, adj_entry=m.adj_entry)


def upload(torch, dev, g):
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
    return m, pos, vel, keep


def allocating(fem, g):
    return fem.TetSolver(g["start"], g["index"], mode="ref32", mass=g["mass"], fixed=g["fixed"],
                         rest_inv=g["rest_inv"], rest_volume=g["rest_volume"], adjacency_offset=g["adj_offset"],
                         adjacency_entry=g["adj_entry"])


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


def test_noalloc_at_the_size_limit_then_a_second_mesh(fem):
    """65,536 tets (256 blocks per launch), then the small spike mesh on the same
    stream: each bit-identical to the allocating step, two calls each."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    step = bind(fem)
    spike = dict(np.load(os.path.join(GOLDEN, "tet32_spike.npz")))
    for g, dt in ((limit_mesh(), 2e-7), (spike, float(spike["dt"]))):
        m, pos, vel, keep = upload(torch, dev, g)
        assert m.tets <= 65536
        params = fem.TetParamsC(210e9, 0.3, 0.0, 0.0, dt, 9.80665, 1.0, 0)
        ref = allocating(fem, g)
        for steps in (7, 20):
            assert step(C.byref(m), steps, C.byref(params), C.c_void_p(stream.cuda_stream)) == 0, \
                fem.lib.femstep_last_error()
            torch.cuda.synchronize(dev)
            ref.run(steps, youngs=210e9, poisson=0.3, dt=dt, gravity=9.80665, damping=1.0)
            p_ref, v_ref = ref.readback()
            assert np.array_equal(pos.cpu().numpy(), p_ref), (m.tets, steps)
            assert np.array_equal(vel.cpu().numpy(), v_ref), (m.tets, steps)
            assert np.abs(v_ref).max() > 0
        ref.close()


# Run in a child process: a context of the caller's own, made with the driver API on
# device 0, with the mesh in that context's memory.  The entry point must look its
# scratch up again there, and again when the library's own context is current once
# more.  Each result is checked against the allocating step.
CONTEXT_SCRIPT = r"""
import ctypes as C, os, sys
import numpy as np
sys.path[:0] = [os.path.join(ROOT, "sinking-simulator_b200"), os.path.join(ROOT, "tests")]
import femstep as fem
from test_zz_no_alloc import DeviceMesh, bind, GOLDEN
g = dict(np.load(os.path.join(GOLDEN, "tet32_spike.npz")))
dt = float(g["dt"])
params = fem.TetParamsC(210e9, 0.3, 0.0, 0.0, dt, 9.80665, 1.0, 0)
step = bind(fem)
ref = fem.TetSolver(g["start"], g["index"], mode="ref32", mass=g["mass"], fixed=g["fixed"],
                    rest_inv=g["rest_inv"], rest_volume=g["rest_volume"], adjacency_offset=g["adj_offset"],
                    adjacency_entry=g["adj_entry"])
cu = C.CDLL("libcuda.so.1")
def ok(rc, what):
    assert rc == 0, (what, rc)
ok(cu.cuInit(0), "cuInit")
dev = C.c_int()
ok(cu.cuDeviceGet(C.byref(dev), 0), "cuDeviceGet")
cu.cuMemAlloc_v2.argtypes = [C.POINTER(C.c_uint64), C.c_size_t]
cu.cuMemcpyHtoD_v2.argtypes = [C.c_uint64, C.c_void_p, C.c_size_t]
cu.cuMemcpyDtoH_v2.argtypes = [C.c_void_p, C.c_uint64, C.c_size_t]
cu.cuMemFree_v2.argtypes = [C.c_uint64]
def put(a):
    a = np.ascontiguousarray(a)
    d = C.c_uint64()
    ok(cu.cuMemAlloc_v2(C.byref(d), a.nbytes), "cuMemAlloc")
    ok(cu.cuMemcpyHtoD_v2(d.value, a.ctypes.data, a.nbytes), "cuMemcpyHtoD")
    return d.value
def get(d, like):
    out = np.empty_like(like)
    ok(cu.cuMemcpyDtoH_v2(out.ctypes.data, d, out.nbytes), "cuMemcpyDtoH")
    return out
def run_in_current_context(steps, state):
    start, vel0 = state
    arrays = [put(start.astype(np.float32)), put(vel0.astype(np.float32)), put(g["mass"].astype(np.float32)),
              put(g["fixed"].astype(np.uint32)), put(g["index"].astype(np.uint32)),
              put(g["rest_inv"].astype(np.float32)), put(g["rest_volume"].astype(np.float32)),
              put(g["adj_offset"].astype(np.uint32)), put(g["adj_entry"].astype(np.uint32))]
    m = DeviceMesh()
    m.nodes, m.tets = start.size // 3, g["index"].size // 4
    (m.position, m.velocity, m.mass, m.fixed, m.index, m.rest_inv, m.rest_volume, m.adjacency_offset,
     m.adjacency_entry) = arrays
    assert step(C.byref(m), steps, C.byref(params), None) == 0, fem.lib.femstep_last_error()
    ok(cu.cuCtxSynchronize(), "cuCtxSynchronize")
    out = get(arrays[0], start.astype(np.float32)), get(arrays[1], start.astype(np.float32))
    for a in arrays:
        ok(cu.cuMemFree_v2(a), "cuMemFree")
    return out
state = (g["start"].astype(np.float32), np.zeros(g["start"].size, np.float32))
# 1: the library's own (primary) context, current after the allocating handle's set-up
state = run_in_current_context(10, state)
ref.run(10, youngs=210e9, poisson=0.3, dt=dt, gravity=9.80665, damping=1.0)
assert all(np.array_equal(a, b) for a, b in zip(state, ref.readback())), "primary context"
# 2: a context of the caller's own, current while the entry point runs; the allocating
# handle lives in the library's context, so that one is current again for it
ctx = C.c_void_p()
ok(cu.cuCtxCreate_v2(C.byref(ctx), 0, dev), "cuCtxCreate")
state = run_in_current_context(10, state)
old = C.c_void_p()
ok(cu.cuCtxPopCurrent_v2(C.byref(old)), "cuCtxPopCurrent")
assert old.value == ctx.value
ref.run(10, youngs=210e9, poisson=0.3, dt=dt, gravity=9.80665, damping=1.0)
assert all(np.array_equal(a, b) for a, b in zip(state, ref.readback())), "caller's context"
# 3: back in the primary context
state = run_in_current_context(10, state)
ok(cu.cuCtxDestroy_v2(ctx), "cuCtxDestroy")
ref.run(10, youngs=210e9, poisson=0.3, dt=dt, gravity=9.80665, damping=1.0)
assert all(np.array_equal(a, b) for a, b in zip(state, ref.readback())), "primary context again"
ref.close()
print("contexts ok")
"""


def test_noalloc_in_a_context_of_the_callers_own():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", f"ROOT = {root!r}\n" + CONTEXT_SCRIPT], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and "contexts ok" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]


def test_noalloc_refuses_plastic_and_ramped_parameters(fem):
    torch = pytest.importorskip("torch")
    g = dict(np.load(os.path.join(GOLDEN, "tet32_spike.npz")))
    m, pos, vel, keep = upload(torch, torch.device("cuda", 0), g)
    step = bind(fem)
    before = pos.cpu().numpy()
    for bad in (fem.TetParamsC(210e9, 0.3, 235e6, 0.0, 1e-7, 0.0, 1.0, 0),
                fem.TetParamsC(210e9, 0.3, 0.0, 1e9, 1e-7, 0.0, 1.0, 0),
                fem.TetParamsC(210e9, 0.3, 0.0, 0.0, 1e-7, 0.0, 1.0, 100)):
        assert step(C.byref(m), 1, C.byref(bad), None) == fem.EINVAL
        assert b"elastic" in fem.lib.femstep_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(pos.cpu().numpy(), before)


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
