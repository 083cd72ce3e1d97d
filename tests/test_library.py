"""The C-ABI library, without a GPU: it loads, exports what include/femstep.h
declares, validates meshes on the host, and reports a missing device as a skip."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "femstep.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(femstep_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(fem):
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(fem.lib, name), name


def test_binding_constants_match_the_header(fem):
    """The status codes and the pool's schedule codes the Python binding passes through
    the C ABI are the header's own values."""
    text = open(HEADER).read()
    defines = {k: int(v) for k, v in re.findall(r"#define\s+(FEMSTEP_[A-Z0-9_]+)\s+(-?\d+)", text)}
    pairs = {"FEMSTEP_POOL_AUTO": fem.POOL_AUTO, "FEMSTEP_POOL_GRAPH": fem.POOL_GRAPH,
             "FEMSTEP_POOL_PERSISTENT": fem.POOL_PERSISTENT, "FEMSTEP_POOL_GRAPH_STAGED": fem.POOL_GRAPH_STAGED,
             "FEMSTEP_POOL_GRAPH_TILED": fem.POOL_GRAPH_TILED, "FEMSTEP_OK": fem.OK, "FEMSTEP_SKIP": fem.SKIP,
             "FEMSTEP_EINVAL": fem.EINVAL, "FEMSTEP_ENOMEM": fem.ENOMEM, "FEMSTEP_ECUDA": fem.ECUDA,
             "FEMSTEP_ESTATE": fem.ESTATE, "FEMSTEP_ETIMEOUT": fem.ETIMEOUT}
    for name, value in pairs.items():
        assert defines.get(name) == value, (name, defines.get(name), value)
    assert set(fem.POOL_MODE_NAMES) == {fem.POOL_GRAPH, fem.POOL_PERSISTENT, fem.POOL_GRAPH_STAGED,
                                        fem.POOL_GRAPH_TILED}


def _has_gpu(fem):
    buf = C.create_string_buffer(64)
    return fem.lib.femstep_device_name(buf, 64) == 0


def test_no_device_is_a_skip(fem):
    if _has_gpu(fem):
        pytest.skip("a GPU is present")
    pos, idx = fem.box_tet_mesh(0.4, 0.1, 0.02, 4, 2, 2)
    with pytest.raises(fem.NoDevice):
        fem.TetSolver(pos, idx, mode="f32k", density=7850.0)


def test_bad_meshes_are_rejected_on_the_host(fem):
    pos, idx = fem.box_tet_mesh(0.4, 0.1, 0.02, 4, 2, 2)
    bad = idx.copy()
    bad[5] = pos.size // 3 + 7
    with pytest.raises(fem.FemStepError) as e:
        fem.TetSolver(pos, bad, mode="f32k", density=7850.0)
    assert e.value.code == fem.EINVAL
    with pytest.raises(fem.FemStepError) as e:
        fem.TetSolver(pos, idx, mode="f32k", density=0.0)
    assert e.value.code == fem.EINVAL
    off, ent = fem.csr(pos.size // 3, idx, 4)
    ent2 = ent.copy()
    ent2[0], ent2[-1] = ent2[-1], ent2[0]  # a corner of the last node filed under node 0
    with pytest.raises(fem.FemStepError) as e:
        fem.TetSolver(pos, idx, mode="f32k", density=7850.0, adjacency_offset=off, adjacency_entry=ent2)
    assert e.value.code == fem.EINVAL
    with pytest.raises(fem.FemStepError) as e:
        fem.TetSolver(pos, idx, mode="ref32")
    assert e.value.code == fem.EINVAL


def test_mesher_matches_reference_generator(fem, port):
    import oracle as O

    for dims in ((1.0, 0.1, 0.1, 40, 4, 4), (2.0, 0.5, 0.05, 20, 4, 2), (0.3, 0.2, 0.1, 3, 5, 2)):
        a = fem.box_tet_mesh(*dims)
        b = O.box_tet_mesh(port, *dims)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        m = O.TetMesh32(port, b[0], b[1])
        m.rest_state(210e9, 0.3, 7850.0)
        off, ent = fem.csr(m.nodes, a[1], 4)
        assert np.array_equal(off, m.adj_offset) and np.array_equal(ent, m.adj_entry)


def test_plate_mesher_matches_reference_generator(fem, port):
    import oracle as O

    for dims in ((0.06, 0.04, 0.012, 6, 4, 1), (1.0, 0.5, 0.02, 3, 5, 2)):
        a = fem.plate_mesh(*dims)
        b = O.plate_mesh(port, *dims)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        load = fem.plate_pressure_load(a[0], a[1], 2.5e5)
        if dims[-1] == 1:
            ref = np.zeros(a[0].size)
            port.plate_pressure_load(b[0], b[1], b[0].size // 3, b[1].size // 8, 2.5e5, ref)
            assert np.allclose(load, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_workload_builders_load_no_gpu_library():
    """The workload generators and the oracle's batch (the CPU baselines' inputs) never
    load libfemstep.so, so the reference arm of the benchmark runs without it."""
    import subprocess
    import sys

    code = ("import sys; sys.path[:0] = [%r, %r, %r]\n"
            "import workloads as W, meshes, oracle\n"
            "b = W.build(W.batch_meshes(3)[0]); meshes.stiffened_panel(nx=4, ny=3, lx=0.04, ly=0.03)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'femstep' not in sys.modules and 'libfemstep' not in maps\n"
            "print('clean')\n") % (os.path.join(ROOT, "sinking-simulator_b200"), os.path.join(ROOT, "oracle"), ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "clean" in r.stdout, r.stderr
