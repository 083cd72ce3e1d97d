"""The multi-mesh pool (batched and served step) on the GPU, through the C ABI.

A pool mesh runs the J2_F32K tet arithmetic: its displacement, velocity and plastic
state must be bit-identical to a single-mesh FEMSTEP_TET_J2_F32K handle given the same
time step, whatever else is in the pool, whichever schedule (graph or persistent) and
tile size runs it, and whenever it was admitted.  Against the FP64 oracle (the
reference's tet kinematics with plasticity::update, in double) each mesh keeps the
target tolerance: 1e-5 relative displacement and energy within 0.5 %.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def beam(fem, nx, ny, nz, length=1.0, load=100e3, clamp_end=0):
    pos, idx = fem.box_tet_mesh(length, 0.1, 0.1, nx, ny, nz)
    x = pos[0::3]
    fixed = ((x < 1e-6) if clamp_end == 0 else (x > length - 1e-6)).astype(np.uint32)
    tip = (x > length - 1e-6) if clamp_end == 0 else (x < 1e-6)
    fext = np.zeros(pos.size)
    fext[2::3][tip] = -load / tip.sum()
    return dict(position=pos, index=idx, fixed=fixed, external_force=fext)


MATS = [dict(yield_strength=235e6, hardening=1e9), dict(yield_strength=355e6, hardening=0.5e9),
        dict(yield_strength=300e6, hardening=2e9)]


def crit(fem, mesh):
    """0.9 x the FP64 element bound of the mesh (what the single-mesh handle reports)."""
    s = fem.TetSolver(mesh["position"], mesh["index"], mode="f32k", fixed=mesh["fixed"], density=7850.0)
    dt = s.critical_dt(210e9, 0.3, 7850.0, 0.9)
    s.close()
    return dt


def single(fem, mesh, steps, dt, mat, ramp):
    s = fem.TetSolver(mesh["position"], mesh["index"], mode="f32k", fixed=mesh["fixed"],
                      external_force=mesh["external_force"], density=7850.0)
    s.run(steps, dt=dt, ramp_steps=ramp, **mat)
    p, v = s.readback64()
    out = (p, v, s.plastic())
    s.close()
    return out


def test_pool_mesh_bit_identical_to_single_mesh_step(fem):
    meshes = [beam(fem, 24, 3, 3, load=300e3), beam(fem, 10, 2, 2, length=0.5, load=200e3, clamp_end=1),
              beam(fem, 40, 4, 4, load=250e3)]
    dts = [crit(fem, m) for m in meshes]
    steps = [1200, 937, 1201]
    for mode in (fem.POOL_GRAPH, fem.POOL_PERSISTENT, fem.POOL_GRAPH_STAGED):
        pool = fem.TetPool(200000, 50000, max_meshes=8)
        ids = [pool.admit(steps=steps[k], dt=dts[k], ramp_steps=400, **MATS[k], **meshes[k]) for k in range(3)]
        # uneven chunks, more steps than some meshes want
        for chunk in (17, 100, 5, 200, 900):
            pool.run(chunk, mode)
        for k, i in enumerate(ids):
            assert pool.status(i) == (steps[k], steps[k])
            p, v = pool.readback(i)
            pe, ve, ple = single(fem, meshes[k], steps[k], dts[k], MATS[k], 400)
            assert np.array_equal(p, pe), (mode, k)
            assert np.array_equal(v, ve), (mode, k)
            assert np.array_equal(pool.plastic(i), ple), (mode, k)
            assert (ple[:, 6] > 0).any(), "the case must exercise plasticity"
        assert sorted(pool.finished()) == sorted(ids)
        pool.close()


def test_result_is_the_same_alone_and_in_the_mix(fem):
    """A mesh admitted into a busy pool mid-run, next to meshes at other steps, gets the
    same bits (state and FP64 energy account) as when it runs alone."""
    a = beam(fem, 30, 3, 3, load=400e3)
    others = [beam(fem, 16, 2, 2, load=80e3), beam(fem, 50, 4, 4, length=2.0, load=120e3)]
    alone = fem.TetPool(100000, 30000, max_meshes=4)
    ia = alone.admit(steps=1500, ramp_steps=500, **MATS[0], **a)  # dt: the device bound
    alone.run(1500)
    pa, va = alone.readback(ia)
    ea = alone.energy(ia)
    assert (alone.plastic(ia)[:, 6] > 0).mean() > 0.05, "the case must exercise plasticity"

    mix = fem.TetPool(300000, 90000, max_meshes=8)
    j0 = mix.admit(steps=3000, ramp_steps=300, **MATS[1], **others[0])
    mix.run(37)
    j1 = mix.admit(steps=3000, ramp_steps=300, **MATS[2], **others[1])
    mix.run(50, fem.POOL_PERSISTENT)
    ib = mix.admit(steps=1500, ramp_steps=500, **MATS[0], **a)  # mid-run
    assert mix.dt(ib) == alone.dt(ia)
    for k, chunk in enumerate((3, 64, 200, 133, 1100)):
        mix.run(chunk, (fem.POOL_GRAPH, fem.POOL_PERSISTENT, fem.POOL_GRAPH_STAGED)[k % 3])
    assert mix.status(ib)[0] == 1500
    pb, vb = mix.readback(ib)
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert np.array_equal(ea, mix.energy(ib))
    assert mix.status(j0)[0] == 37 + 50 + 1500 and mix.status(j1)[0] == 50 + 1500


def test_async_admission_behind_a_running_chunk(fem):
    """admit / release while a chunk is in flight land behind it: the in-flight meshes
    are unaffected and the new mesh starts from rest at the next chunk."""
    a, b = beam(fem, 20, 2, 2, load=90e3), beam(fem, 12, 3, 3, load=70e3)
    da, db = crit(fem, a), crit(fem, b)
    ref = fem.TetPool(60000, 20000, max_meshes=4)
    ra = ref.admit(steps=500, dt=da, ramp_steps=100, **MATS[0], **a)
    ref.run(500)
    rb = ref.admit(steps=200, dt=db, ramp_steps=100, **MATS[1], **b)
    ref.run(200)
    pool = fem.TetPool(60000, 20000, max_meshes=4)
    ia = pool.admit(steps=500, dt=da, ramp_steps=100, **MATS[0], **a)
    pool.run_async(250)
    junk = pool.admit(steps=10, dt=db, **MATS[2], **b)        # admitted while running
    pool.release(junk)                                        # and dropped again
    ib = pool.admit(steps=200, dt=db, ramp_steps=100, **MATS[1], **b)
    pool.wait()
    assert pool.finished() == []
    pool.run(250)
    assert sorted(pool.finished()) == sorted([ia, ib])
    assert pool.status(ib)[0] == 200
    assert np.array_equal(pool.readback(ia)[0], ref.readback(ra)[0])
    assert np.array_equal(pool.readback(ib)[0], ref.readback(rb)[0])


def test_tile_sizes_and_autotune_leave_results_unchanged(fem):
    m = beam(fem, 36, 3, 3, load=170e3)
    base = None
    for tile, mode in ((128, fem.POOL_GRAPH), (256, fem.POOL_GRAPH), (512, fem.POOL_GRAPH),
                       (128, fem.POOL_GRAPH_STAGED), (256, fem.POOL_GRAPH_STAGED), (512, fem.POOL_PERSISTENT)):
        pool = fem.TetPool(50000, 15000, max_meshes=2, tile=tile)
        i = pool.admit(steps=300, ramp_steps=150, **MATS[0], **m)
        pool.run(300, mode)
        p, v = pool.readback(i)
        e = pool.energy(i)
        if base is None:
            base = (p, v, e)
        else:
            assert np.array_equal(p, base[0]) and np.array_equal(v, base[1])
            assert np.allclose(e, base[2], rtol=1e-12, atol=0.0)
            if tile == 128:
                assert np.array_equal(e, base[2])  # the same tiles: the same energy bits
        pool.close()
    pool = fem.TetPool(50000, 15000, max_meshes=2)
    i = pool.admit(steps=300, ramp_steps=150, **MATS[0], **m)
    pool.run(100)
    best = pool.autotune(steps=20)
    assert best["tile"] in (128, 256, 512) and best["ms_per_step"] > 0
    assert pool.status(i)[0] == 100  # tuning rolled its trial steps back
    pool.run(200)
    p, v = pool.readback(i)
    # the same 300 steps with no tuning in between: 100 in the pool's first schedule,
    # 200 in the one the autotuner picked (the tiled schedule has its own association,
    # so this, not the graph schedule's bits, is what tuning must leave unchanged)
    ref = fem.TetPool(50000, 15000, max_meshes=2)
    j = ref.admit(steps=300, ramp_steps=150, **MATS[0], **m)
    ref.run(100)
    ref.set_schedule(best["tile"], {n: c for c, n in fem.POOL_MODE_NAMES.items()}[best["mode"]])
    ref.run(200)
    pr, vr = ref.readback(j)
    assert np.array_equal(p, pr) and np.array_equal(v, vr)
    assert np.allclose(pool.energy(i), ref.energy(j), rtol=1e-12, atol=0.0)
    if best["mode"] != "graph-tiled":
        assert np.array_equal(p, base[0]) and np.array_equal(v, base[1])


def test_admission_against_capacity(fem):
    m = beam(fem, 10, 2, 2)  # 240 tets, 99 nodes
    pool = fem.TetPool(600, 400, max_meshes=8)
    i1 = pool.admit(steps=10, dt=1e-7, **m)
    i2 = pool.admit(steps=10, dt=1e-7, **m)
    with pytest.raises(fem.PoolFull):
        pool.admit(steps=10, dt=1e-7, **m)  # 720 tets > 600
    pool.run(10)
    assert sorted(pool.finished()) == sorted([i1, i2])
    pool.release(i1)
    i3 = pool.admit(steps=5, dt=1e-7, **m)
    pool.run(5)
    assert sorted(pool.finished()) == sorted([i2, i3])
    bad = dict(m)
    bad["index"] = m["index"].copy()
    bad["index"][3] = 10_000
    with pytest.raises(fem.FemStepError) as e:
        pool.admit(steps=1, **bad)
    assert e.value.code == fem.EINVAL


def test_admit_many_is_admit_in_order(fem):
    """admit_many (host work on all cores) gives the same pool as admitting one by one,
    and admits the prefix that fits."""
    meshes = [beam(fem, 12 + 2 * k, 2 + k % 2, 2, load=60e3 + 10e3 * k, clamp_end=k % 2) for k in range(6)]
    kw = [dict(ramp_steps=100, **MATS[k % 3], **m) for k, m in enumerate(meshes)]
    a = fem.TetPool(40000, 12000, max_meshes=8)
    ia = [a.admit(steps=300, **k) for k in kw]
    b = fem.TetPool(40000, 12000, max_meshes=8)
    ib = b.admit_many(kw, [300] * len(kw))
    assert ib == ia
    a.run(300)
    b.run(300)
    for i in ia:
        assert np.array_equal(a.readback(i)[0], b.readback(i)[0])
        assert np.array_equal(a.energy(i), b.energy(i))
    tets = [m["index"].size // 4 for m in meshes]
    small = fem.TetPool(sum(tets[:3]) + 10, 12000, max_meshes=8)
    got = small.admit_many(kw, [10] * len(kw))
    assert got == [0, 1, 2]  # the rest did not fit now
    bad = dict(kw[0])
    bad["index"] = kw[0]["index"].copy()
    bad["index"][0] = 99999
    with pytest.raises(fem.FemStepError) as e:
        b.admit_many([kw[1], bad], [1, 1])
    assert e.value.code == fem.EINVAL and b.info()["meshes"] == len(ia)


def test_device_critical_dt_matches_single_mesh_bound(fem):
    m = beam(fem, 20, 3, 3)
    pool = fem.TetPool(20000, 5000)
    i = pool.admit(steps=1, **m)
    # the pool bounds the FP32 Dm^-1 the kernels use; the single mesh the FP64 one
    assert abs(pool.dt(i) / crit(fem, m) - 1.0) < 1e-6


@pytest.mark.parametrize("k,mode", [(0, "graph"), (1, "graph"), (2, "graph"), (0, "graph-tiled"),
                                    (1, "graph-tiled")])
def test_pool_meshes_against_fp64_oracle(fem, port, k, mode):
    """Per-mesh materials, 2,000 steps, against O-tet64 (fem.cpp kinematics with the
    J2 return in double): 1e-5 relative displacement; energy account within 0.5 %.  In
    the graph schedule and in the tiled one (its own association of the node sums)."""
    loads = [200e3, 260e3, 230e3]
    m = beam(fem, 40, 4, 4, load=loads[k], clamp_end=k % 2)
    ref = O.TetMesh64(port, m["position"], m["index"], m["fixed"], m["external_force"])
    dt = port.tet64_critical_dt(C.byref(ref._s), 210e9, 0.3, 7850.0, 0.9)
    ref.step(O.tet64_params(dt=dt, ramp_steps=1000, yield_=MATS[k]["yield_strength"],
                            hardening=MATS[k]["hardening"]), 2000)
    code = {v: c for c, v in fem.POOL_MODE_NAMES.items()}[mode]
    pool = fem.TetPool(100000, 30000, max_meshes=4, tile=128)
    pool.admit(steps=2000, dt=dt, **beam(fem, 8, 2, 2))  # a neighbour, so the mesh runs in a mix
    i = pool.admit(steps=2000, dt=dt, ramp_steps=1000, **MATS[k], **m)
    pool.run(2000, code)
    p, _ = pool.readback(i)
    rest = m["position"].astype(np.float64)
    u, ur = p - rest, ref.position - rest
    err = np.abs(u - ur).max() / np.abs(ur).max()
    yielded = (ref.plastic.reshape(-1, 7)[:, 6] > 0).mean()
    assert yielded > 0.2, "the case must exercise plasticity"
    assert err < 1e-5, err
    e, er = pool.energy(i), ref.energy
    assert abs(e[0] - er[0]) / er[0] < 5e-3
    for j in (1, 2, 3):
        assert abs(e[j] - er[j]) <= 5e-3 * er[0]


def test_workload_meshes_against_fp64_oracle(fem, port):
    """Eight meshes of the batched workload itself (workloads.batch_meshes as the bench
    draws it; workloads.drift_sample picks them): the largest, a 197,106-tet beam under
    pressure, and the smallest plate of each clamped face and load kind -- x0, x1, y0,
    y1, tip and pressure -- all in one pool for the 1,000-step ramp plus 1,000 steps.
    Each against O-tet64 (in double, on all host cores): 1e-5 relative displacement, and
    every energy term within 0.5 % of the external work."""
    import workloads as W

    specs = W.batch_meshes(256)
    picks = W.drift_sample(specs)
    assert len(picks) == 8
    chosen = [specs[i] for i in picks]
    assert {s.clamp for s in chosen} == {"x0", "x1", "y0", "y1"}
    assert sum(s.load_kind == "pressure" and s.cells[1] > s.cells[2] for s in chosen) >= 2
    assert max(s.tets for s in chosen) > 190000
    built = [W.build(sp) for sp in chosen]
    threads = os.cpu_count() or 1
    refs, dts = [], []
    for b in built:
        r = O.TetMesh64(port, b.position, b.index, b.fixed, b.external_force)
        dt = port.tet64_critical_dt(C.byref(r._s), W.YOUNGS, W.POISSON, W.DENSITY, 0.9)
        r.step(O.tet64_params(dt=dt, ramp_steps=1000, yield_=b.spec.yield_strength, hardening=b.spec.hardening),
               2000, threads=threads)
        refs.append(r)
        dts.append(dt)
    T = sum(sp.tets for sp in chosen)
    N = sum(sp.nodes for sp in chosen)
    pool = fem.TetPool(T, N + len(chosen) + 1, max_meshes=len(chosen) + 1)
    ids = [pool.admit(steps=2000, dt=dt, **b.admit_kwargs()) for b, dt in zip(built, dts)]
    for chunk in (1000, 7, 993):
        pool.run(chunk)
    yielded = []
    for b, r, i in zip(built, refs, ids):
        assert pool.status(i)[0] == 2000
        p, _ = pool.readback(i)
        rest = b.position.astype(np.float64)
        u, ur = p - rest, r.position - rest
        err = np.abs(u - ur).max() / np.abs(ur).max()
        assert err < 1e-5, (b.spec, err)
        e, er = pool.energy(i), r.energy
        for j in (0, 1, 2, 3):
            assert abs(e[j] - er[j]) <= 5e-3 * er[0], (b.spec, j, e, er)
        yielded.append((r.plastic.reshape(-1, 7)[:, 6] > 0).mean())
    assert sum(y > 0.01 for y in yielded) >= 5, yielded
    pool.close()


def test_evict_and_resume_is_bit_identical(fem):
    """A mesh checkpointed mid-run, released, and admitted again later (elsewhere in the
    pool, next to other meshes, after the others moved on) ends with the same bits --
    state and FP64 energy account -- as when it never left."""
    a = beam(fem, 30, 3, 3, load=400e3)
    others = [beam(fem, 16, 2, 2, load=80e3), beam(fem, 50, 4, 4, length=2.0, load=120e3)]
    alone = fem.TetPool(100000, 30000, max_meshes=4)
    ia = alone.admit(steps=1500, ramp_steps=500, **MATS[0], **a)
    alone.run(1500)
    pa, va = alone.readback(ia)
    ea, pla = alone.energy(ia), alone.plastic(ia)
    assert (pla[:, 6] > 0).mean() > 0.05, "the case must exercise plasticity"

    pool = fem.TetPool(300000, 90000, max_meshes=8)
    j0 = pool.admit(steps=4000, ramp_steps=300, **MATS[1], **others[0])
    ib = pool.admit(steps=1500, ramp_steps=500, **MATS[0], **a)
    pool.run(333)
    ck = pool.checkpoint(ib)
    pool.release(ib)
    # someone else takes the space, the pool moves on without the mesh
    j1 = pool.admit(steps=4000, ramp_steps=300, **MATS[2], **others[1])
    pool.run(71, fem.POOL_PERSISTENT)
    with pytest.raises(fem.FemStepError):
        pool.admit_resume(ck, 100, ramp_steps=500, **MATS[0], **a)  # below the steps taken
    ic = pool.admit_resume(ck, 1500, ramp_steps=500, **MATS[0], **a)
    assert pool.status(ic) == (333, 1500)
    for k, chunk in enumerate((5, 400, 29, 900)):
        pool.run(chunk, (fem.POOL_GRAPH, fem.POOL_GRAPH_STAGED, fem.POOL_PERSISTENT, fem.POOL_GRAPH)[k])
    assert pool.status(ic)[0] == 1500
    pc, vc = pool.readback(ic)
    assert np.array_equal(pa, pc) and np.array_equal(va, vc)
    assert np.array_equal(pla, pool.plastic(ic))
    assert np.array_equal(ea, pool.energy(ic))
    assert pool.status(j0)[0] == 333 + 71 + 1334 and pool.status(j1)[0] == 71 + 1334
    # a checkpoint of another mesh is refused
    with pytest.raises(fem.FemStepError):
        pool.admit_resume(ck, 1500, **MATS[0], **others[0])


def test_readback_many_is_readback(fem):
    """The batch readback gives each mesh exactly what the per-mesh readback gives."""
    meshes = [beam(fem, 12, 2, 2, load=80e3), beam(fem, 30, 3, 3, load=300e3), beam(fem, 7, 2, 2, length=0.4)]
    pool = fem.TetPool(100000, 30000, max_meshes=8)
    ids = [pool.admit(steps=300, ramp_steps=100, **MATS[k], **meshes[k]) for k in range(3)]
    pool.run(300)
    many = pool.readback_many(ids[::-1])
    for i, (p, v) in zip(ids[::-1], many):
        pe, ve = pool.readback(i)
        assert np.array_equal(p, pe) and np.array_equal(v, ve)
    assert np.abs(many[1][0] - meshes[1]["position"]).max() > 0
    pool.close()


def test_many_workload_meshes_same_bits_in_every_schedule(fem):
    """A pool of 48 of the batched workload's own meshes (uneven sizes, every clamp face,
    tip and pressure loads), admitted together: more element tiles than the staged
    pass's persistent grid holds at once, so its blocks walk several tiles each.  Every
    mesh's state and FP64 energy account are the same in every schedule, over chunks
    that straddle the meshes' step counts."""
    import workloads as W

    specs = W.batch_meshes(count=48, lo=2e3, hi=3e4, seed=77)
    built = [W.build(s) for s in specs]
    kw = [dict(m.admit_kwargs(), ramp_steps=40) for m in built]
    steps = [60 + 7 * (k % 5) for k in range(len(kw))]
    tets = sum(m.index.size // 4 for m in built)
    nodes = sum(m.position.size // 3 + 1 for m in built)
    out = []
    for mode in (fem.POOL_GRAPH, fem.POOL_GRAPH_STAGED, fem.POOL_PERSISTENT):
        pool = fem.TetPool(tets + 1000, nodes + 1000, max_meshes=64, tile=128)
        ids = pool.admit_many(kw, steps)
        assert len(ids) == len(kw)
        for chunk in (25, 41, 3, 30):  # 99 steps: every mesh reaches its count (60 to 88)
            pool.run(chunk, mode)
        out.append([(pool.readback(i), pool.plastic(i), pool.energy(i), pool.status(i)) for i in ids])
        pool.close()
    for other in out[1:]:
        for (ra, pa, ea, sa), (rb, pb, eb, sb) in zip(out[0], other):
            assert sa == sb and sa[0] == sa[1]
            assert np.array_equal(ra[0], rb[0]) and np.array_equal(ra[1], rb[1])
            assert np.array_equal(pa, pb)
            assert np.array_equal(ea, eb)


def test_tiled_schedule_same_bits_alone_in_the_mix_and_resumed(fem):
    """The tiled schedule associates each node's force sum per tile; its tiles are
    aligned to the mesh's first tet, so a mesh's bits do not depend on its place in the
    pool, its neighbours, the chunking or an eviction in between."""
    a = beam(fem, 30, 3, 3, load=400e3)
    others = [beam(fem, 16, 2, 2, load=80e3), beam(fem, 50, 4, 4, length=2.0, load=120e3)]
    T = fem.POOL_GRAPH_TILED
    alone = fem.TetPool(100000, 30000, max_meshes=4, tile=128)
    ia = alone.admit(steps=1500, ramp_steps=500, **MATS[0], **a)
    alone.run(1500, T)
    pa, va = alone.readback(ia)
    ea, pla = alone.energy(ia), alone.plastic(ia)
    assert (pla[:, 6] > 0).mean() > 0.05, "the case must exercise plasticity"
    mix = fem.TetPool(300000, 90000, max_meshes=8, tile=128)
    j0 = mix.admit(steps=3000, ramp_steps=300, **MATS[1], **others[0])
    mix.run(37, T)
    ib = mix.admit(steps=1500, ramp_steps=500, **MATS[0], **a)  # mid-run, at another place
    mix.run(400, T)
    ck = mix.checkpoint(ib)
    mix.release(ib)
    j1 = mix.admit(steps=3000, ramp_steps=300, **MATS[2], **others[1])
    mix.run(29, T)
    ic = mix.admit_resume(ck, 1500, ramp_steps=500, **MATS[0], **a)
    for chunk in (3, 64, 500, 533, 100):
        mix.run(chunk, T)
    assert mix.status(ic)[0] == 1500
    pc, vc = mix.readback(ic)
    assert np.array_equal(pa, pc) and np.array_equal(va, vc)
    assert np.array_equal(pla, mix.plastic(ic))
    assert np.array_equal(ea, mix.energy(ic))
    assert mix.status(j0)[0] > 1500 and mix.status(j1)[0] > 1000


def test_tiled_schedule_against_graph_on_workload_meshes(fem):
    """48 of the batched workload's meshes (every clamp face, tip and pressure loads,
    uneven sizes) in the tiled schedule against the graph schedule, after the ramp has
    yielded several of them: the two sum the same terms in a different association, so
    they agree to rounding -- 1e-6 of each mesh's largest displacement -- and their
    energy accounts to 1e-6 of the external work."""
    import workloads as W

    specs = W.batch_meshes(count=48, lo=2e3, hi=3e4, seed=77)
    built = [W.build(s) for s in specs]
    kw = [dict(m.admit_kwargs(), ramp_steps=200) for m in built]
    tets = sum(m.index.size // 4 for m in built)
    nodes = sum(m.position.size // 3 + 1 for m in built)
    out = []
    for mode in (fem.POOL_GRAPH, fem.POOL_GRAPH_TILED):
        pool = fem.TetPool(tets + 1000, nodes + 1000, max_meshes=64, tile=128)
        ids = pool.admit_many(kw, [400] * len(kw))
        pool.run(400, mode)
        out.append([(pool.readback(i)[0], pool.energy(i), pool.plastic(i)) for i in ids])
        pool.close()
    yielded = 0
    for b, (pg, eg, plg), (pt, et, plt) in zip(built, *out):
        rest = b.position.astype(np.float64)
        ug, ut = pg - rest, pt - rest
        assert np.abs(ug - ut).max() <= 1e-6 * np.abs(ug).max(), b.spec
        for j in (0, 1, 2, 3):
            assert abs(eg[j] - et[j]) <= 1e-6 * abs(eg[0]), (b.spec, j)
        yielded += (plg[:, 6] > 0).any()
    assert yielded >= 5, yielded


def test_tiled_schedule_refuses_other_tile_sizes(fem):
    """The tiled schedule's tables are built for tiles of 128 tets: asking for it at
    another tile size is refused with FEMSTEP_EINVAL, by set_schedule and by run, and the
    pool keeps working in the schedules it has."""
    m = beam(fem, 12, 2, 2, load=50e3)
    pool = fem.TetPool(20000, 6000, max_meshes=2, tile=256)
    pool.admit(steps=20, ramp_steps=10, **MATS[0], **m)
    with pytest.raises(fem.FemStepError) as e:
        pool.set_schedule(256, fem.POOL_GRAPH_TILED)
    assert e.value.code == fem.EINVAL
    with pytest.raises(fem.FemStepError) as e:
        pool.run(5, fem.POOL_GRAPH_TILED)
    assert e.value.code == fem.EINVAL
    pool.run(5, fem.POOL_GRAPH)
    pool.set_schedule(128, fem.POOL_GRAPH_TILED)
    pool.run(15)
    assert pool.status(0) == (20, 20)
    pool.close()
