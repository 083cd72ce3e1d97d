"""The serving loop (serving.Server) driving a real TetPool on the GPU.

A short seeded burst of Poisson arrivals (workloads.request_trace: about 40 requests
within 0.1 s; small meshes and step counts so the test takes seconds) is served by
continuous batching into a pool that holds about a fifth of them at once, so requests
wait in the queue for releases and join while others are stepping.  Every completed request's positions,
velocities and plastic state must be bit-identical to the same mesh stepped alone in
a fresh pool: the result of a solve does not depend on what else was on the GPU, when
it was admitted, or how the chunks fell.
"""
import numpy as np
import pytest

import serving as S
import workloads as W

pytestmark = pytest.mark.gpu


def test_served_results_are_the_same_alone_and_in_the_mix(fem):
    trace = W.request_trace(rate=400.0, duration=0.1, lo=1e3, hi=2e4, steps=(150, 600), seed=7)
    assert len(trace) >= 30
    built = {k: W.build(sp) for k, sp in enumerate(trace)}
    reqs = [S.Request(key=k, arrival=sp.arrival, tets=sp.tets, steps=sp.steps,
                      build=(lambda k=k: built[k].admit_kwargs())) for k, sp in enumerate(trace)]
    # room for about a fifth of the trace's tets at once: admissions wait for releases
    cap_t = max(sum(sp.tets for sp in trace) // 5, max(sp.tets for sp in trace))
    cap_n = max(sum(sp.nodes for sp in trace) // 5, max(sp.nodes for sp in trace)) + 64
    pool = fem.TetPool(cap_t, cap_n, max_meshes=64)
    rep = S.Server(pool, chunk=48, keep_results=True, full_error=fem.PoolFull).serve(reqs)
    pool.close()
    assert rep.completed == len(reqs)
    assert rep.admit_retries > 0, "some request must wait for room"
    assert max(r.admitted - r.arrival for r in reqs) > 0
    assert rep.element_updates == sum(r.tets * r.steps for r in reqs)
    yielded = 0
    for r in reqs:
        b = built[r.key]
        alone = fem.TetPool(b.spec.tets, b.spec.nodes + 2, max_meshes=2)
        i = alone.admit(steps=r.steps, **b.admit_kwargs())
        alone.run(r.steps)
        p, v = alone.readback(i)
        pl = alone.plastic(i)
        alone.close()
        rp, rv, rpl = r.result
        assert np.array_equal(rp, p) and np.array_equal(rv, v), r.key
        assert np.array_equal(rpl, pl), r.key
        yielded += bool((pl[:, 6] > 0).any())
    assert yielded > 0, "the trace must exercise plasticity"
    s = rep.summary()
    assert s["p50_step_ms"] is not None and s["p99_step_ms"] >= s["p50_step_ms"]
