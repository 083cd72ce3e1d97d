"""The serving loop's host logic, on the CPU against a fake pool.

The fake keeps the pool's contract (admit raises when the tets do not fit, a chunk
advances every admitted mesh by up to `chunk` steps, finished() lists those at their
count, admissions made while a chunk runs join at the next chunk) and a simulated
clock, so the loop's admission order, requeueing, accounting and latency statistics
can be checked exactly.
"""
import numpy as np
import pytest

import serving as S
import workloads as W


class Full(Exception):
    pass


class FakePool:
    def __init__(self, capacity, clock, step_ms=1.0):
        self.capacity, self.used = capacity, 0
        self.clock = clock
        self.step_ms = step_ms
        self.meshes = {}      # id -> [tets, done, target]
        self.next_id = 0
        self.running = None   # ids stepping in the current chunk
        self.log = []         # ("admit", id, time, chunk in flight) / ("release", id, time)

    def admit(self, steps, tets, **_):
        if self.used + tets > self.capacity:
            raise Full()
        i = self.next_id
        self.next_id += 1
        self.meshes[i] = [tets, 0, steps]
        self.used += tets
        self.log.append(("admit", i, self.clock.t, self.running is not None))
        return i

    def release(self, i):
        self.used -= self.meshes.pop(i)[0]
        self.log.append(("release", i, self.clock.t))

    def run_async(self, chunk):
        assert self.running is None
        self.running = [i for i, m in self.meshes.items() if m[1] < m[2]]
        self.chunk = chunk

    def wait(self):
        for i in self.running:
            m = self.meshes[i]
            m[1] += min(self.chunk, m[2] - m[1])
        self.running = None
        ms = self.chunk * self.step_ms
        self.clock.t += ms / 1e3
        return ms

    def finished(self):
        return [i for i, m in self.meshes.items() if m[1] >= m[2]]

    def readback(self, i):
        return ("result", i)


class FakeBatchPool(FakePool):
    """The same, with the real pool's admit_many: the admitted prefix's ids."""

    def admit_many(self, meshes, steps):
        ids = []
        for m, n in zip(meshes, steps):
            try:
                ids.append(self.admit(steps=n, **m))
            except Full:
                break
        return ids


@pytest.fixture(params=[FakePool, FakeBatchPool], ids=["admit", "admit_many"])
def Pool(request):
    return request.param


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, s):
        self.t += s


def make_requests(spec):
    return [S.Request(key=k, arrival=a, tets=t, steps=n, build=(lambda t=t: {"tets": t})) for k, (a, t, n) in
            enumerate(spec)]


def events(pool, kind):
    return {e[1]: e[2] for e in pool.log if e[0] == kind}


def test_all_requests_complete_and_work_is_accounted(Pool):
    clock = Clock()
    pool = Pool(capacity=1000, clock=clock)
    reqs = make_requests([(0.0, 300, 100), (0.01, 500, 64), (0.02, 400, 10), (0.5, 100, 1)])
    srv = S.Server(pool, chunk=16, clock=clock, sleep=clock.sleep, keep_results=True, full_error=Full)
    rep = srv.serve(reqs)
    assert rep.completed == 4
    assert rep.element_updates == sum(r.tets * r.steps for r in reqs)
    assert all(r.result == ("result", r.mesh_id) for r in reqs)
    assert all(r.admitted >= r.arrival and r.finished > r.admitted for r in reqs)
    assert pool.used == 0 and not pool.meshes


def test_a_request_that_does_not_fit_waits_for_a_release(Pool):
    clock = Clock()
    pool = Pool(capacity=1000, clock=clock)
    # 600 + 500 > 1000: the second waits for the first to finish; the third (small)
    # goes in beside the first meanwhile (no head-of-line blocking)
    reqs = make_requests([(0.0, 600, 48), (0.001, 500, 16), (0.002, 300, 16)])
    srv = S.Server(pool, chunk=16, clock=clock, sleep=clock.sleep, full_error=Full)
    rep = srv.serve(reqs)
    assert rep.completed == 3 and rep.admit_retries > 0
    admits, releases = events(pool, "admit"), events(pool, "release")
    first, second, third = reqs
    assert admits[second.mesh_id] >= releases[first.mesh_id]
    assert admits[third.mesh_id] < releases[first.mesh_id]


def test_arrivals_join_while_a_chunk_runs(Pool):
    clock = Clock()
    pool = Pool(capacity=10_000, clock=clock, step_ms=1.0)
    reqs = make_requests([(0.0, 100, 1000), (0.010, 100, 50), (0.020, 100, 50)])
    srv = S.Server(pool, chunk=32, clock=clock, sleep=clock.sleep, full_error=Full)
    rep = srv.serve(reqs)
    assert rep.completed == 3
    # the later requests were admitted with a chunk in flight (continuous batching),
    # not after the long first one finished
    busy = [e[3] for e in pool.log if e[0] == "admit" and e[1] != reqs[0].mesh_id]
    assert busy and all(busy)
    assert reqs[1].finished < reqs[0].finished and reqs[2].finished < reqs[0].finished
    s = rep.summary()
    assert s["p50_step_ms"] == pytest.approx(1.0) and s["p99_step_ms"] == pytest.approx(1.0)


def test_request_that_can_never_fit_is_reported(Pool):
    clock = Clock()
    pool = Pool(capacity=100, clock=clock)
    srv = S.Server(pool, chunk=8, clock=clock, sleep=clock.sleep, full_error=Full)
    with pytest.raises(RuntimeError):
        srv.serve(make_requests([(0.0, 500, 10)]))


def test_trace_and_batch_generators_are_seeded():
    a, b = W.request_trace(duration=5.0), W.request_trace(duration=5.0)
    assert [(r.arrival, r.tets, r.steps) for r in a] == [(r.arrival, r.tets, r.steps) for r in b]
    assert 100 < len(a) < 300  # Poisson, 40/s over 5 s
    assert all(500 <= r.steps <= 5000 for r in a)
    specs = W.batch_meshes()
    t = np.array([s.tets for s in specs])
    assert len(specs) == 256 and t.min() >= 1500 and t.max() <= 2.2e5
    assert 9e6 < t.sum() < 13e6  # E[n] ~ 43 k tets
    assert all(235e6 <= s.yield_strength <= 355e6 and 0.5e9 <= s.hardening <= 2e9 for s in specs)
    m = W.build(specs[0])
    assert m.index.size == 4 * specs[0].tets and m.position.size == 3 * specs[0].nodes
    assert m.fixed.sum() > 0 and np.abs(m.external_force).sum() > 0
