"""Serving loop over a TetPool: continuous batching of FEM solves on one GPU.

Requests (tet meshes with a step count) arrive over time.  The loop admits each
into the pool as soon as its arrays fit in the pool's free device memory, keeps every
admitted solve resident, and steps all of them together in chunks of `chunk` steps;
a solve that reaches its step count is read back and released, which frees room for
the queue.  Admission runs on the host while the GPU works through the current chunk
(the pool queues its uploads behind the chunk), so arrivals join at the next chunk
boundary without stopping the solves already running.

Reported: per-step latency (the wall time of each chunk over its steps, one sample per
live solve per chunk), request latency (arrival to result), queue wait, and aggregate
element-updates/s.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    key: int
    arrival: float
    tets: int
    steps: int
    build: object             # callable -> dict of TetPool.admit keyword arguments
    admitted: float = -1.0
    finished: float = -1.0
    mesh_id: int = -1
    done: int = 0             # steps taken so far
    result: object = None


@dataclass
class Report:
    requests: int = 0
    completed: int = 0
    element_updates: float = 0.0
    wall_s: float = 0.0
    device_ms: float = 0.0
    chunks: int = 0
    step_latency_ms: list = field(default_factory=list)   # one per (live solve, chunk)
    request_latency_s: list = field(default_factory=list)
    queue_wait_s: list = field(default_factory=list)
    max_resident: int = 0
    admit_retries: int = 0
    launches: int = 0                                     # kernel launches of the chunks

    def summary(self):
        def pct(a, q):
            return float(np.percentile(a, q)) if len(a) else None

        return {
            "requests": self.requests, "completed": self.completed, "element_updates": self.element_updates,
            "wall_s": self.wall_s, "elem_upd_per_s": self.element_updates / self.wall_s if self.wall_s else 0.0,
            "device_elem_upd_per_s": self.element_updates / (self.device_ms / 1e3) if self.device_ms else 0.0,
            "device_busy": self.device_ms / 1e3 / self.wall_s if self.wall_s else 0.0,
            "chunks": self.chunks, "p50_step_ms": pct(self.step_latency_ms, 50),
            "p99_step_ms": pct(self.step_latency_ms, 99), "p50_request_s": pct(self.request_latency_s, 50),
            "p99_request_s": pct(self.request_latency_s, 99), "p50_queue_s": pct(self.queue_wait_s, 50),
            "p99_queue_s": pct(self.queue_wait_s, 99), "max_resident": self.max_resident,
            "admit_retries": self.admit_retries, "launches": self.launches,
        }


class Server:
    """Continuous batching over `pool` (a femstep.TetPool or anything with its face).

    clock: seconds since an arbitrary origin (time.perf_counter by default).
    keep_results: read each finished solve back before release: (positions, velocities),
                  and its plastic state where the pool keeps one.
    full_error: the exception the pool raises when a mesh does not fit now.
    """

    def __init__(self, pool, chunk=64, clock=time.perf_counter, sleep=time.sleep, keep_results=False,
                 full_error=Exception, max_tries=8, batch=32):
        self.pool = pool
        self.chunk = int(chunk)
        self.clock = clock
        self.sleep = sleep
        self.keep_results = keep_results
        self.full_error = full_error
        self.max_tries = max_tries
        self.batch = batch

    def _admit_queue(self, queue, live, now, report):
        """Admit queued requests in arrival order while they fit.  A request that does
        not fit stays queued; later, smaller ones may still go in (no head-of-line
        blocking), up to `max_tries` failed admissions per chunk boundary.  A pool with
        admit_many takes the head of the queue in one call (its host work in parallel)."""
        if queue and hasattr(self.pool, "admit_many"):
            head = [queue.popleft() for _ in range(min(len(queue), self.batch))]
            ids = self.pool.admit_many([r.build() for r in head], [r.steps for r in head])
            t = now()
            for r, i in zip(head, ids):
                r.mesh_id, r.admitted = i, t
                live[i] = r
            rest = head[len(ids):]
            if rest:
                # the first of the rest did not fit: it keeps its place at the head; the
                # others (and the rest of the queue) are tried one by one behind it
                report.admit_retries += 1
                others = collections.deque(rest[1:] + list(queue))
                queue.clear()
                self._admit_one_by_one(others, live, now, report, tries=1)
                queue.append(rest[0])
                queue.extend(others)
            return
        self._admit_one_by_one(queue, live, now, report)

    def _admit_one_by_one(self, queue, live, now, report, tries=0):
        kept = collections.deque()
        while queue:
            r = queue.popleft()
            if tries >= self.max_tries:
                kept.append(r)
                continue
            try:
                r.mesh_id = self.pool.admit(steps=r.steps, **r.build())
            except self.full_error:
                report.admit_retries += 1
                tries += 1
                kept.append(r)
                continue
            r.admitted = now()
            live[r.mesh_id] = r
        queue.extend(kept)

    def serve(self, requests, time_limit=None):
        """Serve `requests` (arrival in seconds from the start); returns a Report."""
        report = Report(requests=len(requests))
        arrivals = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue = collections.deque()
        live = {}
        t0 = self.clock()

        def now():
            return self.clock() - t0

        def arrive():
            t = now()
            while arrivals and arrivals[0].arrival <= t:
                queue.append(arrivals.popleft())

        while arrivals or queue or live:
            if time_limit is not None and now() > time_limit:
                break
            arrive()
            if not live:
                self._admit_queue(queue, live, now, report)
                if not live:
                    if arrivals:
                        self.sleep(max(0.0, arrivals[0].arrival - now()))
                        continue
                    if queue:
                        raise RuntimeError("a queued request can never fit in the pool")
                    break
            # one chunk for everything resident; admissions overlap it on the host
            start = now()
            stepping = list(live.values())
            self.pool.run_async(self.chunk)
            arrive()
            self._admit_queue(queue, live, now, report)
            ms = self.pool.wait()
            end = now()
            report.device_ms += ms
            report.chunks += 1
            if hasattr(self.pool, "info"):
                report.launches += self.pool.info()["launches"]
            report.max_resident = max(report.max_resident, len(live))
            for r in stepping:
                taken = min(self.chunk, r.steps - r.done)
                if taken <= 0:
                    continue
                r.done += taken
                report.element_updates += float(r.tets) * taken
                report.step_latency_ms.append((end - start) * 1e3 / self.chunk)
            for mid in self.pool.finished():
                r = live.pop(mid, None)
                if r is None:
                    continue
                if self.keep_results:
                    r.result = self.pool.readback(mid)
                    if hasattr(self.pool, "plastic"):
                        r.result = tuple(r.result) + (self.pool.plastic(mid),)
                self.pool.release(mid)
                r.finished = now()
                report.completed += 1
                report.request_latency_s.append(r.finished - r.arrival)
                report.queue_wait_s.append(r.admitted - r.arrival)
        report.wall_s = now()
        return report
