"""Serving loop: a stream of simulation requests on one GPU with continuous
batching.

Requests (``ensemble.Box`` plus an arrival time) of mixed grid size, step
count and cosmology are admitted into slots of a resident ``Ensemble``.
Slot capacity per size class comes from an HBM budget and the per-slot
footprint (``hgpm_ens_footprint_bytes``), so admission is by footprint: a
request waits until a slot of its class is free.  Every tick advances all
admitted requests by one PM step in one batched launch per phase per class;
requests that arrive while others run are admitted at the next tick, their
ICs generated in place, and a request that finishes frees its slot after its
P(k) is taken.  Particle and grid state stay on the device throughout.

``serve_one_at_a_time`` is the comparison: the same requests, first come
first served, each through its own context and the plain step.
"""
from __future__ import annotations

import collections
import time

import numpy as np

from .binding import Simulation
from .ensemble import Box, Ensemble, _result, _ts_for, prepare_tables


def request_stream(n: int, rate: float = 20.0, seed: int = 7, sizes=(32, 48, 64, 96, 128, 192, 256),
                   steps=(20, 200), z_ini: float = 50.0):
    """Poisson arrivals (mean `rate` per second) of requests with ng = np
    log-uniform over `sizes`, steps ~ U[steps], Om ~ U[0.25, 0.35],
    sigma8 ~ U[0.7, 0.9], L = ng Mpc/h and a seed of their own.  Every
    request runs on the same step grid (N_STEPS = steps[1], z_ini -> 0) and
    stops after its own number of steps, so short requests end at z > 0."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        b = Box(ng=int(rng.choice(sizes)), rl=0.0, seed=5000 + i, nsteps=int(rng.integers(steps[0], steps[1] + 1)),
                n_total=steps[1], z_ini=z_ini, sigma8=float(rng.uniform(0.7, 0.9)), omega_m=float(rng.uniform(0.25, 0.35)), tag=i)
        b.rl = float(b.ng)
        b.arrival = t
        out.append(b)
    return out


def class_capacity(sizes, hbm_budget: float, max_slots: int = 64):
    """Slots per size class: the budget split evenly over the classes, each
    share divided by the class's per-slot footprint."""
    share = hbm_budget / len(sizes)
    caps = []
    for ng in sizes:
        per = Ensemble.footprint_bytes(ng, ng, 1)
        caps.append((ng, ng, int(max(1, min(max_slots, share // per)))))
    return caps


class Server:
    def __init__(self, sizes, hbm_budget: float = 40e9, device: int = 0, graph: bool = True, max_slots: int = 64):
        self.classes = class_capacity(sizes, hbm_budget, max_slots)
        self.index = {c[0]: i for i, c in enumerate(self.classes)}
        self.ens = Ensemble(self.classes, device=device, graph=graph)
        self.free = {i: collections.deque(range(c[2])) for i, c in enumerate(self.classes)}
        self.running = {}  # (cls, slot) -> request
        self.ticks = 0

    def close(self):
        self.ens.close()

    def admit(self, req: Box) -> bool:
        ci = self.index[req.ng]
        if not self.free[ci]:
            return False
        si = self.free[ci].popleft()
        p = req.params()
        v = self.ens.slot(ci, si, p)
        v.generate_ic(req.table, req.k_delta)
        self.ens.start(ci, si, _ts_for(p), req.nsteps)
        self.running[(ci, si)] = req
        return True

    def tick(self):
        """One batched step of every running request; returns the finished
        requests with their results."""
        self.ens.step(1)
        self.ens.sync()
        self.ticks += 1
        done = []
        for (ci, si), req in list(self.running.items()):
            running, nd = self.ens.status(ci, si)
            if not running:
                v = self.ens.views[(ci, si)]
                req.result = _result(v, req)
                self.ens.release(ci, si)
                self.free[ci].append(si)
                del self.running[(ci, si)]
                done.append(req)
        return done


def serve(requests, hbm_budget: float = 40e9, device: int = 0, graph: bool = True, realtime: bool = True,
          max_slots: int = 64):
    """Run the request stream through a Server.  realtime: requests become
    visible at their arrival times (wall clock from the start); otherwise all
    are queued at t = 0 (saturated throughput).  Returns (requests with
    .latency and .result, makespan seconds, server stats)."""
    prepare_tables(requests)
    sizes = sorted({r.ng for r in requests})
    srv = Server(sizes, hbm_budget, device, graph, max_slots)
    try:
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        finished = []
        t0 = time.perf_counter()
        while len(finished) < len(requests):
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                waiting.append(pending.popleft())
            # first come first served within what fits
            still = collections.deque()
            while waiting:
                r = waiting.popleft()
                if not srv.admit(r):
                    still.append(r)
            waiting = still
            if srv.running:
                for r in srv.tick():
                    r.finish = time.perf_counter() - t0
                    r.latency = r.finish - (r.arrival if realtime else 0.0)
                    finished.append(r)
            elif pending:
                time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.01)))
        makespan = time.perf_counter() - t0
        return finished, makespan, {"ticks": srv.ticks, "classes": srv.classes,
                                    "launches": srv.ens.kernel_launches()}
    finally:
        srv.close()


def serve_one_at_a_time(requests, device: int = 0, realtime: bool = True):
    """The same requests, first come first served, one context at a time."""
    prepare_tables(requests)
    finished = []
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda q: q.arrival):
        if realtime:
            wait = r.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        p = r.params()
        with Simulation(p, device=device) as s:
            s.generate_ic(r.table, r.k_delta)
            s.run_steps(_ts_for(p), r.nsteps)
            r.result = _result(s, r)
        r.finish = time.perf_counter() - t0
        r.latency = r.finish - (r.arrival if realtime else 0.0)
        finished.append(r)
    return finished, time.perf_counter() - t0


def latency_summary(reqs, makespan):
    lat = np.array([r.latency for r in reqs])
    return {"n": len(reqs), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": makespan, "sims_per_hour": len(reqs) / makespan * 3600.0}
