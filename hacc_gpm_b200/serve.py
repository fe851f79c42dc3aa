"""Serving loop: a stream of simulation requests on one GPU with continuous
batching.

Requests (``ensemble.Box`` plus an arrival time) of mixed grid size, step
count and cosmology are admitted into slots of a resident ``Ensemble``.
Slot capacity per size class comes from an HBM budget and the per-slot
footprint (``hgpm_ens_footprint_bytes``), so admission is by footprint: a
request waits until a slot of its class is free.  Each class advances on its
own stream at its own pace, all its admitted requests one PM step at a time
in one batched launch per phase; requests that arrive while others run are
admitted between their class's batches, their ICs generated in place, and a
request that finishes frees its slot after its P(k) is taken.  Particle and
grid state stay on the device throughout.

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


# GPU milliseconds of one PM step per particle + cell, for the concurrency
# cap below: the mid-run 512^3 step on one B200 (5.2 ms for 512^3 particles
# on a 512^3 grid, bench.py).
STEP_MS_PER_UNIT = 5.2 / (2 * 512 ** 3)


def class_capacity(sizes, hbm_budget: float, max_slots: int = 64, step_ms: float = None,
                   ms_per_unit: float = STEP_MS_PER_UNIT):
    """Slots per size class by footprint: every class first gets one slot,
    then the budget left is split evenly over the classes, and what a class
    leaves unused (it stops at its cap) is split again over the classes that
    can still take a slot, until no share buys one.  If one slot of every
    class does not fit the budget, ValueError (admission is by footprint: no
    class is given memory it does not have).  The cap is max_slots and, with
    step_ms, the slots whose batched step takes about step_ms of GPU time
    (ms_per_unit per particle + cell): more large boxes at once would only
    share the GPU further and lengthen every one of their runs (the serving
    p99)."""
    per = {ng: Ensemble.footprint_bytes(ng, ng, 1) for ng in sizes}
    one = sum(per.values())
    if one > hbm_budget:
        raise ValueError("one slot of each size class (%s) needs %.3g GB, above the %.3g GB budget"
                         % (", ".join("%d^3" % ng for ng in sizes), one / 1e9, hbm_budget / 1e9))
    cap = {ng: max_slots if step_ms is None else
           int(max(1, min(max_slots, round(step_ms / (ms_per_unit * 2 * ng ** 3))))) for ng in sizes}
    n = {ng: 1 for ng in sizes}
    left = float(hbm_budget) - one
    open_ = [ng for ng in sizes if n[ng] < cap[ng]]
    while open_:
        share = left / len(open_)
        gave = False
        for ng in open_:
            k = int(min(cap[ng] - n[ng], share // per[ng]))
            if k > 0:
                n[ng] += k
                left -= k * per[ng]
                gave = True
        open_ = [ng for ng in open_ if n[ng] < cap[ng] and per[ng] <= left]
        if not gave:
            break
    return [(ng, ng, int(n[ng])) for ng in sizes]


class Server:
    """Continuous batching over the size classes of one resident Ensemble.

    Each class advances on its own stream at its own pace: when a class's
    queued steps have run (a poll, no wait), its finished requests are
    collected, waiting requests of that class are admitted into its free
    slots, and its next batch of steps is queued.  A batch is sized to about
    ``batch_ms`` of GPU time from the class's measured step time (at most
    ``max_batch`` steps, and no more than the fewest steps a running request
    still needs), so small boxes are not held to the pace of large ones and
    the host loop keeps up with them.

    With ``segment_steps``, a request holds its slot for at most that many
    steps at a time: at the end of a segment its exact state and time
    stepper go to a host checkpoint (``Simulation.checkpoint``), the slot is
    freed, and the request queues again to resume from the checkpoint
    (pre-emption; the result is bit-identical to an uninterrupted run)."""

    def __init__(self, sizes, hbm_budget: float = 40e9, device: int = 0, graph: bool = True, max_slots: int = 64,
                 batch_ms: float = 1.0, max_batch: int = 8, step_ms: float = 2.0, segment_steps: int = None):
        self.classes = class_capacity(sizes, hbm_budget, max_slots, step_ms)
        self.index = {c[0]: i for i, c in enumerate(self.classes)}
        self.ens = Ensemble(self.classes, device=device, graph=graph)
        n = len(self.classes)
        self.free = {i: collections.deque(range(c[2])) for i, c in enumerate(self.classes)}
        self.running = {}  # (cls, slot) -> request
        self.busy = [False] * n      # steps queued on the class's stream
        self.queued = [0] * n        # steps in the current batch
        self.t_launch = [0.0] * n
        self.step_ms = [None] * n    # measured seconds per step, per class (ms)
        self.steps = [0] * n         # class steps run
        self.batch_ms, self.max_batch = batch_ms, max_batch
        self.segment_steps = segment_steps
        self.preemptions = 0
        self.requeue = []

    def close(self):
        self.ens.close()

    def admit(self, req: Box) -> bool:
        ci = self.index[req.ng]
        if self.busy[ci] or not self.free[ci]:
            return False
        si = self.free[ci].popleft()
        p = req.params()
        v = self.ens.slot(ci, si, p)
        ckpt = getattr(req, "ckpt", None)
        if ckpt is None:
            v.generate_ic(req.table, req.k_delta)
            ts = _ts_for(p)
            req.steps_before = 0
        else:
            ts = v.restore(ckpt)  # a pre-empted request resumes exactly
            req.ckpt = None
        left = req.nsteps - req.steps_before
        req.segment = min(left, self.segment_steps) if self.segment_steps else left
        self.ens.start(ci, si, ts, req.segment)  # ts leaves advanced through the segment
        req.ts_end = ts
        req.done_steps = 0
        self.running[(ci, si)] = req
        return True

    def poll(self):
        """Finished requests (with results) of every class whose queued
        steps have run; requests whose segment ended with steps left are
        checkpointed and listed in ``self.requeue``."""
        done = []
        self.requeue = []
        for ci in range(len(self.classes)):
            if not self.busy[ci] or not self.ens.class_done(ci):
                continue
            self.ens.sync_class(ci)
            self.busy[ci] = False
            ms = 1e3 * (time.perf_counter() - self.t_launch[ci]) / self.queued[ci]
            self.step_ms[ci] = ms if self.step_ms[ci] is None else 0.5 * (self.step_ms[ci] + ms)
            for (c, si), req in list(self.running.items()):
                if c != ci:
                    continue
                running, req.done_steps = self.ens.status(ci, si)
                if not running:
                    v = self.ens.views[(ci, si)]
                    req.steps_before += req.segment
                    if req.steps_before < req.nsteps:
                        req.ckpt = v.checkpoint(req.ts_end)
                        self.requeue.append(req)
                        self.preemptions += 1
                    else:
                        req.result = _result(v, req)
                        done.append(req)
                    self.ens.release(ci, si)
                    self.free[ci].append(si)
                    del self.running[(ci, si)]
        return done

    def launch(self):
        """Queue the next batch of every idle class that has running requests."""
        for ci in range(len(self.classes)):
            if self.busy[ci]:
                continue
            rem = [r.segment - r.done_steps for (c, _), r in self.running.items() if c == ci]
            if not rem:
                continue
            k = 1 if self.step_ms[ci] is None else int(self.batch_ms / max(self.step_ms[ci], 1e-3))
            k = max(1, min(k, self.max_batch, min(rem)))
            self.ens.step_class(ci, k)
            self.busy[ci] = True
            self.queued[ci] = k
            self.t_launch[ci] = time.perf_counter()
            self.steps[ci] += k


def serve(requests, hbm_budget: float = 40e9, device: int = 0, graph: bool = True, realtime: bool = True,
          max_slots: int = 64, segment_steps: int = None, **server_kw):
    """Run the request stream through a Server.  realtime: requests become
    visible at their arrival times (wall clock from the start); otherwise all
    are queued at t = 0 (saturated throughput).  segment_steps: pre-empt
    every request after that many steps (see Server); server_kw: the other
    Server settings (batch_ms, max_batch, step_ms).  Returns (requests with
    .latency and .result, makespan seconds, server stats)."""
    prepare_tables(requests)
    sizes = sorted({r.ng for r in requests})
    srv = Server(sizes, hbm_budget, device, graph, max_slots, segment_steps=segment_steps, **server_kw)
    try:
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        finished = []
        t0 = time.perf_counter()
        while len(finished) < len(requests):
            now = time.perf_counter() - t0
            while pending and (not realtime or pending[0].arrival <= now):
                waiting.append(pending.popleft())
            for r in srv.poll():
                r.finish = time.perf_counter() - t0
                r.latency = r.finish - (r.arrival if realtime else 0.0)
                finished.append(r)
            waiting.extend(srv.requeue)  # pre-empted: back of the queue
            # first come first served within what fits (a class takes new
            # requests between its batches)
            still = collections.deque()
            while waiting:
                r = waiting.popleft()
                if not srv.admit(r):
                    still.append(r)
            waiting = still
            srv.launch()
            if not srv.running and not waiting and pending:
                time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.01)))
        makespan = time.perf_counter() - t0
        return finished, makespan, {"ticks": max(srv.steps), "steps_per_class": list(srv.steps),
                                    "preemptions": srv.preemptions,
                                    "classes": srv.classes, "launches": srv.ens.kernel_launches()}
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
