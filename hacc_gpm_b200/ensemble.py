"""Batched ensembles of PM boxes (C-ABI ``hgpm_ens_*``).

Many boxes of mixed grid sizes advance together: every PM phase is ONE
kernel launch per size class covering all of the class's boxes, classes run
on parallel streams, and a step can be replayed from one CUDA graph.  Each
box keeps its own cosmology, seed, box size and step count; its results are
bit-identical to running it alone through ``Simulation.run_steps``.

``Box`` describes one run, ``run_batched`` runs a list of boxes as one
ensemble, ``run_serial`` runs them one at a time through the plain step (the
comparison the batched form is measured against).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import ipk as ipkmod
from .binding import HgpmError, Params, Simulation, Timestepper, lib, parse_params


@dataclass
class Box:
    """One simulation request: flat LCDM, EH no-wiggle ICs, steps uniform in a.

    nsteps: steps run.  n_total: N_STEPS of the params, which sets the step
    size (z_ini -> 0 in n_total steps); 0 means nsteps.  A run much shorter
    than its z_ini needs a finer step grid: the reference's IC velocities are
    taken at a_ini - da/2, which must stay positive."""
    ng: int
    rl: float
    seed: int
    nsteps: int
    n_total: int = 0
    z_ini: float = 100.0
    sigma8: float = 0.81
    omega_m: float = 0.31
    np_side: int = 0          # 0: np = ng
    pk_bins: int = 32
    tag: object = None
    table: np.ndarray = field(default=None, repr=False)
    k_delta: float = 0.0

    def params_text(self) -> str:
        return ipkmod.lcdm_params_text(self.ng, self.np_side or self.ng, self.rl, self.z_ini,
                                       self.n_total or self.nsteps, seed=self.seed, omega_m=self.omega_m,
                                       sigma8=self.sigma8)

    def params(self) -> Params:
        return parse_params(self.params_text())


def prepare_tables(boxes):
    """Fill each box's P(k) table (the .ipk body: EH no-wiggle normalised to
    its sigma8, at its z_ini) on the host, covering the grid's largest |k|."""
    for b in boxes:
        if b.table is None:
            n = b.np_side or b.ng
            k_max = np.sqrt(3.0) * (n / 2) * 2 * np.pi / b.rl * 1.05 + 0.1
            header, table = ipkmod.make_ipk(ipkmod.cosmo_from_params(b.params()), b.z_ini, k_max=k_max, k_bins=4000)
            b.table, b.k_delta = table, float(header[3])
    return boxes


def _ts_for(params: Params) -> Timestepper:
    ts = Timestepper(params)
    ts.set_initial_z(params.z_ini)
    ts.reverse_half_step()
    ts.advance_half_step()
    return ts


class Ensemble:
    """Size classes of slots on one GPU (``hgpm_ensemble``)."""

    def __init__(self, classes, device: int = 0, graph: bool = True, multi: bool = True):
        """classes: list of (ng, np, nslots).  multi: one launch per phase
        across all classes where every class allows it (hgpm_ens_multi_launch),
        else one per phase per class; ``self.multi`` says which runs."""
        self.L = lib()
        self.classes = [(int(a), int(b), int(c)) for a, b, c in classes]
        n = len(self.classes)
        ng = (C.c_int * n)(*[c[0] for c in self.classes])
        npp = (C.c_int * n)(*[c[1] for c in self.classes])
        ns = (C.c_int * n)(*[c[2] for c in self.classes])
        h = C.c_void_p()
        rc = self.L.hgpm_ens_create(n, ng, npp, ns, device, C.byref(h))
        self._h = h
        if rc:
            msg = self.L.hgpm_ens_last_error(h).decode() if h.value else ""
            self.close()
            raise HgpmError("hgpm_ens_create status %d: %s" % (rc, msg))
        self.views = {}
        rc = self.L.hgpm_ens_multi_launch(self._h, 1 if multi else 0)
        if rc < 0:
            self._ck(rc)
        self.multi = rc == 1
        if graph:
            self._ck(self.L.hgpm_ens_use_graph(self._h, 1))

    def _ck(self, rc):
        if rc:
            raise HgpmError("hgpm_ens status %d: %s" % (rc, self.L.hgpm_ens_last_error(self._h).decode()))

    def close(self):
        if getattr(self, "_h", None):
            self.L.hgpm_ens_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def footprint_bytes(ng: int, np_side: int, nslots: int) -> int:
        return lib().hgpm_ens_footprint_bytes(ng, np_side, nslots)

    def slot(self, cls: int, slot: int, params: Params) -> Simulation:
        """Bind params to a slot; the slot as a (borrowed) Simulation."""
        v = C.c_void_p()
        self._ck(self.L.hgpm_ens_slot(self._h, cls, slot, C.byref(params._raw), C.byref(v)))
        sim = Simulation._borrow(v, params)
        self.views[(cls, slot)] = sim
        return sim

    def start(self, cls: int, slot: int, ts: Timestepper, nsteps: int):
        self._ck(self.L.hgpm_ens_start(self._h, cls, slot, C.byref(ts._raw), nsteps))

    def release(self, cls: int, slot: int):
        self._ck(self.L.hgpm_ens_release(self._h, cls, slot))

    def step(self, n: int = 1):
        self._ck(self.L.hgpm_ens_step(self._h, n))

    def sync(self):
        self._ck(self.L.hgpm_ens_sync(self._h))

    def step_class(self, cls: int, n: int = 1):
        """n steps of one class on its own stream (returns at once)."""
        self._ck(self.L.hgpm_ens_step_class(self._h, cls, n))

    def class_done(self, cls: int) -> bool:
        d = C.c_int()
        self._ck(self.L.hgpm_ens_class_done(self._h, cls, C.byref(d)))
        return bool(d.value)

    def sync_class(self, cls: int):
        self._ck(self.L.hgpm_ens_sync_class(self._h, cls))

    def status(self, cls: int, slot: int):
        r, d = C.c_int(), C.c_int()
        self._ck(self.L.hgpm_ens_status(self._h, cls, slot, C.byref(r), C.byref(d)))
        return bool(r.value), d.value

    def kernel_launches(self, reset=False) -> int:
        return self.L.hgpm_ens_kernel_launches(self._h, int(reset))


def _result(sim: Simulation, box: Box):
    k, P, n = sim.power_spectrum(box.pk_bins)
    return {"k": k, "P": P, "n": n}


class _Clock:
    """Wall-clock seconds per stage (synchronising before each reading)."""

    def __init__(self, sync):
        self.sync = sync
        self.t = {}
        self.last = time.perf_counter()

    def mark(self, name):
        self.sync()
        now = time.perf_counter()
        self.t[name] = self.t.get(name, 0.0) + now - self.last
        self.last = now


def run_serial(boxes, device: int = 0, keep_state: bool = False, stages: dict = None):
    """Each box alone: its own context, ICs, run_steps, P(k) (the plain step).
    stages (optional dict) receives seconds per stage."""
    out = []
    clk = None
    for b in boxes:
        p = b.params()
        with Simulation(p, device=device) as s:
            if stages is not None:
                clk = clk or _Clock(s.sync)
                clk.sync = s.sync
                clk.mark("create")
            s.generate_ic(b.table, b.k_delta)
            if clk:
                clk.mark("ics")
            ts = _ts_for(p)
            s.run_steps(ts, b.nsteps)
            if clk:
                clk.mark("steps")
            r = _result(s, b)
            if keep_state:
                r["x"], r["v"] = s.store_state()
            if clk:
                clk.mark("pk")
        out.append(r)
    if stages is not None and clk:
        stages.update(clk.t)
    return out


def class_layout(boxes):
    """Size classes (ng, np, nslots) holding every box at once, and each box's
    (class, slot)."""
    keys = sorted({(b.ng, b.np_side or b.ng) for b in boxes})
    count = {k: 0 for k in keys}
    where = []
    for b in boxes:
        k = (b.ng, b.np_side or b.ng)
        where.append((keys.index(k), count[k]))
        count[k] += 1
    return [(k[0], k[1], count[k]) for k in keys], where


def run_batched(boxes, device: int = 0, graph: bool = True, keep_state: bool = False, ens: Ensemble = None,
                stages: dict = None, multi: bool = True):
    """All boxes as one ensemble: ICs per slot, batched steps until every box
    has run its steps, then P(k) per slot.  stages (optional dict) receives
    seconds per stage; multi: one launch per phase across the classes where
    they allow it (Ensemble)."""
    classes, where = class_layout(boxes)
    own = ens is None
    t0 = time.perf_counter()
    ens = ens or Ensemble(classes, device=device, graph=graph, multi=multi)
    clk = _Clock(ens.sync) if stages is not None else None
    if clk:
        clk.last = t0
        clk.mark("create")
    try:
        for b, (ci, si) in zip(boxes, where):
            p = b.params()
            v = ens.slot(ci, si, p)
            v.generate_ic(b.table, b.k_delta)
            ens.start(ci, si, _ts_for(p), b.nsteps)
        if clk:
            clk.mark("ics")
        ens.step(max(b.nsteps for b in boxes))
        ens.sync()
        if clk:
            clk.mark("steps")
        out = []
        for b, (ci, si) in zip(boxes, where):
            running, done = ens.status(ci, si)
            if running or done != b.nsteps:
                raise HgpmError("slot (%d, %d) ran %d of %d steps" % (ci, si, done, b.nsteps))
            v = ens.views[(ci, si)]
            r = _result(v, b)
            if keep_state:
                r["x"], r["v"] = v.store_state()
            ens.release(ci, si)
            out.append(r)
        if clk:
            clk.mark("pk")
            stages.update(clk.t)
        return out
    finally:
        if own:
            ens.close()


def shard(boxes, rank: int, world: int):
    """This rank's share of an ensemble (or a request stream) on `world` GPUs
    (replicas: whole boxes per GPU, split by predicted cost; no collective on
    the data path).  Every rank computes the same split."""
    from .replicas import box_cost, partition

    parts = partition([box_cost(b.ng, b.np_side or b.ng, b.nsteps) for b in boxes], world)
    return [boxes[i] for i in parts[rank]]


def ensemble_boxes(n: int = 96, master_seed: int = 20240601, sizes=(32, 48, 64, 96, 128), nsteps: int = 64,
                   z_ini: float = 100.0):
    """The batched-ensemble workload: n boxes, ng = np uniform over sizes,
    L ~ U[64, 512] Mpc/h, sigma8 ~ U[0.7, 0.9], seed 1000 + i, z_ini 100,
    nsteps steps each."""
    rng = np.random.default_rng(master_seed)
    boxes = []
    for i in range(n):
        boxes.append(Box(ng=int(rng.choice(sizes)), rl=float(rng.uniform(64.0, 512.0)), seed=1000 + i,
                         nsteps=nsteps, z_ini=z_ini, sigma8=float(rng.uniform(0.7, 0.9)), tag=i))
    return boxes


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0
