"""Batched ensembles and the serving loop on the GPU: every box's final state
and P(k) are bit-identical to the same box run alone through the plain step,
with mixed sizes, box lengths, cosmologies and step counts, with and without
the CUDA graph, and for requests admitted while others run."""
import numpy as np
import pytest

import hacc_gpm_b200 as H
from hacc_gpm_b200 import ensemble as E
from hacc_gpm_b200 import serve as S

pytestmark = pytest.mark.gpu


def _boxes():
    spec = [(32, 40.0, 7), (48, 96.0, 5), (32, 64.0, 9), (64, 128.0, 4), (48, 50.0, 6), (32, 32.0, 3)]
    boxes = [E.Box(ng=ng, rl=rl, seed=300 + i, nsteps=n, n_total=100, z_ini=100.0, sigma8=0.75 + 0.02 * i,
                   omega_m=0.28 + 0.01 * i) for i, (ng, rl, n) in enumerate(spec)]
    return E.prepare_tables(boxes)


def _same(a, b):
    assert np.isfinite(a["x"]).all() and np.isfinite(a["v"]).all()
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["v"], b["v"])
    assert np.array_equal(a["n"], b["n"]) and np.array_equal(a["P"], b["P"])


@pytest.mark.parametrize("graph,multi", [(True, True), (False, True), (True, False), (False, False)])
def test_batched_equals_alone(graph, multi):
    """Batched steps, as one launch per phase across all classes (multi) or
    one per phase per class, give every box its state and P(k) alone."""
    boxes = _boxes()
    alone = E.run_serial(boxes, keep_state=True)
    batched = E.run_batched(boxes, graph=graph, keep_state=True, multi=multi)
    for a, b in zip(alone, batched):
        _same(a, b)


def test_multi_class_step_launches():
    """The multi-class step is ten launches whatever the number of classes
    (here three); the per-class step launches every phase once per class."""
    boxes = _boxes()
    classes, where = E.class_layout(boxes)
    assert len(classes) == 3
    counts = {}
    for multi in (True, False):
        with E.Ensemble(classes, graph=False, multi=multi) as ens:
            assert ens.multi == multi
            for b, (ci, si) in zip(boxes, where):
                p = b.params()
                ens.slot(ci, si, p).generate_ic(b.table, b.k_delta)
                ens.start(ci, si, E._ts_for(p), b.nsteps)
            ens.kernel_launches(reset=True)
            ens.step(2)
            ens.sync()
            counts[multi] = ens.kernel_launches()
    assert counts[True] == 2 * 10
    assert counts[False] > counts[True]


@pytest.mark.parametrize("graph", [True, False])
def test_per_class_stepping_equals_alone(graph):
    """Classes advanced one at a time on their own streams, in batches of
    different sizes and interleaved, give each box the state and P(k) of the
    box run alone."""
    boxes = _boxes()
    alone = E.run_serial(boxes, keep_state=True)
    classes, where = E.class_layout(boxes)
    with E.Ensemble(classes, graph=graph) as ens:
        for b, (ci, si) in zip(boxes, where):
            p = b.params()
            ens.slot(ci, si, p).generate_ic(b.table, b.k_delta)
            ens.start(ci, si, E._ts_for(p), b.nsteps)
        left = {ci: max(b.nsteps for b, (c, _) in zip(boxes, where) if c == ci) for ci in range(len(classes))}
        batch = {ci: 1 + ci for ci in left}
        while any(left.values()):
            for ci in left:
                if left[ci] and ens.class_done(ci):
                    k = min(batch[ci], left[ci])
                    ens.step_class(ci, k)
                    left[ci] -= k
        got = []
        for ci in range(len(classes)):
            ens.sync_class(ci)
        for b, (ci, si) in zip(boxes, where):
            assert ens.status(ci, si) == (False, b.nsteps)
            v = ens.views[(ci, si)]
            r = E._result(v, b)
            r["x"], r["v"] = v.store_state()
            got.append(r)
    for a, b in zip(alone, got):
        _same(a, b)


def test_serving_preemption_equals_alone():
    """Requests pre-empted every 4 steps (checkpoint to host, slot freed,
    resumed later from the checkpoint) end bit-identical to runs alone."""
    reqs = S.request_stream(8, rate=500.0, seed=13, sizes=(32, 48), steps=(5, 11))
    got, _, stats = S.serve(reqs, hbm_budget=1e9, realtime=False, max_slots=2, segment_steps=4)
    assert len(got) == 8 and stats["preemptions"] >= 8
    alone, _ = S.serve_one_at_a_time(S.request_stream(8, rate=500.0, seed=13, sizes=(32, 48), steps=(5, 11)),
                                     realtime=False)
    by_tag = {r.tag: r for r in got}
    for r in alone:
        g = by_tag[r.tag].result
        assert np.array_equal(g["n"], r.result["n"]) and np.array_equal(g["P"], r.result["P"])


def test_slot_reuse_and_errors():
    boxes = _boxes()[:2]
    classes, _ = E.class_layout(boxes)
    with E.Ensemble([(32, 32, 1), (48, 48, 1)]) as ens:
        with pytest.raises(H.HgpmError, match="do not fit"):
            ens.slot(0, 0, boxes[1].params())
        v = ens.slot(0, 0, boxes[0].params())
        ts = E._ts_for(boxes[0].params())
        with pytest.raises(H.HgpmError, match="no particle state"):
            ens.start(0, 0, ts, 3)
        first = E.run_batched(boxes, keep_state=True, ens=ens)
        again = E.run_batched(boxes, keep_state=True, ens=ens)  # slots released and reused
        for a, b in zip(first, again):
            _same(a, b)
        v.generate_ic(boxes[0].table, boxes[0].k_delta)
        ens.start(0, 0, E._ts_for(boxes[0].params()), 3)
        with pytest.raises(H.HgpmError, match="still has steps"):
            ens.release(0, 0)
        ens.step(3)
        ens.sync()
        assert ens.status(0, 0) == (False, 3)
        ens.release(0, 0)


def test_serving_mix_equals_alone():
    reqs = S.request_stream(14, rate=200.0, seed=11, sizes=(32, 48, 64), steps=(3, 12))
    # two slots per class: later requests are admitted as earlier ones finish,
    # into slots of a class whose other slot is mid-run
    got, makespan, stats = S.serve(reqs, hbm_budget=2e9, realtime=False, max_slots=2)
    assert len(got) == 14 and stats["ticks"] >= max(r.nsteps for r in reqs)
    ref = S.request_stream(14, rate=200.0, seed=11, sizes=(32, 48, 64), steps=(3, 12))
    alone, _ = S.serve_one_at_a_time(ref, realtime=False)
    by_tag = {r.tag: r for r in got}
    for r in alone:
        g = by_tag[r.tag].result
        assert np.array_equal(g["n"], r.result["n"]) and np.array_equal(g["P"], r.result["P"])
