"""Host logic of the batched ensemble and the serving loop (no kernels):
slot layout, the request stream, capacity by footprint, argument checks."""
import numpy as np
import pytest

import hacc_gpm_b200 as H
from hacc_gpm_b200 import ensemble as E
from hacc_gpm_b200 import serve as S


def test_class_layout_covers_every_box_once():
    boxes = E.ensemble_boxes(96)
    classes, where = E.class_layout(boxes)
    assert [c[0] for c in classes] == sorted({b.ng for b in boxes})
    assert sum(c[2] for c in classes) == 96
    assert len(set(where)) == 96
    for b, (ci, si) in zip(boxes, where):
        assert classes[ci][0] == b.ng and 0 <= si < classes[ci][2]


def test_ensemble_workload_distribution():
    boxes = E.ensemble_boxes(96)
    assert all(b.ng in (32, 48, 64, 96, 128) and 64 <= b.rl <= 512 and 0.7 <= b.sigma8 <= 0.9 for b in boxes)
    assert [b.seed for b in boxes] == list(range(1000, 1096))
    assert all(b.nsteps == 64 and b.z_ini == 100.0 for b in boxes)
    assert E.ensemble_boxes(96)[5].rl == boxes[5].rl  # seeded


def test_tables_cover_grid():
    b = E.ensemble_boxes(3)[0]
    E.prepare_tables([b])
    kmax_grid = np.sqrt(3.0) * (b.ng / 2) * 2 * np.pi / b.rl
    assert b.k_delta * (len(b.table) - 1) > kmax_grid


def test_request_stream():
    reqs = S.request_stream(400, rate=20.0, seed=7)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0)
    assert 15.0 < len(reqs) / t[-1] < 25.0  # mean rate 20/s
    assert {r.ng for r in reqs} <= {32, 48, 64, 96, 128, 192, 256}
    assert all(20 <= r.nsteps <= 200 and 0.25 <= r.omega_m <= 0.35 and 0.7 <= r.sigma8 <= 0.9 for r in reqs)
    assert len({r.seed for r in reqs}) == 400


def test_capacity_by_footprint():
    caps = S.class_capacity([32, 64, 128, 256], 8e9, max_slots=64)
    per = [E.Ensemble.footprint_bytes(ng, npp, 1) for ng, npp, _ in caps]
    used = sum(n * f for (_, _, n), f in zip(caps, per))
    assert all(1 <= n <= 64 for _, _, n in caps) and used <= 8e9
    assert [c[2] for c in caps] == sorted([c[2] for c in caps], reverse=True)
    # what the small classes cannot use goes to the large ones: no class
    # below its cap could still take a slot from what is left
    assert all(n == 64 or f > 8e9 - used for (_, _, n), f in zip(caps, per))
    assert caps[2][2] > 2e9 // per[2]
    # every slot carries a box's whole device state: particles, int64
    # density, four half spectra and the float4 force grid
    n = 64
    per_slot = (E.Ensemble.footprint_bytes(n, n, 8) - E.Ensemble.footprint_bytes(n, n, 4)) / 4
    state = 28 * n ** 3 + 8 * n ** 3 + 4 * 8 * n * n * ((n // 2 + 1 + 15) // 16 * 16) + 16 * n ** 3
    assert per_slot >= state
    assert H.footprint_bytes(n, n) >= state


def test_capacity_refuses_a_budget_below_one_slot_each():
    per = E.Ensemble.footprint_bytes(256, 256, 1)
    with pytest.raises(ValueError, match="budget"):
        S.class_capacity([32, 256], per * 0.5)
    caps = S.class_capacity([32, 256], per * 1.5)
    assert [c[2] for c in caps][1] == 1 and caps[0][2] >= 1


def test_bad_class_rejected_without_gpu():
    with pytest.raises(H.HgpmError, match="NG/NP must be one of"):
        E.Ensemble([(20, 20, 2)])


def test_capacity_capped_by_batched_step_time():
    """With step_ms the large classes hold only the slots whose batched step
    takes about that long (256^3: ~0.7 ms each, so 3 at 2 ms); the small
    classes keep their memory share."""
    sizes = (32, 64, 128, 256)
    free = S.class_capacity(sizes, 40e9, max_slots=64)
    capped = S.class_capacity(sizes, 40e9, max_slots=64, step_ms=2.0)
    by = {ng: n for ng, _, n in capped}
    for ng in (128, 256):
        assert by[ng] == round(2.0 / (S.STEP_MS_PER_UNIT * 2 * ng ** 3))
    assert by[256] == 3
    assert by[32] == 64 and by[64] == 64
    assert all(c[2] <= f[2] for c, f in zip(capped, free))
