"""GPU parity of whole PM steps, P(k) and the IC pipeline against the FP64
oracle, through the C-ABI.

Bars: final positions within 1e-4 of the box side after N steps (north
star), P(k) within 0.1 % per bin with identical mode counts, IC positions
and velocities within float rounding, whole steps bit-exact run to run.
"""
import numpy as np
import pytest

import hacc_gpm_b200 as H
from oracle import pm_oracle as O
from tests.helpers import PK_RTOL, POS_BOX_TOL, box_pos_err, oracle_ics, params_text, rel_max_err

pytestmark = pytest.mark.gpu


def _pair(ng, np_side=None, rl=None, z_ini=50.0, nsteps=100, extra=""):
    # N_STEPS sets the step size (a run of nsteps from z_ini to 0); tests run fewer
    txt = params_text(ng, np_side, rl, z_ini=z_ini, nsteps=nsteps, extra=extra)
    return H.parse_params(txt), O.parse_params_text(txt)


@pytest.mark.parametrize("ng,np_side,rl,z,n", [(32, 32, 32.0, 50.0, 10), (48, 48, 96.0, 100.0, 8),
                                               (64, 32, 64.0, 50.0, 5), (32, 64, 32.0, 50.0, 5),
                                               (40, 40, 40.0, 50.0, 6), (80, 40, 160.0, 50.0, 5),
                                               (160, 80, 160.0, 50.0, 4)])
def test_run_steps_match_oracle(ng, np_side, rl, z, n):
    hp, op = _pair(ng, np_side, rl, z_ini=z)
    x0, v0, *_ = oracle_ics(op)
    with H.Simulation(hp) as s:
        s.load_state(x0, v0)
        ts = H.Timestepper(hp)
        ts.set_initial_z(hp.z_ini)
        ts.reverse_half_step()
        ts.advance_half_step()
        s.run_steps(ts, n)
        xg, vg = s.store_state()
    xo, vo, tso = O.run(x0.astype(np.float64), v0.astype(np.float64), op, n)
    assert ts.aa == pytest.approx(tso.aa, rel=1e-14)
    assert box_pos_err(xg, xo, ng) < POS_BOX_TOL
    assert rel_max_err(vg, vo) < 1e-3


def test_run_steps_equals_unfused_phase_calls():
    """hgpm_run_steps (fused kick + two drifts) against the reference's call
    sequence driver_pm.cpp:114-125 issued phase by phase."""
    hp, op = _pair(32)
    x0, v0, *_ = oracle_ics(op)
    with H.Simulation(hp) as a, H.Simulation(hp) as b:
        ta, tb = H.Timestepper(hp), H.Timestepper(hp)
        for s, t in ((a, ta), (b, tb)):
            s.load_state(x0, v0)
            t.set_initial_z(hp.z_ini)
            t.reverse_half_step()
            t.advance_half_step()
        a.run_steps(ta, 6)
        for _ in range(6):
            b.update_positions(tb, 0.5)
            b.cic()
            b.solve_gradient()
            tb.advance_half_step()
            b.update_velocities(tb)
            tb.advance_half_step()
            b.update_positions(tb, 0.5)
        xa, va = a.store_state()
        xb, vb = b.store_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_whole_step_deterministic():
    hp, op = _pair(48)
    x0, v0, *_ = oracle_ics(op)
    outs = []
    for _ in range(2):
        with H.Simulation(hp) as s:
            s.load_state(x0, v0)
            ts = H.Timestepper(hp)
            ts.set_initial_z(hp.z_ini)
            ts.reverse_half_step()
            ts.advance_half_step()
            s.run_steps(ts, 4)
            outs.append(s.store_state())
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("ng,nbins,log_bins", [(32, 221, False), (48, 40, False), (64, 32, True), (40, 60, False)])
def test_power_spectrum_matches_oracle(ng, nbins, log_bins):
    hp, op = _pair(ng, rl=2.0 * ng, z_ini=20.0)
    x0, v0, *_ = oracle_ics(op)
    with H.Simulation(hp) as s:
        s.load_state(x0, v0)
        k, P, n = s.power_spectrum(nbins, log_bins)
    if log_bins:
        # oracle restated with log edges
        xo = x0.astype(np.float64)
        rho = O.cic_deposit(xo, ng, O.cic_mass(ng, ng))
        rk = np.fft.fftn(rho)
        pw = (rk.real ** 2 + rk.imag ** 2) * (1.0 / ng ** 3) * (op.rl / ng) * O.pk_cic_filter(ng)
        d = 2 * np.pi / op.rl
        kf = O.kmodes_f32(ng, d).astype(np.float64)
        kk = np.sqrt(kf[:, None, None] ** 2 + kf[None, :, None] ** 2 + kf[None, None, :] ** 2)
        maxk = np.sqrt(3 * ((ng // 2) ** 2 * d * d))
        dl = np.log(maxk / d) / nbins
        with np.errstate(divide="ignore"):
            b = np.trunc(np.log(kk / d) / dl)  # (int) truncation, as the kernel
        m = np.ones_like(kk, bool)
        m[0, 0, 0] = False
        m[ng // 2, ng // 2, ng // 2] = False
        m &= (b >= 0) & (b < nbins)
        no = np.bincount(b[m].astype(int), minlength=nbins)
        so = np.bincount(b[m].astype(int), weights=pw[m], minlength=nbins)
        with np.errstate(invalid="ignore"):
            Po = so / no
    else:
        ko, Po, no = O.power_spectrum(x0.astype(np.float64), ng, ng, op.rl, nbins)
        assert np.allclose(k, ko, rtol=1e-12)
    assert np.array_equal(n, no)
    ok = no > 0
    assert np.max(np.abs(P[ok] / Po[ok] - 1)) < PK_RTOL


@pytest.mark.parametrize("ng,fold,quirks", [(32, 1, True), (32, 2, True), (48, 1, False), (32, 2, False)])
def test_folded_power_spectrum_matches_oracle(ng, fold, quirks):
    """One fold of GetPowerSpectrum's PK_FOLDS loop: positions folded `fold`
    times (x -> 2x mod ng), binned with the reference's edges (from the most
    folded box, unfolded scale) or the fold's own box."""
    hp, op = _pair(ng, rl=2.0 * ng, z_ini=20.0, extra="PK_FOLDS 2\nREF_QUIRKS %d\n" % int(quirks))
    x0, v0, *_ = oracle_ics(op)
    with H.Simulation(hp) as s:
        s.load_state(x0, v0)
        k, P, n = s.power_spectrum(64, fold=fold)
        x1, _ = s.store_state()
    ko, Po, no = O.power_spectrum(x0.astype(np.float64), ng, ng, op.rl, 64, folds=2, fold=fold, ref_quirks=quirks)
    assert np.array_equal(x1, x0)  # the state is not folded
    assert np.allclose(k, ko, rtol=1e-12)
    assert np.array_equal(n, no) and n.sum() > 0
    ok = no > 0
    assert np.max(np.abs(P[ok] / Po[ok] - 1)) < PK_RTOL


def test_power_spectrum_deterministic_and_leaves_state():
    hp, op = _pair(32)
    x0, v0, *_ = oracle_ics(op)
    with H.Simulation(hp) as s:
        s.load_state(x0, v0)
        a = s.power_spectrum()
        b = s.power_spectrum()
        x1, v1 = s.store_state()
    for u, w in zip(a, b):
        assert np.array_equal(u, w)
    assert np.array_equal(x1, x0) and np.array_equal(v1, v0)


@pytest.mark.parametrize("ng,np_side,rl", [(32, 32, 32.0), (48, 48, 64.0), (64, 32, 128.0), (32, 64, 64.0),
                                         (40, 40, 80.0), (80, 80, 80.0)])
def test_ic_from_noise_matches_oracle(ng, np_side, rl):
    hp, op = _pair(ng, np_side, rl, z_ini=50.0)
    xo, vo, noise, table, header = oracle_ics(op)
    with H.Simulation(hp) as s:
        s.ic_from_noise(noise, table, header[3])
        xg, vg = s.store_state()
    assert box_pos_err(xg, xo, ng) < 1e-6
    assert rel_max_err(vg, vo) < 1e-5


def test_ic_philox_noise_matches_oracle():
    hp, op = _pair(32, extra="NOISE PHILOX\n")
    assert hp.noise == 1
    with H.Simulation(hp) as s:
        g = s.ic_noise().reshape(-1)
    o = O.philox_normal(32 ** 3, op.seed)
    assert np.abs(g - o).max() <= 2 * np.finfo(np.float32).eps * np.abs(o).max()


def test_ic_generate_equals_from_noise():
    hp, op = _pair(32)
    _, _, noise, table, header = oracle_ics(op)
    with H.Simulation(hp) as a, H.Simulation(hp) as b:
        a.generate_ic(table, header[3])
        b.ic_from_noise(a.ic_noise(), table, header[3])
        xa, va = a.store_state()
        xb, vb = b.store_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)


def test_ic_table_too_short_is_an_error():
    hp, op = _pair(32, rl=8.0)
    k = np.linspace(0, 1.0, 100)
    with H.Simulation(hp) as s:
        with pytest.raises(H.HgpmError, match="ipk"):
            s.generate_ic(np.ones(100), k[1] - k[0])


def test_checkpoint_resume_is_bit_identical(tmp_path):
    """s steps, checkpoint to a host buffer, restore in a fresh context and n
    more steps equal s + n steps at once; the float3 dump reader restores
    exactly what the dump holds."""
    hp, op = _pair(32)
    x0, v0, *_ = oracle_ics(op)

    def ts0():
        t = H.Timestepper(hp)
        t.set_initial_z(hp.z_ini)
        t.reverse_half_step()
        t.advance_half_step()
        return t

    with H.Simulation(hp) as a:
        a.load_state(x0, v0)
        ta = ts0()
        a.run_steps(ta, 7)
        xa, va = a.store_state()
    with H.Simulation(hp) as b:
        b.load_state(x0, v0)
        tb = ts0()
        b.run_steps(tb, 3)
        buf = b.checkpoint(tb)
        b.write_output(str(tmp_path / "dump"))
        xd, vd = b.store_state()
    with H.Simulation(hp) as c:
        tc = c.restore(buf)
        assert tc.aa == tb.aa
        c.run_steps(tc, 4)
        xc, vc = c.store_state()
        c.read_output(str(tmp_path / "dump"))
        xr, vr = c.store_state()
    assert np.array_equal(xa, xc) and np.array_equal(va, vc)
    assert np.array_equal(xr, xd) and np.array_equal(vr, vd)
    hp48, _ = _pair(48)
    with H.Simulation(hp48) as d:
        with pytest.raises(H.HgpmError, match="does not fit"):
            d.restore(buf)


def test_step_host_roundtrip_equals_device_resident():
    hp, op = _pair(32)
    x0, v0, *_ = oracle_ics(op)
    with H.Simulation(hp) as a, H.Simulation(hp) as b:
        ta, tb = H.Timestepper(hp), H.Timestepper(hp)
        for t in (ta, tb):
            t.set_initial_z(hp.z_ini)
            t.reverse_half_step()
            t.advance_half_step()
        a.load_state(x0, v0)
        a.run_steps(ta, 3)
        xa, va = a.store_state()
        xh, vh = x0.copy(), v0.copy()
        for _ in range(3):
            b.step_host(tb, xh, vh)
    # host round trips re-split positions from float3 each step, so agree to
    # float rounding of the position, not bit for bit
    assert box_pos_err(xh, xa, 32) < 1e-6
    assert rel_max_err(vh, va) < 1e-5
