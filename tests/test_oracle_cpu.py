"""CPU tests of the FP64 oracle against known answers and the reference's
own fixtures (no GPU)."""
import math
import os

import numpy as np
import pytest

from oracle import pm_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_reference_example_params_parse():
    p = O.read_params(os.path.join(GOLD, "ref_test_run_params"))
    assert (p.ng, p.np, p.nsteps, p.seed, p.block_size, p.pk_folds) == (32, 32, 625, 21082001, 64, 1)
    assert p.rl == 8.0 and p.z_ini == 200.0 and p.z_fin == 0.0
    assert p.omega_cdm == float(np.float32(0.22)) and p.hubble == float(np.float32(0.71))
    assert p.prefix == "runs/test3" and p.last_step == 625
    assert [i for i in range(1000) if p.pks[i]] == [0, 1, 3, 5, 10, 20, 30, 40, 59, 66, 74, 86, 101, 122, 153,
                                                     175, 205, 247, 310, 415, 610, 624]
    assert not any(p.dumps) and not p.dump_init and not p.dump_final
    assert p.omega_baryon == pytest.approx(p.deut / p.hubble ** 2, rel=1e-15)


def test_reference_example_ipk_header():
    h, t = O.read_ipk(os.path.join(GOLD, "ref_test_run_ipk.ipk"))
    assert h[0] == 0.0 and h[1] == 1000.0 and int(h[2]) == 20000 and t.size == 20000
    assert h[3] == pytest.approx(1000.0 / 19999.0, rel=1e-12)
    assert h[15] == 200.0 and np.all(t[1:] > 0)


def test_cic_single_particle_weights():
    ng = 8
    x = np.array([[1.25, 2.5, 7.75]])
    rho = O.cic_deposit(x, ng, 1.0)
    assert rho.sum() == pytest.approx(1.0, abs=1e-15)
    wx = {1: 0.75, 2: 0.25}
    wy = {2: 0.5, 3: 0.5}
    wz = {7: 0.25, 0: 0.75}  # periodic wrap of the +1 corner
    for i, a in wx.items():
        for j, b in wy.items():
            for k, c in wz.items():
                assert rho[i, j, k] == pytest.approx(a * b * c, abs=1e-15)
    assert np.count_nonzero(rho) == 8


def test_cic_mass_conservation_and_mean():
    ng = 16
    rng = np.random.default_rng(0)
    x = rng.uniform(0, ng, (8 ** 3, 3))
    rho = O.cic_deposit(x, ng, O.cic_mass(ng, 8))
    assert rho.mean() == pytest.approx(1.0, rel=1e-13)


@pytest.mark.parametrize("m", [1, 3])
def test_plane_wave_force_analytic(m):
    """rho = 1 + A cos(2 pi m x / ng): the discrete G and sin gradient give
    F_x = -(A/2) cot(pi m/ng) sin(2 pi m x/ng), F_y = F_z = 0."""
    ng, A = 32, 0.3
    xs = np.arange(ng)
    rho = 1 + A * np.cos(2 * np.pi * m * xs / ng)[:, None, None] * np.ones((1, ng, ng))
    f = O.solve_gradient(rho)
    expect = -(A / 2) / math.tan(math.pi * m / ng) * np.sin(2 * np.pi * m * xs / ng)
    assert np.allclose(f[0], expect[:, None, None], atol=1e-12)
    assert np.abs(f[1]).max() < 1e-12 and np.abs(f[2]).max() < 1e-12


def test_greens_quirk_is_small_but_nonzero():
    g = O.greens(64)
    q = O.greens(64, ref_quirks=True)
    rel = np.abs(q - g)[g != 0] / np.abs(g[g != 0])
    assert 0 < rel.max() < 1e-4


def test_growth_einstein_de_sitter_is_a():
    for a in (0.01, 0.1, 0.5):
        assert O.growth_delta(a, 1.0, 0.0, ref_quirks=False, bins=20000) == pytest.approx(a, rel=1e-6)


def test_timestepper_reaches_final_redshift():
    p = O.read_params(os.path.join(GOLD, "ref_test_run_params"))
    ts = O.Timestepper(p, ref_quirks=False)
    ts.set_initial_z(p.z_ini)
    ts.reverse_half_step()
    ts.advance_half_step()
    for _ in range(p.nsteps):
        ts.advance_half_step()
        ts.advance_half_step()
    assert ts.aa == pytest.approx(1.0 / (1.0 + p.z_fin), rel=1e-12)


PHILOX_KAT = [
    # Random123 known-answer vectors for philox4x32 with 10 rounds:
    # counter (4 words), key (2 words) -> output (4 words)
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def _philox4x32_10(ctr, key):
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF, ((p0 >> 32) ^ c3 ^ k1) & 0xFFFFFFFF, p0 & 0xFFFFFFFF
        k0, k1 = (k0 + W0) & 0xFFFFFFFF, (k1 + W1) & 0xFFFFFFFF
    return c0, c1, c2, c3


@pytest.mark.parametrize("ctr,key,out", PHILOX_KAT)
def test_philox_known_answers(ctr, key, out):
    assert _philox4x32_10(ctr, key) == out


def test_philox_normal_matches_scalar_restatement_and_moments():
    n = O.philox_normal(4096, 7)
    for i in (0, 1, 77, 4095):
        c = _philox4x32_10((i, 0, 0, 0), (7, 0x4850474D))
        u1 = (((c[0] >> 5) << 26 | (c[1] >> 6)) + 0.5) / 2.0 ** 53
        u2 = (((c[2] >> 5) << 26 | (c[3] >> 6)) + 0.5) / 2.0 ** 53
        assert n[i] == np.float32(math.sqrt(-2 * math.log(u1)) * math.cos(2 * math.pi * u2))
    big = O.philox_normal(1 << 18, 3).astype(np.float64)
    assert abs(big.mean()) < 0.01 and abs(big.std() - 1) < 0.01


def test_power_spectrum_counts_cover_all_modes():
    ng = 16
    rng = np.random.default_rng(2)
    x = rng.uniform(0, ng, (16 ** 3, 3))
    k, P, n = O.power_spectrum(x, ng, 16, 16.0, nbins=40)
    assert n.sum() == ng ** 3 - 2  # all modes but DC and the (ng/2)^3 corner
    assert np.all(np.diff(k) > 0)


def test_pk_lines_format():
    txt = O.format_pk_lines([0.1, 0.2, 0.3], [1.5, 0.0, float("nan")], [4, 3, 2])
    assert txt == "0.1,1.5,4\n"


def test_ic_zeldovich_displacement_is_gradient_of_potential():
    """The Zel'dovich field s = -i k delta/k^2 is curl free and its divergence
    is -delta/delta_growth (transform_density_field_initializer.cu:72-112)."""
    n, rl = 16, 32.0
    rng = np.random.default_rng(4)
    noise = rng.standard_normal((n, n, n))
    k = np.linspace(0, 10, 2000)
    table = 1.0 + 0.0 * k
    s = O.displacement_from_noise(noise, table, k[1] - k[0], rl, delta=2.0)
    kf = O.kmodes_f32(n, 2 * np.pi / rl).astype(np.float64)
    sk = [np.fft.fftn(s[d]) for d in range(3)]
    div = 1j * (kf[:, None, None] * sk[0] + kf[None, :, None] * sk[1] + kf[None, None, :] * sk[2])
    dk = np.fft.fftn(noise) * np.sqrt(O.interp_pk(table, k[1] - k[0], n, rl))
    # modes with a Nyquist component are not representable as real fields
    mask = np.ones((n, n, n), bool)
    for ax in range(3):
        sl = [slice(None)] * 3
        sl[ax] = n // 2
        mask[tuple(sl)] = False
    mask[0, 0, 0] = False
    assert np.allclose(div[mask], (dk / 2.0)[mask], rtol=1e-6, atol=1e-9 * np.abs(dk).max())


@pytest.mark.parametrize("fold", [1, 2, 3])
def test_fold_positions_is_doubling_mod_ng(fold):
    """foldParticles (fold_particles_power.cu:3-27) applied `fold` times is
    x -> 2^fold x mod ng; exact for dyadic positions."""
    ng = 32
    rng = np.random.default_rng(5)
    x = np.floor(rng.uniform(0, ng, (500, 3)) * 256) / 256.0
    y = O.fold_positions(x, ng, fold)
    assert np.array_equal(y, np.mod(x * 2 ** fold, ng))
    assert (y >= 0).all() and (y < ng).all()


def test_folded_pk_quirk_bins_drop_modes_below_the_first_edge():
    """With the reference's bins (edges from the most folded box) the low-k
    modes of an unfolded P(k) fall before bin 0: those less than one bin
    below land in bin 0 (truncation), the rest are dropped; with the fold's
    own bins every mode but DC and the corner is binned."""
    ng = 16
    rng = np.random.default_rng(9)
    x = rng.uniform(0, ng, (ng ** 3, 3))
    _, _, nq = O.power_spectrum(x, ng, ng, 16.0, 32, folds=2, fold=0, ref_quirks=True)
    _, _, nc = O.power_spectrum(x, ng, ng, 16.0, 32, folds=2, fold=0, ref_quirks=False)
    assert nc.sum() == ng ** 3 - 2
    assert 0 < nq.sum() < nc.sum()
    d = 2 * np.pi / 16.0
    min_k, delta, _ = O.pk_bin_edges(ng, 16.0, 32, 2)
    assert min_k == pytest.approx(4 * d)
    kf = O.kmodes_f32(ng, d).astype(np.float64)
    kk = np.sqrt(kf[:, None, None] ** 2 + kf[None, :, None] ** 2 + kf[None, None, :] ** 2)
    keep = (kk - min_k) / delta > -1.0
    keep[0, 0, 0] = keep[ng // 2, ng // 2, ng // 2] = False
    keep &= np.trunc((kk - min_k) / delta) < 32
    assert nq.sum() == keep.sum()
