"""Reference match: the B200 path against outputs of the reference's own
serial CUDA path on identical inputs (its cuRAND noise and its ICs), through
the C-ABI.  Bars in tests/refgpu.py (1e-5 on fields, 1e-4 of the box on
positions after N steps, 0.1 % per P(k) bin)."""
import numpy as np
import pytest

import hacc_gpm_b200 as H
from oracle import pm_oracle as O
from tests import refgpu as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=R.CASES)
def case(request):
    return R.Case(request.param)


def _sim(case):
    return H.Simulation(H.parse_params(case.params_text))


def test_ics_from_reference_noise(case):
    with _sim(case) as s:
        s.ic_from_noise(case["noise"], case.ipk_table, case.ipk_header[3])
        x, v = s.store_state()
    assert np.abs(O.periodic_diff(x, case["ics_x"], case.ng)).max() < R.IC_POS_CELLS
    assert np.abs(v - case["ics_v"]).max() / np.abs(case["ics_v"]).max() < R.IC_VEL_REL


def test_curand_noise_is_the_references(case):
    """Default NOISE (CURAND): the same SEED draws the reference's white
    noise bit for bit (rng_initializer.cu:38-49)."""
    with _sim(case) as s:
        assert s.params.noise == 0
        g = s.ic_noise().reshape(case["noise"].shape)
    assert np.array_equal(g, case["noise"])


def test_curand_noise_of_a_larger_box_starts_with_the_references():
    """A cell's draw depends only on SEED and its linear index (its state is
    curand_init(seed, cell, 0)), so the first 32^3 cells of a 128^3 box's
    noise are the reference's 32^3 noise; at 128^3 each thread draws 8 cells,
    reaching each next one by skipahead_sequence, where 32^3 draws one."""
    case = R.Case("a32")
    from tests.helpers import params_text
    with H.Simulation(H.parse_params(params_text(128, seed=case.p.seed))) as s:
        g = s.ic_noise().reshape(-1)
    ref = case["noise"].reshape(-1)
    assert np.array_equal(g[:ref.size], ref)


def test_seeded_ics_are_the_references(case):
    """hgpm_ic_generate from the params file and .ipk alone (no noise
    replay) lands on the reference's ICs within the IC bars."""
    with _sim(case) as s:
        s.generate_ic(case.ipk_table, case.ipk_header[3])
        x, v = s.store_state()
    assert np.abs(O.periodic_diff(x, case["ics_x"], case.ng)).max() < R.IC_POS_CELLS
    assert np.abs(v - case["ics_v"]).max() / np.abs(case["ics_v"]).max() < R.IC_VEL_REL


def test_cells_density_force(case):
    with _sim(case) as s:
        s.load_state(case["ics_x"], case["ics_v"])
        cells = s.get_cells()
        s.cic()
        rho = s.get_density()
        s.solve_gradient()
        f = s.get_force()
    i = np.trunc(case["ics_x"]).astype(np.int64) % case.ng
    assert np.array_equal(cells, (i[:, 0] * case.ng + i[:, 1]) * case.ng + i[:, 2])
    ref = case["rho"]
    assert np.abs(rho - ref).max() / ref.max() < R.RHO_REL
    assert np.abs(f - case["force"]).max() / np.abs(case["force"]).max() < R.FORCE_REL


def test_steps(case):
    hp = H.parse_params(case.params_text)
    with H.Simulation(hp) as s:
        s.load_state(case["ics_x"], case["ics_v"])
        ts = H.Timestepper(hp)
        ts.set_initial_z(hp.z_ini)
        ts.reverse_half_step()
        ts.advance_half_step()
        s.run_steps(ts, case.nsteps)
        x, v = s.store_state()
    assert np.abs(O.periodic_diff(x, case["fin_x"], case.ng)).max() / case.ng < R.POS_BOX
    assert np.abs(v - case["fin_v"]).max() / np.abs(case["fin_v"]).max() < 1e-4


@pytest.mark.parametrize("which", ["pk_ini", "pk_fin"])
def test_power_spectrum(case, which):
    xs = case["ics_x"] if which == "pk_ini" else case["fin_x"]
    with _sim(case) as s:
        s.load_state(xs, case["ics_v"])
        k, P, n = R.nonempty(*s.power_spectrum(221))
    kr, Pr, nr = R.parse_pk(case[which])
    assert len(k) == len(kr) and np.array_equal(n, nr)
    assert np.abs(k / kr - 1).max() < 1e-5
    assert np.abs(P / Pr - 1).max() < R.PK_REL
