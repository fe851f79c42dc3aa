"""Pins the FP64 oracle against outputs of the reference's own serial CUDA
path (fixtures made on a B200 by tests/golden/make_refgpu_fixtures.py):
ICs from the reference's white noise, the density, the force grids, N whole
steps, P(k), and the byte layout of the .params echo."""
import os

import numpy as np
import pytest

import hacc_gpm_b200 as H
from oracle import pm_oracle as O
from tests import refgpu as R


@pytest.fixture(scope="module", params=R.CASES)
def case(request):
    return R.Case(request.param)


def test_ics_from_reference_noise(case):
    x, v = O.generate_ic_from_noise(case["noise"].astype(np.float64), case.p, case.ipk_table, case.ipk_header[3])
    assert np.abs(O.periodic_diff(x, case["ics_x"], case.ng)).max() < R.IC_POS_CELLS
    assert np.abs(v - case["ics_v"]).max() / np.abs(case["ics_v"]).max() < R.IC_VEL_REL


def test_density(case):
    rho = O.cic_deposit(case["ics_x"].astype(np.float64), case.ng, O.cic_mass(case.ng, case.ng))
    assert np.abs(rho - case["rho"]).max() / rho.max() < R.RHO_REL


def test_force(case):
    f = O.solve_gradient(case["rho"].astype(np.float64), ref_quirks=True)
    ref = case["force"]
    assert np.abs(f - ref).max() / np.abs(ref).max() < R.FORCE_REL


def test_steps(case):
    x, v, _ = O.run(case["ics_x"].astype(np.float64), case["ics_v"].astype(np.float64), case.p, case.nsteps)
    assert np.abs(O.periodic_diff(x, case["fin_x"], case.ng)).max() / case.ng < R.POS_BOX
    assert np.abs(v - case["fin_v"]).max() / np.abs(case["fin_v"]).max() < 1e-4


@pytest.mark.parametrize("which", ["pk_ini", "pk_fin"])
def test_power_spectrum(case, which):
    xs = case["ics_x"] if which == "pk_ini" else case["fin_x"]
    k, P, n = R.nonempty(*O.power_spectrum(xs.astype(np.float64), case.ng, case.ng, case.p.rl, 221))
    kr, Pr, nr = R.parse_pk(case[which])
    assert len(k) == len(kr) and np.array_equal(n, nr)
    assert np.abs(k / kr - 1).max() < 1e-5  # %g prints 6 significant digits
    assert np.abs(P / Pr - 1).max() < R.PK_REL


def test_params_echo_byte_compatible(case, tmp_path):
    p = H.parse_params(case.params_text)
    prefix = str(case.p.prefix)
    p.prefix = str(tmp_path / "echo")
    p.save()
    got = open(str(tmp_path / "echo") + ".params").read()
    want = str(case["params_echo"]).replace("OUTPUT_BASE_NAME %s\n" % prefix, "OUTPUT_BASE_NAME %s\n" % p.prefix)
    assert got == want
