"""CPU tests of the C-ABI library: it loads, exports every symbol the header
declares, and its host-side logic (params, time stepper, growth, file
formats) agrees with the oracle.  No kernels run here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import hacc_gpm_b200 as H
from hacc_gpm_b200 import binding, ipk as ipkmod
from oracle import pm_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def header_functions(path):
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hgpm_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(built_lib):
    names = header_functions(os.path.join(ROOT, "include", "hgpm_c.h"))
    assert len(names) > 40
    missing = [n for n in names if not hasattr(built_lib, n)]
    assert not missing, missing


def test_struct_layout_matches(built_lib):
    assert built_lib.hgpm_sizeof_params() == C.sizeof(binding._Params)
    assert built_lib.hgpm_sizeof_timestepper() == C.sizeof(binding._Timestepper)


FIELDS = ["ng", "np", "rl", "seed", "z_ini", "z_fin", "nsteps", "last_step", "pk_folds", "hubble", "omega_cdm",
          "omega_nu", "deut", "ss8", "ns", "w_de", "wa_de", "t_cmb", "neff_massless", "neff_massive", "omega_baryon",
          "omega_cb", "omega_matter", "omega_radiation", "f_nu_massless", "f_nu_massive", "overload"]


def test_params_match_oracle(built_lib):
    path = os.path.join(GOLD, "ref_test_run_params")
    a = H.read_params(path)
    b = O.read_params(path)
    for f in FIELDS:
        assert getattr(a, f) == getattr(b, f), f
    assert a.prefix == b.prefix
    assert [i for i in range(1000) if a._raw.pks[i]] == [i for i in range(1000) if b.pks[i]]


def test_params_errors(built_lib):
    with pytest.raises(H.HgpmError):
        H.parse_params("NG 32\n")  # NP missing (params.cpp:228)
    with pytest.raises(H.HgpmError):
        H.read_params("/nonexistent/params")
    with pytest.raises(H.HgpmError):
        H.parse_params("NG 32\nNP 32\nPK_DUMP 5,2000\n")  # step outside MAX_STEPS


def test_params_noise_key(built_lib):
    """NOISE selects the IC white noise: the reference's cuRAND draws by
    default, Philox on request; anything else is an error."""
    assert H.parse_params("NG 32\nNP 32\n").noise == 0
    assert H.parse_params("NG 32\nNP 32\nNOISE CURAND\n").noise == 0
    assert H.parse_params("NG 32\nNP 32\nNOISE PHILOX\n").noise == 1
    with pytest.raises(H.HgpmError, match="NOISE"):
        H.parse_params("NG 32\nNP 32\nNOISE MT19937\n")


def test_params_save_format(built_lib, tmp_path):
    p = H.read_params(os.path.join(GOLD, "ref_test_run_params"))
    p.prefix = str(tmp_path / "echo")
    p.save()
    lines = open(str(tmp_path / "echo") + ".params").read().splitlines()
    assert lines[0] == "OMEGA_CDM 0.22" and lines[3] == "HUBBLE 0.71"
    assert lines[-6:] == ["NG 32", "NP 32", "RL 8", "SEED 21082001", "BLOCK_SIZE 64", "PK_FOLDS 1"]
    assert len(lines) == 27


@pytest.mark.parametrize("quirks", [1, 0])
def test_timestepper_matches_oracle_whole_run(built_lib, quirks):
    path = os.path.join(GOLD, "ref_test_run_params")
    a = H.read_params(path)
    a.ref_quirks = quirks
    b = O.read_params(path)
    ta, tb = H.Timestepper(a), O.Timestepper(b, ref_quirks=bool(quirks))
    for t in (ta, tb):
        t.set_initial_z(b.z_ini)
        t.reverse_half_step()
        t.advance_half_step()
    for step in range(b.nsteps):
        # the C-ABI prefactor is the kernels' float (pm_actions.cpp:291)
        assert ta.drift_prefactor(0.5) == pytest.approx(float(np.float32(tb.drift_prefactor(0.5))), rel=1e-15)
        ta.advance_half_step(); tb.advance_half_step()
        assert ta.fscal == pytest.approx(tb.fscal, rel=1e-14)
        ta.advance_half_step(); tb.advance_half_step()
        assert ta.aa == pytest.approx(tb.aa, rel=1e-14)


def test_growth_matches_oracle(built_lib):
    a = H.read_params(os.path.join(GOLD, "ref_test_run_params"))
    b = O.read_params(os.path.join(GOLD, "ref_test_run_params"))
    assert H.growth(a, 200.0, 200.5) == O.growth_pair(b, 200.0, 200.5, ref_quirks=True)
    a.ref_quirks = 0
    d, dd = H.growth(a, 200.0, 200.5)
    d2, dd2 = O.growth_pair(b, 200.0, 200.5, ref_quirks=False)
    assert d == pytest.approx(d2, rel=1e-6) and dd == pytest.approx(dd2, rel=1e-3)


def test_ipk_roundtrip_and_eh_normalisation(built_lib, tmp_path):
    p = O.parse_params_text(ipkmod.lcdm_params_text(64, 64, 128.0, 200.0, 50))
    cos = ipkmod.cosmo_from_params(p)
    path = ipkmod.write_ipk(str(tmp_path / "t.ipk"), cos, 0.0, k_max=50.0, k_bins=5000)
    h1, t1 = H.read_ipk(path)
    h2, t2 = O.read_ipk(path)
    assert np.array_equal(h1, h2) and np.array_equal(t1, t2)
    assert h1[15] == 0.0 and int(h1[2]) == 5000
    k = np.linspace(0, 50, 5000)
    assert ipkmod.sigma_r(k[1:], t1[1:]) == pytest.approx(cos["SS8"], rel=2e-3)
    tk = ipkmod.eh_nowiggle_transfer(np.array([1e-5, 0.1, 1.0]), 0.31, 0.048, 0.68)
    assert tk[0] == pytest.approx(1.0, abs=1e-3) and tk[0] > tk[1] > tk[2] > 0


def test_write_pk_format_matches_oracle(built_lib, tmp_path):
    k = np.array([0.1, 0.25, 0.5, 1.0])
    P = np.array([12.5, 0.0, 3.25e-7, float("nan")])
    n = np.array([6, 0, 12, 3], np.int64)
    rc = built_lib.hgpm_write_pk(str(tmp_path / "pk").encode(), 4, binding._d(k), binding._d(P),
                                 n.ctypes.data_as(C.POINTER(C.c_int64)))
    assert rc == 0
    got = open(str(tmp_path / "pk") + ".fold.0").read()
    assert got == O.format_pk_lines(k, P, n)


@pytest.mark.parametrize("ng", [20, 44, 56, 1008, 1280])
def test_create_rejects_bad_sizes_without_touching_gpu(built_lib, ng):
    """Sides outside the compiled 2^a 3^b 5^c multiples of 8 up to 1024 (20:
    not a multiple of 8; 44, 56: factors 11, 7; 1008: a factor 7; 1280: above
    the 10-bit packed cell) are refused before any device work."""
    p = H.parse_params(ipkmod.lcdm_params_text(ng, ng, float(ng), 50.0, 5))
    with pytest.raises(H.HgpmError, match="NG must be one of"):
        H.Simulation(p)


def _alloc_sizes(ng, np_side):
    """The buffers hgpm_create makes and the ones made on first use (float3
    staging, P(k) partial sums), sized as runtime.cu sizes them."""
    pad = lambda v: (v + 15) // 16 * 16
    ncell, npart = ng ** 3, np_side ** 3
    spec = max(ng * ng * pad(ng // 2 + 1), np_side ** 2 * pad(np_side // 2 + 1))
    b = 16 if (np_side % 16 == 0 and ng <= np_side) else 8
    nblocks = (np_side // b) ** 3
    return [(npart * 4 + 255) // 256 * 256 * 7, ncell * 8, spec * 8, 3 * spec * 8, 16 * max(ncell, npart),
            nblocks * 8 * 4, (4 + 2 * nblocks) * 4, npart * 24, 4 * 148 * 1024 * 16]


def test_footprint_covers_the_allocations(built_lib):
    """The admission model counts every buffer a context allocates, with the
    spectra and force grid sized by the larger of the ng and np grids."""
    for ng, np_side in ((32, 32), (32, 64), (64, 32), (48, 96), (512, 512), (1024, 512)):
        need = sum(_alloc_sizes(ng, np_side))
        got = H.footprint_bytes(ng, np_side)
        assert need <= got <= need + 32 * 2 ** 21, (ng, np_side, need, got)
    assert H.footprint_bytes(32, 64) > H.footprint_bytes(32, 32)


def test_footprint_model_monotone(built_lib):
    a = H.footprint_bytes(64, 64)
    b = H.footprint_bytes(128, 128)
    assert 4 * a < b < 9 * a
    assert 7 * b < H.footprint_bytes(256, 256) < 9 * b
    assert H.footprint_bytes(512, 512) / 2 ** 30 < 12


def test_drop_in_header_compiles_the_reference_fft_calls(tmp_path):
    """A caller of the reference's serial::forward_fft / backward_fft on a
    floatFFT_t (cufftComplex) grid compiles against the drop-in header."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    src = tmp_path / "caller.cpp"
    src.write_text('#include "haccgpm.hpp"\n'
                   "void f(floatFFT_t* g, int ng) {\n"
                   "    HACCGPM::serial::forward_fft(g, ng);\n"
                   "    HACCGPM::serial::backward_fft(g, ng, 1);\n"
                   "}\n")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), "-I",
                        os.path.join(ROOT, "hacc_gpm_b200", "host"), "-I", cuda_inc, str(src)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
