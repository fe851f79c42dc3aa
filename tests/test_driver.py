"""The C++ drop-in (hacc_gpm_b200/host): the reference's serial() run over
the HACCGPM::serial:: shim.  CPU: usage, the .params echo and the
reference's exit-on-error behaviour.  GPU: the files it writes against the
Python API on the same seeded run, and the --fused loop against the
per-phase loop."""
import filecmp
import os
import subprocess

import numpy as np
import pytest

import hacc_gpm_b200 as H
from hacc_gpm_b200 import build as B
from hacc_gpm_b200 import ipk as ipkmod
from oracle import pm_oracle as O


def _driver():
    if not os.path.exists(B.DRIVER):
        B.build()
    return B.DRIVER


def _case(tmp, name, ng=32, extra="LAST_STEP 6\nPK_DUMP 2\nPARTICLE_DUMP 3\nDUMP_INIT\nDUMP_FINAL\n"):
    d = tmp / name
    d.mkdir()
    txt = ipkmod.lcdm_params_text(ng, ng, float(ng), 50.0, 100, prefix=str(d / "run"), ipk=str(tmp / "run.ipk"),
                                  extra=extra)
    if not (tmp / "run.ipk").exists():
        op = O.parse_params_text(txt)
        header, table = ipkmod.make_ipk(ipkmod.cosmo_from_params(op), op.z_ini, k_max=20.0)
        np.concatenate([header, table]).astype("<f8").tofile(str(tmp / "run.ipk"))
    (d / "input.params").write_text(txt)
    return d, txt


def test_usage():
    r = subprocess.run([_driver()], capture_output=True, text=True)
    assert r.returncode == 1 and "USAGE" in r.stdout


def test_echo_and_exit_on_error(tmp_path):
    # NG 20 is not a supported FFT size: read_params prints and echoes, then
    # MemoryManager fails and the process exits 1 with the message
    d, txt = _case(tmp_path, "bad", extra="")
    (d / "input.params").write_text(txt.replace("NG 32", "NG 20"))
    r = subprocess.run([_driver(), str(d / "input.params")], capture_output=True, text=True)
    assert r.returncode == 1
    assert "MemoryManager" in r.stderr and "NG must be one of" in r.stderr
    assert "OUTPUT_BASE_NAME" in r.stdout
    p = H.parse_params(txt.replace("NG 32", "NG 20"))
    p.prefix = str(d / "py")
    p.save()
    assert (d / "run.params").read_text() == (d / "py.params").read_text().replace(str(d / "py"), str(d / "run"))


REF_DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_driver")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_DRIVER), reason="the reference driver was not built (make -C oracle refdrv)")
def test_reference_driver_on_the_drop_in(tmp_path):
    """The reference's own src/driver_pm.cpp (main and serial(), compiled
    unchanged with -DNOPYTHON against host/haccgpm.hpp and libhgpm.so by
    oracle/Makefile) runs on the B200 path and writes the same files, byte
    for byte, as this project's driver on the same params."""
    extra = "LAST_STEP 5\nPK_DUMP 1,3\nPARTICLE_DUMP 2\nDUMP_INIT\nDUMP_FINAL\n"
    da, _ = _case(tmp_path, "ref", extra=extra)
    db, _ = _case(tmp_path, "ours", extra=extra)
    ra = subprocess.run([REF_DRIVER, str(da / "input.params")], capture_output=True, text=True, timeout=300)
    assert ra.returncode == 0, ra.stderr[-2000:]
    assert "RUNNING IN SERIAL MODE" in ra.stdout
    rb = subprocess.run([_driver(), str(db / "input.params")], capture_output=True, text=True, timeout=300)
    assert rb.returncode == 0, rb.stderr[-2000:]
    files = ("run.pk.ini.fold.0", "run.pk.1.fold.0", "run.pk.3.fold.0", "run.pk.fin.fold.0", "run.particles.ini",
             "run.particles.2", "run.particles.fin")
    for f in files:
        assert (da / f).exists() and filecmp.cmp(da / f, db / f, shallow=False), f
    echo_a = (da / "run.params").read_text().replace(str(da), "DIR")
    echo_b = (db / "run.params").read_text().replace(str(db), "DIR")
    assert echo_a == echo_b


@pytest.mark.gpu
def test_driver_files_match_api(tmp_path):
    d, txt = _case(tmp_path, "plain")
    r = subprocess.run([_driver(), str(d / "input.params")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for f in ("run.params", "run.pk.ini.fold.0", "run.pk.2.fold.0", "run.pk.fin.fold.0", "run.particles.ini",
              "run.particles.3", "run.particles.fin"):
        assert (d / f).exists(), f
    hp = H.parse_params(txt)
    n3 = 32 ** 3
    header, table = H.read_ipk(str(tmp_path / "run.ipk"))
    with H.Simulation(hp) as s:
        s.generate_ic(table, header[3])
        k, P, n = s.power_spectrum(221)
        H.write_pk(str(tmp_path / "api.pk.ini"), k, P, n)
        ts = H.Timestepper(hp)
        ts.set_initial_z(hp.z_ini)
        ts.reverse_half_step()
        ts.advance_half_step()
        for _ in range(6):
            s.update_positions(ts, 0.5)
            s.cic()
            s.solve_gradient()
            ts.advance_half_step()
            s.update_velocities(ts)
            ts.advance_half_step()
            s.update_positions(ts, 0.5)
        x, v = s.store_state()
    assert (d / "run.pk.ini.fold.0").read_text() == (tmp_path / "api.pk.ini.fold.0").read_text()
    fin = np.fromfile(str(d / "run.particles.fin"), dtype="<f4")
    assert fin.size == 6 * n3
    assert np.array_equal(fin[:3 * n3].reshape(-1, 3), x) and np.array_equal(fin[3 * n3:].reshape(-1, 3), v)


@pytest.mark.gpu
def test_driver_writes_every_fold(tmp_path):
    """PK_FOLDS 2: one pk file per fold (power.cu:189-227), each equal to the
    API's fold through hgpm_write_pk_fold."""
    d, txt = _case(tmp_path, "folds", extra="PK_FOLDS 2\n")
    r = subprocess.run([_driver(), str(d / "input.params")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    hp = H.parse_params(txt)
    header, table = H.read_ipk(str(tmp_path / "run.ipk"))
    with H.Simulation(hp) as s:
        s.generate_ic(table, header[3])
        for fold in range(3):
            k, P, n = s.power_spectrum(221, fold=fold)
            H.write_pk(str(tmp_path / "api.pk.ini"), k, P, n, fold=fold)
    for fold in range(3):
        name = "run.pk.ini.fold.%d" % fold
        assert (d / name).exists(), name
        assert (d / name).read_text() == (tmp_path / ("api.pk.ini.fold.%d" % fold)).read_text()


@pytest.mark.gpu
def test_analysis_hook_and_python_driver(tmp_path):
    """DO_ANALYSIS / ANALYSIS_STEPS (PyAnalysis, py_analysis.cu:3-27): the C++
    driver writes the rows (tag, x, y, z, vx, vy, vz) of the marked steps;
    the Python driver hands the same rows to a callable and writes the same
    pk and particle files."""
    from hacc_gpm_b200 import driver as D

    extra = "LAST_STEP 5\nPK_DUMP 2\nPARTICLE_DUMP 3\nDUMP_FINAL\nPK_FOLDS 1\nDO_ANALYSIS\nANALYSIS_STEPS 1,3\n"
    dc, _ = _case(tmp_path, "cpp", extra=extra + "ANALYSIS_DIR %s\n" % (tmp_path / "cpp"))
    r = subprocess.run([_driver(), str(dc / "input.params"), "--fused"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dp, _ = _case(tmp_path, "py", extra=extra)
    seen = {}
    D.serial(str(dp / "input.params"), analysis=lambda rows, step, a, z: seen.__setitem__(step, (rows.copy(), a, z)))
    assert sorted(seen) == [1, 3]
    n3 = 32 ** 3
    for step, (rows, a, z) in seen.items():
        assert rows.shape == (n3, 7) and np.array_equal(rows[:, 0], np.arange(n3, dtype=np.float32))
        assert 0 < a < 1 and z > 0
        cpp = np.fromfile(str(dc / ("analysis.%d" % step)), dtype="<f4").reshape(n3, 7)
        assert np.array_equal(cpp, rows)
    dump3 = np.fromfile(str(dp / "run.particles.3"), dtype="<f4")
    assert np.array_equal(seen[3][0][:, 1:4].reshape(-1), dump3[:3 * n3])
    for f in ("run.pk.ini.fold.0", "run.pk.ini.fold.1", "run.pk.2.fold.0", "run.pk.fin.fold.1", "run.particles.3",
              "run.particles.fin"):
        assert (dc / f).read_bytes() == (dp / f).read_bytes(), f


@pytest.mark.gpu
def test_driver_fused_equals_plain(tmp_path):
    runs = []
    for name, flags in (("a", []), ("b", ["--fused"])):
        d, _ = _case(tmp_path, name)
        r = subprocess.run([_driver(), str(d / "input.params"), *flags], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        runs.append(d)
    for f in ("run.pk.ini.fold.0", "run.pk.2.fold.0", "run.pk.fin.fold.0", "run.particles.ini", "run.particles.3",
              "run.particles.fin"):
        assert filecmp.cmp(str(runs[0] / f), str(runs[1] / f), shallow=False), f
