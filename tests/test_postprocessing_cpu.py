"""The run's files read back with the reference's own post-processing reader
(postprocessing/run.py: Run.read_params, Run.find_pks, Run.read_pk,
:60-113), where the HACC_GPM sources are on this machine.  The files come
from this project's writers (hgpm_params_save, hgpm_write_pk_fold), the
same host code the driver and the GPU path use; the P(k) values are the
oracle's for a seeded state with two folds.  run.py imports matplotlib for
its plotting helpers only, so a stand-in module is installed when matplotlib
is absent."""
import importlib.util
import os
import sys
import types

import numpy as np
import pytest

import hacc_gpm_b200 as H
from hacc_gpm_b200 import ipk as ipkmod
from oracle import pm_oracle as O
from tests.helpers import lattice_state

RUN_PY = "/root/reference/postprocessing/run.py"
pytestmark = pytest.mark.skipif(not os.path.exists(RUN_PY), reason="the reference's postprocessing/run.py is absent")


def _load_run_py():
    if "matplotlib" not in sys.modules:
        try:
            import matplotlib  # noqa: F401
        except ImportError:
            mpl = types.ModuleType("matplotlib")
            mpl.cm = types.ModuleType("matplotlib.cm")
            mpl.pyplot = types.ModuleType("matplotlib.pyplot")
            sys.modules.update({"matplotlib": mpl, "matplotlib.cm": mpl.cm, "matplotlib.pyplot": mpl.pyplot})
    spec = importlib.util.spec_from_file_location("hacc_run_py", RUN_PY)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_reader_reads_our_files(tmp_path, built_lib):
    ng, folds = 32, 1
    base = str(tmp_path / "run")
    txt = ipkmod.lcdm_params_text(ng, ng, 64.0, 50.0, 10, prefix=base, extra="PK_FOLDS %d\nLAST_STEP 4\n" % folds)
    p = H.parse_params(txt)
    p.save()  # <base>.params, the reference's echo format
    x, _ = lattice_state(ng, ng, disp=1.0, seed=4)
    written = {}
    for step in ("ini", 2, "fin"):
        for fold in range(folds + 1):
            k, P, n = O.power_spectrum(x.astype(np.float64) * (1.0 + 0.01 * (step == 2)), ng, ng, 64.0, 221,
                                       folds=folds, fold=fold)
            ok = (n > 0) & np.isfinite(P) & (P > 0)
            H.write_pk("%s.pk.%s" % (base, step), np.where(ok, k, 0), np.where(ok, P, 0), np.where(ok, n, 0),
                       fold=fold)
            written[(step, fold)] = (k[ok], P[ok], n[ok])
    R = _load_run_py()
    run = R.Run(base)
    assert run.params["NG"] == ng and run.params["PK_FOLDS"] == folds and run.params["SEED"] == p.seed
    assert abs(run.params["RL"] - 64.0) < 1e-6
    assert [pk.step for pk in run.pks] == ["ini", 2, "fin"]
    for pk in run.pks:
        assert len(pk.folds) == folds + 1
        for fold, df in enumerate(pk.folds):
            k, P, n = written[(pk.step, fold)]
            assert list(df.columns) == ["k", "P_0(k)", "nmodes"]
            assert np.array_equal(df["nmodes"].to_numpy(), n)
            # "%g" keeps 6 significant digits
            assert np.allclose(df["k"].to_numpy(), k, rtol=1e-5) and np.allclose(df["P_0(k)"].to_numpy(), P, rtol=1e-5)
