"""bench.py's bookkeeping on the CPU: the algorithmic bytes behind the
roofline figures and the phase names the JSON line reports."""
import importlib.util
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("hgpm_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_step_algorithmic_bytes():
    """72 B per particle (the precision-form state read and written by the
    kick, read by the deposit) and 56 B per cell (density, spectra, potential
    and the float4 force grid's 12 useful bytes) per step."""
    b = _bench()
    for n in (64, 256, 512):
        a = b.alg_bytes(n ** 3, n ** 3)
        assert sum(a.values()) == 72 * n ** 3 + 56 * n ** 3
    assert sum(b.alg_bytes(512 ** 3, 512 ** 3).values()) == 17179869184
    a = b.alg_bytes(512 ** 3, 1024 ** 3)  # more cells than particles
    assert sum(a.values()) == 72 * 512 ** 3 + 56 * 1024 ** 3


def test_every_phase_has_kernels_named():
    b = _bench()
    assert set(b.KERNEL_NAMES) == set(b.alg_bytes(8, 8))


def test_help_runs_without_a_gpu():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and "--impl" in r.stdout


def test_both_arms_report_the_same_config():
    """The b200 line and the --impl reference line carry the same config
    dict for the same --steps/--warmup: the timed steps start at the same
    step of the same run."""
    b = _bench()
    assert b.bench_config(20, 5) == b.bench_config(20, 5)
    assert b.first_warmup_step(20, 5) == 40 and b.first_warmup_step(10, 3) == 42
    c = b.bench_config(20, 5)
    assert "steps 45-64" in c["timed"] and c["np"] == 512 and c["ng"] == 512


def test_config_c_box():
    b = _bench()
    ng, np_side, rl, nrun, mid = b.CONFIGS["C"]
    assert (ng, np_side, rl, nrun) == (1024, 512, 1000.0, 200)
    assert mid < nrun
