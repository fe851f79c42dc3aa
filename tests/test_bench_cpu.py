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
    kick, read by the deposit) and per cell 32 B with a kick that gathers
    the potential (density, spectra, potential) or 56 B with the force-grid
    kick (the float4 grid's 12 useful bytes written and read)."""
    b = _bench()
    for n in (64, 256, 512):
        assert sum(b.alg_bytes(n ** 3, n ** 3).values()) == 72 * n ** 3 + 32 * n ** 3
        assert sum(b.alg_bytes(n ** 3, n ** 3, False).values()) == 72 * n ** 3 + 56 * n ** 3
    assert sum(b.alg_bytes(512 ** 3, 512 ** 3, False).values()) == 17179869184
    a = b.alg_bytes(512 ** 3, 1024 ** 3)  # more cells than particles
    assert sum(a.values()) == 72 * 512 ** 3 + 32 * 1024 ** 3


def test_every_phase_has_kernels_named():
    """Every phase is named for every deposit and kick candidate of both
    block sides (the candidate lists of particles.cu)."""
    b = _bench()
    for np_side, ng, nd in ((512, 512, 12), (512, 1024, 8)):
        for dep in range(nd):
            for kick in range(8):
                for yx in (0, 1, 2):
                    t = {"deposit": dep, "kick": kick, "y_pass": min(yx, 1), "x_pass": yx}
                    names = b.kernel_names(t, np_side, ng)
                    assert set(names) == set(b.alg_bytes(8, 8)) and all("NG" not in v for v in names.values())
    t = {"deposit": {"choice": 8, "ms": 1.0}, "kick": {"choice": 7, "ms": 2.0}, "y_pass": {"choice": 1, "ms": 0.2},
         "x_pass": {"choice": 1, "ms": 0.5}}
    n = b.kernel_names(t, 512, 512)
    assert n["kick_drift"].startswith("kick_phi_kernel<16,1024,4,1>")
    assert n["fft_z_inv"].startswith("zpass_c2r_pair_kernel<512>")
    assert n["deposit"].startswith("deposit_col_kernel<16,4,4,1>")


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
