"""Generate the reference-output fixtures tests/golden/refgpu_*.npz.

Runs the reference's own serial CUDA path (oracle/_ref/refpm, built from the
HACC_GPM sources by `make -C oracle ref`) on a B200 for small seeded cases and
packs its outputs:

  params   the run file given to the reference; params_echo its .params echo
  noise    the reference's cuRAND white noise (GenerateFourierAmplitudes)
  ipk      the .ipk table the run reads (EH no-wiggle, hacc_gpm_b200.ipk)
  ics_x/v  its Zel'dovich ICs (DUMP_INIT of `refpm run` with LAST_STEP 0)
  rho      Re of its density grid after serial::CIC of those ICs
  force    its force grids after serial::SolveGradient
  fin_x/v  positions/velocities after NSTEPS steps of its run loop
  pk_ini   its P(k) CSV lines of the ICs, pk_fin of the final state

Usage (on a machine with a B200 and the built refpm, from the repository
root; the .npz files then go to tests/golden/):
    python tests/golden/make_refgpu_fixtures.py --out refgpu_out
Every input is seeded; PK_FOLDS is 0 (fold > 0 writes out of bounds in the
reference's BinPower).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hacc_gpm_b200 import ipk as ipkmod  # noqa: E402

REFPM = os.path.join(ROOT, "oracle", "_ref", "refpm")

CASES = {
    # name: (ng = np, rl, z_ini, run length N_STEPS, steps run from the ICs)
    "a32": (32, 32.0, 50.0, 100, 10),
    "b24": (24, 48.0, 100.0, 60, 8),
}


def params_text(ng, rl, z, nsteps, prefix, ipk_path, last_step=None, dump_init=False):
    extra = ""
    if last_step is not None:
        extra += "LAST_STEP %d\n" % last_step
    if dump_init:
        extra += "DUMP_INIT\n"
    return ipkmod.lcdm_params_text(ng, ng, rl, z, nsteps, seed=21082001, prefix=prefix, ipk=ipk_path, extra=extra)


def run(cmd, log):
    with open(log, "a") as f:
        r = subprocess.run(cmd, stdout=f, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("%s failed (rc %d), see %s" % (" ".join(cmd), r.returncode, log))


def make_case(name, out):
    ng, rl, z, nsteps, nrun = CASES[name]
    work = os.path.join(out, name)
    os.makedirs(work, exist_ok=True)
    log = os.path.join(work, "refpm.log")
    from oracle import pm_oracle as O  # cosmology derivation only

    cosmo = ipkmod.cosmo_from_params(O.parse_params_text(params_text(ng, rl, z, nsteps, "x", "x")))
    ipk_path = os.path.join(work, "run.ipk")
    header, table = ipkmod.make_ipk(cosmo, z, k_max=20.0, k_bins=20000)
    np.concatenate([header, table]).astype("<f8").tofile(ipk_path)
    prefix = os.path.join(work, "run")
    # the reference writes "<prefix>.params" (save_params), so the input lives elsewhere
    pfile = os.path.join(work, "input.params")
    ptxt = params_text(ng, rl, z, nsteps, prefix, ipk_path, last_step=0, dump_init=True)
    with open(pfile, "w") as f:
        f.write(ptxt)
    run([REFPM, "run", pfile], log)
    run([REFPM, "noise", pfile, prefix + ".noise"], log)
    ics = prefix + ".particles.ini"
    run([REFPM, "load", pfile, ics, str(nrun), prefix + ".load"], log)
    n3 = ng ** 3
    xv = np.fromfile(ics, dtype="<f4")
    fin = np.fromfile(prefix + ".load.fin", dtype="<f4")
    with open(prefix + ".params") as f:
        echo = f.read()
    data = dict(
        params=np.array(ptxt),
        params_echo=np.array(echo),
        nsteps_run=np.array(nrun),
        ipk=np.fromfile(ipk_path, dtype="<f8"),
        noise=np.fromfile(prefix + ".noise", dtype="<f4").reshape(ng, ng, ng),
        ics_x=xv[: 3 * n3].reshape(-1, 3), ics_v=xv[3 * n3:].reshape(-1, 3),
        rho=np.fromfile(prefix + ".load.rho", dtype="<f4").reshape(ng, ng, ng),
        force=np.fromfile(prefix + ".load.force", dtype="<f4").reshape(3, ng, ng, ng),
        fin_x=fin[: 3 * n3].reshape(-1, 3), fin_v=fin[3 * n3:].reshape(-1, 3),
        pk_ini=np.array(open(prefix + ".load.pk.ini.fold.0").read()),
        pk_fin=np.array(open(prefix + ".load.pk.fin.fold.0").read()),
        pk_ics_run=np.array(open(prefix + ".pk.ini.fold.0").read()),
    )
    path = os.path.join(out, "refgpu_%s.npz" % name)
    np.savez_compressed(path, **data)
    return path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="refgpu_out")
    ap.add_argument("--cases", default=",".join(CASES))
    a = ap.parse_args()
    if not os.path.exists(REFPM):
        sys.exit("build the reference harness first: make -C oracle ref")
    os.makedirs(a.out, exist_ok=True)
    for c in a.cases.split(","):
        print(make_case(c, a.out))


if __name__ == "__main__":
    main()
