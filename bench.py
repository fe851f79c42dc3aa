#!/usr/bin/env python
"""Headline benchmark: PM steps per second of particles at 512^3.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--config NS|C] [--workload step|ensemble|serve]

One process per GPU (torchrun for N > 1).  Each rank advances its own
independent box (replicas: the step itself has no collective), so scaling
is weak.  --config NS (default): 512^3 particles on a 512^3 grid, L = 512
Mpc/h, a 100-step run from z = 50 to z = 0.  --config C: 512^3 particles on a
1024^3 grid, L = 1000 Mpc/h, a 200-step run from z = 50.  The cost of a step
grows as the particles cluster and the middle of the run costs about the
run's average, so the run is advanced untimed to step MID - W (45 of 100, 90
of 200), then W warm-up steps, then exactly K timed steps (CUDA events on
the box's stream, barrier + synchronize on both sides, max over ranks;
per-kernel events inside the same region).  value = particle updates of all
ranks / that time.  The ICs are the reference's own: EH no-wiggle Zel'dovich
displacements from its cuRAND white noise for SEED 21082001 (+ rank).  The
whole run is also timed once ("full_run").

Also reported (rank 0): per-kernel timings and the roofline of the dominant
kernel against the measured HBM peak, the end-to-end number through the
C-ABI with host buffers (hgpm_step_host: H2D of the state, one step, D2H of
the state, every step), the CPU baseline (the OpenMP C++ transcription of
the reference's serial step on this host's cores, on the same state), kernel
launch count, SM clocks sampled during the timed region, and (N = 1,
--config NS) the batched forms: the 96-box ensemble and the serving loop
against the same work one box at a time ("forms"; --no-forms skips them).

--impl reference times the reference's algorithm on the host cores (the
reference has no CPU path; oracle/_bin/cpu_pm is its OpenMP transcription)
on the same state and steps: the reference's own serial CUDA code
(oracle/_ref/refpm, built from its sources) makes the ICs from the same SEED
and advances them to the first warm-up step, then the transcription runs
the W warm-up and K timed steps.  Its line carries the same config.

--workload ensemble | serve print only the batched form's line (under
torchrun each rank takes its share of the boxes / requests, whole boxes by
predicted cost; makespans are the slowest rank's):
  ensemble  96 boxes, ng = np from {32, 48, 64, 96, 128}, L ~ U[64, 512],
            sigma8 ~ U[0.7, 0.9], z 100, 64 steps each: sims/hour batched
            (one launch per phase per size class, CUDA graph) against the
            same boxes one at a time through the plain step;
  serve     a Poisson request stream (20/s, ng log-uniform over 32..256,
            steps U[20, 200], own cosmology and seed) through the
            continuous-batching server and one at a time: p50/p99 latency
            and sims/hour, plus the saturated (all queued) throughput.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

UNIT = "particle-updates/s"
SEED = 21082001
Z_INI = 50.0
# the box of each --config: (ng, np, rl, steps in the run, first timed step)
CONFIGS = {"NS": (512, 512, 512.0, 100, 45), "C": (1024, 512, 1000.0, 200, 90)}
NG, NP, RL, NSTEPS_RUN, MID_STEP = CONFIGS["NS"]


def metric_name():
    if NG == NP:
        return "particle-updates/s at %d^3" % NP
    return "particle-updates/s at %d^3 particles on a %d^3 grid" % (NP, NG)


def first_warmup_step(steps, warmup):
    """The run is advanced untimed to this step; W warm-up steps follow, then
    the K timed steps."""
    return max(0, min(MID_STEP, NSTEPS_RUN - steps) - warmup)

# Algorithmic bytes per launch of each kernel (precision-form state:
# x = 12 B offset + 4 B cell, v = 12 B; FP32 grids).
def alg_bytes(np3, ng3, potential_kick=True):
    """Algorithmic bytes per phase: each input read once, each output
    written once (FP32).  The gradient is taken in real space, so the x pass
    moves one spectrum in and one out (8 B/cell).  With a kick that gathers
    the potential, the inverse z phase is the C2R of the potential (4 + 4
    B/cell) and the kick reads the potential (4 B/cell): 72 Np + 32 Ng per
    step; with the force-grid kick the inverse z phase adds the gradient (4
    + 12 B/cell) and the kick reads the force (12 B/cell): 72 Np + 56 Ng."""
    return {
        "deposit": 16 * np3 + 4 * ng3,
        "fft_z_fwd": 8 * ng3,
        "fft_y_fwd": 0,
        "poisson_x": 8 * ng3,
        "fft_y_inv": 0,
        "fft_z_inv": (8 if potential_kick else 24) * ng3,
        "kick_drift": 56 * np3 + (4 if potential_kick else 12) * ng3,
    }


# The kernels of each phase (one launch each per step, unless noted); the
# deposit and kick entries follow the candidate lists of particles.cu.
DEPOSIT_NAMES = {
    16: ["deposit_tiled_kernel<16,S,256,3>", "deposit_tiled_kernel<16,S,512,2>", "deposit_tiled_kernel<16,S,1024,1>",
         "deposit_w32_kernel<16,512,2,1>", "deposit_w32_kernel<16,256,4,1,4>", "deposit_col_kernel<16,4,4,0>",
         "deposit_col_kernel<16,4,2,0>", "deposit_col_kernel<16,3,4,0>",
         "deposit_col_kernel<16,4,4,1> (32-bit windows, x-half split, wraps from the atomics' returned values)",
         "deposit_direct_kernel<16,S,512>", "deposit_col_kernel<16,4,4,2>",
         "deposit_col_kernel<16,4,4,1,1> (32-bit windows, x-half split, returned-value wraps, x-chain merge)"],
    8: ["deposit_tiled_kernel<8,S,256,3>", "deposit_w32_kernel<8,256,4,1,2> (32-bit windows, 13312 cells)",
        "deposit_col_kernel<8,12,4,0>", "deposit_w32_kernel<8,512,2,1,1>", "deposit_col_kernel<8,12,4,1>",
        "deposit_direct_kernel<8,S,256>", "deposit_col_kernel<8,12,4,2>", "deposit_col_kernel<8,12,4,1,1>"],
}
KICK_NAMES = {
    16: ["kick_flat_nt_kernel<16,1024,4> (float4 force gathers)", "kick_flat_nt_kernel<16,1024,2>",
         "kick_flat_nt_kernel<16,1024,1>", "kick_spill_kernel<16>", "kick_win4_kernel<16,512> + kick_spill_kernel<16>",
         "kick_phi_kernel<16,1024,4,0> (potential gathers)", "kick_phi_kernel<16,1024,2,0>",
         "kick_phi_kernel<16,1024,4,1> (one particle per thread, a 16^3 block per CTA as four units of four "
         "x-planes; 16 paired-potential gathers form the 8 corner forces)"],
    8: ["kick_spill_kernel<8>", "kick_flat_nt_kernel<8,512,1>", "kick_flat_nt_kernel<8,512,2>",
        "kick_flat_nt_kernel<8,256,4>", "kick_win4_kernel<8,512> + kick_spill_kernel<8>",
        "kick_phi_kernel<8,512,1,0> (32 potential gathers form the 8 corner forces)", "kick_phi_kernel<8,512,2,0>",
        "kick_phi_kernel<8,512,1,1> (paired potential)"],
}


def kernel_names(tuned, np_side, ng, plane=None):
    if plane is None:
        plane = os.environ.get("HGPM_PLANE") == "1"
    blk = 16 if np_side % 16 == 0 and ng <= np_side else 8
    dep, kick = tuned["deposit"]["choice"] if isinstance(tuned["deposit"], dict) else tuned["deposit"], \
        tuned["kick"]["choice"] if isinstance(tuned["kick"], dict) else tuned["kick"]
    ypass = tuned["y_pass"]["choice"] if isinstance(tuned["y_pass"], dict) else tuned["y_pass"]
    xpass = tuned["x_pass"]["choice"] if isinstance(tuned["x_pass"], dict) else tuned["x_pass"]
    zinv = {7: "zpass_c2r_pair_kernel<NG> (the paired potential)", 5: "zpass_c2r_kernel<NG> (the potential)",
            6: "zpass_c2r_kernel<NG> (the potential)"}.get(
        kick, "zpass_c2r_kernel<NG> (the potential) + gradient_kernel<8,3,2> (central differences, float4 force)")
    spill = "deposit_spill_kernel<%d,S,%d>" % (blk, 1024 if blk == 16 else 512)
    names = {
        "deposit": "%s + %s (queued blocks)" % (DEPOSIT_NAMES[blk][dep], spill),
        "fft_z_fwd": "zpass_r2c_kernel<NG,1>",
        "fft_y_fwd": "strided_tma_kernel<NG,0,0>" if ypass else "strided_kernel<NG,0>",
        "poisson_x": {0: "xfused_kernel<NG,PotentialOp>", 1: "xpotential_tma_kernel<NG,256>"}.get(
            xpass, "xpot_wide_kernel<NG> (twice the columns per CTA)") +
                     " (forward x, Green's function, inverse x)",
        "fft_y_inv": "strided_tma_kernel<NG,1,0>" if ypass else "strided_kernel<NG,1>",
        "fft_z_inv": zinv,
        "kick_drift": KICK_NAMES[blk][kick],
    }
    if plane and ng in (256, 512, 1024):
        # HGPM_PLANE=1: the z and y passes in one kernel, a cluster per x plane
        names["fft_z_fwd"] = "zy_fwd_kernel<NG,3> (z and y passes, an 8-CTA cluster per x plane)"
        names["fft_y_fwd"] = "(in zy_fwd_kernel)"
        if kick == 7:
            names["fft_z_inv"] = "yz_inv_pair_kernel<NG,3> (y and z inverse passes, the paired potential)"
            names["fft_y_inv"] = "(in yz_inv_pair_kernel)"
    small = "1" if ng <= np_side else "0"
    return {k: v.replace("NG", str(ng)).replace(",S,", "," + small + ",") for k, v in names.items()}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 50 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for nm, val in zip(names, r[5:9]):
                    if val.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cosmo_args(params):
    """Cosmology of the run for the CPU transcription's time stepper."""
    return ["--omega-cb", repr(params.omega_cb), "--omega-m", repr(params.omega_matter),
            "--omega-r", repr(params.omega_radiation), "--f-nu", repr(params.f_nu_massless)]


def cpu_baseline(steps=1, warmup=0, load=None, start_step=0, cosmo=()):
    """The OpenMP C++ transcription of the reference's serial step on all host
    threads: `warmup` + `steps` steps from `load` (x then v, float3, lattice
    order) at step `start_step` of the run, or from a seeded lattice."""
    exe = os.path.join(ROOT, "oracle", "_bin", "cpu_pm")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "cpu"], check=True)
    cmd = [exe, "--ng", str(NG), "--np", str(NP), "--rl", str(RL), "--zini", str(Z_INI),
           "--nsteps-total", str(NSTEPS_RUN), "--steps", str(steps), "--warmup", str(warmup), *cosmo]
    if load:
        cmd += ["--load", load, "--start-step", str(start_step)]
    out = subprocess.run(cmd, capture_output=True, text=True, check=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def run_params_text(rank=0, prefix="run", ipk="run.ipk", extra=""):
    from hacc_gpm_b200 import ipk as ipkmod
    return ipkmod.lcdm_params_text(NG, NP, RL, Z_INI, NSTEPS_RUN, seed=SEED + rank, prefix=prefix, ipk=ipk,
                                   extra=extra)


def run_ipk(params):
    """The .ipk of the run (EH no-wiggle, sigma8-normalised, at z_ini)."""
    from hacc_gpm_b200 import ipk as ipkmod
    return ipkmod.make_ipk(ipkmod.cosmo_from_params(params), Z_INI, k_max=20.0, k_bins=20000)


def reference_state(start, d):
    """The reference's own serial CUDA path (oracle/_ref/refpm, compiled from
    its sources; GPU) makes the ICs of SEED and runs `start` steps of its
    serial() loop, dumping x, v (writeOutput's float3 layout) after the last.
    Returns the dump's path, or None when the harness or a GPU is absent."""
    exe = os.path.join(ROOT, "oracle", "_ref", "refpm")
    if not os.path.exists(exe) or start < 1:
        return None
    import numpy as np
    from oracle import pm_oracle as O
    pre = os.path.join(d, "r")
    txt = run_params_text(prefix=pre, ipk=pre + ".ipk",
                          extra="LAST_STEP %d\nPARTICLE_DUMP %d\n" % (start, start - 1))
    h, tab = run_ipk(O.parse_params_text(txt))
    np.concatenate([h, tab]).astype("<f8").tofile(pre + ".ipk")
    pf = pre + ".in"
    with open(pf, "w") as f:
        f.write(txt)
    r = subprocess.run([exe, "run", pf], capture_output=True, text=True, timeout=900)
    dump = "%s.particles.%d" % (pre, start - 1)
    if r.returncode != 0 or not os.path.exists(dump):
        return None
    return dump


def reference_gpu():
    """The reference's own serial CUDA step (oracle/_ref/refpm, compiled from
    the HACC_GPM sources when they were present at build time) on this GPU:
    the same run, K = 10 steps from the first timed step (mid-run) and the
    whole run.  Context for the GPU-to-GPU comparison; None when the harness
    is absent."""
    exe = os.path.join(ROOT, "oracle", "_ref", "refpm")
    if not os.path.exists(exe):
        return None
    import numpy as np
    from oracle import pm_oracle as O
    out = {}
    with tempfile.TemporaryDirectory() as d:
        pre = os.path.join(d, "r")
        txt = run_params_text(prefix=pre, ipk=pre + ".ipk")
        h, tab = run_ipk(O.parse_params_text(txt))
        np.concatenate([h, tab]).astype("<f8").tofile(pre + ".ipk")
        pf = pre + ".in"
        with open(pf, "w") as f:
            f.write(txt)
        for key, (w, k) in (("mid", (MID_STEP, 10)), ("full", (0, NSTEPS_RUN))):
            r = subprocess.run([exe, "time", pf, str(w), str(k)], capture_output=True, text=True, timeout=900)
            line = [l for l in r.stderr.splitlines() if l.startswith("REFPM_TIME")]
            if r.returncode != 0 or not line:
                return {"error": "refpm %s failed (rc %d)" % (key, r.returncode)}
            ms = float(line[-1].split("ms_per_step=")[1])
            out[key] = {"ms_per_step": ms, "value": NP ** 3 / (ms * 1e-3), "unit": UNIT}
    out["what"] = ("the reference's serial CUDA path (HACCGPM::serial::UpdatePositions/CIC/SolveGradient/"
                   "UpdateVelocities, cuFFT C2C, float atomics) compiled from its sources for sm_100a, CUDA events")
    return out


def bench_config(steps, warmup):
    """The workload both arms report (identical dicts)."""
    start = first_warmup_step(steps, warmup)
    return {"workload": "PM step (deposit, R2C FFT, Poisson+gradient, C2R FFT, gather+kick+drift), "
                        "%d^3 particles on a %d^3 grid, L=%g Mpc/h, flat LCDM (Om 0.31, h 0.68, ns 0.96, "
                        "sigma8 0.81), %d-step run from z=%g" % (NP, NG, RL, NSTEPS_RUN, Z_INI),
            "np": NP, "ng": NG, "rl": RL,
            "ics": "EH no-wiggle Zel'dovich from the reference's cuRAND white noise, SEED %d (+ rank)" % SEED,
            "timed": "steps %d-%d of the run after %d warm-up steps (mid-run cost = run average)"
                     % (start + warmup, start + warmup + steps - 1, warmup),
            "l2": "inputs larger than L2 (%.2g GB particle state, %.2g GB grids)" % (28 * NP ** 3 / 1e9,
                                                                                    40 * NG ** 3 / 1e9)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from hacc_gpm_b200 import binding as Bd
    params = Bd.parse_params(run_params_text())
    start = first_warmup_step(args.steps, args.warmup)
    gpu = None
    with tempfile.TemporaryDirectory() as d:
        dump = None
        try:
            import torch
            if torch.cuda.is_available():
                dump = reference_state(start, d)
        except Exception:
            dump = None
        r = cpu_baseline(steps=args.steps, warmup=args.warmup, load=dump, start_step=start,
                         cosmo=cosmo_args(params))
    try:
        import torch
        if torch.cuda.is_available() and not args.no_full:
            gpu = reference_gpu()
    except Exception as e:  # the CPU arm stands on its own
        gpu = {"error": str(e)[:200]}
    v = NP ** 3 / r["sec_per_step"]
    state = ("the run's state after %d steps from the reference's own serial CUDA path (refpm) on the same SEED"
             % start) if dump else "a seeded perturbed lattice (the reference harness was not available)"
    print(json.dumps({
        "impl": "reference", "metric": metric_name(), "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": r["steps"], "warmup": args.warmup, "ms_per_step": r["sec_per_step"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded EH no-wiggle Zel'dovich ICs (the reference's cuRAND white noise)",
        "config": bench_config(args.steps, args.warmup),
        "execution": "the OpenMP C++ transcription of the reference's serial step on %d host threads" % r["threads"],
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["threads"], "kind": "port",
                         "sample": "%d full %d^3 steps (after %d warm-up) of the OpenMP C++ transcription of the "
                                   "reference's serial step (float3 layout, float atomics, C2C FFTs) from %s"
                                   % (r["steps"], NP, args.warmup, state)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "same_state": bool(dump),
        "reference_gpu": gpu,
    }))


def _check_same(a, b):
    """Largest relative P(k) difference and whether the mode counts agree."""
    worst, counts = 0.0, True
    for ra, rb in zip(a, b):
        ra = ra.result if hasattr(ra, "result") else ra
        rb = rb.result if hasattr(rb, "result") else rb
        counts &= bool((ra["n"] == rb["n"]).all())
        ok = ra["n"] > 0
        if ok.any():
            worst = max(worst, float(abs(ra["P"][ok] / rb["P"][ok] - 1).max()))
    return worst, counts


def form_ensemble(rk=None):
    """96 mixed boxes batched against the same boxes one at a time.  Under
    torchrun each rank takes its share of the boxes (ensemble.shard: whole
    boxes by predicted cost, no collective on the data path); times are the
    slowest rank's."""
    import torch

    from hacc_gpm_b200 import ensemble as E
    from hacc_gpm_b200.replicas import Ranks
    rk = rk or Ranks("nccl")
    boxes = E.prepare_tables(E.shard(E.ensemble_boxes(96), rk.rank, rk.world))
    warm = E.prepare_tables(E.ensemble_boxes(10, master_seed=1))
    for b in warm:
        b.nsteps = 3
    E.run_serial(warm)
    E.run_batched(warm)
    E.run_batched(warm, multi=False)
    torch.cuda.synchronize()
    # each arm twice, alternately; the faster of each is kept (the first pass
    # after a large box is freed can pay one-time allocation costs).  Batched:
    # one launch per phase across the size classes (the default); the same
    # with one launch per phase per class on parallel streams beside it
    reps = {"one_at_a_time": [], "batched": [], "batched_per_class": []}
    for _ in range(2):
        rk.barrier()
        serial, t = E.timed(E.run_serial, boxes)
        reps["one_at_a_time"].append(rk.allmax(t))
        rk.barrier()
        batched, t = E.timed(E.run_batched, boxes)
        reps["batched"].append(rk.allmax(t))
        rk.barrier()
        _, t = E.timed(lambda b: E.run_batched(b, multi=False), boxes)
        reps["batched_per_class"].append(rk.allmax(t))
    t_serial, t_batch = min(reps["one_at_a_time"]), min(reps["batched"])
    st_serial, st_batch, st_pc = {}, {}, {}
    E.run_serial(boxes, stages=st_serial)
    E.run_batched(boxes, stages=st_batch)
    E.run_batched(boxes, stages=st_pc, multi=False)
    worst, counts = _check_same(batched, serial)
    worst = rk.allmax(worst)
    counts = rk.allsum(0.0 if counts else 1.0) == 0.0
    classes, _ = E.class_layout(boxes)
    return {
        "metric": "ensemble sims/hour (96 mixed boxes, 64 steps each)", "value": 96 / t_batch * 3600.0,
        "unit": "sims/hour", "higher_is_better": True, "n_gpus": rk.world,
        "one_at_a_time": {"value": 96 / t_serial * 3600.0, "seconds": t_serial},
        "batched_seconds": t_batch, "speedup_vs_one_at_a_time": t_serial / t_batch, "seconds_per_pass": reps,
        "stages_s": {"batched": st_batch, "batched_per_class": st_pc, "one_at_a_time": st_serial},
        "batched_per_class_seconds": min(reps["batched_per_class"]),
        "speedup_steps_only": st_serial["steps"] / st_batch["steps"],
        "speedup_compute_only": (sum(v for k, v in st_serial.items() if k != "create") /
                                 sum(v for k, v in st_batch.items() if k != "create")),
        "pk_max_rel_diff_vs_one_at_a_time": worst, "pk_counts_equal": counts,
        "config": {"workload": "96 boxes, ng = np uniform over {32,48,64,96,128}, L ~ U[64,512] Mpc/h, "
                               "sigma8 ~ U[0.7,0.9], seeds 1000+i, EH ICs at z=100, 64 steps, P(k) 32 bins",
                   "classes_rank0": classes, "timed": "ICs + 64 steps + final P(k) of every box (host-side "
                                                      ".ipk tables prepared beforehand for both)",
                   "batched": "one launch per phase across all size classes (deposit and kick persistent, "
                              "FFT passes one CTA per unit), CUDA graph per step",
                   "batched_per_class": "one launch per phase per size class, classes on parallel streams, "
                                        "CUDA graph per step",
                   "parallelism": "replicas: %d rank(s), whole boxes per rank by predicted cost" % rk.world},
        "dtype": "f32", "data": "synthetic: seeded EH no-wiggle Zel'dovich ICs",
    }


def form_serve(nreq, rk=None):
    """A Poisson request stream served with continuous batching against the
    same stream one request at a time.  Under torchrun each rank serves its
    share of the requests (ensemble.shard) on its own GPU, from a common
    start after a barrier; latencies are gathered, makespans are the
    slowest rank's."""
    import torch

    from hacc_gpm_b200 import ensemble as E
    from hacc_gpm_b200 import serve as S
    from hacc_gpm_b200.replicas import Ranks
    rk = rk or Ranks("nccl")

    def mine():
        return E.shard(S.request_stream(nreq), rk.rank, rk.world)

    warm = S.request_stream(8, rate=1000.0, seed=3, steps=(2, 3))
    S.serve(warm, realtime=False)
    S.serve_one_at_a_time(S.request_stream(8, rate=1000.0, seed=3, steps=(2, 3)), realtime=False)
    torch.cuda.synchronize()
    rk.barrier()
    got, mk, stats = S.serve(mine())
    mk = rk.allmax(mk)
    rk.barrier()
    one, mk1 = S.serve_one_at_a_time(mine())
    mk1 = rk.allmax(mk1)
    rk.barrier()
    sat, mks, _ = S.serve(mine(), realtime=False)
    mks = rk.allmax(mks)
    # one at a time, saturated, twice: its per-request context allocation
    # makes passes differ by up to 2x; the faster pass is the baseline
    passes = []
    for _ in range(2):
        rk.barrier()
        sat1, t1 = S.serve_one_at_a_time(mine(), realtime=False)
        passes.append(rk.allmax(t1))
    mks1 = min(passes)
    worst, counts = _check_same(sorted(got, key=lambda r: r.tag), sorted(one, key=lambda r: r.tag))
    worst = rk.allmax(worst)
    counts = rk.allsum(0.0 if counts else 1.0) == 0.0

    class _L:
        def __init__(self, lat):
            self.latency = lat

    def everyone(reqs):
        return [_L(x) for part in rk.gather([r.latency for r in reqs]) for x in part]

    out = S.latency_summary(everyone(got), mk)
    return {
        "metric": "serving p99 completion latency (Poisson 20 req/s)", "value": out["p99_s"], "unit": "s",
        "higher_is_better": False, "n_gpus": rk.world, "batched": out,
        "one_at_a_time": S.latency_summary(everyone(one), mk1),
        "saturated": {"batched_sims_per_hour": nreq / mks * 3600.0,
                      "one_at_a_time_sims_per_hour": nreq / mks1 * 3600.0, "speedup": mks1 / mks,
                      "one_at_a_time_seconds_per_pass": passes, "batched_seconds": mks},
        "pk_max_rel_diff_vs_one_at_a_time": worst, "pk_counts_equal": counts,
        "config": {"workload": "%d requests, Poisson arrivals 20/s (seed 7), ng = np log-uniform over "
                               "{32,48,64,96,128,192,256}, L = ng Mpc/h, steps U[20,200], Om U[0.25,0.35], "
                               "sigma8 U[0.7,0.9], EH ICs at z=50" % nreq,
                   "classes_rank0": stats["classes"],
                   "admission": "slots per size class from a 40 GB HBM budget split over the classes by footprint "
                                "per slot, at most the slots whose batched step is ~2 ms of GPU time",
                   "scheduling": "each class on its own stream at its own pace (batches of ~1 ms), stream "
                                 "priority by box size (smaller first)",
                   "parallelism": "replicas: %d rank(s), whole requests per rank by predicted cost" % rk.world},
        "dtype": "f32", "data": "synthetic",
    }


def run_forms(args):
    """--workload ensemble | serve: the batched form's own line (one rank per
    GPU under torchrun; rank 0 prints)."""
    import torch

    from hacc_gpm_b200.replicas import Ranks
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rk = Ranks("nccl")
    out = form_ensemble(rk) if args.workload == "ensemble" else form_serve(args.requests, rk)
    rk.close()
    if rk.rank == 0:
        print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="NS", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-full", action="store_true", help="skip the whole-run timing")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched ensemble and serving forms")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (built-in or cached choices)")
    ap.add_argument("--size", type=int, default=0, help="np = ng = rl (profiling runs use a smaller box)")
    ap.add_argument("--workload", default="step", choices=["step", "ensemble", "serve"])
    ap.add_argument("--requests", type=int, default=160, help="serve: requests in the stream")
    args = ap.parse_args()
    if args.workload != "step":
        run_forms(args)
        return
    global NG, NP, RL, NSTEPS_RUN, MID_STEP
    NG, NP, RL, NSTEPS_RUN, MID_STEP = CONFIGS[args.config]
    if args.size:
        NG = NP = args.size
        RL = float(args.size)
    if args.impl == "reference":
        run_reference(args)
        return

    import numpy as np
    import torch

    from hacc_gpm_b200.replicas import Ranks

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rk = Ranks("nccl")  # replicas: NCCL only for the barrier and max-over-ranks timing
    world, rank, local = rk.world, rk.rank, rk.local
    barrier, allmax = rk.barrier, rk.allmax

    import hacc_gpm_b200 as H

    params = H.parse_params(run_params_text(rank))
    header, table = run_ipk(params)
    sim = H.Simulation(params, device=local)
    sim.generate_ic(table, header[3])
    ts = H.Timestepper(params)
    ts.set_initial_z(params.z_ini)
    ts.reverse_half_step()
    ts.advance_half_step()
    stream = torch.cuda.ExternalStream(sim.stream)

    # untimed advance to the middle of the run, the autotuner on that state
    # (it times every configuration of the tunable phases and leaves the
    # state unchanged), then warm-up
    start = first_warmup_step(args.steps, args.warmup)
    sim.run_steps(ts, start)
    tuned = sim.autotune(reps=3) if not args.no_tune else sim.tuned_choices()
    sim.run_steps(ts, args.warmup)
    sim.sync()

    # timed region (per-kernel events on the same stream, inside the region)
    clocks = ClockSampler(local)
    sim.enable_timing(True)
    sim.phase_times()
    barrier()
    torch.cuda.synchronize()
    sim.sync()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = sim.kernel_launches()
    e0.record(stream)
    sim.run_steps(ts, args.steps)
    e1.record(stream)
    e1.synchronize()
    launches = sim.kernel_launches() - launches0
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ph_ms, ph_n = sim.phase_times()
    sim.enable_timing(False)
    ms = e0.elapsed_time(e1)
    ms_max = allmax(ms)
    np3, ng3 = NP ** 3, NG ** 3
    value = world * np3 * args.steps / (ms_max * 1e-3)
    run_state = {"first_timed_step": start + args.warmup, "a_after": ts.aa}
    peak, peak_kind = measured_peak()
    kick_choice = tuned["kick"]["choice"] if isinstance(tuned["kick"], dict) else tuned["kick"]
    potential_kick = kick_choice >= 5
    names = kernel_names(tuned, NP, NG)
    ab = alg_bytes(np3, ng3, potential_kick)
    phases = {}
    for k, b in ab.items():
        n = int(ph_n.get(k, 0))
        if n == 0:
            continue
        # events bracket the phase (all its kernels) once per step
        avg = ph_ms[k] / args.steps
        phases[k] = {"ms_per_step": avg, "kernels": n, "kernel": names[k], "alg_bytes": b,
                     "alg_gbs": b / (avg * 1e-3) / 1e9 if b else 0.0,
                     "frac_of_peak": (b / (avg * 1e-3) / 1e9 / peak) if b else None}
    dom = max(phases, key=lambda k: phases[k]["ms_per_step"])
    d = phases[dom]
    roofline = {"bound": "hbm", "kernel": names[dom], "phase": dom,
                "achieved": d["alg_gbs"], "peak": peak, "unit": "GB/s", "frac": d["alg_gbs"] / peak,
                "peak_kind": peak_kind, "traffic": None, "alg_bytes_per_launch": d["alg_bytes"],
                "ms_per_launch": d["ms_per_step"]}
    step_ms = ms_max / args.steps
    b_step = sum(ab.values())  # 72 Np + 32 Ng (potential kick) or 72 Np + 56 Ng
    step_roof = {"alg_bytes_per_step": b_step, "achieved_gbs": b_step / (step_ms * 1e-3) / 1e9,
                 "frac": b_step / (step_ms * 1e-3) / 1e9 / peak, "peak": peak,
                 "survey_bytes_per_step": 72 * np3 + 64 * ng3,
                 "survey_frac": (72 * np3 + 64 * ng3) / (step_ms * 1e-3) / 1e9 / peak}
    # DRAM bytes per launch from an ncu capture (profiles/traffic_<NG>.json:
    # per phase the kernel captured and its bytes), used only when the
    # captured kernel is the one this run timed
    tp = os.path.join(ROOT, "profiles", "traffic_%d.json" % NG)
    if os.path.exists(tp) and NG == NP:
        with open(tp) as f:
            traf = json.load(f)
        t = traf.get(dom)
        if isinstance(t, dict) and names[dom].startswith(t.get("kernel", "?")):
            roofline["traffic"] = t["bytes"]

    # the CPU baseline on this state (rank 0, N = 1): 2 steps of the OpenMP
    # transcription from the state the timed steps ended with
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        with tempfile.TemporaryDirectory() as dtmp:
            dump = os.path.join(dtmp, "state")
            xh, vh = sim.store_state()
            np.concatenate([xh.ravel(), vh.ravel()]).astype("<f4").tofile(dump)
            del xh, vh
            at = start + args.warmup + args.steps
            r = cpu_baseline(steps=2, warmup=0, load=dump, start_step=at, cosmo=cosmo_args(params))
        cpu = {"value": np3 / r["sec_per_step"], "unit": UNIT, "cores": r["threads"], "kind": "port",
               "sample": "2 full %d^3 steps (steps %d-%d of the run, the state this GPU run reached) of the "
                         "OpenMP C++ transcription of the reference's serial step (float3 layout, float atomics, "
                         "C2C FFTs) on %d host threads" % (NP, at, at + 1, r["threads"])}

    # end to end through the C-ABI with pinned host buffers, every step:
    # H2D state -> one step -> D2H state
    e2e = None
    if not args.no_e2e:
        x_h, v_h = sim.store_state()
        xp = torch.from_numpy(x_h).pin_memory()
        vp = torch.from_numpy(v_h).pin_memory()
        xn, vn = xp.numpy(), vp.numpy()
        sim.step_host(ts, xn, vn)  # warm-up
        barrier()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.e2e_steps):
            sim.step_host(ts, xn, vn)
        t1.record(stream)
        t1.synchronize()
        barrier()
        ems = allmax(t0.elapsed_time(t1))
        e2e = {"value": world * np3 * args.e2e_steps / (ems * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": 24 * np3, "d2h_bytes_per_step": 24 * np3, "steps": args.e2e_steps,
               "path": "hgpm_step_host (C-ABI, pinned float3 x,v in and out every step)"}

    # the whole run once (fresh ICs), for the run-average cost
    full = None
    if not args.no_full:
        sim.generate_ic(table, header[3])
        tsf = H.Timestepper(params)
        tsf.set_initial_z(params.z_ini)
        tsf.reverse_half_step()
        tsf.advance_half_step()
        sim.sync()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        sim.run_steps(tsf, NSTEPS_RUN)
        f1.record(stream)
        f1.synchronize()
        fms = allmax(f0.elapsed_time(f1))
        full = {"steps": NSTEPS_RUN, "ms_per_step": fms / NSTEPS_RUN,
                "value": world * np3 * NSTEPS_RUN / (fms * 1e-3), "unit": UNIT, "z": "%g -> 0" % Z_INI}

    sim.close()
    forms = None
    if rank == 0 and world == 1 and args.config == "NS" and not args.size and not args.no_forms:
        forms = {"ensemble": form_ensemble(rk), "serve": form_serve(args.requests, rk)}
    rk.close()
    if rank != 0:
        return
    out = {
        "metric": metric_name(), "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded EH no-wiggle Zel'dovich ICs (the reference's cuRAND white noise), seed + rank",
        "config": bench_config(args.steps, args.warmup),
        "execution": "replicas (one independent box per GPU)",
        "roofline": roofline, "step_roofline": step_roof, "phases": phases, "cpu_baseline": cpu, "e2e": e2e,
        "full_run": full, "timed_steps": run_state, "gpu_launches": int(launches), "clocks": clk,
        "autotuned": tuned, "forms": forms,
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
