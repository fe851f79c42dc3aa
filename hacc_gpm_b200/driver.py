"""The reference's serial() run (src/driver_pm.cpp:32-163) from Python, with
its Python analysis hook.

``serial(path)`` reads the params file and writes what the reference's run
writes (``<prefix>.params``, ``<prefix>.pk.{ini,<step>,fin}.fold.<f>``,
``<prefix>.particles.{ini,<step>,fin}``), the same files as the C++ driver
``_lib/haccgpm``.  With DO_ANALYSIS, at the steps ANALYSIS_STEPS marks the
particles' rows go to ``analysis(rows, step, a, z)`` (PyAnalysis,
py_analysis.cu:3-27): rows is a (np^3, 7) float32 array, columns tag
(lattice index), x, y, z, vx, vy, vz.  Without an ``analysis`` argument the
function ``analysis_step`` of the module at ANALYSIS_PY is called (the
reference reaches its Python module through pycosmotools, a submodule absent
here, so this calling convention is this project's own); with neither, the
rows are written as ``<ANALYSIS_DIR>/analysis.<step>`` like the C++ driver.
"""
from __future__ import annotations

import importlib.util
import os

import numpy as np

from .binding import Simulation, Timestepper, read_ipk, read_params, write_pk


def _load_hook(path: str):
    spec = importlib.util.spec_from_file_location("hgpm_analysis_module", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.analysis_step


def _pk(sim: Simulation, p, name: str):
    for fold in range(p.pk_folds + 1):
        k, P, n = sim.power_spectrum(p.pk_bins or 221, bool(p.pk_log), fold=fold)
        write_pk(name, k, P, n, fold=fold)


def serial(params_path: str, analysis=None, fused: bool = True, device: int = 0):
    """One run of serial(); returns the final (x, v) as float3 arrays.
    fused: steps between two outputs run through run_steps (bit-identical
    to the phase-by-phase loop)."""
    p = read_params(params_path)
    p.save()
    hook = analysis
    if hook is None and p.do_analysis and p.analysis_py:
        hook = _load_hook(p.analysis_py)
    if hook is None:
        out_dir = p.analysis_dir or "."

        def hook(rows, step, a, z):
            rows.tofile(os.path.join(out_dir, "analysis.%d" % step))

    header, table = read_ipk(p.ipk)
    with Simulation(p, device=device) as sim:
        ts = Timestepper(p)
        ts.set_initial_z(p.z_ini)
        ts.reverse_half_step()
        sim.generate_ic(table, header[3])
        _pk(sim, p, "%s.pk.ini" % p.prefix)
        if p.dump_init:
            sim.write_output("%s.particles.ini" % p.prefix)
        ts.advance_half_step()
        step = 0
        while step < p.last_step:
            end = step
            if fused:
                while (end < p.last_step - 1 and not p.pks[end] and not p.dumps[end]
                       and not (p.do_analysis and p.analysis[end])):
                    end += 1
            sim.run_steps(ts, end - step + 1)
            step = end
            if p.pks[step]:
                _pk(sim, p, "%s.pk.%d" % (p.prefix, step))
            if p.dumps[step]:
                sim.write_output("%s.particles.%d" % (p.prefix, step))
            if p.do_analysis and p.analysis[step]:
                hook(sim.analysis_rows(), step, ts.aa, ts.z)
            step += 1
        _pk(sim, p, "%s.pk.fin" % p.prefix)
        if p.dump_final:
            sim.write_output("%s.particles.fin" % p.prefix)
        return sim.store_state()


if __name__ == "__main__":
    import sys

    if len(sys.argv) < 2:
        print("USAGE: python -m hacc_gpm_b200.driver <params>")
        sys.exit(1)
    serial(sys.argv[1])
