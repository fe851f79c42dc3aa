"""Shared test helpers: seeded synthetic states, run files and tolerances."""
from __future__ import annotations

import os
import tempfile

import numpy as np

from hacc_gpm_b200 import ipk as ipkmod
from oracle import pm_oracle as O

# Parity bars: fields 1e-5 relative to the field's max, final
# positions 1e-4 of the box side, P(k) 0.1 % per bin.
FIELD_RTOL = 1e-5
POS_BOX_TOL = 1e-4
PK_RTOL = 1e-3


def params_text(ng, np_side=None, rl=None, z_ini=50.0, nsteps=10, seed=21082001, extra=""):
    np_side = np_side or ng
    rl = rl if rl is not None else float(ng)
    return ipkmod.lcdm_params_text(ng, np_side, rl, z_ini, nsteps, seed=seed, extra=extra)


def lattice_state(np_side: int, ng: int, disp: float = 0.7, vel: float = 2.0, seed: int = 1):
    """Lattice positions (Lagrangian order, get_index) plus seeded Gaussian
    displacements/velocities, wrapped into [0, ng), as float32."""
    rng = np.random.default_rng(seed)
    q = np.stack(np.meshgrid(np.arange(np_side), np.arange(np_side), np.arange(np_side), indexing="ij"),
                 axis=-1).reshape(-1, 3).astype(np.float64) * (ng / np_side)
    x = np.mod(q + disp * rng.standard_normal(q.shape), ng).astype(np.float32)
    x[x >= ng] = 0.0
    v = (vel * rng.standard_normal(q.shape)).astype(np.float32)
    return x, v


def eh_table(cosmo_params, z, k_max=20.0, k_bins=20000):
    header, table = ipkmod.make_ipk(ipkmod.cosmo_from_params(cosmo_params), z, k_max=k_max, k_bins=k_bins)
    return header, table


def oracle_ics(p: O.Params, seed_noise=None, k_max=20.0):
    """Realistic ICs from the oracle: Philox noise + EH table + Zel'dovich."""
    header, table = eh_table(p, p.z_ini, k_max=k_max)
    noise = O.philox_normal(p.np ** 3, p.seed if seed_noise is None else seed_noise).reshape(p.np, p.np, p.np)
    x, v = O.generate_ic_from_noise(noise.astype(np.float64), p, table, header[3])
    return x.astype(np.float32), v.astype(np.float32), noise, table, header


def rel_max_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def box_pos_err(x, y, ng):
    return float(np.max(np.abs(O.periodic_diff(x, y, ng))) / ng)
