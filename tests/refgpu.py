"""Access to the reference-output fixtures tests/golden/refgpu_*.npz (made by
tests/golden/make_refgpu_fixtures.py from the reference's own serial CUDA
path) and the tolerances the parity tests hold against them."""
from __future__ import annotations

import os

import numpy as np

from oracle import pm_oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("a32", "b24")

# bars against the reference's own outputs
IC_POS_CELLS = 1e-5      # Zel'dovich positions, absolute, in cells
IC_VEL_REL = 1e-5        # velocities, relative to the max
RHO_REL = 1e-6           # density, relative to the max (reference: float atomics)
FORCE_REL = 1e-5         # force grids, relative to the max (the 1e-5 field bar)
POS_BOX = 1e-4           # positions after N steps, fraction of the box
PK_REL = 1e-3            # P(k) per bin (0.1 %)


class Case:
    def __init__(self, name):
        self.name = name
        self.d = np.load(os.path.join(GOLD, "refgpu_%s.npz" % name))
        self.params_text = str(self.d["params"])
        self.p = O.parse_params_text(self.params_text)
        self.ng = self.p.ng
        self.nsteps = int(self.d["nsteps_run"])
        ipk = self.d["ipk"]
        self.ipk_header, self.ipk_table = ipk[:20], ipk[20:]

    def __getitem__(self, k):
        return self.d[k]


def parse_pk(text):
    rows = [r.split(",") for r in str(text).strip().splitlines()]
    k = np.array([float(r[0]) for r in rows])
    p = np.array([float(r[1]) for r in rows])
    n = np.array([int(r[2]) for r in rows])
    return k, p, n


def nonempty(k, p, n):
    """Bins writePkOutput would print (power.cu:19-26)."""
    m = (n > 0) & (p == p) & (p != 0)
    return k[m], p[m], n[m]
