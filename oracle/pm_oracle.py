"""FP64 CPU restatement of HACC_GPM's serial particle-mesh path.

TEST INFRASTRUCTURE ONLY.  This module is the oracle that the CUDA path is
compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it; the
product (``hacc_gpm_b200`` and its C-ABI library) never does.

Every function restates one piece of the reference's serial path in float64
NumPy, citing the reference file:line it follows (paths are relative to the
HACC_GPM project root).  FFTs are complex128 (``scipy.fft`` on all host
threads when SciPy is present, else ``numpy.fft``: the same transforms) with
the same sign and normalisation conventions as the reference's cuFFT calls
(``src/fft_tools/cuda/ffts.cu:271`` forward = e^{-ikx}, ``:423`` inverse,
unnormalised).

Where the reference rounds through float32 on purpose (``atof`` into a float
in the params parser, ``float dtdy`` in the time stepper, the float growth
integral) the oracle follows it when ``ref_quirks=True`` (the default), so
that its scalars equal the reference's; ``ref_quirks=False`` gives the pure
FP64 value.  Bulk particle/grid arithmetic is always float64.

Parity pinning: the reference ships no tests or golden vectors.  This oracle
is pinned against outputs of the reference's own CUDA serial path compiled
from its sources (``oracle/ref_harness``), committed as fixtures under
``tests/golden/`` together with the script that generated them.
"""
from __future__ import annotations

import math
import os
import struct
from dataclasses import dataclass, field

import numpy as np

try:
    import scipy.fft as _sfft

    def _fftn(a):
        return _sfft.fftn(a, workers=-1)

    def _ifftn(a):
        return _sfft.ifftn(a, workers=-1)
except ImportError:  # pragma: no cover
    _fftn, _ifftn = np.fft.fftn, np.fft.ifftn

MAX_STEPS = 1000  # src/haccgpm.hpp:106


def _f32(v: float) -> float:
    """Round a Python float through IEEE float32 (the reference's ``float``)."""
    return float(np.float32(v))


# ---------------------------------------------------------------------------
# Params (src/simulation/params.cpp:72-250, src/haccgpm.hpp:118-174)
# ---------------------------------------------------------------------------

_FLOAT_KEYS = {
    "OMEGA_CDM": "omega_cdm", "DEUT": "deut", "OMEGA_NU": "omega_nu",
    "HUBBLE": "hubble", "SS8": "ss8", "NS": "ns", "W_DE": "w_de",
    "WA_DE": "wa_de", "T_CMB": "t_cmb", "N_EFF_MASSLESS": "neff_massless",
    "N_EFF_MASSIVE": "neff_massive", "Z_IN": "z_ini", "Z_FIN": "z_fin",
    "RL": "rl",
}
_INT_KEYS = {
    "N_STEPS": "nsteps", "NG": "ng", "NP": "np", "SEED": "seed",
    "BLOCK_SIZE": "block_size", "LAST_STEP": "last_step", "PK_FOLDS": "pk_folds",
    "PK_BINS": "pk_bins", "PK_LOG": "pk_log",
}


@dataclass
class Params:
    """Mirror of ``HACCGPM::Params`` (src/haccgpm.hpp:118-174)."""
    omega_cdm: float = 0.0
    deut: float = 0.0
    omega_nu: float = 0.0
    hubble: float = 0.0
    ss8: float = 0.0
    ns: float = 0.0
    w_de: float = -1.0
    wa_de: float = 0.0
    t_cmb: float = 2.726
    neff_massless: float = 3.04
    neff_massive: float = 0.0
    z_ini: float = 200.0
    z_fin: float = 0.0
    rl: float = 0.0
    nsteps: int = 0
    ng: int = 0
    np: int = 0
    seed: int = 0
    block_size: int = 64
    last_step: int = -1
    pk_folds: int = 0
    pk_bins: int = 221  # params.cpp:91 (fixed in the reference)
    pk_log: int = 0
    prefix: str = ""
    ipk: str = ""
    ol: float = 1.0
    dump_init: bool = False
    dump_final: bool = False
    pks: list = field(default_factory=lambda: [False] * MAX_STEPS)
    dumps: list = field(default_factory=lambda: [False] * MAX_STEPS)
    # derived (params.cpp:237-245)
    omega_baryon: float = 0.0
    omega_cb: float = 0.0
    omega_matter: float = 0.0
    omega_radiation: float = 0.0
    f_nu_massless: float = 0.0
    f_nu_massive: float = 0.0
    overload: int = 0


def derive(p: Params) -> Params:
    """Derived cosmology, params.cpp:237-245 (pow(T/2.725f, 4.0f) in float)."""
    p.overload = int(math.ceil(p.ng / p.rl * p.ol)) if p.rl else 0
    p.omega_baryon = p.deut / p.hubble / p.hubble
    p.omega_cb = p.omega_cdm + p.omega_baryon
    p.omega_matter = p.omega_cb + p.omega_nu
    # pow(m_Tcmb/2.725f, 4.0f)/pow(m_hubble, 2.0f): double-precision pow of
    # (double/float-promoted) arguments.
    p.omega_radiation = 2.471e-5 * (p.t_cmb / _f32(2.725)) ** 4.0 / (p.hubble ** 2.0)
    c = 7.0 / 8.0 * (4.0 / 11.0) ** (4.0 / 3.0)
    p.f_nu_massless = p.neff_massless * c
    p.f_nu_massive = p.neff_massive * c
    if p.last_step == -1:
        p.last_step = p.nsteps
    return p


def parse_params_text(text: str) -> Params:
    """Parse ``KEY VALUE`` lines like params.cpp:102-226.

    Float values go through ``float val = atof(value)`` (float32 rounding,
    params.cpp:109); unknown keys are ignored; ``PK_DUMP``/``PARTICLE_DUMP``
    take comma lists (``all`` for dumps).  ``PK_BINS``/``PK_LOG`` are keys this
    project adds (the reference fixes 221 linear bins, params.cpp:91).
    """
    p = Params()
    for raw in text.splitlines():
        toks = raw.split()
        if len(toks) < 1:
            continue
        key = toks[0]
        val = toks[1] if len(toks) > 1 else ""
        if key in _FLOAT_KEYS:
            setattr(p, _FLOAT_KEYS[key], _f32(float(val)))
        elif key in _INT_KEYS:
            setattr(p, _INT_KEYS[key], int(float(val)) if val else 0)
        elif key == "OUTPUT_BASE_NAME":
            p.prefix = val
        elif key == "IPK":
            p.ipk = val
        elif key == "OL":
            p.ol = float(val)
        elif key == "DUMP_INIT":
            p.dump_init = True
        elif key == "DUMP_FINAL":
            p.dump_final = True
        elif key == "PK_DUMP":
            for t in val.split(","):
                if t:
                    p.pks[int(t)] = True
        elif key == "PARTICLE_DUMP":
            if val == "all":
                p.dumps = [True] * MAX_STEPS
            else:
                for t in val.split(","):
                    if t:
                        p.dumps[int(t)] = True
    if p.np == 0:
        raise ValueError("NP missing or zero (params.cpp:228 asserts np != 0)")
    return derive(p)


def read_params(path: str) -> Params:
    with open(path) as f:
        return parse_params_text(f.read())


# ---------------------------------------------------------------------------
# Time stepper (src/simulation/timestepper.cpp:7-68)
# ---------------------------------------------------------------------------

def omega_nu_massive(a, p: Params):
    """timestepper.cpp:7-11."""
    mat = p.omega_nu / a ** 3.0
    rad = p.f_nu_massive * p.omega_radiation / a ** 4.0
    return mat if mat >= rad else rad


def get_adot(a, p: Params):
    """timestepper.cpp:13-21."""
    pp1 = a ** (-3.0 * (p.w_de + p.wa_de)) * math.exp(-3.0 * p.wa_de * (1.0 - a))
    tmp = (p.omega_cb + (1.0 + p.f_nu_massless) * p.omega_radiation / a
           + omega_nu_massive(a, p) * a ** 3.0
           + (1.0 - p.omega_matter - (1.0 + p.f_nu_massless) * p.omega_radiation) * pp1)
    tmp /= a
    return math.sqrt(tmp)


def get_fscal(a, adot, omega_cb, ref_quirks=True):
    """timestepper.cpp:23-28; ``float dtdy`` at :24 when ``ref_quirks``."""
    dtdy = a / (a * adot)
    if ref_quirks:
        dtdy = _f32(dtdy)
    return 1.5 * omega_cb * dtdy * (1.0 / a)


class Timestepper:
    """timestepper.cpp:31-68: uniform step in a, leapfrog half steps."""

    def __init__(self, p: Params, ref_quirks=True):
        self.p = p
        self.ref_quirks = ref_quirks
        self.deltaT = ((1.0 / (p.z_fin + 1.0)) - (1.0 / (p.z_ini + 1.0))) / float(p.nsteps)
        self.aa = 0.0
        self.adot = 0.0
        self.fscal = 0.0

    def _update(self):
        self.adot = get_adot(self.aa, self.p)
        self.fscal = get_fscal(self.aa, self.adot, self.p.omega_cb, self.ref_quirks)

    def set_initial_z(self, z):
        self.aa = 1.0 / (z + 1.0)
        self._update()

    def advance_half_step(self):
        self.aa += self.deltaT * 0.5
        self._update()

    def reverse_half_step(self):
        self.aa -= self.deltaT * 0.5
        self._update()

    def drift_prefactor(self, frac=0.5):
        """pm_actions.cpp:291 ``float prefactor = deltaT/(a*a*adot)*frac``."""
        v = (self.deltaT / (self.aa * self.aa * self.adot)) * frac
        return _f32(v) if self.ref_quirks else v


# ---------------------------------------------------------------------------
# Index helpers (src/haccgpm.hpp:255-274, :423-429)
# ---------------------------------------------------------------------------

def signed_index(ng: int) -> np.ndarray:
    """get_kmodes: index > ng/2-1 maps to index-ng (haccgpm.hpp:255-274)."""
    i = np.arange(ng)
    return np.where(i > ng // 2 - 1, i - ng, i)


def kmodes_f32(ng: int, d: float) -> np.ndarray:
    """1D k values as the reference forms them: ``float l = idx; l *= d``
    (float*double product stored to float, haccgpm.hpp:256-260)."""
    return (signed_index(ng).astype(np.float64) * d).astype(np.float32)


# ---------------------------------------------------------------------------
# Particle actions
# ---------------------------------------------------------------------------

def drift(x: np.ndarray, v: np.ndarray, prefactor: float, ng: int) -> np.ndarray:
    """UpdatePosKernel: x <- fmod(x + v*pf + ng, ng) (update_positions_pm.cu:3-20)."""
    return np.fmod(x + v * prefactor + ng, ng)


def cic_corners(x: np.ndarray, ng: int):
    """Base cell and fractional offsets as in cic_pm.cu:51-58 (``int i = x``,
    truncation, then ``diff = x - i``); corners wrap with ``% ng`` (:63-66)."""
    i = np.trunc(x).astype(np.int64)
    diff = x - i
    return i, diff


def _corner_iter():
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                yield dx, dy, dz


def cic_deposit(x: np.ndarray, ng: int, mass: float) -> np.ndarray:
    """CICKernel (cic_pm.cu:46-87): 8 weights (1-d or d) * mass, periodic wrap.
    Returns the real density grid (mean (np/ng)^3*mass*... = 1 when mass=(ng/np)^3)."""
    i, diff = cic_corners(x, ng)
    rho = np.zeros(ng ** 3, dtype=np.float64)
    for cx, cy, cz in _corner_iter():
        wx = diff[:, 0] if cx else 1.0 - diff[:, 0]
        wy = diff[:, 1] if cy else 1.0 - diff[:, 1]
        wz = diff[:, 2] if cz else 1.0 - diff[:, 2]
        w = wx * wy * wz * mass
        nx = (i[:, 0] + cx) % ng
        ny = (i[:, 1] + cy) % ng
        nz = (i[:, 2] + cz) % ng
        idx = (nx * ng + ny) * ng + nz  # get_index row-major, z fastest
        rho += np.bincount(idx, weights=w, minlength=ng ** 3)
    return rho.reshape(ng, ng, ng)


def cic_mass(ng: int, np_side: int) -> float:
    """pm_actions.cpp:229-230: mass = (float(ng)/float(np))^3 in float."""
    g = np.float32(ng) / np.float32(np_side)
    return float(g * g * g)


def greens(ng: int, ref_quirks: bool = False) -> np.ndarray:
    """calcGreens (calcGreens.hpp:11-25): G = 0.5/ng^3 / (cos kx + cos ky + cos kz - 3),
    G(0) = 0; the cos arguments are unsigned index*2pi/ng.  The reference
    forms the argument in float (``idx3d * d`` with ``float d``) and calls
    ``cos`` on a float, i.e. the float overload; ``ref_quirks`` reproduces
    that rounding (it moves G by up to ~1e-4 relative at the lowest k)."""
    if ref_quirks:
        d = np.float32(2.0 * np.pi / np.float32(ng))
        arg = np.arange(ng).astype(np.float32) * d
        c = np.cos(arg).astype(np.float32).astype(np.float64)
    else:
        c = np.cos(2.0 * np.pi * np.arange(ng) / ng)
    s = c[:, None, None] + c[None, :, None] + c[None, None, :] - 3.0
    with np.errstate(divide="ignore"):
        g = (0.5 / ng ** 3) / s
    g[0, 0, 0] = 0.0
    return g


def solve_gradient(rho: np.ndarray, ref_quirks: bool = False) -> np.ndarray:
    """serial::SolveGradient one-grid path (solver.cpp:144-170):
    forward C2C FFT, then per dim F_k = -i sin(k_dim) G rho_k
    (kspace_solver.cu:55-90: c = -sin(k)*G, out = (-c*Im, c*Re)), inverse C2C
    (unnormalised, 1/ng^3 sits in G), real part into the force grid
    (transform_density_field_initializer.cu:14-28).  Returns (3, ng, ng, ng)."""
    ng = rho.shape[0]
    rk = _fftn(rho.astype(np.complex128))
    g = greens(ng, ref_quirks)
    k1 = signed_index(ng) * (2.0 * np.pi / ng)
    sk = np.sin(k1)
    out = np.empty((3,) + rho.shape, dtype=np.float64)
    shapes = [(ng, 1, 1), (1, ng, 1), (1, 1, ng)]
    for dim in range(3):
        c = -sk.reshape(shapes[dim]) * g
        fk = 1j * c * rk  # (-c*Im, c*Re) == i*c*rho
        out[dim] = _ifftn(fk).real * ng ** 3  # unnormalised inverse
    return out


def interp_kick(x: np.ndarray, v: np.ndarray, force: np.ndarray, deltaT: float,
                fscal: float) -> np.ndarray:
    """ICICKernel (icic_pm.cu:72-127): v += sum_8 w * grad[corner] * deltaT * fscal."""
    ng = force.shape[1]
    i, diff = cic_corners(x, ng)
    f = force.reshape(3, -1)
    dv = np.zeros_like(v)
    for cx, cy, cz in _corner_iter():
        wx = diff[:, 0] if cx else 1.0 - diff[:, 0]
        wy = diff[:, 1] if cy else 1.0 - diff[:, 1]
        wz = diff[:, 2] if cz else 1.0 - diff[:, 2]
        w = wx * wy * wz * deltaT * fscal
        nx = (i[:, 0] + cx) % ng
        ny = (i[:, 1] + cy) % ng
        nz = (i[:, 2] + cz) % ng
        idx = (nx * ng + ny) * ng + nz
        dv += w[:, None] * f[:, idx].T
    return v + dv


def pm_step(x, v, ts: Timestepper, ng: int, np_side: int):
    """One DKD step as sequenced in driver_pm.cpp:114-125."""
    x = drift(x, v, ts.drift_prefactor(0.5), ng)
    rho = cic_deposit(x, ng, cic_mass(ng, np_side))
    force = solve_gradient(rho, ts.ref_quirks)
    ts.advance_half_step()
    v = interp_kick(x, v, force, ts.deltaT, ts.fscal)
    ts.advance_half_step()
    x = drift(x, v, ts.drift_prefactor(0.5), ng)
    return x, v


def run(x, v, p: Params, nsteps: int | None = None, ref_quirks=True):
    """driver_pm.cpp:63-142 minus ICs and I/O: the time stepper starts at
    a(z_ini) then steps half forward before the loop."""
    ts = Timestepper(p, ref_quirks)
    ts.set_initial_z(p.z_ini)
    ts.reverse_half_step()
    ts.advance_half_step()
    n = p.last_step if nsteps is None else nsteps
    for _ in range(n):
        x, v = pm_step(x, v, ts, p.ng, p.np)
    return x, v, ts


# ---------------------------------------------------------------------------
# Power spectrum (src/power_spectrum/cuda/power.cu:152-246 and kernels)
# ---------------------------------------------------------------------------

def pk_bin_edges(ng: int, rl: float, nbins: int, folds: int = 0):
    """power.cu:174-187: minK = 2pi/rl_f, maxK = sqrt(3 (ng/2)^2 d^2), centres."""
    new_rl = rl / (2.0 ** folds)
    d = 2.0 * np.pi / new_rl
    min_k = d
    max_k = math.sqrt(3 * ((ng // 2) * (ng // 2) * d * d))
    delta = (max_k - min_k) / float(nbins)
    centres = np.array([min_k + delta * (_f32(i) + 0.5) for i in range(nbins)])
    return min_k, delta, centres


def pk_log_bin_edges(ng: int, rl: float, nbins: int):
    """Log-spaced bins over the reference's k range (power.cu:174-187:
    minK = 2pi/rl, maxK = sqrt(3 (ng/2)^2 d^2)): width ln(maxK/minK)/nbins in
    ln k, centres minK exp((i + 1/2) width).  The reference bins linearly
    only; PK_LOG is a key this project adds (config C's 64 log bins)."""
    d = 2.0 * np.pi / rl
    min_k = d
    max_k = math.sqrt(3 * ((ng // 2) * (ng // 2) * d * d))
    dl = math.log(max_k / min_k) / nbins
    centres = np.array([min_k * math.exp(dl * (i + 0.5)) for i in range(nbins)])
    return min_k, dl, centres


def pk_cic_filter(ng: int) -> np.ndarray:
    """get_pk_cic_filter (filter_power.cu:3-32): prod_axis [sin(k/2)/(k/2)]^-4,
    k = signed index * 2pi/ng, factor 1 at k = 0."""
    k = signed_index(ng) * (2.0 * np.pi / ng)
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.sin(0.5 * k) / (0.5 * k)
        f = 1.0 / s ** 4
    f[k == 0] = 1.0
    return f[:, None, None] * f[None, :, None] * f[None, None, :]


def pk_bin_index(ng: int, rl_fold: float, min_k: float, delta: float) -> np.ndarray:
    """calc_power_bins (bin_power.cu:3-17): float kmodes, sqrtf of the float
    sum of squares, then (int)((|k| - minK)/delta) in double (truncation:
    a mode less than one bin below minK lands in bin 0; further below the
    index is negative, which the reference writes before its arrays and
    callers here drop)."""
    kf = kmodes_f32(ng, 2.0 * np.pi / rl_fold)
    kx = kf[:, None, None]
    ky = kf[None, :, None]
    kz = kf[None, None, :]
    s = (kx * kx + ky * ky).astype(np.float32) + kz * kz
    kmag = np.sqrt(s.astype(np.float32)).astype(np.float32)
    return np.trunc((kmag.astype(np.float64) - min_k) / delta).astype(np.int64)


def fold_positions(x: np.ndarray, ng: int, fold: int) -> np.ndarray:
    """foldParticles (fold_particles_power.cu:3-27) applied `fold` times:
    x -> 2x - ng [x >= ng/2], i.e. 2x mod ng, per axis (in float64)."""
    y = np.array(x, dtype=np.float64)
    for _ in range(fold):
        y = 2.0 * y
        y = np.where(y >= ng, y - ng, y)
    return y


def power_spectrum(x: np.ndarray, ng: int, np_side: int, rl: float, nbins: int = 221,
                   folds: int = 0, fold: int = 0, ref_quirks: bool = True, log_bins: bool = False):
    """One fold of serial::GetPowerSpectrum (power.cu:152-246): CIC of the
    particles folded `fold` times, forward FFT, scalePower (|d|^2 (1/ng^3)
    (rl/ng), scale_power.cu:3-12), PkCICFilter, BinPower (k in the fold's
    box rl/2^fold) skipping DC and the (ng/2)^3 corner.  ref_quirks: bin
    edges from rl/2^max(folds, fold) and the scale from the unfolded rl, as
    the reference (power.cu:174-187, 215); otherwise both from the fold's
    box.  Negative bin indices (reference: writes before its arrays) are
    dropped.  Sums in float64 (the reference sums in float).  log_bins:
    pk_log_bin_edges over the fold's box, index (int)(ln(|k|/minK)/width)
    with |k| formed in float as calc_power_bins does.  Returns
    (k_centres, P, counts) for all bins (empty bins give P=nan)."""
    rl_f = rl / (2.0 ** fold)
    nf = max(folds, fold)
    xf = fold_positions(x, ng, fold) if fold else x
    rho = cic_deposit(xf, ng, cic_mass(ng, np_side))
    rk = _fftn(rho)
    scale = (1.0 / float(ng * ng * ng)) * ((rl if ref_quirks else rl_f) / ng)
    pw = (rk.real ** 2 + rk.imag ** 2) * scale * pk_cic_filter(ng)
    if log_bins:
        min_k, dl, centres = pk_log_bin_edges(ng, rl / (2.0 ** nf) if ref_quirks else rl_f, nbins)
        kf = kmodes_f32(ng, 2.0 * np.pi / rl_f)
        s2 = (kf[:, None, None] * kf[:, None, None] + kf[None, :, None] * kf[None, :, None]).astype(np.float32) \
            + kf[None, None, :] * kf[None, None, :]
        kmag = np.sqrt(s2.astype(np.float32)).astype(np.float64)
        with np.errstate(divide="ignore"):
            idx = np.trunc(np.log(kmag / min_k) / dl)
        idx = np.where(np.isfinite(idx), idx, -1).astype(np.int64)
    elif ref_quirks:
        min_k, delta, centres = pk_bin_edges(ng, rl, nbins, nf)
        idx = pk_bin_index(ng, rl_f, min_k, delta)
    else:
        min_k, delta, centres = pk_bin_edges(ng, rl_f, nbins, 0)
        idx = pk_bin_index(ng, rl_f, min_k, delta)
    mask = np.ones((ng, ng, ng), dtype=bool)
    mask[0, 0, 0] = False
    mask[ng // 2, ng // 2, ng // 2] = False
    mask &= idx >= 0
    ii = idx[mask]
    sums = np.bincount(ii, weights=pw[mask], minlength=nbins)[:nbins]
    counts = np.bincount(ii, minlength=nbins)[:nbins]
    with np.errstate(invalid="ignore", divide="ignore"):
        P = sums / counts
    return centres, P, counts


def format_pk_lines(k, P, counts) -> str:
    """writePkOutput (power.cu:13-28): ``%g,%g,%d`` skipping empty/zero/nan."""
    out = []
    for kk, pp, nn in zip(k, P, counts):
        if nn != 0 and pp == pp and pp != 0:
            out.append("%g,%g,%d\n" % (kk, pp, nn))
    return "".join(out)


# ---------------------------------------------------------------------------
# Initial conditions (src/initial_conditions/*)
# ---------------------------------------------------------------------------

def read_ipk(path: str):
    """CosmoClass::read_ipk (cosmo.cpp:26-79): 20-double header
    (k_min, k_max, k_bins, k_delta, cosmology...) then k_bins doubles."""
    with open(path, "rb") as f:
        header = np.frombuffer(f.read(160), dtype="<f8")
        nb = int(header[2])
        table = np.frombuffer(f.read(8 * nb), dtype="<f8")
    return header, table


def interp_pk(table: np.ndarray, k_delta: float, n: int, rl: float) -> np.ndarray:
    """interpolatePowerSpectrum / do_pk_interpolation
    (interpolation_initializer.cu:3-41): log-log interpolation between table
    bins (int)(k/k_delta) and +1, times n^3/rl^3; bin 0 uses table[1]; k=0 -> 0.
    |k| uses the float kmodes of get_kmodes with d = 2pi/rl."""
    kf = kmodes_f32(n, 2.0 * np.pi / rl).astype(np.float64)
    kx, ky, kz = kf[:, None, None], kf[None, :, None], kf[None, None, :]
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    left = (kk / k_delta).astype(np.int64)
    right = left + 1
    with np.errstate(divide="ignore", invalid="ignore"):
        ly1 = np.log(table[left])
        lx1 = np.log(k_delta * left)
        ly2 = np.log(table[right])
        lx2 = np.log(k_delta * right)
        lx = np.log(kk)
        y = np.exp(ly1 + (ly2 - ly1) / (lx2 - lx1) * (lx - lx1))
    scale = float(n * n * n) / (rl * rl * rl)
    y = y * scale
    y = np.where(left == 0, table[right] * scale, y)
    y[0, 0, 0] = 0.0
    return y


def growth_delta(a, om, ol, ref_quirks=True, bins=100):
    """CosmoClass::delta (cosmo.cpp:81-111): D(a) = 5 Om/(2a) * da_dtau(a) *
    int_0^a da'/da_dtau^3, trapezoid with ``bins`` bins; float arithmetic when
    ``ref_quirks`` (the reference's CosmoClass works in float)."""
    f = np.float32 if ref_quirks else np.float64
    a = f(a); om = f(om); ol = f(ol)

    def da_dtau(x):
        return f(np.sqrt(f(f(1) + om * (f(1) / x - f(1)) + ol * (x * x - f(1)))))

    def da_dtau_3(x):
        d1 = da_dtau(x)
        return f(f(1) / (d1 * d1 * d1))

    start = f(0)
    delta = (a - start) / f(bins)
    s = f(0)
    with np.errstate(divide="ignore"):
        for k in range(1, bins):
            s = f(s + da_dtau_3(start + f(k) * delta))
        s = f(s + (da_dtau_3(start) + da_dtau_3(a)) / f(2.0))
    s = f(s * delta)
    diff = da_dtau(a)
    mul = f(f(5) * om) / f(f(2) * a)
    return float(f(mul * diff * s))


def growth_pair(p: Params, z_ini: float, z_vel: float, ref_quirks=True):
    """get_delta_and_dotDelta (cosmo.cpp:133-139): delta at z_ini and the
    central difference (h = 1e-4) of delta at z_vel; Om = Omega_m,
    OL = 1 - (Om + Omega_nu)."""
    f = np.float32 if ref_quirks else np.float64
    om = f(p.omega_matter)
    ol = f(f(1) - (om + f(p.omega_nu)))

    def z2a(z):
        return f(f(1.0) / (f(1.0) + f(z)))

    # FP64 mode: same integral, 20000 bins and h = 1e-6 (as the C-ABI's FP64 growth)
    bins = 100 if ref_quirks else 20000
    d = growth_delta(z2a(z_ini), om, ol, ref_quirks, bins)
    h = f(0.0001) if ref_quirks else 1e-6
    a1 = z2a(z_vel)
    dd = f((f(growth_delta(f(a1 + h), om, ol, ref_quirks, bins))
            - f(growth_delta(f(a1 - h), om, ol, ref_quirks, bins))) / (f(2.0) * h))
    return float(d), float(dd)


def displacement_from_noise(noise: np.ndarray, table, k_delta, rl, delta):
    """GenerateFourierAmplitudes + transformDensityField + ScaleFFT
    (initializer.cpp:10-117): FFT the white noise, scale by sqrt(P n^3/rl^3),
    s_dim = -i k_dim delta_k / (k^2 delta), inverse FFT, times 1/n^3.
    Returns s with shape (3, n, n, n)."""
    n = noise.shape[0]
    dk = _fftn(noise.astype(np.complex128))
    dk *= np.sqrt(interp_pk(table, k_delta, n, rl))
    kf = kmodes_f32(n, 2.0 * np.pi / rl).astype(np.float64)
    kx, ky, kz = kf[:, None, None], kf[None, :, None], kf[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    with np.errstate(divide="ignore"):
        k2mul = np.where(k2 == 0, 0.0, 1.0 / k2)
    mul = (1.0 / delta) * k2mul
    cur = dk * mul
    s = np.empty((3, n, n, n))
    for dim, kd in enumerate((kx, ky, kz)):
        sk = -1j * cur * kd  # (Im*k, -Re*k)
        s[dim] = (_ifftn(sk) * n ** 3).real / float(n ** 3)
    return s


def place_particles(s: np.ndarray, ng: int, delta: float, dotDelta: float,
                    z_ini: float, deltaT: float, fscal: float):
    """placeParticles / init_pos / init_vel (place_particles_initializer.cu:23-65):
    x = fmod(q*(ng/np) + delta*s + ng, ng), v = (a - deltaT/2)^2 dotDelta fscal s
    with a = 1/(1+z_ini).  Particle order = lattice index (get_index)."""
    n = s.shape[1]
    q = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), axis=-1)
    q = q.reshape(-1, 3).astype(np.float64)
    sv = s.reshape(3, -1).T
    x = np.fmod(q * (ng / n) + delta * sv + ng, ng)
    a = 1.0 / (1.0 + z_ini)
    vel_a = a - deltaT * 0.5
    v = (vel_a * vel_a * dotDelta * fscal) * sv
    return x, v


def generate_ic_from_noise(noise, p: Params, table, k_delta, ref_quirks=True):
    """serial::GenerateDisplacementIC (initializer.cpp:65-166) given the
    white-noise grid (the reference draws it with cuRAND; identical noise
    bytes are shared with the reference harness for parity)."""
    ts = Timestepper(p, ref_quirks)
    ts.set_initial_z(p.z_ini)
    ts.reverse_half_step()
    this_a = (1.0 / (p.z_ini + 1.0)) - (ts.deltaT / 2.0)
    vel_z = (1.0 / this_a) - 1.0
    delta, dot_delta = growth_pair(p, p.z_ini, vel_z, ref_quirks)
    s = displacement_from_noise(noise, table, k_delta, p.rl, delta)
    return place_particles(s, p.ng, delta, dot_delta, p.z_ini, ts.deltaT, ts.fscal)


def philox_normal(n_cells: int, seed: int) -> np.ndarray:
    """White noise of the B200 IC path: Philox4x32-10 (Salmon et al., SC'11)
    with counter (cell, 0, 0, 0) and key (seed, 0x4850474D); two 53-bit
    uniforms u1, u2 -> sqrt(-2 ln u1) cos(2 pi u2), rounded to float32.  (The
    reference draws cuRAND XORWOW normals instead, rng_initializer.cu:38-49.)"""
    M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    mask = np.uint64(0xFFFFFFFF)
    idx = np.arange(n_cells, dtype=np.uint64)
    c0 = idx & mask
    c1 = idx >> np.uint64(32)
    c2 = np.zeros_like(c0)
    c3 = np.zeros_like(c0)
    k0 = np.uint64(seed & 0xFFFFFFFF)
    k1 = np.uint64(0x4850474D)
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & mask, lo1, (hi0 ^ c3 ^ k1) & mask, lo0
        k0 = (k0 + np.uint64(0x9E3779B9)) & mask
        k1 = (k1 + np.uint64(0xBB67AE85)) & mask
    u1 = (((c0 >> np.uint64(5)) << np.uint64(26)) | (c1 >> np.uint64(6))).astype(np.float64)
    u2 = (((c2 >> np.uint64(5)) << np.uint64(26)) | (c3 >> np.uint64(6))).astype(np.float64)
    u1 = (u1 + 0.5) / 9007199254740992.0
    u2 = (u2 + 0.5) / 9007199254740992.0
    return (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)).astype(np.float32)


# ---------------------------------------------------------------------------
# Particle dumps (src/simulation/cuda/io.cu:12-44)
# ---------------------------------------------------------------------------

def read_dump(path: str, n_particles: int):
    """writeOutput layout: float3 x[n] then float3 v[n], no header."""
    raw = np.fromfile(path, dtype="<f4")
    if raw.size != 6 * n_particles:
        raise ValueError("dump %s has %d floats, expected %d" % (path, raw.size, 6 * n_particles))
    return raw[: 3 * n_particles].reshape(-1, 3), raw[3 * n_particles:].reshape(-1, 3)


def periodic_diff(a: np.ndarray, b: np.ndarray, ng: float) -> np.ndarray:
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    return d - ng * np.round(d / ng)
