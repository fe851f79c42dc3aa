"""Write ``.ipk`` initial power-spectrum tables without CAMB.

The reference reads a binary ``.ipk`` (20 float64 header values, then
``k_bins`` float64 P(k) samples at ``linspace(k_min, k_max, k_bins)``), laid
out by its ``generate_ipk.py:192-202`` and read by ``CosmoClass::read_ipk``
(cosmo.cpp:26-79).  The reference fills the table from CAMB, which is not
available here; this module fills it from the Eisenstein & Hu (1998,
ApJ 496, 605) "no-wiggle" transfer function (their eqs. 26-31), normalised
to sigma_8 with a real-space top-hat of radius 8 Mpc/h at z = 0 and scaled
to the requested redshift with the linear growth factor
D(a) = 5 Om/(2a) E(a) int_0^a da'/(a' E(a'))^3 (the same growth integral the
reference's CosmoClass uses, here in FP64).

Units: k in h/Mpc, P in (Mpc/h)^3, as CAMB's matter power in the reference.
"""
from __future__ import annotations

import math

import numpy as np

HEADER_KEYS = ["OMEGA_CDM", "DEUT", "OMEGA_NU", "HUBBLE", "SS8", "NS", "W_DE", "WA_DE", "T_CMB",
               "N_EFF_MASSLESS", "N_EFF_MASSIVE", "Z_IN"]


def eh_nowiggle_transfer(k_hmpc: np.ndarray, omega_m: float, omega_b: float, h: float, t_cmb: float = 2.7255):
    """Eisenstein & Hu 1998 zero-baryon-oscillation transfer function."""
    k = np.asarray(k_hmpc, dtype=np.float64) * h  # 1/Mpc
    omh2 = omega_m * h * h
    obh2 = omega_b * h * h
    fb = omega_b / omega_m
    theta = t_cmb / 2.7
    s = 44.5 * math.log(9.83 / omh2) / math.sqrt(1.0 + 10.0 * obh2 ** 0.75)  # Mpc
    alpha = 1.0 - 0.328 * math.log(431.0 * omh2) * fb + 0.38 * math.log(22.3 * omh2) * fb * fb
    gamma_eff = omh2 * (alpha + (1.0 - alpha) / (1.0 + (0.43 * k * s) ** 4))
    with np.errstate(divide="ignore", invalid="ignore"):
        q = k * theta * theta / gamma_eff
        l0 = np.log(2.0 * math.e + 1.8 * q)
        c0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
        t = l0 / (l0 + c0 * q * q)
    return np.where(k == 0, 1.0, t)


def growth_factor(a: float, omega_m: float, omega_l: float, n: int = 20000) -> float:
    """D(a) = 5 Om/(2a) E(a) int_0^a (a' E(a'))^-3 da' with E = da/dtau
    normalised as in cosmo.cpp:81-111 (Simpson rule, FP64)."""
    def dadtau(x):
        return np.sqrt(1.0 + omega_m * (1.0 / x - 1.0) + omega_l * (x * x - 1.0))

    xs = np.linspace(0.0, a, n + 1)[1:]
    f = 1.0 / dadtau(xs) ** 3
    f = np.concatenate([[0.0], f])  # integrand -> 0 as a -> 0
    hstep = a / n
    integral = hstep / 3.0 * (f[0] + f[-1] + 4.0 * f[1:-1:2].sum() + 2.0 * f[2:-1:2].sum())
    return 5.0 * omega_m / (2.0 * a) * float(dadtau(a)) * integral


def sigma_r(k: np.ndarray, pk: np.ndarray, r: float = 8.0) -> float:
    x = k * r
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.where(x > 1e-6, 3.0 * (np.sin(x) - x * np.cos(x)) / x ** 3, 1.0)
    integrand = k * k * pk * w * w / (2.0 * math.pi ** 2)
    return math.sqrt(np.trapezoid(integrand, k))


def eh_power(k_hmpc: np.ndarray, cosmo: dict, z: float) -> np.ndarray:
    """Linear P(k, z) in (Mpc/h)^3 from EH no-wiggle, sigma_8-normalised."""
    h = cosmo["HUBBLE"]
    omega_b = cosmo["DEUT"] / h / h
    omega_m = cosmo["OMEGA_CDM"] + omega_b + cosmo.get("OMEGA_NU", 0.0)
    ns = cosmo["NS"]
    tcmb = cosmo.get("T_CMB", 2.7255)
    kk = np.logspace(-5, 2.5, 8000)
    p0 = kk ** ns * eh_nowiggle_transfer(kk, omega_m, omega_b, h, tcmb) ** 2
    amp = (cosmo["SS8"] / sigma_r(kk, p0)) ** 2
    omega_l = 1.0 - omega_m
    dz = growth_factor(1.0 / (1.0 + z), omega_m, omega_l) / growth_factor(1.0, omega_m, omega_l)
    k = np.asarray(k_hmpc, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        p = amp * np.where(k > 0, k ** ns, 0.0) * eh_nowiggle_transfer(k, omega_m, omega_b, h, tcmb) ** 2
    return p * dz * dz


def make_ipk(cosmo: dict, z: float, k_max: float = 100.0, k_bins: int = 20000, k_min: float = 0.0):
    """Return (header[20], table) in the generate_ipk.py:192-202 layout."""
    ks = np.linspace(k_min, k_max, k_bins).astype(np.float64)
    header = np.zeros(20)
    header[0], header[1], header[2], header[3] = k_min, k_max, k_bins, ks[1] - ks[0]
    for i, key in enumerate(HEADER_KEYS):
        header[4 + i] = z if key == "Z_IN" else float(cosmo.get(key, 0.0))
    return header, eh_power(ks, cosmo, z)


def write_ipk(path: str, cosmo: dict, z: float, k_max: float = 100.0, k_bins: int = 20000) -> str:
    header, table = make_ipk(cosmo, z, k_max, k_bins)
    np.concatenate([header, table]).astype("<f8").tofile(path)
    return path


def cosmo_from_params(p) -> dict:
    """Cosmology dict from a Params-like object (binding or oracle)."""
    g = (lambda k: getattr(p, k))
    return {"OMEGA_CDM": g("omega_cdm"), "DEUT": g("deut"), "OMEGA_NU": g("omega_nu"), "HUBBLE": g("hubble"),
            "SS8": g("ss8"), "NS": g("ns"), "W_DE": g("w_de"), "WA_DE": g("wa_de"), "T_CMB": g("t_cmb"),
            "N_EFF_MASSLESS": g("neff_massless"), "N_EFF_MASSIVE": g("neff_massive")}


def lcdm_params_text(ng: int, np_side: int, rl: float, z_ini: float, nsteps: int, seed: int = 21082001,
                     omega_m: float = 0.31, h: float = 0.68, ns: float = 0.96, sigma8: float = 0.81,
                     deut: float = 0.0224, prefix: str = "run", ipk: str = "run.ipk", extra: str = "") -> str:
    """A params file in the reference's KEY VALUE format for flat LCDM."""
    omega_cdm = omega_m - deut / (h * h)
    return ("OMEGA_CDM %.8g\nDEUT %.8g\nOMEGA_NU 0.0\nHUBBLE %.8g\nSS8 %.8g\nNS %.8g\nW_DE -1.0\nWA_DE 0.0\n"
            "T_CMB 2.726\nN_EFF_MASSLESS 3.04\nN_EFF_MASSIVE 0.0\nOUTPUT_BASE_NAME %s\nIPK %s\nZ_IN %.8g\n"
            "Z_FIN 0\nN_STEPS %d\nPK_FOLDS 0\nNG %d\nNP %d\nRL %.8g\nSEED %d\nBLOCK_SIZE 64\n%s"
            % (omega_cdm, deut, h, sigma8, ns, prefix, ipk, z_ini, nsteps, ng, np_side, rl, seed, extra))
