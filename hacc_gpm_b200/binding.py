"""ctypes binding of the PM step's C-ABI (``include/hgpm_c.h``).

Host-side mirror of the reference's ``HACCGPM`` serial interface for Python
callers (tests, benchmarks, notebooks): ``read_params`` (params.cpp:72),
``Timestepper`` (timestepper.cpp:31-68), and ``Simulation`` which stands for
``serial::MemoryManager`` plus the phase functions ``UpdatePositions``,
``CIC``, ``SolveGradient``, ``UpdateVelocities``, ``GetPowerSpectrum``,
``GenerateDisplacementIC`` and ``writeOutput``.  Every call goes through the
native library ``_lib/libhgpm.so``; a non-zero status raises ``HgpmError``
with the library's message (the reference exits instead).  There is no
Python fallback: if the library is missing, importing this module fails.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libhgpm.so")

HGPM_MAX_STEPS = 1000
HGPM_PATH_MAX = 300
HGPM_NPHASE = 9
TUNE_KNOBS = 4
TUNE_NAMES = ("deposit", "kick", "y_pass", "x_pass")
PHASES = ("drift", "deposit", "fft_z_fwd", "fft_y_fwd", "poisson_x", "fft_y_inv", "fft_z_inv", "kick_drift", "pk")


class HgpmError(RuntimeError):
    pass


class _Params(C.Structure):
    _fields_ = [
        ("fname", C.c_char * HGPM_PATH_MAX),
        ("prefix", C.c_char * HGPM_PATH_MAX),
        ("ipk", C.c_char * HGPM_PATH_MAX),
        ("ng", C.c_int), ("np", C.c_int),
        ("rl", C.c_double),
        ("block_size", C.c_int), ("seed", C.c_int),
        ("z_ini", C.c_double), ("z_fin", C.c_double),
        ("nsteps", C.c_int), ("last_step", C.c_int), ("pk_folds", C.c_int),
        ("pk_bins", C.c_int), ("pk_log", C.c_int),
        ("ol", C.c_double), ("overload", C.c_int),
        ("hubble", C.c_double), ("omega_cdm", C.c_double), ("omega_nu", C.c_double),
        ("deut", C.c_double), ("ss8", C.c_double), ("ns", C.c_double),
        ("w_de", C.c_double), ("wa_de", C.c_double), ("t_cmb", C.c_double),
        ("neff_massless", C.c_double), ("neff_massive", C.c_double),
        ("omega_baryon", C.c_double), ("omega_cb", C.c_double),
        ("omega_matter", C.c_double), ("omega_radiation", C.c_double),
        ("f_nu_massless", C.c_double), ("f_nu_massive", C.c_double),
        ("pks", C.c_ubyte * HGPM_MAX_STEPS), ("dumps", C.c_ubyte * HGPM_MAX_STEPS),
        ("dump_init", C.c_int), ("dump_final", C.c_int),
        ("ref_quirks", C.c_int),
        ("do_analysis", C.c_int),
        ("analysis", C.c_ubyte * HGPM_MAX_STEPS),
        ("analysis_dir", C.c_char * HGPM_PATH_MAX),
        ("analysis_py", C.c_char * HGPM_PATH_MAX),
        ("noise", C.c_int),
    ]


class _Timestepper(C.Structure):
    _fields_ = [("aa", C.c_double), ("z", C.c_double), ("deltaT", C.c_double),
                ("adot", C.c_double), ("fscal", C.c_double), ("params", _Params)]


_lib = None


def _f(p):
    return p.ctypes.data_as(C.POINTER(C.c_float))


def _d(p):
    return p.ctypes.data_as(C.POINTER(C.c_double))


def lib() -> C.CDLL:
    """Load ``libhgpm.so`` and declare its prototypes (once)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise HgpmError("native library %s is missing; run python -m hacc_gpm_b200.build" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "hgpm_params_read": (C.c_int, [C.c_char_p, P(_Params), C.c_char_p, C.c_size_t]),
        "hgpm_params_parse": (C.c_int, [C.c_char_p, P(_Params), C.c_char_p, C.c_size_t]),
        "hgpm_params_derive": (None, [P(_Params)]),
        "hgpm_params_save": (C.c_int, [P(_Params)]),
        "hgpm_ts_init": (None, [P(_Timestepper), P(_Params)]),
        "hgpm_ts_set_initial_z": (None, [P(_Timestepper), C.c_double]),
        "hgpm_ts_advance_half": (None, [P(_Timestepper)]),
        "hgpm_ts_reverse_half": (None, [P(_Timestepper)]),
        "hgpm_ts_drift_prefactor": (C.c_float, [P(_Timestepper), C.c_float]),
        "hgpm_get_adot": (C.c_double, [C.c_double, P(_Params)]),
        "hgpm_get_fscal": (C.c_double, [C.c_double, C.c_double, C.c_double, C.c_int]),
        "hgpm_growth": (None, [P(_Params), C.c_double, C.c_double, P(C.c_double), P(C.c_double)]),
        "hgpm_create": (C.c_int, [P(_Params), C.c_int, P(vp)]),
        "hgpm_destroy": (None, [vp]),
        "hgpm_last_error": (C.c_char_p, [vp]),
        "hgpm_footprint_bytes": (C.c_size_t, [C.c_int, C.c_int]),
        "hgpm_stream": (vp, [vp]),
        "hgpm_sync": (C.c_int, [vp]),
        "hgpm_ng": (C.c_int, [vp]),
        "hgpm_np": (C.c_int, [vp]),
        "hgpm_load_state": (C.c_int, [vp, P(C.c_float), P(C.c_float)]),
        "hgpm_store_state": (C.c_int, [vp, P(C.c_float), P(C.c_float)]),
        "hgpm_load_state_device": (C.c_int, [vp, vp, vp]),
        "hgpm_store_state_device": (C.c_int, [vp, vp, vp]),
        "hgpm_get_cells": (C.c_int, [vp, P(C.c_int32)]),
        "hgpm_drift": (C.c_int, [vp, C.c_float]),
        "hgpm_deposit": (C.c_int, [vp]),
        "hgpm_get_density": (C.c_int, [vp, P(C.c_float)]),
        "hgpm_solve_gradient": (C.c_int, [vp]),
        "hgpm_get_force": (C.c_int, [vp, P(C.c_float)]),
        "hgpm_kick": (C.c_int, [vp, C.c_double, C.c_double]),
        "hgpm_kick_drift": (C.c_int, [vp, C.c_double, C.c_double, C.c_float, C.c_float, C.c_int]),
        "hgpm_run_steps": (C.c_int, [vp, P(_Timestepper), C.c_int]),
        "hgpm_step_host": (C.c_int, [vp, P(_Timestepper), P(C.c_float), P(C.c_float)]),
        "hgpm_power_spectrum": (C.c_int, [vp, C.c_int, C.c_int, P(C.c_double), P(C.c_double), P(C.c_int64)]),
        "hgpm_write_pk": (C.c_int, [C.c_char_p, C.c_int, P(C.c_double), P(C.c_double), P(C.c_int64)]),
        "hgpm_read_output": (C.c_int, [vp, C.c_char_p]),
        "hgpm_analysis_rows": (C.c_int, [vp, P(C.c_float)]),
        "hgpm_checkpoint_bytes": (C.c_size_t, [vp]),
        "hgpm_checkpoint_save": (C.c_int, [vp, P(_Timestepper), vp, C.c_size_t]),
        "hgpm_checkpoint_load": (C.c_int, [vp, P(_Timestepper), vp, C.c_size_t]),
        "hgpm_power_spectrum_fold": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, P(C.c_double), P(C.c_double),
                                               P(C.c_int64)]),
        "hgpm_write_pk_fold": (C.c_int, [C.c_char_p, C.c_int, C.c_int, P(C.c_double), P(C.c_double), P(C.c_int64)]),
        "hgpm_write_output": (C.c_int, [vp, C.c_char_p]),
        "hgpm_read_ipk": (C.c_int, [C.c_char_p, P(C.c_double), P(C.c_double), C.c_int, P(C.c_int)]),
        "hgpm_ic_generate": (C.c_int, [vp, P(C.c_double), C.c_int, C.c_double]),
        "hgpm_ic_from_noise": (C.c_int, [vp, P(C.c_float), P(C.c_double), C.c_int, C.c_double]),
        "hgpm_ic_noise": (C.c_int, [vp, P(C.c_float)]),
        "hgpm_enable_timing": (C.c_int, [vp, C.c_int]),
        "hgpm_phase_times": (C.c_int, [vp, P(C.c_double), P(C.c_int64)]),
        "hgpm_kernel_launches": (C.c_int64, [vp, C.c_int]),
        "hgpm_ens_create": (C.c_int, [C.c_int, P(C.c_int), P(C.c_int), P(C.c_int), C.c_int, P(vp)]),
        "hgpm_ens_destroy": (None, [vp]),
        "hgpm_ens_last_error": (C.c_char_p, [vp]),
        "hgpm_ens_footprint_bytes": (C.c_size_t, [C.c_int, C.c_int, C.c_int]),
        "hgpm_ens_stream": (vp, [vp]),
        "hgpm_ens_slot": (C.c_int, [vp, C.c_int, C.c_int, P(_Params), P(vp)]),
        "hgpm_ens_start": (C.c_int, [vp, C.c_int, C.c_int, P(_Timestepper), C.c_int]),
        "hgpm_ens_release": (C.c_int, [vp, C.c_int, C.c_int]),
        "hgpm_ens_step": (C.c_int, [vp, C.c_int]),
        "hgpm_ens_use_graph": (C.c_int, [vp, C.c_int]),
        "hgpm_ens_multi_launch": (C.c_int, [vp, C.c_int]),
        "hgpm_fft_c2c": (C.c_int, [vp, C.c_int, C.c_int, vp]),
        "hgpm_ens_sync": (C.c_int, [vp]),
        "hgpm_ens_status": (C.c_int, [vp, C.c_int, C.c_int, P(C.c_int), P(C.c_int)]),
        "hgpm_ens_kernel_launches": (C.c_int64, [vp, C.c_int]),
        "hgpm_ens_step_class": (C.c_int, [vp, C.c_int, C.c_int]),
        "hgpm_ens_class_done": (C.c_int, [vp, C.c_int, P(C.c_int)]),
        "hgpm_ens_sync_class": (C.c_int, [vp, C.c_int]),
        "hgpm_autotune": (C.c_int, [vp, C.c_int, C.c_int, P(C.c_int), P(C.c_double)]),
        "hgpm_tuned_choices": (C.c_int, [vp, P(C.c_int)]),
        "hgpm_tune_pick": (C.c_int, [P(C.c_double), C.c_int, C.c_int, C.c_double]),
        "hgpm_tune_cache_lookup": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, P(C.c_int)]),
        "hgpm_tune_cache_store": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, P(C.c_int),
                                            P(C.c_double)]),
        "hgpm_test_wait_timeout": (C.c_int, [vp, C.c_uint]),
        "hgpm_sizeof_params": (C.c_size_t, []),
        "hgpm_sizeof_timestepper": (C.c_size_t, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.hgpm_sizeof_params() != C.sizeof(_Params) or L.hgpm_sizeof_timestepper() != C.sizeof(_Timestepper):
        raise HgpmError("hgpm_params/hgpm_timestepper layout mismatch between binding and library")
    _lib = L
    return L


# ---------------------------------------------------------------------------
class Params:
    """``HACCGPM::Params`` (src/haccgpm.hpp:118-174) backed by the C struct."""

    def __init__(self, raw: _Params):
        object.__setattr__(self, "_raw", raw)

    def __getattr__(self, k):
        v = getattr(self._raw, k)
        if isinstance(v, bytes):
            return v.decode()
        return v

    def __setattr__(self, k, v):
        if isinstance(v, str):
            v = v.encode()
        setattr(self._raw, k, v)
        if k in ("hubble", "omega_cdm", "omega_nu", "deut", "t_cmb", "neff_massless", "neff_massive", "rl", "ng", "ol"):
            lib().hgpm_params_derive(C.byref(self._raw))

    def copy(self) -> "Params":
        r = _Params()
        C.pointer(r)[0] = self._raw
        return Params(r)

    def save(self):
        _check(None, lib().hgpm_params_save(C.byref(self._raw)))


def _check(ctx, rc):
    if rc != 0:
        msg = lib().hgpm_last_error(ctx).decode() if ctx else ""
        raise HgpmError("hgpm status %d: %s" % (rc, msg))


def parse_params(text: str) -> Params:
    r = _Params()
    err = C.create_string_buffer(512)
    rc = lib().hgpm_params_parse(text.encode(), C.byref(r), err, 512)
    if rc:
        raise HgpmError("params: " + err.value.decode())
    return Params(r)


def read_params(path: str) -> Params:
    """``HACCGPM::read_params`` (params.cpp:72-250)."""
    r = _Params()
    err = C.create_string_buffer(512)
    rc = lib().hgpm_params_read(path.encode(), C.byref(r), err, 512)
    if rc:
        raise HgpmError("params: " + err.value.decode())
    return Params(r)


class Timestepper:
    """``HACCGPM::Timestepper`` (timestepper.cpp:31-68)."""

    def __init__(self, params: Params):
        self._raw = _Timestepper()
        lib().hgpm_ts_init(C.byref(self._raw), C.byref(params._raw))

    aa = property(lambda s: s._raw.aa)
    z = property(lambda s: s._raw.z)
    adot = property(lambda s: s._raw.adot)
    fscal = property(lambda s: s._raw.fscal)
    deltaT = property(lambda s: s._raw.deltaT)

    def set_initial_z(self, z):
        lib().hgpm_ts_set_initial_z(C.byref(self._raw), z)

    def advance_half_step(self):
        lib().hgpm_ts_advance_half(C.byref(self._raw))

    def reverse_half_step(self):
        lib().hgpm_ts_reverse_half(C.byref(self._raw))

    def drift_prefactor(self, frac=0.5) -> float:
        return lib().hgpm_ts_drift_prefactor(C.byref(self._raw), frac)

    def copy(self) -> "Timestepper":
        t = Timestepper.__new__(Timestepper)
        t._raw = _Timestepper()
        C.pointer(t._raw)[0] = self._raw
        return t


def growth(params: Params, z: float, z_vel: float):
    d = C.c_double()
    dd = C.c_double()
    lib().hgpm_growth(C.byref(params._raw), z, z_vel, C.byref(d), C.byref(dd))
    return d.value, dd.value


def read_ipk(path: str):
    """``CosmoClass::read_ipk`` (cosmo.cpp:26-79): (header[20], table)."""
    L = lib()
    h = np.zeros(20)
    nb = C.c_int()
    _check(None, L.hgpm_read_ipk(path.encode(), _d(h), None, 0, C.byref(nb)))
    t = np.zeros(nb.value)
    _check(None, L.hgpm_read_ipk(path.encode(), _d(h), _d(t), nb.value, C.byref(nb)))
    return h, t


def footprint_bytes(ng: int, np_side: int) -> int:
    return lib().hgpm_footprint_bytes(ng, np_side)


def fft_c2c(data_ptr: int, ng: int, inverse: bool = False, stream: int = 0):
    """``serial::forward_fft`` / ``backward_fft`` (ffts.cu:244-294, 397-445) on a
    device complex64 grid [ng][ng][ng] at data_ptr, in place, unnormalised
    (hgpm_fft_c2c); stream-ordered on the CUDA stream handle `stream`."""
    _check(None, lib().hgpm_fft_c2c(C.c_void_p(data_ptr), ng, int(inverse), C.c_void_p(stream)))


def write_pk(fname: str, k: np.ndarray, pk: np.ndarray, count: np.ndarray, fold: int = 0):
    """``writePkOutput`` (power.cu:13-28): "<fname>.fold.<fold>" lines "%g,%g,%d"."""
    k = np.ascontiguousarray(k, np.float64)
    pk = np.ascontiguousarray(pk, np.float64)
    n = np.ascontiguousarray(count, np.int64)
    _check(None, lib().hgpm_write_pk_fold(fname.encode(), fold, k.size, _d(k), _d(pk),
                                          n.ctypes.data_as(C.POINTER(C.c_int64))))


class Simulation:
    """One box on one GPU: ``serial::MemoryManager`` plus the serial phase
    functions, all running on the context's CUDA stream."""

    def __init__(self, params: Params, device: int = 0):
        self.params = params.copy()
        self.L = lib()
        h = C.c_void_p()
        rc = self.L.hgpm_create(C.byref(self.params._raw), device, C.byref(h))
        self._h = h
        if rc:
            msg = self.L.hgpm_last_error(h).decode() if h.value else ""
            if h.value:
                self.L.hgpm_destroy(h)
            self._h = None
            raise HgpmError("hgpm_create status %d: %s" % (rc, msg))
        self.ng = params.ng
        self.np = params.np
        self.npart = params.np ** 3
        self._owned = True

    @classmethod
    def _borrow(cls, handle: C.c_void_p, params: Params) -> "Simulation":
        """A context owned elsewhere (an ensemble slot); close() leaves it."""
        s = cls.__new__(cls)
        s.params = params.copy()
        s.L = lib()
        s._h = handle
        s.ng, s.np, s.npart = params.ng, params.np, params.np ** 3
        s._owned = False
        return s

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                self.L.hgpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, rc):
        _check(self._h, rc)

    @property
    def stream(self) -> int:
        return self.L.hgpm_stream(self._h)

    def sync(self):
        self._ck(self.L.hgpm_sync(self._h))

    # state ---------------------------------------------------------------
    def load_state(self, x: np.ndarray, v: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3)
        if x.shape[0] != self.npart or v.shape[0] != self.npart:
            raise HgpmError("state must hold np^3 = %d particles" % self.npart)
        self._ck(self.L.hgpm_load_state(self._h, _f(x), _f(v)))

    def store_state(self):
        x = np.empty((self.npart, 3), np.float32)
        v = np.empty((self.npart, 3), np.float32)
        self._ck(self.L.hgpm_store_state(self._h, _f(x), _f(v)))
        return x, v

    def load_state_device(self, x_ptr: int, v_ptr: int):
        self._ck(self.L.hgpm_load_state_device(self._h, C.c_void_p(x_ptr), C.c_void_p(v_ptr)))

    def store_state_device(self, x_ptr: int, v_ptr: int):
        self._ck(self.L.hgpm_store_state_device(self._h, C.c_void_p(x_ptr), C.c_void_p(v_ptr)))

    def analysis_rows(self) -> np.ndarray:
        """PyAnalysis's rows (py_analysis.cu:10-22): (np^3, 7) float32,
        columns tag, x, y, z, vx, vy, vz."""
        out = np.empty((self.npart, 7), np.float32)
        self._ck(self.L.hgpm_analysis_rows(self._h, _f(out)))
        return out

    def read_output(self, fname: str):
        """Load the state from a ``serial::writeOutput`` dump (io.cu:12-44)."""
        self._ck(self.L.hgpm_read_output(self._h, fname.encode()))

    def checkpoint(self, ts: Timestepper) -> np.ndarray:
        """The exact device state and ``ts`` as one byte array (resume with
        ``restore``: bit-identical continuation)."""
        buf = np.empty(self.L.hgpm_checkpoint_bytes(self._h), np.uint8)
        self._ck(self.L.hgpm_checkpoint_save(self._h, C.byref(ts._raw), buf.ctypes.data_as(C.c_void_p), buf.size))
        return buf

    def restore(self, buf: np.ndarray) -> Timestepper:
        """Load a ``checkpoint`` byte array; returns its time stepper."""
        buf = np.ascontiguousarray(buf, np.uint8)
        ts = Timestepper.__new__(Timestepper)
        ts._raw = _Timestepper()
        self._ck(self.L.hgpm_checkpoint_load(self._h, C.byref(ts._raw), buf.ctypes.data_as(C.c_void_p), buf.size))
        return ts

    def get_cells(self) -> np.ndarray:
        out = np.empty(self.npart, np.int32)
        self._ck(self.L.hgpm_get_cells(self._h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    # phases (serial:: names) ---------------------------------------------
    def update_positions(self, ts: Timestepper, frac: float = 0.5):
        """``serial::UpdatePositions`` (pm_actions.cpp:287-314)."""
        self._ck(self.L.hgpm_drift(self._h, ts.drift_prefactor(frac)))

    def drift(self, prefactor: float):
        self._ck(self.L.hgpm_drift(self._h, prefactor))

    def cic(self):
        """``serial::CIC`` (pm_actions.cpp:251-258)."""
        self._ck(self.L.hgpm_deposit(self._h))

    def get_density(self) -> np.ndarray:
        out = np.empty(self.ng ** 3, np.float32)
        self._ck(self.L.hgpm_get_density(self._h, _f(out)))
        return out.reshape(self.ng, self.ng, self.ng)

    def solve_gradient(self):
        """``serial::SolveGradient`` (solver.cpp:84-170)."""
        self._ck(self.L.hgpm_solve_gradient(self._h))

    def get_force(self) -> np.ndarray:
        out = np.empty(3 * self.ng ** 3, np.float32)
        self._ck(self.L.hgpm_get_force(self._h, _f(out)))
        return out.reshape(3, self.ng, self.ng, self.ng)

    def update_velocities(self, ts: Timestepper):
        """``serial::UpdateVelocities`` (pm_actions.cpp:260-285)."""
        self._ck(self.L.hgpm_kick(self._h, ts.deltaT, ts.fscal))

    def kick_drift(self, deltaT, fscal, pf_a, pf_b, ndrift):
        self._ck(self.L.hgpm_kick_drift(self._h, deltaT, fscal, pf_a, pf_b, ndrift))

    def run_steps(self, ts: Timestepper, nsteps: int):
        """nsteps of the loop in driver_pm.cpp:110-142 (no outputs)."""
        self._ck(self.L.hgpm_run_steps(self._h, C.byref(ts._raw), nsteps))

    def step_host(self, ts: Timestepper, x: np.ndarray, v: np.ndarray):
        """One step with the state in host arrays (updated in place)."""
        assert x.dtype == np.float32 and v.dtype == np.float32 and x.flags.c_contiguous and v.flags.c_contiguous
        self._ck(self.L.hgpm_step_host(self._h, C.byref(ts._raw), _f(x), _f(v)))

    def power_spectrum(self, nbins: int = 221, log_bins: bool = False, fold: int = 0):
        """One fold of ``serial::GetPowerSpectrum`` (fold 0 by default):
        (k, P, counts); see hgpm_power_spectrum_fold for folds > 0."""
        k = np.zeros(nbins)
        p = np.zeros(nbins)
        n = np.zeros(nbins, np.int64)
        self._ck(self.L.hgpm_power_spectrum_fold(self._h, fold, nbins, int(log_bins), _d(k), _d(p),
                                                 n.ctypes.data_as(C.POINTER(C.c_int64))))
        return k, p, n

    def write_output(self, fname: str):
        self._ck(self.L.hgpm_write_output(self._h, fname.encode()))

    # initial conditions ---------------------------------------------------
    def generate_ic(self, table: np.ndarray, k_delta: float):
        """``serial::GenerateDisplacementIC`` with Philox noise."""
        t = np.ascontiguousarray(table, np.float64)
        self._ck(self.L.hgpm_ic_generate(self._h, _d(t), t.size, k_delta))

    def ic_from_noise(self, noise: np.ndarray, table: np.ndarray, k_delta: float):
        t = np.ascontiguousarray(table, np.float64)
        nz = np.ascontiguousarray(noise, np.float32).reshape(-1)
        if nz.size != self.npart:
            raise HgpmError("noise must hold np^3 values")
        self._ck(self.L.hgpm_ic_from_noise(self._h, _f(nz), _d(t), t.size, k_delta))

    def ic_noise(self) -> np.ndarray:
        out = np.empty(self.npart, np.float32)
        self._ck(self.L.hgpm_ic_noise(self._h, _f(out)))
        return out.reshape(self.np, self.np, self.np)

    # timing ------------------------------------------------------------------
    def enable_timing(self, on=True):
        self._ck(self.L.hgpm_enable_timing(self._h, int(on)))

    def phase_times(self):
        ms = np.zeros(HGPM_NPHASE)
        n = np.zeros(HGPM_NPHASE, np.int64)
        self._ck(self.L.hgpm_phase_times(self._h, _d(ms), n.ctypes.data_as(C.POINTER(C.c_int64))))
        return dict(zip(PHASES, ms)), dict(zip(PHASES, n))

    def kernel_launches(self, reset=False) -> int:
        return self.L.hgpm_kernel_launches(self._h, int(reset))

    def test_wait_timeout(self, polls: int = 1000):
        """Queue a bounded wait that nothing completes (the time-out path of
        the TMA passes); the next sync() raises HgpmError."""
        self._ck(self.L.hgpm_test_wait_timeout(self._h, int(polls)))

    def autotune(self, reps: int = 3, store: bool = False) -> dict:
        """Time every configuration of the tunable phases on the current
        state (left unchanged), apply the winners (hgpm_autotune); store:
        also append them to the tuning cache."""
        ch = (C.c_int * TUNE_KNOBS)()
        ms = (C.c_double * TUNE_KNOBS)()
        self._ck(self.L.hgpm_autotune(self._h, int(reps), int(store), ch, ms))
        return {k: {"choice": int(ch[i]), "ms": float(ms[i])} for i, k in enumerate(TUNE_NAMES)}

    def tuned_choices(self) -> dict:
        ch = (C.c_int * TUNE_KNOBS)()
        self._ck(self.L.hgpm_tuned_choices(self._h, ch))
        return {k: int(ch[i]) for i, k in enumerate(TUNE_NAMES)}
