"""The autotuner's host logic on the CPU: the pick rule (the default stays
unless another configuration is faster by more than the noise margin) and
the cache file keyed by (device, SM count, ng, np).  The timing itself runs
on the GPU (tests/test_gpu_phases.py)."""
import ctypes as C

import pytest

from hacc_gpm_b200 import binding


def _pick(lib, ms, default, tol=0.02):
    arr = (C.c_double * len(ms))(*ms)
    return lib.hgpm_tune_pick(arr, len(ms), default, tol)


def test_pick_keeps_the_default_within_noise(built_lib):
    assert _pick(built_lib, [2.0, 1.99, 2.5], 0) == 0      # 0.5 % faster: noise
    assert _pick(built_lib, [2.0, 1.90, 2.5], 0) == 1      # 5 % faster: taken
    assert _pick(built_lib, [2.0, 1.90, 1.80], 1) == 2
    assert _pick(built_lib, [1.5, 1.90, 1.80], 1) == 0
    assert _pick(built_lib, [-1.0, 3.0, 2.0], 0) == 2      # unmeasured default
    assert _pick(built_lib, [2.0], 5) == 0                  # default out of range
    assert _pick(built_lib, [], 0) == -1


def _store(lib, path, dev, sms, ng, np_side, ch, ms=(1.0, 2.0, 3.0, 4.0)):
    a = (C.c_int * 4)(*ch)
    m = (C.c_double * 4)(*ms)
    return lib.hgpm_tune_cache_store(str(path).encode(), dev.encode(), sms, ng, np_side, a, m)


def _lookup(lib, path, dev, sms, ng, np_side):
    a = (C.c_int * 4)()
    rc = lib.hgpm_tune_cache_lookup(str(path).encode(), dev.encode(), sms, ng, np_side, a)
    return rc, list(a)


def test_cache_keyed_by_device_sms_and_size(built_lib, tmp_path):
    f = tmp_path / "tune.txt"
    assert _lookup(built_lib, f, "NVIDIA_B200", 148, 512, 512)[0] == 0   # no file yet
    assert _store(built_lib, f, "NVIDIA_B200", 148, 512, 512, [5, 0, 1, 1]) == 0
    assert _store(built_lib, f, "NVIDIA_B200", 148, 256, 256, [4, 2, 0, 1]) == 0
    assert _store(built_lib, f, "NVIDIA_B200", 132, 512, 512, [1, 1, 1, 0]) == 0
    assert _lookup(built_lib, f, "NVIDIA_B200", 148, 512, 512) == (1, [5, 0, 1, 1])
    assert _lookup(built_lib, f, "NVIDIA_B200", 148, 256, 256) == (1, [4, 2, 0, 1])
    assert _lookup(built_lib, f, "NVIDIA_B200", 132, 512, 512) == (1, [1, 1, 1, 0])
    assert _lookup(built_lib, f, "NVIDIA_H100", 148, 512, 512)[0] == 0
    assert _lookup(built_lib, f, "NVIDIA_B200", 148, 512, 1024)[0] == 0
    # a later entry for the same key wins
    assert _store(built_lib, f, "NVIDIA_B200", 148, 512, 512, [6, 3, 1, 1]) == 0
    assert _lookup(built_lib, f, "NVIDIA_B200", 148, 512, 512) == (1, [6, 3, 1, 1])
    # malformed lines are skipped
    with open(f, "a") as fh:
        fh.write("garbage line\nv1 NVIDIA_B200 148 512\n")
    assert _lookup(built_lib, f, "NVIDIA_B200", 148, 512, 512) == (1, [6, 3, 1, 1])


def test_cache_rejects_blank_device_names(built_lib, tmp_path):
    assert _store(built_lib, tmp_path / "t.txt", "NVIDIA B200", 148, 64, 64, [0, 0, 1, 1]) == 1  # HGPM_ERR_ARG


def test_binding_names_the_knobs():
    assert binding.TUNE_NAMES == ("deposit", "kick", "y_pass", "x_pass") and binding.TUNE_KNOBS == 4
