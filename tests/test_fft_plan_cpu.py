"""The shared-memory FFT engine's index algebra, restated in numpy (CPU).

The radix plans are read from csrc/fft_engine.cuh, and each stage moves data
with the same formulas as fft_stage / fft_turn_stage.  Element j + r*NB goes
in, twiddle tw[r*m] with m = k*N/(NS*R) and k = j % NS, and the output goes
to (j/NS)*NS*R + k + r*NS.  For every supported length this checks that:
  * the forward plan is the DFT,
  * the inverse, with the radices in reverse order, is the unnormalised
    inverse DFT,
  * forward, then a per-mode operator in the turn stage, then inverse equals
    N * ifft(op * fft(x)), which is what the fused x pass computes.
The GPU tests compare the kernels with the oracle at 16-128 and 512; this
also covers 192, 256, 384, 768 and 1024.
"""
import os
import re

import numpy as np
import pytest

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "hacc_gpm_b200", "csrc",
                   "fft_engine.cuh")


def plans():
    txt = open(HDR).read()
    out = {}
    for n, rs in re.findall(r"struct Plan<(\d+)>\s*\{\s*using type = RSeq<([\d,\s]+)>;", txt):
        out[int(n)] = [int(r) for r in rs.split(",")]
    return out


def dft(v, inv):
    R = len(v)
    s = 1.0 if inv else -1.0
    w = np.exp(s * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
    return w @ v


def stage(buf, N, NS, R, inv, tw):
    NB = N // R
    out = np.empty_like(buf)
    for j in range(NB):
        k = j % NS
        v = np.array([buf[j + r * NB] for r in range(R)])
        if NS > 1:
            m = k * (N // (NS * R))
            w = np.array([tw[(r * m) % N] for r in range(R)])
            v = v * (np.conj(w) if inv else w)
        v = dft(v, inv)
        base = (j // NS) * NS * R + k
        for r in range(R):
            out[base + r * NS] = v[r]
    return out


def turn(buf, N, R, tw, op):
    NB = NS = N // R
    out = np.empty_like(buf)
    for j in range(NB):
        v = np.array([buf[j + r * NB] for r in range(R)])
        m = j * (N // (NS * R))
        v = v * np.array([tw[(r * m) % N] for r in range(R)])
        v = dft(v, False)
        v = np.array([op(j + r * NS, v[r]) for r in range(R)])
        v = dft(v, True)  # NS = 1: no twiddles
        for r in range(R):
            out[j * R + r] = v[r]
    return out


def run(x, N, radices, inv, tw, ns=1):
    for R in radices:
        x = stage(x, N, ns, R, inv, tw)
        ns *= R
    return x


@pytest.mark.parametrize("N", sorted(plans()))
def test_plan_forward_inverse_and_turn(N):
    P = plans()[N]
    assert int(np.prod(P)) == N and all(r in (2, 3, 4, 8) for r in P)
    tw = np.exp(-2j * np.pi * np.arange(N) / N)
    rng = np.random.default_rng(N)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    fx = run(x, N, P, False, tw)
    assert np.allclose(fx, np.fft.fft(x), atol=1e-9 * N)
    assert np.allclose(run(fx, N, P[::-1], True, tw), N * x, atol=1e-9 * N * N)
    g = rng.standard_normal(N)
    y = run(x, N, P[:-1], False, tw)
    y = turn(y, N, P[-1], tw, lambda e, v: g[e] * v)
    y = run(y, N, P[-2::-1], True, tw, ns=P[-1])
    assert np.allclose(y, N * np.fft.ifft(g * np.fft.fft(x)), atol=1e-9 * N * N)


def test_every_supported_grid_side_has_a_plan():
    assert set(plans()) >= {16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024}
