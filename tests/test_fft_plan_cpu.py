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
The GPU tests compare the kernels with the oracle at 16-160 and 512; this
also covers every other compiled length up to 1024.  The radix-5
butterfly's algebra (Dft<5> in fft_engine.cuh) is restated too and checked
against the DFT definition.
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
    assert int(np.prod(P)) == N and all(r in (2, 3, 4, 5, 8) for r in P)
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


def compiled_sizes():
    txt = open(os.path.join(os.path.dirname(HDR), "hgpm_internal.h")).read()
    body = txt[txt.index("#define HGPM_SIZES(X)"):txt.index("#define HGPM_SIZES_TEXT")]
    return sorted(int(n) for n in re.findall(r"X\((\d+)\)", body))


def test_every_supported_grid_side_has_a_plan():
    """Every compiled grid side and its half (the z passes' complex length)
    has a plan; the sides are 2^a 3^b 5^c multiples of 8 up to 1024."""
    sides = compiled_sizes()
    assert set(sides) >= {16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 40, 80, 160, 320, 640, 1000}
    for n in sides:
        m = n
        for r in (2, 3, 5):
            while m % r == 0:
                m //= r
        assert m == 1 and n % 8 == 0 and n <= 1024
    assert set(plans()) >= set(sides) | {n // 2 for n in sides}


def test_radix5_butterfly_algebra():
    """Dft<5>: t1 = v1 + v4, t2 = v2 + v3, t3 = v1 - v4, t4 = v2 - v3;
    X0 = v0 + t1 + t2, X1/X4 = a1 -/+ i b1, X2/X3 = a2 -/+ i b2 with
    a1 = v0 + c1 t1 + c2 t2, a2 = v0 + c2 t1 + c1 t2, b1 = s1 t3 + s2 t4,
    b2 = s2 t3 - s1 t4 (forward; the inverse flips i)."""
    c1, c2 = np.cos(2 * np.pi / 5), np.cos(4 * np.pi / 5)
    s1, s2 = np.sin(2 * np.pi / 5), np.sin(4 * np.pi / 5)
    rng = np.random.default_rng(5)
    for inv in (False, True):
        v = rng.standard_normal(5) + 1j * rng.standard_normal(5)
        t1, t2, t3, t4 = v[1] + v[4], v[2] + v[3], v[1] - v[4], v[2] - v[3]
        a1, a2 = v[0] + c1 * t1 + c2 * t2, v[0] + c2 * t1 + c1 * t2
        rot = (1j if inv else -1j)
        b1, b2 = rot * (s1 * t3 + s2 * t4), rot * (s2 * t3 - s1 * t4)
        X = np.array([v[0] + t1 + t2, a1 + b1, a2 + b2, a2 - b2, a1 - b1])
        assert np.allclose(X, dft(v, inv), atol=1e-12)
