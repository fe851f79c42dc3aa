"""gradient_kernel's thread layout, restated in numpy (CPU).

A thread q makes the 8 z-consecutive cells z0..z0+7 of row (x, y) at XR
consecutive x.  It carries phi(x-1) and phi(x) from one x to the next.  The
z neighbours of its run's ends come from lanes q-1 and q+1 of its warp, and
it loads them itself at the warp's ends and at the row's periodic wrap.
This restatement follows the launcher's choice of XR (8 from 64^3 for sides
that are multiples of 16, else 1) and its warp layout (lane = q mod 32).  It
checks that every cell is written exactly once with
F_d = (phi(x - e_d) - phi(x + e_d)) / 2 in float32, bit for bit, and that the
thread count is a whole number of warps, which the kernel's shuffles need.
"""
import numpy as np
import pytest


def xr_for(ng):
    return 8 if ng % 16 == 0 and ng >= 64 else 1


def emulate(phi, ng):
    XR, n8 = xr_for(ng), ng // 8
    nq = (ng // XR) * ng * n8
    assert nq % 32 == 0
    q = np.arange(nq)
    lane = q & 31
    z0 = (q % n8) * 8
    r = q // n8
    y = r % ng
    x0 = (r // ng) * XR
    ym, yp = (y - 1) % ng, (y + 1) % ng
    zz = z0[:, None] + np.arange(8)[None, :]
    out = np.zeros((ng, ng, ng, 3), np.float32)
    written = np.zeros((ng, ng, ng), np.int32)
    half = np.float32(0.5)
    for k in range(XR):
        x = x0 + k
        a = phi[((x - 1) % ng)[:, None], y[:, None], zz]
        c = phi[x[:, None], y[:, None], zz]
        b = phi[((x + 1) % ng)[:, None], y[:, None], zz]
        d = phi[x[:, None], ym[:, None], zz]
        e = phi[x[:, None], yp[:, None], zz]
        # shuffles: lane l receives lane l-1's c[7] and lane l+1's c[0]
        zm = np.roll(c[:, 7], 1)
        zp = np.roll(c[:, 0], -1)
        own_m = (lane == 0) | (z0 == 0)
        own_p = (lane == 31) | (z0 + 8 == ng)
        zm = np.where(own_m, phi[x, y, (z0 - 1) % ng], zm)
        zp = np.where(own_p, phi[x, y, (z0 + 8) % ng], zp)
        lo = np.concatenate([zm[:, None], c[:, :7]], 1)
        hi = np.concatenate([c[:, 1:], zp[:, None]], 1)
        f = np.stack([half * (a - b), half * (d - e), half * (lo - hi)], -1)
        out[x[:, None], y[:, None], zz] = f
        np.add.at(written, (x[:, None].repeat(8, 1), y[:, None].repeat(8, 1), zz), 1)
    return out, written


@pytest.mark.parametrize("ng", [16, 24, 32, 48, 64, 96, 128])
def test_gradient_layout_matches_central_differences(ng):
    phi = np.random.default_rng(ng).standard_normal((ng, ng, ng)).astype(np.float32)
    out, written = emulate(phi, ng)
    assert (written == 1).all()
    half = np.float32(0.5)
    ref = np.stack([half * (np.roll(phi, 1, a) - np.roll(phi, -1, a)) for a in range(3)], -1)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("ng", [16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024])
def test_gradient_threads_fill_whole_warps(ng):
    XR = xr_for(ng)
    assert ng % XR == 0 and ((ng // XR) * ng * (ng // 8)) % 32 == 0
