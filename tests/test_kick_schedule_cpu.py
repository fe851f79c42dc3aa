"""kick_flat_nt_kernel's work schedule, restated in Python (CPU).

The particles are split into units of NT = 1024 (four Lagrangian x-planes of
a 16^3 block).  CTA c of a persistent grid of G takes the runs of R = 4
consecutive units that start at (c + i G) R, and it loads the next particle
one unit ahead.  This checks that every particle of every block is kicked
exactly once, for grids larger and smaller than the work.
"""
import pytest

B, NT, R = 16, 1024, 4
B3 = B ** 3
SUB = B3 // NT


def schedule(nblocks, grid):
    n = nblocks * SUB
    seen = []
    for c in range(grid):
        if c * R >= n:
            continue
        unit = lambda k: (c + (k // R) * grid) * R + k % R
        k = 0
        while True:
            u = unit(k)
            seen.append(u)
            if unit(k + 1) >= n:
                break
            k += 1
    return seen, n


@pytest.mark.parametrize("np_side,grid", [(32, 148), (48, 148), (64, 148), (64, 5), (128, 148), (512, 148),
                                          (512, 132)])
def test_every_particle_kicked_once(np_side, grid):
    nblocks = (np_side // B) ** 3
    units, n = schedule(nblocks, grid)
    assert n % R == 0
    assert sorted(units) == list(range(n))
    idx = sorted(u // SUB * B3 + u % SUB * NT + t for u in units[:64] for t in range(0, NT, 257))
    assert len(set(idx)) == len(idx) and max(idx) < nblocks * B3
