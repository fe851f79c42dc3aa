"""The allocation-free density entry point, hgpm_cic_density_noalloc.

It serves callers that cannot allocate device memory: code running inside a
host framework that owns every device allocation, or a run that must not
allocate after start-up.  Its int64 accumulation grid is a built-in device
array, so this test checks, through the C-ABI, that two calls in a row give
exactly the density of the allocating path (hgpm_deposit + hgpm_get_density)
and that grids above the built-in limit are refused.  This file is named to
be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import hacc_gpm_b200 as H
from hacc_gpm_b200 import binding
from tests.helpers import lattice_state, params_text

pytestmark = pytest.mark.gpu

HGPM_ERR_ARG = 1


def _noalloc():
    fn = binding.lib().hgpm_cic_density_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    return fn


@pytest.mark.parametrize("ng,np_side", [(32, 32), (48, 48), (64, 32), (128, 128)])
def test_noalloc_density_equals_allocating_path_twice(ng, np_side):
    import torch

    x, v = lattice_state(np_side, ng, disp=1.7, seed=ng + np_side)
    with H.Simulation(H.parse_params(params_text(ng, np_side))) as s:
        s.load_state(x, v)
        s.cic()
        expect = s.get_density()
    fn = _noalloc()
    xd = torch.from_numpy(x).cuda()
    out = []
    for _ in range(2):
        rho = torch.full((ng, ng, ng), -1.0, dtype=torch.float32, device="cuda")
        rc = fn(xd.data_ptr(), np_side, ng, rho.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        out.append(rho.cpu().numpy())
    assert np.array_equal(out[0], expect)
    assert np.array_equal(out[1], expect)


def test_noalloc_rejects_grid_above_limit():
    fn = _noalloc()
    # rejected before any device work, so the pointers are never touched
    rc = fn(C.c_void_p(16), 32, 256, C.c_void_p(16), None)
    assert rc == HGPM_ERR_ARG
    assert fn(None, 32, 32, C.c_void_p(16), None) == HGPM_ERR_ARG
