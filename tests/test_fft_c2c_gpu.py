"""serial::forward_fft / backward_fft on a caller's single-precision complex
grid (hgpm_fft_c2c, ffts.cu:244-294, 397-445): the unnormalised 3D C2C
transform against numpy's FP64 FFT, both directions, radices 2, 3, 5."""
import numpy as np
import pytest
import torch

from hacc_gpm_b200 import binding

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ng", [16, 24, 32, 40, 48, 64, 96])
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_matches_numpy(ng, inverse):
    rng = np.random.default_rng(ng + 7 * inverse)
    a = (rng.standard_normal((ng, ng, ng)) + 1j * rng.standard_normal((ng, ng, ng))).astype(np.complex64)
    d = torch.from_numpy(a.view(np.float32).reshape(ng, ng, ng, 2)).cuda()
    s = torch.cuda.current_stream()
    binding.fft_c2c(d.data_ptr(), ng, inverse, s.cuda_stream)
    s.synchronize()
    got = d.cpu().numpy().view(np.complex64)[..., 0]
    ref = np.fft.ifftn(a.astype(np.complex128)) * ng ** 3 if inverse else np.fft.fftn(a.astype(np.complex128))
    assert np.abs(got - ref).max() < 2e-5 * np.abs(ref).max()


def test_c2c_round_trip_and_legacy_stream():
    """forward then inverse (NULL stream: returns when done) gives ng^3 times
    the input; an unsupported side is refused."""
    ng = 80
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((ng, ng, ng)) + 1j * rng.standard_normal((ng, ng, ng))).astype(np.complex64)
    d = torch.from_numpy(a.view(np.float32).reshape(ng, ng, ng, 2)).cuda()
    torch.cuda.synchronize()
    binding.fft_c2c(d.data_ptr(), ng, False)
    binding.fft_c2c(d.data_ptr(), ng, True)
    back = d.cpu().numpy().view(np.complex64)[..., 0] / ng ** 3
    assert np.abs(back - a).max() < 2e-5 * np.abs(a).max()
    with pytest.raises(binding.HgpmError):
        binding.fft_c2c(d.data_ptr(), 56, False)
