"""The allocation-free FFT entry point (cl_fft3d_noalloc), for callers that cannot call
cudaMalloc: their own pool owns the device memory, or an allocation's device-wide
synchronisation is not acceptable on their path.  The caller allocates the data (here with
torch); the call must give what the allocating entry point cl_fft3d gives, twice in a row
with different shapes (the shared scratch tables are rewritten each call), and reject axes
longer than its fixed scratch.  This file is collected last on purpose."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative to the largest output magnitude, as in the FFT tests


def _device_fft(x, sign):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128)).cuda()
    nz, ny, nx = x.shape[-3:]
    batch = int(np.prod(x.shape[:-3])) if x.ndim > 3 else 1
    cl.fft3d_noalloc_device(t.data_ptr(), (nx, ny, nz), batch, sign)
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_matches_allocating_entry_point_twice_in_a_row():
    rng = np.random.default_rng(2024)
    cases = [((2, 20, 24, 32), -1), ((1, 8, 16, 45), +1)]
    for shape, sign in cases:
        x = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        got = _device_fft(x, sign)
        want = cl.fft3d(x, sign=sign)
        assert np.abs(got - want).max() <= TOL * np.abs(want).max()


def test_rejects_axis_beyond_scratch():
    import torch
    t = torch.zeros(8192, dtype=torch.complex128, device="cuda")
    with pytest.raises(cl.CoulomboError, match="exceeds the 4096-point twiddle scratch"):
        cl.fft3d_noalloc_device(t.data_ptr(), (8192, 1, 1), 1, -1)
