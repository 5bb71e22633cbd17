"""The allocation-free FFT entry point (cl_fft3d_noalloc), for callers that cannot call
cudaMalloc: their own pool owns the device memory, or an allocation's device-wide
synchronisation is not acceptable on their path.  The caller allocates the data (here with
torch).  The call must give NumPy's unnormalised transforms, and the same as the allocating
entry point cl_fft3d, twice in a row with different shapes (the shared scratch tables are
rewritten each call), including a 4096-point axis, the longest its fixed scratch holds; it
must leave the device's free memory unchanged and reject longer axes.  This file is collected
last on purpose."""
import numpy as np
import pytest

import coulombo_lattice_b200 as cl

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative to the largest output magnitude, as in the FFT tests


def _numpy_fft(x, sign):
    """FFTW's conventions: sign -1 forward, +1 backward, both unnormalised."""
    axes = (-3, -2, -1)
    if sign < 0:
        return np.fft.fftn(x, axes=axes)
    return np.fft.ifftn(x, axes=axes, norm="forward")


def _device_fft(x, sign):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128)).cuda()
    nz, ny, nx = x.shape[-3:]
    batch = int(np.prod(x.shape[:-3])) if x.ndim > 3 else 1
    cl.fft3d_noalloc_device(t.data_ptr(), (nx, ny, nz), batch, sign)
    torch.cuda.synchronize()
    return t.cpu().numpy()


CASES = [((2, 20, 24, 32), -1), ((1, 8, 16, 45), +1), ((1, 1, 2, 4096), -1)]


def test_matches_numpy_and_allocating_entry_point_twice_in_a_row():
    rng = np.random.default_rng(2024)
    for _ in range(2):
        for shape, sign in CASES:
            x = rng.normal(size=shape) + 1j * rng.normal(size=shape)
            got = _device_fft(x, sign)
            want = _numpy_fft(x, sign)
            assert np.abs(got - want).max() <= TOL * np.abs(want).max(), shape
            also = cl.fft3d(x, sign=sign)
            assert np.abs(got - also).max() <= TOL * np.abs(want).max(), shape


def test_allocates_no_device_memory():
    import torch
    rng = np.random.default_rng(7)
    shape = (3, 12, 20, 30)
    x = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    t = torch.from_numpy(x).cuda()
    nz, ny, nx = shape[1:]
    cl.fft3d_noalloc_device(t.data_ptr(), (nx, ny, nz), shape[0], -1)  # warm-up: module and kernels loaded
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for sign in (+1, -1):
        cl.fft3d_noalloc_device(t.data_ptr(), (nx, ny, nz), shape[0], sign)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_rejects_axis_beyond_scratch():
    import torch
    t = torch.zeros(8192, dtype=torch.complex128, device="cuda")
    with pytest.raises(cl.CoulomboError, match="exceeds the 4096-point twiddle scratch"):
        cl.fft3d_noalloc_device(t.data_ptr(), (8192, 1, 1), 1, -1)
