"""r3d_fft3d_noalloc: the shifted 3D transform for callers that cannot
allocate device memory (their framework owns the memory pool, or they run in
a loop that must never enter the allocator).  The caller provides the device
input and output; the library works in one fixed array of
R3D_NOALLOC_SCRATCH_BYTES.  Checked against r3d_fft3d, which allocates its
own buffers, on two calls in a row (the fixed array keeps the previous
call's contents, so the second call shows that nothing stale is reused).
This file is collected last on purpose: a failure here stops a -x run only
after every other test has run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-11  # FP64 transform, relative to the largest coefficient


def _call(R, nx, ny, nz, box, direction, d_in, d_out, stream=None):
    b = (ctypes.c_double * 3)(*box)
    return R.lib.r3d_fft3d_noalloc(0, nx, ny, nz, b, direction,
                                   ctypes.c_void_p(d_in.data_ptr()),
                                   ctypes.c_void_p(d_out.data_ptr()),
                                   None if stream is None else ctypes.c_void_p(stream))


def test_noalloc_matches_fft3d_on_two_calls():
    import torch
    import rism3d as R
    nz, ny, nx = 36, 28, 32
    box = (16.0, 14.0, 18.5)
    rng = np.random.default_rng(11)
    for call in range(2):
        f = rng.standard_normal((nz, ny, nx))
        ref = R.fft3d(f, box, -1)  # existing entry point (allocates)
        d_in = torch.from_numpy(f).cuda()
        d_out = torch.empty(2 * (nx // 2) * ny * nz, dtype=torch.float64, device="cuda")
        assert _call(R, nx, ny, nz, box, -1, d_in, d_out) == 0, R.lib.r3d_last_error(None)
        h = d_out.cpu().numpy()
        got = (h[0::2] + 1j * h[1::2]).reshape(nz, ny, nx // 2)
        np.testing.assert_allclose(got, ref, atol=TOL * np.abs(ref).max())
        # and back: the inverse of the existing entry point
        back_ref = R.fft3d(ref, box, +1)
        d_spec = torch.from_numpy(np.ascontiguousarray(h)).cuda()
        d_back = torch.empty(nx * ny * nz, dtype=torch.float64, device="cuda")
        assert _call(R, nx, ny, nz, box, +1, d_spec, d_back) == 0, R.lib.r3d_last_error(None)
        back = d_back.cpu().numpy().reshape(nz, ny, nx)
        np.testing.assert_allclose(back, back_ref, atol=TOL * np.abs(f).max())
        np.testing.assert_allclose(back, f, atol=TOL * 10 * np.abs(f).max())


def test_noalloc_rejects_grids_beyond_the_fixed_array():
    import torch
    import rism3d as R
    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    # 256^3: nx/2*ny*nz = 8.4 million points, above the array's 2.1 million
    rc = _call(R, 256, 256, 256, (128.0, 128.0, 128.0), -1, small, small)
    assert rc == 6  # R3D_EBUDGET
    msg = R.lib.r3d_last_error(None).decode()
    assert "too large for the fixed work array" in msg


def test_noalloc_on_the_callers_stream():
    """The caller fills the input on its own stream and passes that stream:
    the transform is ordered after the fill (no device-wide sync in
    between), on two calls in a row, and matches r3d_fft3d."""
    import torch
    import rism3d as R
    nz, ny, nx = 20, 24, 40
    box = (20.0, 12.0, 10.0)
    rng = np.random.default_rng(23)
    side = torch.cuda.Stream()
    for call in range(2):
        f = rng.standard_normal((nz, ny, nx))
        ref = R.fft3d(f, box, -1)
        host = torch.from_numpy(f).pin_memory()
        d_in = torch.empty(f.shape, dtype=torch.float64, device="cuda")
        d_out = torch.empty(2 * (nx // 2) * ny * nz, dtype=torch.float64, device="cuda")
        with torch.cuda.stream(side):
            d_in.copy_(host, non_blocking=True)  # queued on the caller's stream
            d_in.mul_(1.0)
        rc = _call(R, nx, ny, nz, box, -1, d_in, d_out, stream=side.cuda_stream)
        assert rc == 0, R.lib.r3d_last_error(None)
        side.synchronize()
        h = d_out.cpu().numpy()
        got = (h[0::2] + 1j * h[1::2]).reshape(nz, ny, nx // 2)
        np.testing.assert_allclose(got, ref, atol=TOL * np.abs(ref).max())
    assert torch.cuda.current_device() == 0
