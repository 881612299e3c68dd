"""field::dft / field::ift on the GPU against numpy (pocketfft) in FP64 / FP32."""
import numpy as np
import pytest

from oracle import nsve as O

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n", [16, 32, 64, 128])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_dft_ift_match_numpy(n, precision):
    import torch
    from bfps_b200.solver import vorticity_equation
    from bfps_b200 import _lib
    ve = vorticity_equation(n, precision=precision)
    rng = np.random.default_rng(n)
    r = rng.standard_normal((n, n, n, 3))
    rpad = O.real_to_padded(r).astype(ve.rdtype)
    c_ref = O.dft(r)  # (ny, nz, nx/2+1, 3) transposed layout
    din = _dev(rpad)
    dout = torch.zeros(ve.cshape, dtype=torch.complex64 if precision == "single" else torch.complex128,
                       device="cuda")
    _lib.check(_lib.lib().bfg_dft(ve.handle, din.data_ptr(), dout.data_ptr()), ve.handle)
    c = dout.cpu().numpy()
    tol = 1e-13 if precision == "double" else 2e-6
    assert np.abs(c - c_ref).max() / np.abs(c_ref).max() < tol
    # inverse of a Hermitian spectrum
    back = torch.zeros(rpad.shape, dtype=din.dtype, device="cuda")
    cin = _dev(c_ref.astype(ve.cdtype))
    _lib.check(_lib.lib().bfg_ift(ve.handle, cin.data_ptr(), back.data_ptr()), ve.handle)
    rb = back.cpu().numpy()
    assert np.all(rb[:, :, n:, :] == 0)
    ref = r * n ** 3
    assert np.abs(rb[:, :, :n] - ref).max() / np.abs(ref).max() < tol
    ve.close()


def test_device_buffers_wait_for_the_callers_stream():
    """Device buffers written by work still queued on the caller's stream
    (torch's): the transform reads them only after that work.  The input is
    written behind a GPU sleep of tens of milliseconds, so a call that did
    not wait would read the zeros that precede it."""
    import torch
    from bfps_b200.solver import vorticity_equation
    from bfps_b200 import _lib
    n = 32
    ve = vorticity_equation(n, precision="double")
    try:
        r = np.random.default_rng(5).standard_normal((n, n, n, 3))
        src = _dev(O.real_to_padded(r))
        din = torch.zeros_like(src)
        dout = torch.zeros(ve.cshape, dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        torch.cuda._sleep(100_000_000)   # about 50 ms of device time
        din.copy_(src)                    # queued behind the sleep
        _lib.check(_lib.lib().bfg_dft(ve.handle, din.data_ptr(), dout.data_ptr()), ve.handle)
        c_ref = O.dft(r)
        assert np.abs(dout.cpu().numpy() - c_ref).max() / np.abs(c_ref).max() < 1e-13
        # and the output is not overwritten by work the caller queued before
        back = torch.full(din.shape, 7.0, dtype=din.dtype, device="cuda")
        torch.cuda._sleep(100_000_000)
        back.fill_(3.0)                   # queued behind the sleep, before the call
        _lib.check(_lib.lib().bfg_ift(ve.handle, dout.data_ptr(), back.data_ptr()), ve.handle)
        rb = back.cpu().numpy()
        assert np.abs(rb[:, :, :n] - r * n ** 3).max() / np.abs(r * n ** 3).max() < 1e-13
    finally:
        ve.close()
