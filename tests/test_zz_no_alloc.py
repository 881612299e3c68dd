"""bfg_rspace_stats_noalloc: the entry point for callers that cannot allocate.

Some callers cannot call cudaMalloc (another framework's allocator owns the
device memory, the footprint is fixed at start-up, or the loop cannot take
cudaMalloc's device-wide synchronisation).  This entry point takes the field
and the outputs from the caller and keeps its partial sums in a fixed array
inside the library.  The test checks it against the moments and histograms
of the existing bfg_stats entry point on the same velocity field, for two
calls in a row (the second call reuses the shared array left by the first).
The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes
import math

import numpy as np
import pytest

from bfps_b200 import _lib, ic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["double", "single"])
def test_noalloc_moments_match_bfg_stats(precision):
    import torch
    from bfps_b200.solver import vorticity_equation
    n, nbins, max_u = 32, 64, 2.0
    ve = vorticity_equation(n, precision=precision)
    ve.set_cvorticity(ic.vorticity_ic(n, seed=11, dtype=ve.cdtype))
    _, mom_ref, hist_ref = ve.do_stats(max_velocity_estimate=max_u, max_vorticity_estimate=5.0,
                                       nbins=nbins)["velocity"]
    ve.velocity_rspace()
    field = torch.from_numpy(ve.get_rvelocity()).cuda()  # (nz, ny, nx+2, 3)
    mom = torch.full((40,), float("nan"), dtype=torch.float64, device="cuda")
    hist = torch.full((nbins * 4,), -1, dtype=torch.int64, device="cuda")
    L = _lib.lib()
    for call in range(2):
        rc = L.bfg_rspace_stats_noalloc(field.data_ptr(), n, n, n, ve.real_bytes,
                                        max_u / math.sqrt(3), nbins, mom.data_ptr(),
                                        hist.data_ptr(), None)
        assert rc == _lib.BFG_OK
        torch.cuda.synchronize()
        m = mom.cpu().numpy().reshape(10, 4)
        h = hist.cpu().numpy().reshape(nbins, 4)
        assert np.abs(m - mom_ref).max() <= 1e-12 * np.abs(mom_ref).max(), call
        assert np.array_equal(h, hist_ref), call
    ve.close()


def test_noalloc_rejects_too_many_bins():
    import torch
    field = torch.zeros((16, 16, 18, 3), dtype=torch.float64, device="cuda")
    mom = torch.zeros(40, dtype=torch.float64, device="cuda")
    hist = torch.zeros(8, dtype=torch.int64, device="cuda")
    rc = _lib.lib().bfg_rspace_stats_noalloc(field.data_ptr(), 16, 16, 16, 8, 1.0, 2049,
                                             mom.data_ptr(), hist.data_ptr(), None)
    assert rc == _lib.BFG_EUNSUP


def test_noalloc_non_cubic_against_numpy():
    """nx != ny != nz in the padded layout (nz, ny, nx + 2, 3), the padding
    filled with NaN (it must not be read), checked against the numpy
    restatement of field::compute_rspace_stats (field.cpp:661-889), for two
    calls in a row."""
    import torch
    from oracle import nsve as O
    nx, ny, nz, nbins, me = 32, 16, 8, 48, 1.5
    rng = np.random.default_rng(5)
    r = rng.standard_normal((nz, ny, nx, 3))
    pad = np.full((nz, ny, nx + 2, 3), np.nan)
    pad[:, :, :nx] = r
    mom_ref, hist_ref = O.rspace_stats(r, [me] * 3 + [me * math.sqrt(3)], nbins)
    field = torch.from_numpy(pad).cuda()
    mom = torch.zeros(40, dtype=torch.float64, device="cuda")
    hist = torch.zeros(nbins * 4, dtype=torch.int64, device="cuda")
    for call in range(2):
        rc = _lib.lib().bfg_rspace_stats_noalloc(field.data_ptr(), nx, ny, nz, 8, me, nbins,
                                                 mom.data_ptr(), hist.data_ptr(), None)
        assert rc == _lib.BFG_OK
        torch.cuda.synchronize()
        m = mom.cpu().numpy().reshape(10, 4)
        assert np.abs(m - mom_ref).max() <= 1e-12 * np.abs(mom_ref).max(), call
        assert np.array_equal(hist.cpu().numpy().reshape(nbins, 4), hist_ref), call


def test_noalloc_accepts_the_maximum_bin_count():
    import torch
    from oracle import nsve as O
    n, nbins, me = 16, 2048, 3.0
    rng = np.random.default_rng(6)
    r = rng.standard_normal((n, n, n, 3)).astype(np.float32)
    pad = np.zeros((n, n, n + 2, 3), np.float32)
    pad[:, :, :n] = r
    _, hist_ref = O.rspace_stats(r.astype(np.float64), [me] * 3 + [me * math.sqrt(3)], nbins)
    field = torch.from_numpy(pad).cuda()
    mom = torch.zeros(40, dtype=torch.float64, device="cuda")
    hist = torch.zeros(nbins * 4, dtype=torch.int64, device="cuda")
    rc = _lib.lib().bfg_rspace_stats_noalloc(field.data_ptr(), n, n, n, 4, me, nbins,
                                             mom.data_ptr(), hist.data_ptr(), None)
    assert rc == _lib.BFG_OK
    torch.cuda.synchronize()
    assert np.array_equal(hist.cpu().numpy().reshape(nbins, 4), hist_ref)
