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
