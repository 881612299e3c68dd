"""Failure detection without a GPU fault: a bounded wait that runs out (an
mbarrier that nothing arms) sets the library's status word, the host reports
it as an error, and the same context keeps working afterwards."""
import numpy as np
import pytest

from bfps_b200 import ic

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_stays_usable():
    from bfps_b200 import _lib
    from bfps_b200.solver import vorticity_equation
    ve = vorticity_equation(32, precision="single")
    try:
        rc = _lib.lib().bfg_selftest_wait(ve.handle)
        assert rc == _lib.BFG_ECUDA
        assert b"ran out" in _lib.lib().bfg_last_error(ve.handle)
        # the status word was cleared: steps run and report normally
        w0 = ic.vorticity_ic(32, seed=3, dtype=np.complex64)
        ve.set_cvorticity(w0)
        ve.step(0.01, 2)
        assert ve.last_step_ms() > 0
        w = ve.get_cvorticity()
        assert np.isfinite(w).all() and not np.array_equal(w, w0)
    finally:
        ve.close()
