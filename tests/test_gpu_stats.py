"""NSVE::do_stats quantities on the GPU against the oracle."""
import numpy as np
import pytest

from oracle import nsve as O
from bfps_b200 import ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu


def test_stats_match_oracle():
    from bfps_b200.solver import vorticity_equation
    n = 32
    ve = vorticity_equation(n, precision="double")
    w0 = ic.vorticity_ic(n, seed=5)
    ve.set_cvorticity(w0)
    ref = O.VorticityEquation(n)
    ref.cvorticity = w0.copy()
    got = ve.do_stats(1.0, 5.0, 64)
    want = O.nsve_do_stats(ref, 1.0, 5.0, 64)
    for name in ("velocity", "vorticity"):
        gs, gm, gh = got[name]
        ws, wm, wh = want[name]
        assert rel_err(gs, ws) < 1e-12
        assert np.abs(gm - wm).max() <= 1e-10 * np.abs(wm).max()
        # bin edges may differ by one count under round-off
        assert np.abs(gh - wh).sum() <= 4
        assert gh.sum() == wh.sum()
    # energy from the spectrum: 0.5 by construction of the initial condition
    spec_u = got["velocity"][0]
    assert abs(0.5 * np.trace(spec_u, axis1=1, axis2=2).sum() - 0.5) < 1e-12
    ve.close()
