"""Interpolation kernels: exact restatement vs the reference's compiled tables.

The reference library is built from bfps/cpp/{Lagrange_polys,spline_n*}.cpp
by oracle/build_ref.py into oracle/_ref/ (skipped where it is absent).
"""
import ctypes
from fractions import Fraction

import numpy as np
import pytest

from oracle import build_ref
from oracle.interp import SUPPORTED, beta_coefficients, beta_eval, beta_eval_exact


def _ref():
    build_ref.build()
    lib = build_ref.load()
    if lib is None:
        pytest.skip("reference interpolation library not built")
    lib.ref_beta.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    return lib


@pytest.mark.parametrize("n,m", SUPPORTED)
def test_restatement_matches_reference_tables(n, m):
    lib = _ref()
    xs = np.random.default_rng(n * 10 + m).random(64)
    xs = np.concatenate([xs, [0.0, 0.5, 1.0 - 2 ** -40]])
    for d in range(3):
        for x in xs:
            out = (ctypes.c_double * (2 * n + 2))()
            assert lib.ref_beta(n, m, d, float(x), out) == 0
            ref = np.array(out[:])
            mine = beta_eval(n, m, x, d)
            assert np.allclose(mine, ref, rtol=0, atol=1e-14 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("n,m", SUPPORTED)
def test_partition_of_unity_and_nodes(n, m):
    for x in [Fraction(0), Fraction(1, 3), Fraction(7, 11)]:
        assert sum(beta_eval_exact(n, m, x)) == 1
    # interpolating at a node returns the node value
    w0 = beta_eval_exact(n, m, 0)
    assert w0[n] == 1 and all(w == 0 for i, w in enumerate(w0) if i != n)


@pytest.mark.parametrize("n", range(1, 6))
def test_lagrange_reproduces_polynomials(n):
    # Lagrange with 2n+2 nodes is exact for degree <= 2n+1
    nodes = range(-n, n + 2)
    x = Fraction(2, 7)
    w = beta_eval_exact(n, 0, x)
    for deg in range(2 * n + 2):
        assert sum(wi * Fraction(j) ** deg for wi, j in zip(w, nodes)) == x ** deg


def test_degrees():
    for n, m in SUPPORTED:
        c = beta_coefficients(n, m)
        assert len(c) == 2 * n + 2
        deg = 2 * n + 1 if m == 0 else 2 * m + 1
        assert max(len(p) for p in c) == deg + 1
