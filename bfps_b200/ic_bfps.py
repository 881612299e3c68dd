"""Initial-field helpers derived from bfps/tools.py.

Provenance and licence: the two functions below restate
``generate_data_3D`` (bfps/tools.py:96-144) and ``padd_with_zeros``
(bfps/tools.py:169-203) of bfps (Copyright 2015 Max Planck Institute for
Dynamics and Self-Organization; GNU General Public License version 3 or
later), statement for statement.  They are kept alike on purpose: the
launcher must draw the same numbers from numpy's global legacy generator, in
the same order and with the same arithmetic, to reproduce the initial fields
the reference writes for a given seed bit for bit (pinned by
tests/golden/ic_vector_field_n16.npz, which tests/golden/make_ic_golden.py
writes by running the reference's own tools.py).  This module is therefore
distributed under the same GPL-3.0-or-later terms as its source.
"""
import numpy as np

def generate_data_3D(n0, n1, n2, dtype=np.complex128, p=1.5, amplitude=0.5):
    """Gaussian random scalar field in the transposed FFTW layout (y, z, x),
    modes |k| > min(n)/3 zeroed, kx = 0 plane Hermitian
    (bfps/tools.py:96-144); draws from numpy's global legacy generator."""
    assert n0 % 2 == 0 and n1 % 2 == 0 and n2 % 2 == 0
    a = np.zeros((n1, n0, n2 // 2 + 1), dtype=dtype)
    a[:] = amplitude * (np.random.randn(*a.shape) + 1j * np.random.randn(*a.shape))
    k, j, i = np.mgrid[-n1 // 2 + 1:n1 // 2 + 1, -n0 // 2 + 1:n0 // 2 + 1, 0:n2 // 2 + 1]
    k = (k ** 2 + j ** 2 + i ** 2) ** .5
    k = np.roll(k, n1 // 2 + 1, axis=0)
    k = np.roll(k, n0 // 2 + 1, axis=1)
    k[0, 0, 0] = 1
    a /= k ** p
    a[0, 0, 0] = 0
    for ky in range(1, n1 // 2):
        a[n1 - ky, 0, 0] = np.conj(a[ky, 0, 0])
    for kz in range(1, n0 // 2):
        a[0, n0 - kz, 0] = np.conj(a[0, kz, 0])
    for ky in range(1, n1 // 2):
        for kz in range(1, n0):
            a[n1 - ky, n0 - kz, 0] = np.conj(a[ky, kz, 0])
    a[np.where(k > min(n0, n1, n2) / 3.)] = 0
    return a


def padd_with_zeros(a, n0, n1, n2, odtype=None):
    """Embed a smaller transposed-layout field in an (n1, n0, n2/2+1) grid
    (bfps/tools.py:169-203)."""
    odtype = a.dtype if odtype is None else odtype
    assert a.shape[0] <= n0 and a.shape[1] <= n1 and a.shape[2] <= n2 // 2 + 1
    b = np.zeros((n0, n1, n2 // 2 + 1) + a.shape[3:], dtype=odtype)
    m0, m1, m2 = a.shape[1], a.shape[0], a.shape[2]
    b[:m1 // 2, :m0 // 2, :m2 // 2 + 1] = a[:m1 // 2, :m0 // 2, :m2 // 2 + 1]
    b[:m1 // 2, n0 - m0 // 2:, :m2 // 2 + 1] = a[:m1 // 2, m0 - m0 // 2:, :m2 // 2 + 1]
    b[n1 - m1 // 2:, :m0 // 2, :m2 // 2 + 1] = a[m1 - m1 // 2:, :m0 // 2, :m2 // 2 + 1]
    b[n1 - m1 // 2:, n0 - m0 // 2:, :m2 // 2 + 1] = a[m1 - m1 // 2:, m0 - m0 // 2:, :m2 // 2 + 1]
    return b
