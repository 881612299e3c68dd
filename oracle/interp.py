"""Oracle: exact construction of bfps' particle interpolation kernels.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module; it is
the checker that the CUDA gather kernel and its generated coefficient header
are compared against.

bfps samples a grid field at a particle with a tensor product of 1D weight
polynomials ``beta_i(x)``, ``i = 0 .. 2n+1``, where ``x`` in [0, 1) is the
particle's offset inside its cell and weight ``i`` multiplies grid node
``cell - n + i`` (bfps/cpp/particles/particles_field_computer.hpp:65-157).
The kernel is chosen at run time by (neighbours n, smoothness m)
(bfps/cpp/particles/particles_system_builder.hpp:238-257,
bfps/cpp/particles/particles_generic_interp.hpp:10-313):

* m == 0: Lagrange interpolation through the 2n+2 nodes -n .. n+1
  (bfps/cpp/Lagrange_polys.cpp, e.g. beta_Lagrange_n2 at :53-81).
* m >= 1: the smooth piecewise polynomials of Lalescu, Teaca and Carati
  (J. Comput. Phys. 229, 2010): on [0, 1] the interpolant is the Hermite
  polynomial of degree 2m+1 that matches the value and the first m
  derivatives at both nodes 0 and 1, and each derivative at a node is
  replaced by the centred finite difference over the 2n+1 nodes around it
  (exact for polynomials of degree 2n).  bfps ships these as generated
  tables (bfps/cpp/spline_n1.cpp .. spline_n10.cpp, e.g. beta_n2_m2 at
  spline_n2.cpp:92-121); they are reproduced here from that construction
  with exact rational arithmetic.

Only derivative order 0 is used on the tracer path
(particles_field_computer.hpp:37-39), but derivatives are provided too.
"""
from fractions import Fraction
from functools import lru_cache

__all__ = ["beta_coefficients", "beta_eval", "beta_eval_exact", "SUPPORTED"]

# (neighbours, smoothness) pairs the GPU path supports (1..5 x 0..2).
SUPPORTED = [(n, m) for n in range(1, 6) for m in range(0, 3)]


def _poly_mul(a, b):
    out = [Fraction(0)] * (len(a) + len(b) - 1)
    for i, ai in enumerate(a):
        if ai == 0:
            continue
        for j, bj in enumerate(b):
            out[i + j] += ai * bj
    return out


def _poly_add(a, b, scale=Fraction(1)):
    n = max(len(a), len(b))
    out = [Fraction(0)] * n
    for i, ai in enumerate(a):
        out[i] += ai
    for i, bi in enumerate(b):
        out[i] += scale * bi
    return out


def _solve(mat, rhs):
    """Exact Gauss-Jordan elimination over Fractions."""
    n = len(mat)
    a = [list(row) + [r] for row, r in zip(mat, rhs)]
    for col in range(n):
        piv = next(r for r in range(col, n) if a[r][col] != 0)
        a[col], a[piv] = a[piv], a[col]
        p = a[col][col]
        a[col] = [v / p for v in a[col]]
        for r in range(n):
            if r != col and a[r][col] != 0:
                f = a[r][col]
                a[r] = [vr - f * vc for vr, vc in zip(a[r], a[col])]
    return [a[r][n] for r in range(n)]


def _factorial(k):
    out = 1
    for i in range(2, k + 1):
        out *= i
    return out


@lru_cache(maxsize=None)
def _centred_fd(n, d):
    """Weights c_j (j = -n..n) with sum_j c_j f(j) = f^(d)(0) for deg <= 2n."""
    nodes = list(range(-n, n + 1))
    mat = [[Fraction(j) ** p / _factorial(p) for j in nodes] for p in range(2 * n + 1)]
    rhs = [Fraction(1 if p == d else 0) for p in range(2 * n + 1)]
    return _solve(mat, rhs)


@lru_cache(maxsize=None)
def _hermite_basis(m):
    """Degree 2m+1 polynomials H0[d], H1[d] on [0,1].

    H0[d] has d-th derivative 1 at x=0 and all other derivatives of order
    0..m zero at both ends; H1[d] likewise at x=1.
    """
    deg = 2 * m + 1
    ncoef = deg + 1

    def deriv_row(x, e):
        # row giving the e-th derivative at x of sum_k a_k x^k
        row = []
        for k in range(ncoef):
            if k < e:
                row.append(Fraction(0))
            else:
                c = Fraction(_factorial(k), _factorial(k - e))
                row.append(c * (Fraction(x) ** (k - e) if k - e > 0 else Fraction(1)))
        return row

    rows = [deriv_row(0, e) for e in range(m + 1)] + [deriv_row(1, e) for e in range(m + 1)]
    h0, h1 = [], []
    for d in range(m + 1):
        rhs = [Fraction(0)] * (2 * m + 2)
        rhs[d] = Fraction(1)
        h0.append(_solve(rows, rhs))
        rhs = [Fraction(0)] * (2 * m + 2)
        rhs[m + 1 + d] = Fraction(1)
        h1.append(_solve(rows, rhs))
    return h0, h1


@lru_cache(maxsize=None)
def beta_coefficients(n, m):
    """Monomial coefficients (Fractions) of the 2n+2 weight polynomials.

    Returns a tuple of 2n+2 tuples; entry i holds the coefficients of
    beta_i(x) in increasing powers of x.  beta_i multiplies node i - n.
    """
    npts = 2 * n + 2
    if m == 0:
        nodes = list(range(-n, n + 2))
        out = []
        for j in nodes:
            poly = [Fraction(1)]
            for k in nodes:
                if k == j:
                    continue
                poly = _poly_mul(poly, [Fraction(-k, j - k), Fraction(1, j - k)])
            out.append(tuple(poly))
        return tuple(out)
    h0, h1 = _hermite_basis(m)
    polys = [[Fraction(0)] * (2 * m + 2) for _ in range(npts)]
    for d in range(m + 1):
        if d == 0:
            w0 = {0: Fraction(1)}
        else:
            c = _centred_fd(n, d)
            w0 = {j: c[j + n] for j in range(-n, n + 1)}
        for node, w in w0.items():
            # derivative at 0 uses nodes around 0; at 1 the same stencil shifted by 1
            if w != 0:
                polys[node + n] = _poly_add(polys[node + n], h0[d], w)
                polys[node + 1 + n] = _poly_add(polys[node + 1 + n], h1[d], w)
    return tuple(tuple(p) for p in polys)


def _deriv_coeffs(coeffs, deriv):
    c = list(coeffs)
    for _ in range(deriv):
        c = [k * c[k] for k in range(1, len(c))] or [Fraction(0)]
    return c


def beta_eval_exact(n, m, x, deriv=0):
    """Exact weights at a rational x (list of Fractions)."""
    x = Fraction(x)
    out = []
    for coeffs in beta_coefficients(n, m):
        c = _deriv_coeffs(coeffs, deriv)
        acc = Fraction(0)
        for a in reversed(c):
            acc = acc * x + a
        out.append(acc)
    return out


def beta_eval(n, m, x, deriv=0):
    """Weights at x (scalar or numpy array) in float64, Horner order.

    Returns an array of shape (2n+2,) + shape(x).
    """
    import numpy as np
    x = np.asarray(x, dtype=np.float64)
    out = []
    for coeffs in beta_coefficients(n, m):
        c = [float(v) for v in _deriv_coeffs(coeffs, deriv)]
        acc = np.zeros_like(x)
        for a in reversed(c):
            acc = acc * x + a
        out.append(acc)
    return np.stack(out)
