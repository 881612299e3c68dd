// Test-infrastructure shim: exposes the reference's C++ weight-polynomial
// functions (bfps/cpp/Lagrange_polys.hpp, bfps/cpp/spline.hpp) under one
// C-linkage entry point so that Python tests can call them through ctypes.
// Built only by oracle/build_ref.py together with the reference sources.
#include "Lagrange_polys.hpp"
#include "spline.hpp"

typedef void (*beta_fn)(int, double, double*);

static beta_fn pick(int n, int m) {
    // Same (neighbours, smoothness) -> function mapping as
    // bfps/cpp/particles/particles_generic_interp.hpp:10-313 (m == 0 is Lagrange).
    static const beta_fn lagrange[] = {0, (beta_fn)beta_Lagrange_n1, (beta_fn)beta_Lagrange_n2,
                                       (beta_fn)beta_Lagrange_n3, (beta_fn)beta_Lagrange_n4,
                                       (beta_fn)beta_Lagrange_n5};
    static const beta_fn m1[] = {0, (beta_fn)beta_n1_m1, (beta_fn)beta_n2_m1, (beta_fn)beta_n3_m1,
                                 (beta_fn)beta_n4_m1, (beta_fn)beta_n5_m1};
    static const beta_fn m2[] = {0, (beta_fn)beta_n1_m2, (beta_fn)beta_n2_m2, (beta_fn)beta_n3_m2,
                                 (beta_fn)beta_n4_m2, (beta_fn)beta_n5_m2};
    if (n < 1 || n > 5) return 0;
    if (m == 0) return lagrange[n];
    if (m == 1) return m1[n];
    if (m == 2) return m2[n];
    return 0;
}

extern "C" int ref_beta(int n, int m, int deriv, double x, double* out) {
    beta_fn f = pick(n, m);
    if (!f) return -1;
    f(deriv, x, out);
    return 0;
}
