// Oracle (test infrastructure only): known-answer entry points for the
// building blocks the frequency loops share, so that tests can hold them
// against independent closed forms (scipy Legendre functions, LAPACK
// solves, exact polynomial interpolation, Python complex division).
#include "oracle_common.hpp"

using namespace oracle;

// P_l^m(x) for l = m..lmax by the calplm recurrence (src/SGTsh/trial.f90:85-118)
extern "C" void oracle_kat_plm(int lmax, int m, double x, double* out) {
    double plm[3] = {0.0, 0.0, 0.0};
    for (int l = m; l <= lmax; ++l) {
        calplm(l, m, x, plm);
        out[l - m] = plm[0];
    }
}

// glu + glusub (src/SGTsh/glu2.f90:140-281): a column-major n x n complex
// (re, im interleaved), b n complex; solution replaces b.  Returns ier.
extern "C" int oracle_kat_glu(double* a, double* b, int n) {
    std::vector<cplx> A(n * n), B(n);
    for (int i = 0; i < n * n; ++i) A[i] = cplx(a[2 * i], a[2 * i + 1]);
    for (int i = 0; i < n; ++i) B[i] = cplx(b[2 * i], b[2 * i + 1]);
    std::vector<int> ip(n);
    int ier = glu(A.data(), n, n, B.data(), -1.0, ip.data());
    for (int i = 0; i < n; ++i) { b[2 * i] = B[i].re; b[2 * i + 1] = B[i].im; }
    return ier;
}

// interpolate (src/SGTsh/others.f90:843-891), one real component
extern "C" double oracle_kat_interp(double rsta, const double* rrsta, const double* g, int nderiv) {
    cplx gc[3] = {cplx(g[0]), cplx(g[1]), cplx(g[2])}, u;
    interpolate(1, nderiv, rsta, rrsta, gc, &u);
    return u.re;
}

// complex division as gfortran evaluates it (Smith's rule)
extern "C" void oracle_kat_cdiv(const double* a, const double* b, double* q) {
    cplx r = cplx(a[0], a[1]) / cplx(b[0], b[1]);
    q[0] = r.re;
    q[1] = r.im;
}
