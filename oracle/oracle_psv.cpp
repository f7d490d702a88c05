// Oracle (test infrastructure only): CPU FP64 restatement of the SGTpsv
// frequency loop, src/SGTpsv/SGTpsv-MPI.f90:535-1152.  Parity unpinned:
// see oracle_common.hpp.  Each function names the Fortran routine it
// restates; quirks of the reference are reproduced and marked QUIRK.
#include "oracle_common.hpp"
#include "dsmsgt.h"

#include <chrono>
#include <cstring>

namespace oracle {
namespace {

inline double f32(double x) { return (double)(float)x; }  // Fortran cmplx(x): default kind

// calcoef, src/SGTpsv/calmat.f90:409-447
void calcoef_psv(int nzone, double omega, const double* qmu, const double* qkappa, cplx* c1,
                 cplx* c2, cplx* c) {
    for (int i = 0; i < nzone; ++i) {
        if (qmu[i] <= 0.0) c1[i] = cplx(1.0);
        else {
            double aa = (omega == 0.0) ? 1.0 : 1.0 + std::log(omega / (2.0 * kPi)) / (kPi * qmu[i]);
            double bb = 1.0 / (2.0 * qmu[i]);
            c1[i] = cplx(aa, bb) * cplx(aa, bb);
        }
        if (qkappa[i] <= 0.0) {
            c2[i] = cplx(1.0);
            c[i] = cplx(1.0) / c2[i];
        } else {
            double aa = (omega == 0.0) ? 1.0 : 1.0 + std::log(omega / (2.0 * kPi)) / (kPi * qkappa[i]);
            double bb = 1.0 / (2.0 * qkappa[i]);
            c2[i] = cplx(aa, bb) * cplx(aa, bb);
            c[i] = cplx(1.0) / c2[i];
        }
    }
}

// element array accessor: entry nnn (1-based) of array k of zone z
struct Elem {
    const dsm_psv_setup_t& s;
    double operator()(int k, int off, int nnn) const {
        return s.solid_el[(size_t)k * s.n_sel + (off - 1) + (nnn - 1)];
    }
};

// cala0, src/SGTpsv/calmat.f90:452-494.  a0: 1-based cwork[1..16*nlayer]
void cala0(const Elem& E, int off, int nlayer, double omega, double omegai, cplx coef1, cplx coef2,
           cplx* a0) {
    for (int i = 1; i <= 16 * nlayer; ++i) a0[i] = cplx(0.0);
    cplx comega2 = cplx(omega, -omegai) * cplx(omega, -omegai);
    for (int i = 1; i <= 16 * nlayer - 3; i += 4) {
        int nnn = (i + 3) / 4;
        if (nnn % 4 == 3) continue;
        double tt = E(DSM_PSV_T, off, nnn);
        cplx hh0 = coef2 * cplx(4.0 * E(DSM_PSV_H1X, off, nnn)) +
                   coef1 * cplx(16.0 / 3.0 * E(DSM_PSV_H2N, off, nnn)) +
                   coef1 * cplx(-4.0 * E(DSM_PSV_H2N, off, nnn)) +
                   coef2 * cplx(2.0 * (E(DSM_PSV_H3AY, off, nnn) + E(DSM_PSV_H5AY, off, nnn))) -
                   coef1 * cplx(4.0 / 3.0 * (E(DSM_PSV_H4AN, off, nnn) + E(DSM_PSV_H6AN, off, nnn))) +
                   coef2 * cplx(3.0 * E(DSM_PSV_H7Z, off, nnn) - 2.0 * E(DSM_PSV_H7Y, off, nnn)) +
                   coef1 * cplx(4.0 / 3.0 * E(DSM_PSV_H8N, off, nnn));
        a0[i] = comega2 * cplx(tt) - hh0;
    }
    for (int i = 4; i <= 16 * nlayer; i += 4) {
        int nnn = i / 4;
        if (nnn % 4 == 3) continue;
        double tt = E(DSM_PSV_T, off, nnn);
        cplx hh0 = coef1 * cplx(E(DSM_PSV_H2L, off, nnn)) +
                   coef1 * cplx(-2.0 * E(DSM_PSV_H2N, off, nnn)) -
                   coef1 * cplx(E(DSM_PSV_H4AL, off, nnn) + E(DSM_PSV_H6AL, off, nnn)) +
                   coef1 * cplx(E(DSM_PSV_H8L, off, nnn));
        a0[i] = comega2 * cplx(tt) - hh0;
    }
}

// cala1, src/SGTpsv/calmat.f90:499-537
void cala1(const Elem& E, int off, int nlayer, cplx coef1, cplx coef2, cplx* a1) {
    for (int i = 1; i <= 16 * nlayer; ++i) a1[i] = cplx(0.0);
    for (int i = 2; i <= 16 * nlayer - 2; i += 4) {
        int nnn = (i + 2) / 4;
        if (nnn % 4 == 3) continue;
        cplx hh1 = -coef2 * cplx(2.0 * E(DSM_PSV_H1X, off, nnn)) -
                   coef1 * cplx(8.0 / 3.0 * E(DSM_PSV_H2N, off, nnn)) -
                   coef1 * cplx(E(DSM_PSV_H2L, off, nnn)) -
                   coef1 * cplx(-2.0 * E(DSM_PSV_H2N, off, nnn)) -
                   coef2 * cplx(E(DSM_PSV_H3Y, off, nnn)) -
                   coef1 * cplx(-2.0 / 3.0 * E(DSM_PSV_H4N, off, nnn)) +
                   coef1 * cplx(E(DSM_PSV_H6L, off, nnn));
        a1[i] = -hh1;
    }
    for (int i = 3; i <= 16 * nlayer - 1; i += 4) {
        int nnn = (i + 1) / 4;
        if (nnn % 4 != 2) continue;
        cplx hh1 = -coef2 * cplx(2.0 * E(DSM_PSV_H1X, off, nnn)) -
                   coef1 * cplx(8.0 / 3.0 * E(DSM_PSV_H2N, off, nnn)) -
                   coef1 * cplx(-2.0 * E(DSM_PSV_H2N, off, nnn)) -
                   coef1 * cplx(E(DSM_PSV_H2L, off, nnn)) +
                   coef1 * cplx(E(DSM_PSV_H4L, off, nnn)) -
                   coef2 * cplx(E(DSM_PSV_H5Y, off, nnn)) +
                   coef1 * cplx(2.0 / 3.0 * E(DSM_PSV_H6N, off, nnn));
        a1[i] = -hh1;
    }
}

// cala2, src/SGTpsv/calmat.f90:543-567
void cala2(const Elem& E, int off, int nlayer, cplx coef1, cplx coef2, cplx* a2) {
    for (int i = 1; i <= 16 * nlayer; ++i) a2[i] = cplx(0.0);
    for (int i = 1; i <= 16 * nlayer - 3; i += 4) {
        int nnn = (i + 3) / 4;
        if (nnn % 4 == 3) continue;
        cplx hh2 = coef1 * cplx(E(DSM_PSV_H2L, off, nnn));
        a2[i] = -hh2;
    }
    for (int i = 4; i <= 16 * nlayer; i += 4) {
        int nnn = i / 4;
        if (nnn % 4 == 3) continue;
        cplx hh2 = coef2 * cplx(E(DSM_PSV_H1X, off, nnn)) +
                   coef1 * cplx(4.0 / 3.0 * E(DSM_PSV_H2N, off, nnn));
        a2[i] = -hh2;
    }
}

// calb0 / calb2, src/SGTpsv/calmat.f90:572-622
void calb0(const double* p1, const double* p3, int nlayer, double omega, double omegai, cplx coef,
           cplx* b0) {
    for (int i = 1; i <= 4 * nlayer; ++i) b0[i] = cplx(0.0);
    cplx comega2 = cplx(omega, -omegai) * cplx(omega, -omegai);
    for (int i = 1; i <= 4 * nlayer; ++i) {
        if (i % 4 == 3) continue;
        b0[i] = -(cplx(p1[i - 1]) / comega2) + coef * cplx(p3[i - 1]);
    }
}
void calb2(const double* p2, int nlayer, double omega, double omegai, cplx* b2) {
    for (int i = 1; i <= 4 * nlayer; ++i) b2[i] = cplx(0.0);
    cplx comega2 = cplx(omega, -omegai) * cplx(omega, -omegai);
    for (int i = 1; i <= 4 * nlayer; ++i) {
        if (i % 4 == 3) continue;
        b2[i] = -(cplx(p2[i - 1]) / comega2);
    }
}

// band view (4, ncol) column-major, 1-based
struct Band {
    cplx* p;
    cplx& operator()(int i, int j) { return p[(i - 1) + 4 * (j - 1)]; }
};

// overlapa, src/SGTpsv/calmat.f90:670-714
void overlapa(int nlayer, const cplx* a, Band a2) {
    int nsize = 2 * (nlayer + 1), msize = 16 * nlayer;
    for (int j = 1; j <= nsize; ++j)
        for (int i = 1; i <= 4; ++i) a2(i, j) = cplx(0.0);
    a2(4, 1) = a[1];
    a2(3, 2) = a[2];
    a2(4, 2) = a[4];
    a2(4, nsize - 1) = a[msize - 3];
    a2(3, nsize) = a[msize - 2];
    a2(4, nsize) = a[msize];
    for (int i = 3; i <= nsize - 1; i += 2) {
        int n1 = 16 * (i - 3) / 2 + 5;
        a2(2, i) = a[n1];
        n1 = n1 + 2;
        a2(3, i) = a[n1];
        if (i != nsize - 1) {
            n1 = n1 + 6;
            int n2 = n1 + 4;
            a2(4, i) = a[n1] + a[n2];
        }
    }
    for (int i = 4; i <= nsize; i += 2) {
        int n1 = 16 * (i - 4) / 2 + 6;
        a2(1, i) = a[n1];
        n1 = n1 + 2;
        a2(2, i) = a[n1];
        if (i != nsize) {
            n1 = n1 + 6;
            int n2 = n1 + 4;
            a2(3, i) = a[n1] + a[n2];
            n1 = n1 + 2;
            n2 = n1 + 4;
            a2(4, i) = a[n1] + a[n2];
        }
    }
}

// overlapb, src/SGTpsv/calmat.f90:720-742
void overlapb(int nlayer, const cplx* b, Band b2) {
    for (int j = 1; j <= nlayer + 1; ++j)
        for (int i = 1; i <= 4; ++i) b2(i, j) = cplx(0.0);
    b2(4, 1) = b[1];
    for (int i = 2; i <= nlayer; ++i) {
        int n1 = 4 * (i - 1), n2 = n1 + 1;
        b2(4, i) = b[n1] + b[n2];
    }
    b2(4, nlayer + 1) = b[4 * nlayer];
    for (int i = 2; i <= nlayer + 1; ++i) b2(3, i) = b[4 * (i - 2) + 2];
}

// calhml, src/SGTpsv/calmat.f90:629-664.  hm(k, lo-based row, 1-based col)
void calhml(const dsm_psv_setup_t& s, int hmoff, int nlayer, cplx coef1, cplx coef2, Band a1) {
    auto H = [&](int k, int lo, int m, int n) {
        return s.hm_el[(size_t)k * 4 * s.n_hm + 4 * (hmoff - 1 + n - 1) + (m - lo)];
    };
    for (int j = 2; j <= 2 * (nlayer + 1); j += 2) {
        for (int i = 1; i <= 3; i += 2) {
            if (i == 1 && j == 2) continue;
            int m = (-i + 3) / 2, n = (i + j - 3) / 2;
            a1(i, j) = a1(i, j) - (-(coef2 * cplx(H(DSM_PSV_H3MY, -2, m, n))) +
                                   coef1 * cplx(2.0 / 3.0 * H(DSM_PSV_H4M2N, -2, m, n)) +
                                   coef1 * cplx(H(DSM_PSV_H6M2L, -2, m, n)));
        }
    }
    for (int j = 3; j <= 2 * nlayer + 1; j += 2) {
        for (int i = 1; i <= 3; i += 2) {
            if (i == 1 && j == 3) continue;
            int m = (-i + 5) / 2, n = (i + j - 4) / 2;
            a1(i, j) = a1(i, j) - (coef1 * cplx(H(DSM_PSV_H4M1L, -1, m, n)) -
                                   coef2 * cplx(H(DSM_PSV_H5MY, -1, m, n)) +
                                   coef1 * cplx(2.0 / 3.0 * H(DSM_PSV_H6M1N, -1, m, n)));
        }
    }
}

// calabnum, src/SGTpsv/calmat.f90:815-903.  anum/bnum: [10][4][4] as
// (i,j,k) -> [(k-1)*16 + (j-1)*4 + (i-1)], the Fortran column-major order.
void calabnum(double omega, double omegai, double rmax, const double* poly, const double* ra,
              double r0, cplx coef1, cplx coef2, cplx* anum, cplx* bnum) {
    for (int k = 0; k < 160; ++k) anum[k] = bnum[k] = cplx(0.0);
    auto AN = [&](int i, int j, int k) -> cplx& { return anum[(k - 1) * 16 + (j - 1) * 4 + (i - 1)]; };
    auto BN = [&](int i, int j, int k) -> cplx& { return bnum[(k - 1) * 16 + (j - 1) * 4 + (i - 1)]; };
    for (int i = 1; i <= 10; ++i) {
        double r;
        if (i <= 5) r = ra[0] + (double)(i - 1) / 4.0 * (r0 - ra[0]);
        else r = ra[1] - (double)(10 - i) / 4.0 * (ra[1] - r0);
        double trho = 0, tvpv = 0, tvph = 0, tvsv = 0, tvsh = 0, teta = 0, coef = 1.0;
        for (int j = 1; j <= 4; ++j) {
            if (j == 1) coef = 1.0;
            else coef = coef * (r / rmax);
            trho = trho + poly[0 + j - 1] * coef;
            tvpv = tvpv + poly[4 + j - 1] * coef;
            tvph = tvph + poly[8 + j - 1] * coef;
            tvsv = tvsv + poly[12 + j - 1] * coef;
            tvsh = tvsh + poly[16 + j - 1] * coef;
            teta = teta + poly[20 + j - 1] * coef;
        }
        double tecA = trho * tvph * tvph;
        double tecC = trho * tvpv * tvpv;
        double tecL = trho * tvsv * tvsv;
        double tecN = trho * tvsh * tvsh;
        double tmu = trho * tvsv * tvsv;
        double tAkappa = tecA - tmu * 4.0 / 3.0;
        double tCkappa = tecC - tmu * 4.0 / 3.0;
        cplx xAkappa = cplx(tAkappa) * coef2;
        cplx xCkappa = cplx(tCkappa) * coef2;
        cplx xrho = cplx(trho);
        cplx xmu = cplx(tmu) * coef1;
        cplx xecL = cplx(tecL) * coef1;
        cplx xecN = cplx(tecN) * coef1;
        cplx xecA = xAkappa + xmu * cplx(4.0 / 3.0);
        cplx xecC = xCkappa + xmu * cplx(4.0 / 3.0);
        cplx xecF = cplx(teta) * (xecA - cplx(2.0) * xecL);
        cplx xFdC = xecF / xecC;
        cplx xAmF2dC = xecA - xecF * xFdC;
        double r2 = r * r;
        cplx comega2 = cplx(omega, -omegai) * cplx(omega, -omegai);
        AN(1, 1, i) = -(cplx(2.0 / r) * xFdC);
        AN(1, 2, i) = cplx(1.0) / xecC;
        AN(2, 1, i) = -(xrho * comega2) + cplx(4.0 / r2) * (xAmF2dC - xecN);
        AN(2, 2, i) = cplx(2.0 / r) * (xFdC - cplx(1.0));
        AN(3, 1, i) = -cplx(1.0 / r);
        AN(3, 3, i) = cplx(1.0 / r);
        AN(3, 4, i) = cplx(1.0) / xecL;
        AN(4, 1, i) = -(cplx(2.0 / r2) * (xAmF2dC - xecN));
        AN(4, 2, i) = -(cplx(1.0 / r) * xFdC);
        AN(4, 3, i) = -(xrho * comega2) - cplx(2.0 / r2) * xecN;
        AN(4, 4, i) = -cplx(3.0 / r);
        BN(1, 3, i) = cplx(1.0 / r) * xFdC;
        BN(2, 3, i) = -(cplx(2.0 / r2) * (xAmF2dC - xecN));
        BN(2, 4, i) = cplx(1.0 / r);
        BN(4, 3, i) = xAmF2dC / cplx(r2);
    }
}

// eqmotion1 (src/SGTpsv/calmat.f90:1176-1204) for stage block b (1..10)
void eqmotion(const cplx* anum, const cplx* bnum, int blk, double l2, const cplx* y, cplx* f) {
    cplx c[4][4];
    int mtmp = 16 * (blk - 1);
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i) {
            cplx b = bnum[mtmp];
            c[i][j] = anum[mtmp] + cplx(l2 * b.re, l2 * b.im);
            mtmp++;
        }
    for (int i = 0; i < 4; ++i) {
        f[i] = cplx(0.0);
        for (int j = 0; j < 4; ++j) f[i] = f[i] + c[i][j] * y[j];
    }
}

// rk3 with n = 1 / rkstep, src/SGTpsv/rk3.f90:1-83.  The four stages use
// coefficient blocks blk[0..3].  y is advanced in place; x0 becomes xe.
void rk3_one(const cplx* anum, const cplx* bnum, const int blk[4], double l2, double& x0, double xe,
             cplx* y0) {
    const double c1 = 1.0 / 6.0, c2 = 1.0 / 3.0, c3 = c2, c4 = c1, b2 = 0.5, b3 = b2;
    double h = (xe - x0) / 1.0;
    cplx ak[4], yn[4], w[4];
    eqmotion(anum, bnum, blk[0], l2, y0, ak);
    for (int i = 0; i < 4; ++i) yn[i] = y0[i] + cplx(h * c1) * ak[i];
    for (int i = 0; i < 4; ++i) w[i] = y0[i] + cplx(h * b2) * ak[i];
    eqmotion(anum, bnum, blk[1], l2, w, ak);
    for (int i = 0; i < 4; ++i) yn[i] = yn[i] + cplx(h * c2) * ak[i];
    for (int i = 0; i < 4; ++i) w[i] = y0[i] + cplx(h * b3) * ak[i];
    eqmotion(anum, bnum, blk[2], l2, w, ak);
    for (int i = 0; i < 4; ++i) yn[i] = yn[i] + cplx(h * c3) * ak[i];
    for (int i = 0; i < 4; ++i) w[i] = y0[i] + cplx(h) * ak[i];
    eqmotion(anum, bnum, blk[3], l2, w, ak);
    for (int i = 0; i < 4; ++i) yn[i] = yn[i] + cplx(h * c4) * ak[i];
    x0 = x0 + h;
    for (int i = 0; i < 4; ++i) y0[i] = yn[i];
    x0 = xe;
}

// calya, src/SGTpsv/calmat.f90:908-1009
void calya(const cplx* anum, const cplx* bnum, double l2, const double* ra, double r0, cplx* ya,
           cplx* yb, cplx* yc, cplx* yd) {
    for (int i = 0; i < 4; ++i) ya[i] = yb[i] = yc[i] = yd[i] = cplx(0.0);
    ya[1] = cplx(1.0);
    yb[3] = cplx(1.0);
    double dr = (r0 - ra[0]) / 2.0;
    if (dr > 0.0) {
        double xs = ra[0];
        const int blk[2][4] = {{1, 2, 2, 3}, {3, 4, 4, 5}};
        for (int k = 0; k < 2; ++k) {
            double xe = xs + dr;
            rk3_one(anum, bnum, blk[k], l2, xs, xe, ya);
            xs = xe - dr;
            rk3_one(anum, bnum, blk[k], l2, xs, xe, yb);
        }
    }
    yc[1] = cplx(1.0);
    yd[3] = cplx(1.0);
    dr = (ra[1] - r0) / 2.0;
    if (dr > 0.0) {
        double xs = ra[1];
        const int blk[2][4] = {{10, 9, 9, 8}, {8, 7, 7, 6}};
        for (int k = 0; k < 2; ++k) {
            double xe = xs - dr;
            rk3_one(anum, bnum, blk[k], l2, xs, xe, yc);
            xs = xe + dr;
            rk3_one(anum, bnum, blk[k], l2, xs, xe, yd);
        }
    }
}

// calg, src/SGTpsv/calmat.f90:1075-1171
void calg(int l, int m, cplx coef1, cplx coef2, double lsq, double ecC0, double ecF0, double ecL0,
          const cplx* ya, const cplx* yb, const cplx* yc, const cplx* yd, const double* ra, double r0,
          const double mt[3][3], cplx* g) {
    double sgn = (m >= 0) ? 1.0 : -1.0;
    double b1 = std::sqrt((double)(2 * l + 1) / (16.0 * kPi));
    double b2 = 0.0;
    if (l != 0) b2 = std::sqrt((double)(2 * l + 1) * (double)(l - 1) * (double)(l + 2) / (64.0 * kPi));
    cplx dd, ee, s1, s2;
    int am = std::abs(m);
    if (am == 2) { dd = cplx(0.0); ee = cplx(0.0); }
    if (am == 1) {
        dd = cplx(0.0);
        ee = cplx(-b1 * sgn * mt[0][1], b1 * mt[0][2]) / (cplx(r0 * r0 * ecL0) * coef1);
    }
    if (am == 0) {
        dd = cplx(2.0 * b1 * mt[0][0] / (r0 * r0)) /
             (cplx(ecC0 - 4.0 / 3.0 * ecL0) * coef2 + cplx(4.0 / 3.0 * ecL0) * coef1);
        ee = cplx(0.0);
        double r03 = r0 * r0 * r0;
        cplx xtmp = ((ecF0 + 2.0 / 3.0 * ecL0) * coef2 - 2.0 / 3.0 * ecL0 * coef1) /
                    ((ecC0 - 4.0 / 3.0 * ecL0) * coef2 + 4.0 / 3.0 * ecL0 * coef1);
        s1 = cplx(-2.0 * b1 * (mt[1][1] + mt[2][2]) / r03) + cplx(4.0 * b1 * mt[0][0] / r03) * xtmp;
        s2 = cplx(b1 * lsq * (mt[1][1] + mt[2][2]) / r03) - cplx(2.0 * b1 * lsq * mt[0][0] / r03) * xtmp;
    }
    if (am == 1) { s1 = cplx(0.0); s2 = cplx(0.0); }
    if (am == 2) {
        double r03 = r0 * r0 * r0;
        s1 = cplx(0.0);
        s2 = cplx(-b2 * (mt[1][1] - mt[2][2]) / r03, sgn * 2.0 * b2 * mt[1][2] / r03);
    }
    cplx sv[4];
    sv[0] = dd;
    sv[1] = s1;
    if (l != 0) {
        sv[2] = cplx(ee.re / lsq, ee.im / lsq);
        sv[3] = cplx(s2.re / lsq, s2.im / lsq);
    } else {
        sv[2] = cplx(0.0);
        sv[3] = cplx(0.0);
    }
    cplx a[16], b[4];
    int ip[4];
    if (l != 0) {
        for (int i = 0; i < 4; ++i) {  // sab1
            a[i + 0] = -ya[i];
            a[i + 4] = -yb[i];
            a[i + 8] = yc[i];
            a[i + 12] = yd[i];
            b[i] = sv[i];
        }
        glu(a, 4, 4, b, -1.0, ip);
    } else {
        for (int i = 0; i < 2; ++i) {  // sab2
            a[i + 0] = -ya[i];
            a[i + 4] = yc[i];
            b[i] = sv[i];
        }
        glu(a, 2, 4, b, -1.0, ip);
        b[2] = b[1];
        b[1] = cplx(0.0);
        b[3] = cplx(0.0);
    }
    double dtmp[4];
    dtmp[0] = -ra[0] * ra[0];
    dtmp[1] = dtmp[0] * lsq;
    dtmp[2] = ra[1] * ra[1];
    dtmp[3] = dtmp[2] * lsq;
    for (int i = 0; i < 4; ++i) g[i] = cplx(b[i].re * dtmp[i], b[i].im * dtmp[i]);
}

// dcsymbdl0, src/SGTpsv/dcsymbdl.f90:2-88.  a: packed 1-based a[1..(m+1)n]
void dcsymbdl0(cplx* a, int m, int n) {
    int l[13], li[13], lj[13];
    int ij = 0;
    for (int i = 1; i <= m; ++i) {
        ij++;
        li[ij] = i + 1;
        lj[ij] = 2;
        l[ij] = m * (i - 1) + 1;
        for (int j = i + 1; j <= m; ++j) {
            ij++;
            l[ij] = l[ij - 1] + m + 1;
            li[ij] = li[ij - 1] + 1;
            lj[ij] = lj[ij - 1] + 1;
        }
    }
    int mm = (m + 1) * m / 2;
    cplx z[5], w[5];
    for (int k = 1; k <= n - m; ++k) {
        int nk = (m + 1) * (k - 1) + 1;
        cplx piv = cplx(1.0) / a[nk + m];
        for (int j = 2; j <= m + 1; ++j) {
            z[j] = -a[nk + m * j];
            w[j] = a[nk + m * j] * piv;
            a[nk + m * j] = w[j];
        }
        int kk = nk + m + m;
        for (int i = 1; i <= mm; ++i) a[kk + l[i]] = a[kk + l[i]] + w[lj[i]] * z[li[i]];
    }
    for (int k = n - m + 1; k <= n - 1; ++k) {
        int nk = (m + 1) * (k - 1) + 1;
        int nkk = (m + 1) * k - 1;
        cplx piv = cplx(1.0) / a[nk + m];
        for (int j = 2; j <= n - k + 1; ++j) {
            z[j] = -a[nk + m * j];
            w[j] = a[nk + m * j] * piv;
            a[nk + m * j] = w[j];
            int nki = nkk + m * (j - 1);
            for (int i = 2; i <= j; ++i) a[nki + i] = a[nki + i] + w[j] * z[i];
        }
    }
}

// dcsbdlv0, src/SGTpsv/dcsymbdl.f90:93-166 (also mydcsbdlv3 / mydcsbdlv1,
// src/SGTpsv/dcsymbdl3.f90:151-214, which are the same arithmetic).
// a: packed 1-based, b and z 1-based.
void dcsbdlv0(const cplx* a, cplx* b, int m, int n, cplx* z) {
    auto A = [&](int i, int j) { return a[(m + 1) * (j - 1) + i]; };
    int mm = m + 1;
    if (mm < 3) {
        z[1] = b[1];
        for (int j = 2; j <= n; ++j) z[j] = b[j] - A(1, j) * z[j - 1];
        for (int j = 1; j <= n; ++j) z[j] = z[j] / A(m + 1, j);
        b[n] = z[n];
        for (int j = 1; j <= n - 1; ++j) b[n - j] = z[n - j] - A(1, n - j + 1) * b[n - j + 1];
    } else {
        z[1] = b[1];
        z[2] = b[2] - A(m - 1, 2) * z[1];  // QUIRK: a(m-1,2), not a(m,2)
        for (int j = 3; j <= n; ++j) {
            int i1 = (j > mm) ? 1 : mm - j + 1;
            cplx sum = cplx(0.0);
            for (int k = i1; k <= mm - 1; ++k) sum = sum + A(k, j) * z[j - mm + k];
            z[j] = b[j] - sum;
        }
        for (int j = 1; j <= n; ++j) z[j] = z[j] / A(m + 1, j);
        b[n] = z[n];
        b[n - 1] = z[n - 1] - A(mm - 1, n) * z[n];
        for (int j = 3; j <= n; ++j) {
            int j1 = n - j + 1;
            int i1 = (j < mm) ? mm - j + 1 : 1;
            cplx sum = cplx(0.0);
            for (int k = i1; k <= mm - 1; ++k) sum = sum + A(k, mm - k + j1) * b[mm - k + j1];
            b[j1] = z[j1] - sum;
        }
    }
}

// caldvecphi0_withplm, src/SGTpsv/trial.f90:97-223.  v[(k-1)+3*(m+2)].
void caldvecphi0_withplm(int l, double theta, double* plm, cplx* bvec, cplx* bvecdt, cplx* bvecdp) {
    auto B = [](cplx* v, int k, int m) -> cplx& { return v[(k - 1) + 3 * (m + 2)]; };
    if (theta == 0.0 || theta == kPi) {
        double sign1 = 1.0;
        if (theta == kPi) sign1 = (l % 2 == 0) ? 1.0 : -1.0;
        for (int i = 0; i < 15; ++i) bvec[i] = bvecdt[i] = bvecdp[i] = cplx(0.0);
        double coeff = std::sqrt((double)(2 * l + 1) / (4.0 * kPi));
        B(bvec, 1, 0) = cplx(f32(coeff), 0.0) * sign1;  // QUIRK: cmplx() is single precision
        return;
    }
    double x = std::cos(theta);
    double xl2 = (double)l * (double)(l + 1);
    for (int m = 0; m <= (l < 3 ? l : 3); ++m) calplm(l, m, x, plm + 3 * m);
    double st = std::sin(theta);
    for (int m = 0; m <= (l < 2 ? l : 2); ++m) {
        double fact = 1.0;
        if (m != 0)
            for (int i = l - m + 1; i <= l + m; ++i) fact = fact * (double)i;
        double coef = std::sqrt((double)(2 * l + 1) / (4.0 * kPi) / fact);
        double p = plm[3 * m], pn = plm[3 * (m + 1)];
        double plmdt = (double)m * x / st * p + pn;
        B(bvec, 1, m) = cplx(coef * p);
        B(bvec, 1, -m) = conj(B(bvec, 1, m));
        B(bvec, 2, m) = cplx(coef * plmdt);
        B(bvec, 2, -m) = conj(B(bvec, 2, m));
        B(bvec, 3, m) = cplx(0.0, (double)m) / st * coef * p;
        B(bvec, 3, -m) = conj(B(bvec, 3, m));
        B(bvecdt, 1, m) = cplx(plmdt * coef);
        B(bvecdt, 1, m) = conj(B(bvecdt, 1, m));
        // QUIRK: bvecdt(1,-m) is never assigned for m > 0 (taken as zero)
        if (m != 0) B(bvecdt, 1, -m) = cplx(0.0);
        B(bvecdt, 2, m) = cplx((-x / st * plmdt + (double)m * (double)m / (1 - x * x) * p - xl2 * p) * coef);
        B(bvecdt, 2, -m) = conj(B(bvecdt, 2, m));
        B(bvecdt, 3, m) = cplx(0.0, (double)m) * (-x / (1 - x * x) * p + 1.0 / st * plmdt) * coef;
        B(bvecdt, 3, -m) = conj(B(bvecdt, 3, m));
        B(bvecdp, 1, m) = cplx(0.0, (double)m) * p * coef;
        B(bvecdp, 1, -m) = conj(B(bvecdp, 1, m));
        B(bvecdp, 2, m) = cplx(0.0, (double)m) * plmdt * coef;
        B(bvecdp, 2, -m) = conj(B(bvecdp, 2, m));
        B(bvecdp, 3, m) = cplx(-(double)m * (double)m / st * p * coef);
        B(bvecdp, 3, -m) = conj(B(bvecdp, 3, m));
        if (m % 2 == 1) {
            for (int k = 1; k <= 3; ++k) {
                B(bvec, k, -m) = -B(bvec, k, -m);
                B(bvecdt, k, -m) = -B(bvecdt, k, -m);
                B(bvecdp, k, -m) = -B(bvecdp, k, -m);
            }
        }
    }
}

// caldveczero, src/SGTpsv/trial.f90:326-364
void caldveczero(int l, cplx* bvec) {
    auto B = [&](int k, int m) -> cplx& { return bvec[(k - 1) + 3 * (m + 2)]; };
    for (int i = 0; i < 15; ++i) bvec[i] = cplx(0.0);
    double xl2 = (double)l * (double)(l + 1);
    for (int m = 0; m <= (l < 1 ? l : 1); ++m) {
        double fact = 1.0;
        if (m != 0)
            for (int i = l - m + 1; i <= l + m; ++i) fact = fact * (double)i;
        double coef = std::sqrt((double)(2 * l + 1) / (4.0 * kPi) / fact);
        if (m == 0) B(1, m) = cplx(f32(coef));  // QUIRK: cmplx() single precision
        if (m == 1) {
            B(2, m) = cplx(-1.0, 0.0) * xl2 * coef / 2.0;
            B(2, -m) = conj(B(2, m));
            B(3, m) = cplx(0.0, (double)m) * xl2 * coef / 2.0;
            B(3, -m) = conj(B(3, m));
        }
        if (m % 2 == 1) {
            B(2, -m) = -B(2, -m);
            B(3, -m) = -B(3, -m);
        }
    }
}

// calamp, src/SGTpsv/others.f90:1246-1264 (l >= lsuf)
void calamp_psv(const cplx* g, int l, int lsuf, double& maxamp, int& ismall, double ratl) {
    double ampratio = 0.0;
    double a1 = cabs(g[0]), a2 = cabs(g[1]);
    double amp = std::sqrt(a1 * a1 + a2 * a2);
    if (amp > maxamp) maxamp = amp;
    if (amp != 0.0 && maxamp != 0.0) ampratio = amp / maxamp;
    if (ampratio < ratl && l >= lsuf) ismall = ismall + 1;
    else ismall = 0;
}

// calup (:983-993) / calu (:968-978) with u accumulated
void calup(cplx c1, cplx c2, double lsq, const cplx* bvec, cplx* u) {
    u[0] = u[0] + c1 * bvec[0];
    u[1] = u[1] + c2 * bvec[1] / cplx(lsq);
    u[2] = u[2] + c2 * bvec[2] / cplx(lsq);
}
void calup0(cplx c1, const cplx* bvec, cplx* u) { u[0] = u[0] + c1 * bvec[0]; }

// calupfluid, src/SGTpsv/others.f90:1009-1031
void calupfluid(cplx c1, cplx omega, double lambda, double qkp, cplx ylm, Uder& d) {
    const double deuxsurpi = 0.63661977236, unsurdeuxpi = 0.15915494309,
                 unsurtrois = 0.33333333333333333333;
    cplx fl = cplx(lambda * 1.0, lambda * (1.0 / qkp));
    double fac = 1 + deuxsurpi / qkp * std::log(unsurdeuxpi * omega.re);
    fl = cplx(fl.re * fac, fl.im * fac);
    d.u[0][0] = omega * unsurtrois / fl * c1 * ylm;
    d.u[1][1] = d.u[0][0];
    d.u[2][2] = d.u[0][0];
}

// locallyCartesianDerivatives, src/SGTpsv/others.f90:310-344.
// QUIRK: cmplx(r), cmplx(sin), cmplx(cot) round to single precision.
void lcd_psv(const cplx* u, const cplx* udr, const cplx* udt, const cplx* udp, Uder& d, double r,
             double theta) {
    double rr = f32(r);
    if (theta == 0.0 || theta == kPi) {
        d.u[0][0] = udr[0];
        d.u[1][1] = u[0] / rr;
        d.u[2][2] = u[0] / rr;
        return;
    }
    double ts = std::sin(theta);
    double tc = std::cos(theta) / ts;
    double fs = f32(ts), fc = f32(tc);
    d.u[0][0] = udr[0];
    d.u[0][1] = (udt[0] - u[1]) / rr;
    d.u[0][2] = (udp[0] / fs - u[2]) / rr;
    d.u[1][0] = udr[1];
    d.u[1][1] = (udt[1] + u[0]) / rr;
    d.u[1][2] = (udp[1] / fs - u[2] * fc) / rr;
    d.u[2][0] = udr[2];
    d.u[2][1] = udt[2] / rr;
    d.u[2][2] = (udp[2] / fs + u[0] + u[1] * fc) / rr;
}

#define U(i, j) d.u[(i)-1][(j)-1]
// udertotsgt, src/SGTpsv/others.f90:231-285; t[0..19] = tsgt(1..20)
void udertotsgt(int imt, const Uder& d, cplx* t) {
    if (imt == 1) {
        t[0] = t[0] + U(1, 1);
        t[2] = t[2] - 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
        t[5] = t[5] - 5.e-1 * U(1, 2) - 5.e-1 * U(2, 1);
        t[9] = t[9] + 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
    }
    if (imt == 2) {
        t[1] = t[1] - 5.e-1 * U(1, 1);
        t[3] = t[3] + 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
        t[7] = t[7] + 2.5e-1 * U(1, 2) + 2.5e-1 * U(2, 1);
        t[8] = t[8] + 5.e-1 * U(1, 1);
        t[10] = t[10] - 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
        t[11] = t[11] - 2.5e-1 * U(2, 2) - 2.5e-1 * U(3, 3);
        t[16] = t[16] - 1.25e-1 * U(1, 2) - 1.25e-1 * U(2, 1);
        t[17] = t[17] + 1.25e-1 * U(1, 2) + 1.25e-1 * U(2, 1);
        t[18] = t[18] + 1.25e-1 * U(2, 2) - 1.25e-1 * U(3, 3);
        t[19] = t[19] + 1.25e-1 * U(2, 2) - 1.25e-1 * U(3, 3);
    }
    if (imt == 3) {
        t[1] = t[1] - 5.e-1 * U(1, 1);
        t[3] = t[3] + 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
        t[7] = t[7] - 2.5e-1 * U(1, 2) - 2.5e-1 * U(2, 1);
        t[8] = t[8] - 5.e-1 * U(1, 1);
        t[10] = t[10] - 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
        t[11] = t[11] + 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
        t[16] = t[16] - 1.25e-1 * U(1, 2) - 1.25e-1 * U(2, 1);
        t[17] = t[17] + 1.25e-1 * U(1, 2) + 1.25e-1 * U(2, 1);
        t[18] = t[18] - 1.25e-1 * U(2, 2) + 1.25e-1 * U(3, 3);
        t[19] = t[19] - 1.25e-1 * U(2, 2) + 1.25e-1 * U(3, 3);
    }
    if (imt == 4) {
        t[4] = t[4] + U(1, 1);
        t[6] = t[6] - 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
        t[12] = t[12] - 2.5e-1 * U(1, 2) - 2.5e-1 * U(2, 1);
        t[13] = t[13] + 2.5e-1 * U(1, 2) + 2.5e-1 * U(2, 1);
        t[14] = t[14] + 2.5e-1 * U(2, 2) - 2.5e-1 * U(3, 3);
        t[15] = t[15] - 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
    }
    if (imt == 5) {
        t[12] = t[12] + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t[13] = t[13] + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t[14] = t[14] - 2.5e-1 * U(2, 3) - 2.5e-1 * U(3, 2);
        t[15] = t[15] - 2.5e-1 * U(2, 3) - 2.5e-1 * U(3, 2);
    }
    if (imt == 6) {
        t[16] = t[16] + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t[17] = t[17] + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t[18] = t[18] - 2.5e-1 * U(2, 3) - 2.5e-1 * U(3, 2);
        t[19] = t[19] + 2.5e-1 * U(2, 3) + 2.5e-1 * U(3, 2);
    }
}

// udertorsgt, src/SGTpsv/others.f90:204-227; r[0..9] = rsgt(1..10)
void udertorsgt(int icomp, const Uder& d, cplx* r) {
    if (icomp == 1) {
        r[0] = r[0] + U(1, 1);
        r[1] = r[1] - 5.e-1 * U(2, 1) - 5.e-1 * U(1, 2);
        r[2] = r[2] + 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
        r[3] = r[3] - 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
    }
    if (icomp == 2) {
        r[4] = r[4] + U(1, 1);
        r[5] = r[5] - 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
        r[6] = r[6] - 5.e-1 * U(2, 2) + 5.e-1 * U(3, 3);
        r[8] = r[8] - 5.e-1 * U(1, 2) - 5.e-1 * U(2, 1);
    }
    if (icomp == 3) {
        r[7] = r[7] - 5.e-1 * U(2, 3) - 5.e-1 * U(3, 2);
        r[9] = r[9] + 5.e-1 * U(1, 3) + 5.e-1 * U(3, 1);
    }
}
#undef U

// utosynn, src/SGTpsv/others.f90:161-198; s[0..9] = synn(1..10)
void utosynn(int imt, const cplx* u, cplx* s) {
    if (imt == 1) { s[0] = s[0] + u[0]; s[4] = s[4] + u[1]; }
    if (imt == 2) {
        s[2] = s[2] + 5.e-1 * u[0]; s[3] = s[3] - 5.e-1 * u[0];
        s[5] = s[5] - 5.e-1 * u[1]; s[6] = s[6] - 5.e-1 * u[1];
    }
    if (imt == 3) {
        s[2] = s[2] - 5.e-1 * u[0]; s[3] = s[3] - 5.e-1 * u[0];
        s[5] = s[5] - 5.e-1 * u[1]; s[6] = s[6] + 5.e-1 * u[1];
    }
    if (imt == 4) { s[1] = s[1] + u[0]; s[8] = s[8] + u[1]; }
    if (imt == 5) { s[9] = s[9] + u[2]; }
    if (imt == 6) { s[7] = s[7] - u[2]; }
}

void setmt(int imt, double mt[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) mt[i][j] = 0.0;
    if (imt == 1) mt[0][0] = 1.0;
    if (imt == 2) mt[1][1] = 1.0;
    if (imt == 3) mt[2][2] = 1.0;
    if (imt == 4) mt[0][1] = 1.0;
    if (imt == 5) mt[0][2] = 1.0;
    if (imt == 6) mt[1][2] = 1.0;
}

// rea2 / rea2_back, src/SGTpsv/calmat.f90:1247-1389.  Builds the l = 0
// tridiagonal c(2,nn0) (rea2 only) and rhs d(nn0); sets jsta, kkdr0, nn0.
// QUIRK: rea2_back writes its matrix into a local array, so the caller's c
// keeps the factor of the last forward solve.
void rea2(const dsm_psv_setup_t& s, int nn, const cplx* a /*1-based packed (4,nn)*/, const cplx* g,
          cplx* c /*1-based packed (2,*) or null*/, cplx* d, int* jsta, int& nn0) {
    auto A = [&](int i, int j) { return a[4 * (j - 1) + i]; };
    auto C = [&](int i, int j) -> cplx& { return c[2 * (j - 1) + i]; };
    int itmp = 0;
    const int nzone = s.nzone;
    for (int iz = 1; iz <= nzone; ++iz) {
        for (int ista = 1; ista <= s.r_n; ++ista)
            if (iz == s.istazone[ista - 1]) jsta[ista - 1] = itmp + s.iista[3 * (ista - 1)];
        int kk = s.kkdr[iz - 1];
        int i1 = itmp + 1, i2;
        if (s.iphase[iz - 1] == 1) {
            if (iz != nzone) i2 = i1 + (s.kkdr[iz] - kk) / 2 - 1;
            else i2 = i1 + (nn + 1 - kk) / 2 - 1;
            d[i1] = g[kk];
            if (c) {
                if (iz != 1) C(1, i1) = (s.iphase[iz - 2] == 2) ? A(3, kk) : A(2, kk);
                C(2, i1) = A(4, kk);
            }
            for (int i = i1 + 1; i <= i2; ++i) {
                int mtmp = kk + 2 * (i - i1);
                d[i] = g[mtmp];
                if (c) { C(1, i) = A(2, mtmp); C(2, i) = A(4, mtmp); }
            }
        } else {
            i2 = i1 + (s.kkdr[iz] - kk) - 1;
            d[i1] = g[kk];
            if (c) {
                if (iz != 1) C(1, i1) = (s.iphase[iz - 2] == 1) ? A(2, kk) : A(3, kk);
                C(2, i1) = A(4, kk);
            }
            for (int i = i1 + 1; i <= i2; ++i) {
                int mtmp = kk + (i - i1);
                d[i] = g[mtmp];
                if (c) { C(1, i) = A(3, mtmp); C(2, i) = A(4, mtmp); }
            }
        }
        itmp = i2;
    }
    nn0 = itmp;
}

}  // namespace

// One frequency of src/SGTpsv/SGTpsv-MPI.f90:535-1152.
//
// The reference's l loop interleaves, per order, the banded solves of every
// source and back-propagation right-hand side with their use (the cutoff
// probe, SYNN and the receiver x theta accumulation).  The solves of
// different orders are independent, so orders are taken in blocks:
//   1. the solves of the block's orders run in parallel over orders, each
//      keeping g0 at the rows the rest of the loop reads (the receivers'
//      three-node stencils, which include the probe rows, and the surface
//      rows nn-1, nn);
//   2. in order: the vector-harmonic recurrence of each order (kept per
//      order) and the cutoff test (calamp, the ismall > 20 exit), which
//      fixes the last order of the block that the loop reaches;
//   3. the accumulation of those orders, in parallel over receivers: each
//      receiver owns its outputs and adds its terms in the reference's
//      (l, m, source) order; SYNN is one more task of the same kind.
// Every value is computed by the same operations, in the same order, as in
// the sequential loop, so the results do not depend on the thread count.
// t_theta (optional) receives the wall time of the parts whose cost is
// proportional to the number of epicentral distances (steps 2 and 3 but the
// cutoff test; at l = 0 the same parts of the sequential branch).
struct PsvOrderSol {
    std::vector<cplx> g;  // [rhs][capture row]
};

void psv_one_frequency(const dsm_psv_setup_t& s, int ifreq, cplx* tsgt, cplx* rsgt, cplx* synn,
                       int* llog_out, double* probe_out = nullptr, int probe_n = 0, int nthreads = 1,
                       double* t_theta = nullptr) {
    using clock = std::chrono::steady_clock;
    double theta_s = 0.0;
    if (nthreads < 1) nthreads = 1;
    const int nzone = s.nzone, nn = s.nn, r_n = s.r_n, th_n = s.theta_n;
    const int NT = DSM_PSV_NUM_TSGT, NR = DSM_PSV_NUM_RSGT, NS = DSM_PSV_NUM_SYNN;
    for (long k = 0; k < (long)NT * r_n * th_n; ++k) tsgt[k] = cplx(0.0);
    for (long k = 0; k < (long)NR * r_n * th_n; ++k) rsgt[k] = cplx(0.0);
    for (long k = 0; k < (long)NS * th_n; ++k) synn[k] = cplx(0.0);
    const double omega = 2.0 * kPi * (double)ifreq / s.tlen;
    const cplx comega(omega, -s.omegai);
    // callsuf (src/SGTpsv/others.f90:1269-1287)
    int lsuf;
    {
        double tvs = 0.0;
        for (int i = 0; i < 4; ++i) tvs = tvs + s.vsv[4 * (nzone - 1) + i] * 1.0;
        lsuf = (int)(omega * s.vrmax[nzone - 1] / tvs - 0.5) + 1;
    }
    std::vector<cplx> coef1(nzone), coef2(nzone), coef(nzone);
    calcoef_psv(nzone, omega, s.qmu, s.qkappa, coef1.data(), coef2.data(), coef.data());
    const int spn0 = s.spn - 1;
    std::vector<cplx> anum(160), bnum(160);
    calabnum(omega, s.omegai, s.rmax, s.src_poly, s.ra_src, s.r0, coef1[spn0], coef2[spn0],
             anum.data(), bnum.data());
    // per-zone l-independent blocks (SGTpsv-MPI.f90:562-588)
    Elem E{s};
    std::vector<std::vector<cplx>> A0(nzone), A1(nzone), A2(nzone);
    {
        int maxl = 0;
        for (int j = 0; j < nzone; ++j) maxl = s.nlayer[j] > maxl ? s.nlayer[j] : maxl;
        std::vector<cplx> cwork(16 * maxl + 1);
        for (int j = 0; j < nzone; ++j) {
            int nl = s.nlayer[j];
            if (s.iphase[j] == 1) {
                int ncol = 2 * (nl + 1);
                A0[j].assign(4 * ncol, cplx(0.0));
                A1[j].assign(4 * ncol, cplx(0.0));
                A2[j].assign(4 * ncol, cplx(0.0));
                cala0(E, s.elem[j], nl, omega, s.omegai, coef1[j], coef2[j], cwork.data());
                overlapa(nl, cwork.data(), Band{A0[j].data()});
                cala1(E, s.elem[j], nl, coef1[j], coef2[j], cwork.data());
                overlapa(nl, cwork.data(), Band{A1[j].data()});
                cala2(E, s.elem[j], nl, coef1[j], coef2[j], cwork.data());
                overlapa(nl, cwork.data(), Band{A2[j].data()});
                calhml(s, s.hmoff[j], nl, coef1[j], coef2[j], Band{A1[j].data()});
            } else {
                int ncol = nl + 1;
                A0[j].assign(4 * ncol, cplx(0.0));
                A1[j].assign(4 * ncol, cplx(0.0));
                A2[j].assign(4 * ncol, cplx(0.0));
                const double* p1 = s.fluid_el + (s.elem[j] - 1);
                const double* p2 = s.fluid_el + s.n_fel + (s.elem[j] - 1);
                const double* p3 = s.fluid_el + 2 * (size_t)s.n_fel + (s.elem[j] - 1);
                calb0(p1, p3, nl, omega, s.omegai, coef[j], cwork.data());
                overlapb(nl, cwork.data(), Band{A0[j].data()});
                calb2(p2, nl, omega, s.omegai, cwork.data());
                overlapb(nl, cwork.data(), Band{A2[j].data()});
            }
        }
    }
    // receivers' stack points (l-independent, :621-629)
    std::vector<int> ksta(r_n);
    for (int ir = 0; ir < r_n; ++ir)
        ksta[ir] = s.kkdr[s.istazone[ir] - 1] + 2 * s.iista[3 * ir] - 1;
    // rows of g0 read after a solve: the receivers' stencils g0(ksta-1 ..
    // ksta+4) (the probe rows are those of the top receiver) and nn-1, nn
    std::vector<int> caprow, capidx(nn + 2, -1);
    auto addrow = [&](int j) {
        if (capidx[j] < 0) {
            capidx[j] = (int)caprow.size();
            caprow.push_back(j);
        }
    };
    for (int ir = 0; ir < r_n; ++ir)
        for (int k = 0; k < 6; ++k) addrow(ksta[ir] - 1 + k);
    addrow(nn - 1);
    addrow(nn);
    const int ncap = (int)caprow.size();
    std::vector<double> thr(th_n);
    for (int it = 0; it < th_n; ++it) thr[it] = s.theta[it] / 180.0 * kPi;
    std::vector<double> plm(12 * th_n, 0.0);
    std::vector<cplx> dvec(15 * th_n), dvecdt(15 * th_n), dvecdp(15 * th_n);
    std::vector<cplx> a(4 * nn + 1), g0(nn + 1), z(nn + 1);
    std::vector<cplx> c(2 * nn + 1), d0(nn + 1);
    std::vector<int> jsta(r_n);
    int nn0 = 0;
    const int itmp_l0 = (s.rmin == 0.0) ? 2 : 1;
    const int itmp_l = (s.rmin == 0.0) ? 3 : 1;
    int ismall = 0;
    double maxamp = -1.0;
    int llog = s.maxlmax;
    const double* rsrc = s.ra_src;
    const int jtmp = s.jsrc;

    // receiver x theta terms of one right-hand side for receivers [ir0, ir1)
    // with the harmonics dv / dvt / dvp of the order
    auto receivers_range = [&](int ir0, int ir1, int m, double lsq, const cplx* gsrc, int l0mode, bool back,
                               int id, const cplx* dv, const cplx* dvt, const cplx* dvp) {
        // gsrc: for l != 0 the 1-based g0; for l = 0 the 1-based d0
        for (int ir = ir0; ir < ir1; ++ir) {
            cplx gt[2] = {}, gd[2] = {};
            if (l0mode) {
                const cplx* gp = gsrc + jsta[ir];
                interpolate(1, 0, s.r[ir], s.rrsta + 3 * ir, gp, gt);
                interpolate(1, 1, s.r[ir], s.rrsta + 3 * ir, gp, gd);
            } else {
                const cplx* gp = gsrc + ksta[ir] - 1;
                interpolate(2, 0, s.r[ir], s.rrsta + 3 * ir, gp, gt);
                interpolate(2, 1, s.r[ir], s.rrsta + 3 * ir, gp, gd);
            }
            bool fluid = s.iphase[s.istazone[ir] - 1] == 2;
            for (int it = 0; it < th_n; ++it) {
                Uder d;
                d.zero();
                int bo = 15 * it + 3 * (m + 2);
                if (fluid) {
                    calupfluid(gt[0], comega, s.lambda[ir], s.qkp[ir], dv[bo], d);
                } else {
                    cplx u[3] = {}, udr[3] = {}, udt[3] = {}, udp[3] = {};
                    if (l0mode) {
                        calup0(gt[0], dv + bo, u);
                        calup0(gd[0], dv + bo, udr);
                        calup0(gt[0], dvt + bo, udt);
                        calup0(gt[0], dvp + bo, udp);
                    } else {
                        calup(gt[0], gt[1], lsq, dv + bo, u);
                        calup(gd[0], gd[1], lsq, dv + bo, udr);
                        calup(gt[0], gt[1], lsq, dvt + bo, udt);
                        calup(gt[0], gt[1], lsq, dvp + bo, udp);
                    }
                    lcd_psv(u, udr, udt, udp, d, s.r[ir], thr[it]);
                }
                if (back) udertorsgt(id, d, rsgt + NR * ((long)ir + (long)r_n * it));
                else udertotsgt(id, d, tsgt + NT * ((long)ir + (long)r_n * it));
            }
        }
    };
    auto receivers = [&](int m, double lsq, const cplx* gsrc, int l0mode, bool back, int id) {
        const auto t0 = clock::now();
        receivers_range(0, r_n, m, lsq, gsrc, l0mode, back, id, dvec.data(), dvecdt.data(), dvecdp.data());
        theta_s += std::chrono::duration<double>(clock::now() - t0).count();
    };
    auto synn_terms = [&](int m, int imt, double lsq, cplx g1, cplx g2, bool l0mode, const cplx* dv) {
        if (s.synn_switch != 1) return;
        for (int th = 0; th < th_n; ++th) {
            cplx u[3] = {};
            if (l0mode) calup0(g1, dv + 15 * th + 3 * (m + 2), u);
            else calup(g1, g2, lsq, dv + 15 * th + 3 * (m + 2), u);
            utosynn(imt, u, synn + NS * th);
        }
    };
    // cala (src/SGTpsv/calmat.f90:747-789) + calbc (:795-809) into the band a
    auto assemble = [&](std::vector<cplx>& ab, double l2, double lsq) {
        for (int k = 1; k <= 4 * nn; ++k) ab[k] = cplx(0.0);
        auto Ag = [&](int i, int j) -> cplx& { return ab[4 * (j - 1) + i]; };
        for (int j = 0; j < nzone; ++j) {
            int kk = s.kkdr[j];
            Band b0{A0[j].data()}, b1{A1[j].data()}, b2{A2[j].data()};
            if (s.iphase[j] == 1) {
                int i2 = kk + 2 * s.nlayer[j] + 1;
                for (int jj = kk; jj <= i2; ++jj) {
                    int mt = jj - kk + 1;
                    for (int ii = 2; ii <= 4; ii += 2)
                        Ag(ii, jj) = Ag(ii, jj) + cplx(b0(ii, mt).re + l2 * b2(ii, mt).re,
                                                       b0(ii, mt).im + l2 * b2(ii, mt).im);
                    for (int ii = 1; ii <= 3; ii += 2)
                        Ag(ii, jj) = Ag(ii, jj) + cplx(lsq * b1(ii, mt).re, lsq * b1(ii, mt).im);
                }
            } else {
                int i2 = kk + s.nlayer[j];
                for (int jj = kk; jj <= i2; ++jj) {
                    int mt = jj - kk + 1;
                    for (int ii = 3; ii <= 4; ++ii)
                        Ag(ii, jj) = Ag(ii, jj) + cplx(b0(ii, mt).re + l2 * b2(ii, mt).re,
                                                       b0(ii, mt).im + l2 * b2(ii, mt).im);
                }
            }
        }
        for (int i = 1; i <= nzone - 1; ++i) {
            if (s.iphase[i - 1] == 1 && s.iphase[i] == 2)
                Ag(2, s.kkdr[i]) = cplx(s.vrmax[i - 1] * s.vrmax[i - 1]);
            if (s.iphase[i - 1] == 2 && s.iphase[i] == 1)
                Ag(3, s.kkdr[i]) = -cplx(s.vrmax[i - 1] * s.vrmax[i - 1]);
        }
    };
    // every right-hand side of order l >= 1, in the reference's sequence:
    // m = -2..2 (|m| <= l): imt = 1..6 (calg, the factorisation once per
    // order, dcsbdlv0 for the excited pairs), then the back-propagated
    // sources (m = 0: vertical force; |m| = 1: icomp 2, 3)
    struct Scratch {
        std::vector<cplx> a, g0, z;
    };
    auto solve_order = [&](int l, Scratch& sc, PsvOrderSol& o) {
        double l2 = (double)l * (double)(l + 1);
        double lsq = std::sqrt(l2);
        cplx rdvec[15];
        caldveczero(l, rdvec);
        assemble(sc.a, l2, lsq);
        cplx ya[4], yb[4], yc[4], yd[4];
        calya(anum.data(), bnum.data(), l2, rsrc, s.r0, ya, yb, yc, yd);
        o.g.clear();
        auto keep = [&]() {
            for (int k = 0; k < ncap; ++k) o.g.push_back(sc.g0[caprow[k]]);
        };
        const int it = itmp_l, n1 = nn - it + 1;
        for (int m = -2; m <= 2; ++m) {
            if (!(std::abs(m) <= std::abs(l))) continue;
            int ig2 = 0;
            for (int imt = 1; imt <= 6; ++imt) {
                double mt[3][3];
                setmt(imt, mt);
                for (auto& v : sc.g0) v = cplx(0.0);
                calg(l, m, coef1[spn0], coef2[spn0], lsq, s.ecC0, s.ecF0, s.ecL0, ya, yb, yc, yd, rsrc, s.r0,
                     mt, sc.g0.data() + jtmp);
                if ((m == -2) || (m == -l)) {
                    if (ig2 == 0) {
                        dcsymbdl0(sc.a.data() + 4 * (it - 1), 3, n1);
                        ig2 = 1;
                    }
                }
                int am = std::abs(m);
                bool solve = (am == 0 && imt <= 3) || (am == 1 && (imt == 4 || imt == 5)) ||
                             (am == 2 && (imt == 2 || imt == 3 || imt == 6));
                if (solve) dcsbdlv0(sc.a.data() + 4 * (it - 1), sc.g0.data() + (it - 1), 3, n1, sc.z.data());
                keep();
            }
            if (m == 0 && s.rsgt_switch == 1) {
                for (auto& v : sc.g0) v = cplx(0.0);
                sc.g0[nn - 1] = -conj(rdvec[0 + 3 * (m + 2)]);
                dcsbdlv0(sc.a.data() + 4 * (it - 1), sc.g0.data() + (it - 1), 3, n1, sc.z.data());
                keep();
            }
            if (std::abs(m) == 1 && s.rsgt_switch == 1) {
                for (int icomp = 2; icomp <= 3; ++icomp) {
                    for (auto& v : sc.g0) v = cplx(0.0);
                    sc.g0[nn] = conj(rdvec[(icomp - 1) + 3 * (m + 2)]) / cplx(lsq);
                    dcsbdlv0(sc.a.data() + 4 * (it - 1), sc.g0.data() + (it - 1), 3, n1, sc.z.data());
                    keep();
                }
            }
        }
    };
    // the cutoff test of order l >= 1 (calamp for imt = 1 of every m, in the
    // m order of the loop) from its solutions
    auto cutoff_order = [&](int l, const PsvOrderSol& o) {
        int k = 0;
        for (int m = -2; m <= 2; ++m) {
            if (!(std::abs(m) <= std::abs(l))) continue;
            const cplx* src = o.g.data() + (size_t)k * ncap;
            const cplx gp[2] = {src[capidx[ksta[r_n - 1] - 1]], src[capidx[ksta[r_n - 1]]]};
            calamp_psv(gp, l, lsuf, maxamp, ismall, s.ratl);
            if (probe_out && m == 0 && l < probe_n) {
                double a1 = cabs(gp[0]), a2 = cabs(gp[1]);
                probe_out[l] = std::sqrt(a1 * a1 + a2 * a2);
            }
            k += 6 + (m == 0 && s.rsgt_switch == 1 ? 1 : 0) + (std::abs(m) == 1 && s.rsgt_switch == 1 ? 2 : 0);
        }
    };
    // terms of order l >= 1 for receivers [ir0, ir1) (task ir0 = r_n: SYNN),
    // in the reference's m / source sequence; gb is the task's own g0
    auto accumulate_order = [&](int l, const PsvOrderSol& o, int ir0, int ir1, std::vector<cplx>& gb,
                                const cplx* dv, const cplx* dvt, const cplx* dvp) {
        double l2 = (double)l * (double)(l + 1);
        double lsq = std::sqrt(l2);
        int k = 0;
        auto load = [&]() {
            const cplx* src = o.g.data() + (size_t)k * ncap;
            for (int q = 0; q < ncap; ++q) gb[caprow[q]] = src[q];
            ++k;
        };
        const bool synn_task = ir0 == r_n;
        for (int m = -2; m <= 2; ++m) {
            if (!(std::abs(m) <= std::abs(l))) continue;
            for (int imt = 1; imt <= 6; ++imt) {
                load();
                if (synn_task) synn_terms(m, imt, lsq, gb[nn - 1], gb[nn], false, dv);
                else receivers_range(ir0, ir1, m, lsq, gb.data(), 0, false, imt, dv, dvt, dvp);
            }
            if (m == 0 && s.rsgt_switch == 1) {
                load();
                if (!synn_task) receivers_range(ir0, ir1, m, lsq, gb.data(), 0, true, 1, dv, dvt, dvp);
            }
            if (std::abs(m) == 1 && s.rsgt_switch == 1) {
                for (int icomp = 2; icomp <= 3; ++icomp) {
                    load();
                    if (!synn_task) receivers_range(ir0, ir1, m, lsq, gb.data(), 0, true, icomp, dv, dvt, dvp);
                }
            }
        }
    };
    auto harmonics = [&](int l) {
        const auto t0 = clock::now();
        for (int it = 0; it < th_n; ++it)
            caldvecphi0_withplm(l, thr[it], plm.data() + 12 * it, dvec.data() + 15 * it,
                                dvecdt.data() + 15 * it, dvecdp.data() + 15 * it);
        theta_s += std::chrono::duration<double>(clock::now() - t0).count();
    };

    // ---- l = 0 (the compact tridiagonal of rea2; its factor stays in c)
    harmonics(0);
    {
        const int l = 0;
        double l2 = 0.0, lsq = 0.0;
        cplx rdvec[15];
        caldveczero(l, rdvec);
        assemble(a, l2, lsq);
        cplx ya[4], yb[4], yc[4], yd[4];
        calya(anum.data(), bnum.data(), l2, rsrc, s.r0, ya, yb, yc, yd);
        const int m = 0;
        for (int imt = 1; imt <= 6; ++imt) {
            double mt[3][3];
            setmt(imt, mt);
            for (auto& v : g0) v = cplx(0.0);
            calg(l, m, coef1[spn0], coef2[spn0], lsq, s.ecC0, s.ecF0, s.ecL0, ya, yb, yc, yd, rsrc, s.r0, mt,
                 g0.data() + jtmp);
            rea2(s, nn, a.data(), g0.data(), c.data(), d0.data(), jsta.data(), nn0);
            int it = itmp_l0;
            int n0 = nn0 - it + 1;
            dcsymbdl0(c.data() + 2 * (it - 1), 1, n0);
            bool solve = (imt <= 3);
            if (solve) dcsbdlv0(c.data() + 2 * (it - 1), d0.data() + (it - 1), 1, n0, z.data());
            {
                const auto t0 = clock::now();
                synn_terms(m, imt, lsq, d0[nn0], cplx(0.0), true, dvec.data());
                theta_s += std::chrono::duration<double>(clock::now() - t0).count();
            }
            receivers(m, lsq, d0.data(), 1, false, imt);
        }
        if (s.rsgt_switch == 1) {
            for (auto& v : g0) v = cplx(0.0);
            g0[nn - 1] = -conj(rdvec[0 + 3 * (m + 2)]);
            rea2(s, nn, a.data(), g0.data(), nullptr, d0.data(), jsta.data(), nn0);
            int it = itmp_l0;
            dcsbdlv0(c.data() + 2 * (it - 1), d0.data() + (it - 1), 1, nn0 - it + 1, z.data());
            receivers(m, lsq, d0.data(), 1, true, 1);
        }
    }
    // ---- l >= 1 in blocks
    Pool pool(nthreads);
    std::vector<Scratch> scr(nthreads);
    for (auto& sc : scr) {
        sc.a.assign(4 * nn + 1, cplx(0.0));
        sc.g0.assign(nn + 1, cplx(0.0));
        sc.z.assign(nn + 1, cplx(0.0));
    }
    const int blk = 8 * nthreads;
    std::vector<PsvOrderSol> sol(blk);
    const size_t hv = (size_t)15 * th_n;
    std::vector<cplx> hdv(blk * hv), hdt(blk * hv), hdp(blk * hv);
    // receiver tasks of the accumulation (contiguous ranges) and SYNN
    const int ntask = std::min(r_n, 4 * nthreads);
    std::vector<std::vector<cplx>> gtask(ntask + 1, std::vector<cplx>(nn + 1, cplx(0.0)));
    bool done = false;
    for (int lb = 1; lb <= s.maxlmax && !done; lb += blk) {
        const int le = std::min(s.maxlmax, lb + blk - 1);
        // 1. solves, in parallel over orders (each pool thread owns a scratch)
        pool.run(le - lb + 1, [&](int i, int t) { solve_order(lb + i, scr[t], sol[i]); });
        // 2. harmonics and the cutoff test in order
        int lend = le + 1;
        {
            const auto t0 = clock::now();
            for (int l = lb; l <= le; ++l) {
                for (int it = 0; it < th_n; ++it)
                    caldvecphi0_withplm(l, thr[it], plm.data() + 12 * it, dvec.data() + 15 * it,
                                        dvecdt.data() + 15 * it, dvecdp.data() + 15 * it);
                const size_t o = (size_t)(l - lb) * hv;
                std::copy(dvec.begin(), dvec.end(), hdv.begin() + o);
                std::copy(dvecdt.begin(), dvecdt.end(), hdt.begin() + o);
                std::copy(dvecdp.begin(), dvecdp.end(), hdp.begin() + o);
                if (ismall > 20) {
                    if (llog > l) llog = l;
                    done = true;
                    lend = l;
                    break;
                }
                const auto tc = clock::now();
                cutoff_order(l, sol[l - lb]);
                theta_s -= std::chrono::duration<double>(clock::now() - tc).count();
            }
            theta_s += std::chrono::duration<double>(clock::now() - t0).count();
        }
        // 3. accumulation of orders lb .. lend-1, in parallel over receivers
        const auto t0 = clock::now();
        pool.run(ntask + 1, [&](int task, int) {
            const int ir0 = task < ntask ? (int)((long)task * r_n / ntask) : r_n;
            const int ir1 = task < ntask ? (int)((long)(task + 1) * r_n / ntask) : r_n;
            for (int l = lb; l < lend; ++l) {
                const size_t o = (size_t)(l - lb) * hv;
                accumulate_order(l, sol[l - lb], ir0, ir1, gtask[task], hdv.data() + o, hdt.data() + o,
                                 hdp.data() + o);
            }
        });
        theta_s += std::chrono::duration<double>(clock::now() - t0).count();
    }
    *llog_out = llog;
    if (t_theta) *t_theta = theta_s;
}

}  // namespace oracle

extern "C" int oracle_psv_probe(const dsm_psv_setup_t* s, int ifreq, double* probe, int n) {
    using oracle::cplx;
    long nt = (long)DSM_PSV_NUM_TSGT * s->r_n * s->theta_n;
    long nr = (long)DSM_PSV_NUM_RSGT * s->r_n * s->theta_n;
    long ns = (long)DSM_PSV_NUM_SYNN * s->theta_n;
    std::vector<cplx> t(nt), r(nr), y(ns);
    int lg = 0;
    oracle::psv_one_frequency(*s, ifreq, t.data(), r.data(), y.data(), &lg, probe, n);
    return lg;
}

extern "C" int oracle_psv_run(const dsm_psv_setup_t* s, const int* ilist, int n, double* tsgt,
                              double* rsgt, double* synn, int* llog) {
    using oracle::cplx;
    long nt = (long)DSM_PSV_NUM_TSGT * s->r_n * s->theta_n;
    long nr = (long)DSM_PSV_NUM_RSGT * s->r_n * s->theta_n;
    long ns = (long)DSM_PSV_NUM_SYNN * s->theta_n;
    std::vector<cplx> t(nt), r(nr), y(ns);
    for (int k = 0; k < n; ++k) {
        int lg = 0;
        oracle::psv_one_frequency(*s, ilist[k], t.data(), r.data(), y.data(), &lg);
        if (tsgt) std::memcpy(tsgt + 2 * nt * k, t.data(), sizeof(cplx) * nt);
        if (rsgt) std::memcpy(rsgt + 2 * nr * k, r.data(), sizeof(cplx) * nr);
        if (synn) std::memcpy(synn + 2 * ns * k, y.data(), sizeof(cplx) * ns);
        if (llog) llog[k] = lg;
    }
    return 0;
}

// One frequency after another, each spread over nthreads host threads
// (order-parallel solves, receiver-parallel theta loop); t_theta[k] (if
// given) receives frequency k's time in its theta-proportional parts and
// t_total[k] its whole time.
extern "C" int oracle_psv_run_threads(const dsm_psv_setup_t* s, const int* ilist, int n, double* tsgt,
                                      double* rsgt, double* synn, int* llog, int nthreads, double* t_theta,
                                      double* t_total) {
    using oracle::cplx;
    long nt = (long)DSM_PSV_NUM_TSGT * s->r_n * s->theta_n;
    long nr = (long)DSM_PSV_NUM_RSGT * s->r_n * s->theta_n;
    long ns = (long)DSM_PSV_NUM_SYNN * s->theta_n;
    std::vector<cplx> t(nt), r(nr), y(ns);
    for (int k = 0; k < n; ++k) {
        int lg = 0;
        double tt = 0.0;
        const auto t0 = std::chrono::steady_clock::now();
        oracle::psv_one_frequency(*s, ilist[k], t.data(), r.data(), y.data(), &lg, nullptr, 0, nthreads, &tt);
        if (t_total) t_total[k] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (t_theta) t_theta[k] = tt;
        if (tsgt) std::memcpy(tsgt + 2 * nt * k, t.data(), sizeof(cplx) * nt);
        if (rsgt) std::memcpy(rsgt + 2 * nr * k, r.data(), sizeof(cplx) * nr);
        if (synn) std::memcpy(synn + 2 * ns * k, y.data(), sizeof(cplx) * ns);
        if (llog) llog[k] = lg;
    }
    return 0;
}
