// Oracle (test infrastructure only): CPU FP64 restatement of the SGTsh
// frequency loop, src/SGTsh/SGTsh-MPI.f90:389-613.  Parity unpinned: see
// oracle_common.hpp.  Each function names the Fortran routine it restates.
#include "oracle_common.hpp"
#include "dsmsgt.h"

#include <cstring>

namespace oracle {
namespace {

// calcoef, src/SGTsh/others.f90:772-800
void calcoef_sh(int nzone, double omega, const double* q, cplx* coef) {
    for (int iz = 0; iz < nzone; ++iz) {
        if (q[iz] <= 0.0) {
            coef[iz] = cplx(1.0);
        } else {
            double aa = (omega == 0.0) ? 1.0 : 1.0 + std::log(omega / (2.0 * kPi)) / (kPi * q[iz]);
            double bb = 1.0 / (2.0 * q[iz]);
            coef[iz] = cplx(aa, bb) * cplx(aa, bb);
        }
    }
}

// callsuf, src/SGTsh/others.f90:748-766 (coef stays 1: the sum of the four
// polynomial coefficients of the top zone)
int callsuf_sh(double omega, int nzone, const double* vrmax, const double* vsv) {
    double tvs = 0.0;
    for (int i = 0; i < 4; ++i) tvs = tvs + vsv[4 * (nzone - 1) + i] * 1.0;
    return (int)(omega * vrmax[nzone - 1] / tvs - 0.5) + 1;
}

// cala0, src/SGTsh/calmat.f90:267-285
void cala0(int nlayer, double omega, double omegai, const double* t, const double* h1,
           const double* h2, const double* h3, const double* h4, cplx coef, cplx* a0) {
    cplx comega2 = cplx(omega, -omegai) * cplx(omega, -omegai);
    for (int i = 0; i < 4 * nlayer; ++i) {
        double h = h1[i] - h2[i] + h3[i] - 2.0 * h4[i];
        a0[i] = comega2 * cplx(t[i]) - coef * cplx(h);
    }
}

// cala2, src/SGTsh/calmat.f90:290-304
void cala2(int nlayer, const double* h4, cplx coef, cplx* a2) {
    for (int i = 0; i < 4 * nlayer; ++i) a2[i] = -coef * cplx(h4[i]);
}

// calga, src/SGTsh/calmat.f90:329-353
void calga(int nlayer, double omega, double omegai, int l, const double* t, const double* h1,
           const double* h2, const double* h3, const double* h4, cplx coef, cplx* a) {
    cplx comega2 = cplx(omega, -omegai) * cplx(omega, -omegai);
    double xl2m2 = (double)l * (double)(l + 1) - 2.0;
    for (int i = 0; i < 4 * nlayer; ++i) {
        double h = h1[i] - h2[i] + h3[i] + xl2m2 * h4[i];
        a[i] = comega2 * cplx(t[i]) - coef * cplx(h);
    }
}

// overlap, src/SGTsh/calmat.f90:386-423.  a: 1-based element entries
// a[1..4*nlayer]; a2: 2 x (nlayer+1) band, column-major, accumulated.
void overlap(int nlayer, const cplx* a, cplx* a2) {
    int nsize = nlayer + 1;
    auto A2 = [&](int k, int j) -> cplx& { return a2[(k - 1) + 2 * (j - 1)]; };
    for (int j = 1; j <= nsize; ++j) {
        int i1 = (j - 1 > 1) ? j - 1 : 1;
        for (int i = i1; i <= j; ++i) {
            int k = i - j + 2;
            if (i == j) {
                if (i == 1) A2(k, j) = A2(k, j) + a[1];
                else if (i == nsize) A2(k, j) = A2(k, j) + a[4 * nlayer];
                else {
                    int k1 = 4 * i - 4, k2 = k1 + 1;
                    A2(k, j) = A2(k, j) + a[k1] + a[k2];
                }
            }
            if (i + 1 == j) {
                int k1 = 4 * i - 2;
                A2(k, j) = A2(k, j) + a[k1];
            }
        }
    }
}

// dclisb0 + dcsbsub0 for nud = 1, src/SGTsh/dclib.f90:1-137.
// a: (2,n) band (1-based columns), dr: [n+1], b: [n+1] rhs -> solution.
void dclisb0_factor(cplx* a, int n, cplx* dr) {
    auto A = [&](int i, int j) -> cplx& { return a[(i - 1) + 2 * (j - 1)]; };
    const int m = 2;
    dr[1] = cplx(1.0) / A(m, 1);
    cplx xx = A(m - 1, 2);
    A(m - 1, 2) = A(m - 1, 2) * dr[1];
    cplx s = A(m, 2) - xx * A(m - 1, 2);
    dr[2] = cplx(1.0) / s;
    for (int j = 3; j <= n; ++j) {
        xx = A(1, j);
        A(1, j) = xx * dr[j - 1];
        s = A(2, j) - xx * A(1, j);
        dr[j] = cplx(1.0) / s;
    }
}
void dcsbsub0(const cplx* a, int n, cplx* b, const cplx* dr, cplx* z) {
    auto A = [&](int i, int j) { return a[(i - 1) + 2 * (j - 1)]; };
    z[1] = b[1];
    for (int j = 2; j <= n; ++j) z[j] = b[j] - A(1, j) * z[j - 1];
    for (int j = 1; j <= n; ++j) z[j] = z[j] * dr[j];
    b[n] = z[n];
    for (int j = 1; j <= n - 1; ++j) b[n - j] = z[n - j] - A(1, n - j + 1) * b[n - j + 1];
}

// calg2, src/SGTsh/calmat.f90:427-479.  ga2 is factored in place at the
// first call of an order (ig2 == 0 with m == -2 or m == -l).
void calg2(int l, int m, double spo, double r0, const double mt[3][3], double mu0, cplx coef,
           const cplx* ga, const cplx* a, cplx* ga2, cplx* dr, cplx* g2, int& ig2) {
    cplx cg2[4] = {cplx(0.0), cplx(0.0), cplx(0.0), cplx(0.0)};
    cplx dd = cplx(0.0);
    double sgn = (m >= 0) ? 1.0 : -1.0;
    if (std::abs(m) == 1) {
        double b1 = std::sqrt((double)(2 * l + 1) / (16.0 * kPi));
        dd = cplx(b1) * cplx(sgn * mt[0][2], mt[0][1]) / (cplx(r0 * r0 * mu0) * coef);
        int itmp = 4;
        for (int i = 2; i <= 3; ++i) {
            cg2[i] = -dd * (ga[itmp + 1] + ga[itmp + 2]);
            itmp = itmp + 2;
        }
    } else if (std::abs(m) == 2) {
        double b1 = std::sqrt((double)(2 * l + 1) * (double)(l - 1) * (double)(l + 2) / (64.0 * kPi));
        cg2[2] = cplx(b1 / r0) * cplx(2.0 * mt[1][2], sgn * (mt[1][1] - mt[2][2]));
    }
    cplx z[4];
    if (((m == -2) || (m == -l)) && ig2 == 0) {
        dclisb0_factor(ga2, 3, dr);
        dcsbsub0(ga2, 3, cg2, dr, z);
        ig2 = ig2 + 1;
    } else {
        dcsbsub0(ga2, 3, cg2, dr, z);
    }
    cg2[3] = cg2[3] + dd;
    int itmp = (int)std::trunc(spo);
    g2[itmp + 1] = a[1] * cg2[1] + a[2] * cg2[3];
    g2[itmp + 2] = a[3] * cg2[1] + a[4] * cg2[3];
}

// calbvecphi0, src/SGTsh/trial.f90:1-83.  Index: v[(k-1) + 3*(m+2)].
void calbvecphi0(int l, double theta, double* plm, cplx* bvec, cplx* bvecdt, cplx* bvecdp) {
    auto B = [](cplx* v, int k, int m) -> cplx& { return v[(k - 1) + 3 * (m + 2)]; };
    if (theta == 0.0 || theta == kPi) {
        for (int i = 0; i < 15; ++i) bvec[i] = bvecdt[i] = bvecdp[i] = cplx(0.0);
        return;
    }
    double x = std::cos(theta);
    double xl2 = (double)l * (double)(l + 1);
    for (int m = 0; m <= (l < 3 ? l : 3); ++m) calplm(l, m, x, plm + 3 * m);
    for (int m = 0; m <= (l < 2 ? l : 2); ++m) {
        double fact = 1.0;
        if (m != 0)
            for (int i = l - m + 1; i <= l + m; ++i) fact = fact * (double)i;
        double coef = std::sqrt((double)(2 * l + 1) / (4.0 * kPi) / fact);
        double p = plm[3 * m], pn = plm[3 * (m + 1)];
        double plmdt = (double)m * x / std::sin(theta) * p + pn;
        double st = std::sin(theta);
        B(bvec, 1, m) = cplx(0.0);
        B(bvec, 1, -m) = cplx(0.0);
        B(bvec, 2, m) = cplx(0.0, (double)m) / st * coef * p;
        B(bvec, 2, -m) = conj(B(bvec, 2, m));
        B(bvec, 3, m) = cplx(-coef * plmdt);
        B(bvec, 3, -m) = conj(B(bvec, 3, m));
        B(bvecdt, 1, m) = cplx(0.0);
        B(bvecdt, 1, -m) = cplx(0.0);
        B(bvecdt, 2, m) = cplx(0.0, (double)m) * (plmdt / st - x / (1 - x * x) * p) * coef;
        B(bvecdt, 2, -m) = conj(B(bvecdt, 2, m));
        B(bvecdt, 3, m) = cplx((x / st * plmdt - (double)m * (double)m / (1 - x * x) * p + xl2 * p) * coef);
        B(bvecdt, 3, -m) = conj(B(bvecdt, 3, m));
        B(bvecdp, 1, m) = cplx(0.0);
        B(bvecdp, 1, -m) = cplx(0.0);
        B(bvecdp, 2, m) = cplx(-(double)m * (double)m / st * p * coef);
        B(bvecdp, 2, -m) = conj(B(bvecdp, 2, m));
        B(bvecdp, 3, m) = -cplx(0.0, (double)m) * plmdt * coef;
        B(bvecdp, 3, -m) = conj(B(bvecdp, 3, m));
        if (m % 2 == 1) {
            for (int k = 2; k <= 3; ++k) {
                B(bvec, k, -m) = -B(bvec, k, -m);
                B(bvecdt, k, -m) = -B(bvecdt, k, -m);
                B(bvecdp, k, -m) = -B(bvecdp, k, -m);
            }
        }
    }
}

// calbveczero, src/SGTsh/trial.f90:120-157
void calbveczero(int l, cplx* bvec) {
    auto B = [&](int k, int m) -> cplx& { return bvec[(k - 1) + 3 * (m + 2)]; };
    double xl2 = (double)l * (double)(l + 1);
    for (int m = 0; m <= (l < 1 ? l : 1); ++m) {
        double fact = 1.0;
        if (m != 0)
            for (int i = l - m + 1; i <= l + m; ++i) fact = fact * (double)i;
        double coef = std::sqrt((double)(2 * l + 1) / (4.0 * kPi) / fact);
        B(1, m) = cplx(0.0);
        B(1, -m) = cplx(0.0);
        B(2, m) = cplx(0.0, (double)m) * xl2 * coef / 2.0;
        B(2, -m) = conj(B(2, m));
        B(3, m) = -cplx((double)m, 0.0) * xl2 * coef / 2.0;
        B(3, -m) = conj(B(3, m));
        if (m % 2 == 1) {
            B(2, -m) = -B(2, -m);
            B(3, -m) = -B(3, -m);
        }
    }
}

// calamp, src/SGTsh/others.f90:805-824 (strict l > lsuf)
void calamp_sh(cplx g, int l, int lsuf, double& maxamp, int& ismall, double ratl) {
    double ampratio = 0.0;
    double amp = cabs(g);
    if (amp > maxamp) maxamp = amp;
    if (amp != 0.0 && maxamp != 0.0) ampratio = amp / maxamp;
    if (ampratio < ratl && l > lsuf) ismall = ismall + 1;
    else ismall = 0;
}

// calu, src/SGTsh/others.f90:829-838 (u zeroed by the caller)
void calu(cplx c0, double lsq, const cplx* bvec, cplx* u) {
    u[0] = cplx(0.0);
    u[1] = u[1] + c0 * bvec[1] / cplx(lsq);
    u[2] = u[2] + c0 * bvec[2] / cplx(lsq);
}

// locallyCartesianDerivatives, src/SGTsh/others.f90:336-367
void lcd_sh(const cplx* u, const cplx* udr, const cplx* udt, const cplx* udp, Uder& d, double r,
            double theta) {
    if (theta == 0.0 || theta == kPi) {
        d.u[0][0] = udr[0];
        d.u[1][1] = u[0] / cplx(r);
        d.u[2][2] = u[0] / cplx(r);
        return;
    }
    double ts = std::sin(theta);
    double tc = std::cos(theta) / ts;
    d.u[0][0] = udr[0];
    d.u[0][1] = (udt[0] - u[1]) / cplx(r);
    d.u[0][2] = (udp[0] / cplx(ts) - u[2]) / cplx(r);
    d.u[1][0] = udr[1];
    d.u[1][1] = (udt[1] + u[0]) / cplx(r);
    d.u[1][2] = (udp[1] / cplx(ts) - u[2] * cplx(tc)) / cplx(r);
    d.u[2][0] = udr[2];
    d.u[2][1] = udt[2] / cplx(r);
    d.u[2][2] = (udp[2] / cplx(ts) + u[0] + u[1] * cplx(tc)) / cplx(r);
}

#define U(i, j) d.u[(i)-1][(j)-1]
// udertotsgtSH, src/SGTsh/others.f90:249-332; t = tsgt(1:10) of one point
void udertotsgt_sh(int imt, const Uder& d, cplx* t) {
    // t[0..9] map to the reference's tsgt(7),(12),(13),...,(20)
    cplx& t7 = t[0]; cplx& t12 = t[1]; cplx& t13 = t[2]; cplx& t14 = t[3]; cplx& t15 = t[4];
    cplx& t16 = t[5]; cplx& t17 = t[6]; cplx& t18 = t[7]; cplx& t19 = t[8]; cplx& t20 = t[9];
    if (imt == 2) {
        t12 = t12 - 2.5e-1 * U(2, 2) - 2.5e-1 * U(3, 3);
        t17 = t17 - 1.25e-1 * U(1, 2) - 1.25e-1 * U(2, 1);
        t18 = t18 + 1.25e-1 * U(1, 2) + 1.25e-1 * U(2, 1);
        t19 = t19 + 1.25e-1 * U(2, 2) - 1.25e-1 * U(3, 3);
        t20 = t20 + 1.25e-1 * U(2, 2) - 1.25e-1 * U(3, 3);
    }
    if (imt == 3) {
        t12 = t12 + 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
        t17 = t17 - 1.25e-1 * U(1, 2) - 1.25e-1 * U(2, 1);
        t18 = t18 + 1.25e-1 * U(1, 2) + 1.25e-1 * U(2, 1);
        t19 = t19 - 1.25e-1 * U(2, 2) + 1.25e-1 * U(3, 3);
        t20 = t20 - 1.25e-1 * U(2, 2) + 1.25e-1 * U(3, 3);
    }
    if (imt == 4) {
        t7 = t7 - 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
        t13 = t13 - 2.5e-1 * U(1, 2) - 2.5e-1 * U(2, 1);
        t14 = t14 + 2.5e-1 * U(1, 2) + 2.5e-1 * U(2, 1);
        t15 = t15 + 2.5e-1 * U(2, 2) - 2.5e-1 * U(3, 3);
        t16 = t16 - 2.5e-1 * U(2, 2) + 2.5e-1 * U(3, 3);
    }
    if (imt == 5) {
        t13 = t13 + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t14 = t14 + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t15 = t15 - 2.5e-1 * U(2, 3) - 2.5e-1 * U(3, 2);
        t16 = t16 - 2.5e-1 * U(2, 3) - 2.5e-1 * U(3, 2);
    }
    if (imt == 6) {
        t17 = t17 + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t18 = t18 + 2.5e-1 * U(1, 3) + 2.5e-1 * U(3, 1);
        t19 = t19 - 2.5e-1 * U(2, 3) - 2.5e-1 * U(3, 2);
        t20 = t20 + 2.5e-1 * U(2, 3) + 2.5e-1 * U(3, 2);
    }
}

// udertorsgtSH, src/SGTsh/others.f90:196-245; r[0..4] = rsgt(6..10)
void udertorsgt_sh(int icomp, const Uder& d, cplx* r) {
    if (icomp == 2) {
        r[0] = r[0] - 5.e-1 * U(2, 2) - 5.e-1 * U(3, 3);
        r[1] = r[1] - 5.e-1 * U(2, 2) + 5.e-1 * U(3, 3);
        r[3] = r[3] - 5.e-1 * U(1, 2) - 5.e-1 * U(2, 1);
    }
    if (icomp == 3) {
        r[2] = r[2] - 5.e-1 * U(2, 3) - 5.e-1 * U(3, 2);
        r[4] = r[4] + 5.e-1 * U(1, 3) + 5.e-1 * U(3, 1);
    }
}
#undef U

// utosynnSH, src/SGTsh/others.f90:132-186; s[0..4] = synn(6..10)
void utosynn_sh(int imt, const cplx* u, cplx* s) {
    if (imt == 2) { s[0] = s[0] - 5.e-1 * u[1]; s[1] = s[1] - 5.e-1 * u[1]; }
    if (imt == 3) { s[0] = s[0] - 5.e-1 * u[1]; s[1] = s[1] + 5.e-1 * u[1]; }
    if (imt == 4) { s[3] = s[3] + u[1]; }
    if (imt == 5) { s[4] = s[4] + u[2]; }
    if (imt == 6) { s[2] = s[2] - u[2]; }
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

}  // namespace

// One frequency of src/SGTsh/SGTsh-MPI.f90:389-613.  Outputs are complex128
// column-major (10, r_n, theta_n), (5, r_n, theta_n), (5, theta_n).
void sh_one_frequency(const dsm_sh_setup_t& s, int ifreq, cplx* tsgt, cplx* rsgt, cplx* synn,
                      int* llog_out) {
    const int nzone = s.nzone, nn = s.nnlayer + 1, r_n = s.r_n, th_n = s.theta_n;
    const int NT = DSM_SH_NUM_TSGT, NR = DSM_SH_NUM_RSGT, NS = DSM_SH_NUM_SYNN;
    for (long k = 0; k < (long)NT * r_n * th_n; ++k) tsgt[k] = cplx(0.0);
    for (long k = 0; k < (long)NR * r_n * th_n; ++k) rsgt[k] = cplx(0.0);
    for (long k = 0; k < (long)NS * th_n; ++k) synn[k] = cplx(0.0);
    double omega = 2.0 * kPi * (double)ifreq / s.tlen;
    int lsuf = callsuf_sh(omega, nzone, s.vrmax, s.vsv);
    std::vector<cplx> coef(nzone);
    calcoef_sh(nzone, omega, s.qmu, coef.data());
    std::vector<double> plm(12 * th_n, 0.0);
    std::vector<cplx> a0(2 * nn), a2(2 * nn), a(2 * nn), cwork(4 * s.nnlayer + 1);
    for (int j = 0; j < nzone; ++j) {
        int o = s.jsp[j] - 1;
        cala0(s.nlayer[j], omega, s.omegai, s.t + o, s.h1 + o, s.h2 + o, s.h3 + o, s.h4 + o, coef[j],
              cwork.data() + 1);
        overlap(s.nlayer[j], cwork.data(), a0.data() + 2 * (s.isp[j] - 1));
        cala2(s.nlayer[j], s.h4 + o, coef[j], cwork.data() + 1);
        overlap(s.nlayer[j], cwork.data(), a2.data() + 2 * (s.isp[j] - 1));
    }
    int ismall = 0;
    double maxamp = -1.0;
    int llog = s.maxlmax;
    std::vector<cplx> bvec(15 * th_n), bvecdt(15 * th_n), bvecdp(15 * th_n);
    std::vector<cplx> g0(nn + 1), dr(nn + 1), z(nn + 1);
    std::vector<double> thr(th_n);
    for (int it = 0; it < th_n; ++it) thr[it] = s.theta[it] / 180.0 * kPi;
    const int spn0 = s.spn - 1;
    const int gofs = s.isp[spn0] - 1;  // g0(isp(spn)) base
    for (int l = 0; l <= s.maxlmax; ++l) {
        double lsq = std::sqrt((double)l * (double)(l + 1));
        if (ismall > 20) {  // the reference only keeps refreshing bvec (cycle)
            if (llog > l) llog = l;
            break;
        }
        for (int it = 0; it < th_n; ++it)
            calbvecphi0(l, thr[it], plm.data() + 12 * it, bvec.data() + 15 * it,
                        bvecdt.data() + 15 * it, bvecdp.data() + 15 * it);
        cplx rvec[15];
        calbveczero(l, rvec);
        // cala, src/SGTsh/calmat.f90:309-324
        double xl2 = (double)l * (double)(l + 1);
        for (int k = 0; k < 2 * nn; ++k) a[k] = a0[k] + cplx(xl2) * a2[k];
        cplx aa[5], ga[9], ga2[6];
        for (auto& c : ga2) c = cplx(0.0);
        {
            int o = s.ins - 1;
            calga(1, omega, s.omegai, l, s.t + o, s.h1 + o, s.h2 + o, s.h3 + o, s.h4 + o,
                  coef[spn0], aa + 1);
            calga(2, omega, s.omegai, l, s.gt, s.gh1, s.gh2, s.gh3, s.gh4, coef[spn0], ga + 1);
            overlap(2, ga, ga2);
        }
        cplx gdr[4];
        for (int m = -2; m <= 2; ++m) {
            if (!(m != 0 && std::abs(m) <= std::abs(l))) continue;
            int ig2 = 0;
            for (int imt = 2; imt <= 6; ++imt) {
                for (auto& c : g0) c = cplx(0.0);
                double mt[3][3];
                setmt(imt, mt);
                calg2(l, m, s.spo, s.r0, mt, s.mu0, coef[spn0], ga, aa, ga2, gdr, g0.data() + gofs,
                      ig2);
                if ((m == -2) || (m == -l)) {
                    if (ig2 == 1) {
                        dclisb0_factor(a.data(), nn, dr.data());
                        dcsbsub0(a.data(), nn, g0.data(), dr.data(), z.data());
                        ig2 = ig2 + 1;
                    } else {
                        dcsbsub0(a.data(), nn, g0.data(), dr.data(), z.data());
                    }
                } else {
                    dcsbsub0(a.data(), nn, g0.data(), dr.data(), z.data());
                }
                if (imt == 3) calamp_sh(g0[nn], l, lsuf, maxamp, ismall, s.ratl);
                if (s.synn_switch == 1) {
                    for (int it = 0; it < th_n; ++it) {
                        cplx u[3] = {cplx(0.0), cplx(0.0), cplx(0.0)};
                        calu(g0[nn], lsq, bvec.data() + 15 * it + 3 * (m + 2), u);
                        utosynn_sh(imt, u, synn + NS * it);
                    }
                }
                for (int ir = 0; ir < r_n; ++ir) {
                    cplx gl[3], g0tmp, g0der;
                    for (int k = 0; k < 3; ++k) gl[k] = g0[s.iista[3 * ir + k]];
                    interpolate(1, 0, s.r[ir], s.rrsta + 3 * ir, gl, &g0tmp);
                    interpolate(1, 1, s.r[ir], s.rrsta + 3 * ir, gl, &g0der);
                    for (int it = 0; it < th_n; ++it) {
                        cplx u[3] = {}, udr[3] = {}, udt[3] = {}, udp[3] = {};
                        Uder d;
                        d.zero();
                        int bo = 15 * it + 3 * (m + 2);
                        calu(g0tmp, lsq, bvec.data() + bo, u);
                        calu(g0der, lsq, bvec.data() + bo, udr);
                        calu(g0tmp, lsq, bvecdt.data() + bo, udt);
                        calu(g0tmp, lsq, bvecdp.data() + bo, udp);
                        lcd_sh(u, udr, udt, udp, d, s.r[ir], thr[it]);
                        udertotsgt_sh(imt, d, tsgt + NT * ((long)ir + (long)r_n * it));
                    }
                }
            }
            if (std::abs(m) == 1) {
                for (int icomp = 2; icomp <= 3; ++icomp) {
                    for (auto& c : g0) c = cplx(0.0);
                    g0[nn] = -conj(rvec[(icomp - 1) + 3 * (m + 2)]) / cplx(lsq);
                    dcsbsub0(a.data(), nn, g0.data(), dr.data(), z.data());
                    for (int ir = 0; ir < r_n; ++ir) {
                        cplx gl[3], g0tmp, g0der;
                        for (int k = 0; k < 3; ++k) gl[k] = g0[s.iista[3 * ir + k]];
                        interpolate(1, 0, s.r[ir], s.rrsta + 3 * ir, gl, &g0tmp);
                        interpolate(1, 1, s.r[ir], s.rrsta + 3 * ir, gl, &g0der);
                        for (int it = 0; it < th_n; ++it) {
                            cplx u[3] = {}, udr[3] = {}, udt[3] = {}, udp[3] = {};
                            Uder d;
                            d.zero();
                            int bo = 15 * it + 3 * (m + 2);
                            calu(g0tmp, lsq, bvec.data() + bo, u);
                            calu(g0der, lsq, bvec.data() + bo, udr);
                            calu(g0tmp, lsq, bvecdt.data() + bo, udt);
                            calu(g0tmp, lsq, bvecdp.data() + bo, udp);
                            lcd_sh(u, udr, udt, udp, d, s.r[ir], thr[it]);
                            udertorsgt_sh(icomp, d, rsgt + NR * ((long)ir + (long)r_n * it));
                        }
                    }
                }
            }
        }
    }
    *llog_out = llog;
}

}  // namespace oracle

extern "C" int oracle_sh_run(const dsm_sh_setup_t* s, const int* ilist, int n, double* tsgt,
                             double* rsgt, double* synn, int* llog) {
    using oracle::cplx;
    long nt = (long)DSM_SH_NUM_TSGT * s->r_n * s->theta_n;
    long nr = (long)DSM_SH_NUM_RSGT * s->r_n * s->theta_n;
    long ns = (long)DSM_SH_NUM_SYNN * s->theta_n;
    std::vector<cplx> t(nt), r(nr), y(ns);
    for (int k = 0; k < n; ++k) {
        int lg = 0;
        oracle::sh_one_frequency(*s, ilist[k], t.data(), r.data(), y.data(), &lg);
        if (tsgt) std::memcpy(tsgt + 2 * nt * k, t.data(), sizeof(cplx) * nt);
        if (rsgt) std::memcpy(rsgt + 2 * nr * k, r.data(), sizeof(cplx) * nr);
        if (synn) std::memcpy(synn + 2 * ns * k, y.data(), sizeof(cplx) * ns);
        if (llog) llog[k] = lg;
    }
    return 0;
}
