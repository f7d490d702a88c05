// SH (toroidal) engine: replaces src/SGTsh/SGTsh-MPI.f90:404-555.
//
// Kernels (plain FP64 path; this file is compiled without fused
// multiply-add so every scalar operation rounds as the Fortran does):
//   k_sh_omega   per-omega band pieces a0, a2 (cala0, cala2, overlap,
//                src/SGTsh/calmat.f90:267-304, 386-423; calcoef,
//                src/SGTsh/others.f90:772-800)
//   k_sh_solve   one thread per (omega, l): assembly a = a0 + l(l+1) a2
//                (cala, calmat.f90:309-324) fused with the complex-symmetric
//                tridiagonal LDL^T (dclisb0, src/SGTsh/dclib.f90:1-89) and
//                the substitution (dcsbsub0, :90-137) of three basis
//                right-hand sides: the two source rows and the surface row.
//                Factors live in HBM between the downward and upward sweeps
//                (layout [row][system], coalesced).
//   k_sh_fields  source terms (calga, calg2, calmat.f90:329-353, 427-479),
//                back-propagation sources (calbveczero, trial.f90:120-157),
//                receiver interpolation (interpolate, others.f90:843-891):
//                writes the per-order receiver fields of every active
//                (m, source) slot and the cutoff probe |g0(nn)| of imt = 3.
//   k_sh_scan    the cutoff test (calamp, others.f90:805-824, and the
//                ismall > 20 rule, SGTsh-MPI.f90:431-436) in the
//                reference's order.
//   k_sh_epi     turns the l-contractions into TSGT / RSGT / SYNN
//                (calu, locallyCartesianDerivatives, udertotsgtSH,
//                udertorsgtSH, utosynnSH, others.f90:132-367, 829-838).
#include <algorithm>
#include <cstdlib>
#include <cmath>

#include "engine.cuh"

namespace dsm {
namespace {

constexpr int SH_NSLOT1 = 8;  // |m| = 1: m = -1, +1 x {imt 4, imt 5, back 2, back 3}
constexpr int SH_NSLOT2 = 6;  // |m| = 2: m = -2, +2 x {imt 2, imt 3, imt 6}
constexpr int SH_NF = 3;      // fields: W/lsq, W'/lsq, l(l+1) W/lsq

struct ShDev {
    int nn, nzone, R, ncap, srow, ins, spn;
    double spo, r0, mu0, tlen, omegai;
    const int *nlayer, *isp, *jsp;
    const double *qmu;
    const double *t, *h1, *h2, *h3, *h4;  // [4*nnlayer]
    const double *g;                      // gt, gh1..gh4: [5][8]
    const int* rcap;                      // [R][3] capture index of the stencil nodes
    int cap_nn;                           // capture index of the surface row
    const double *wv, *wd;                // [R][3]
};

__device__ __forceinline__ cd calcoef1(double omega, double q) {
    if (q <= 0.0) return mk(1.0);
    double aa = (omega == 0.0) ? 1.0 : 1.0 + log(omega / (2.0 * kPi)) / (kPi * q);
    double bb = 1.0 / (2.0 * q);
    return mk(aa, bb) * mk(aa, bb);
}

// a0/a2 of one frequency: layout [(nn+1)][2] (k = 0 off-diagonal, 1 diagonal)
__global__ void k_sh_omega(ShDev d, const int* __restrict__ freqs, cd* __restrict__ a0,
                           cd* __restrict__ a2) {
    int w = blockIdx.y;
    int jj = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (jj > d.nn) return;
    double omega = 2.0 * kPi * (double)freqs[w] / d.tlen;
    cd comega2 = mk(omega, -d.omegai) * mk(omega, -d.omegai);
    cd s0d = mk(0.0), s0o = mk(0.0), s2d = mk(0.0), s2o = mk(0.0);
    for (int z = 0; z < d.nzone; ++z) {
        int nl = d.nlayer[z], i = jj - d.isp[z] + 1;
        if (i < 1 || i > nl + 1) continue;
        cd coef = calcoef1(omega, d.qmu[z]);
        const int o = d.jsp[z] - 2;  // element entry n (1-based) -> array index o + n
        auto e0 = [&](int n) {
            double h = d.h1[o + n] - d.h2[o + n] + d.h3[o + n] - 2.0 * d.h4[o + n];
            return comega2 * mk(d.t[o + n]) - coef * mk(h);
        };
        auto e2 = [&](int n) { return -coef * mk(d.h4[o + n]); };
        int nsize = nl + 1;
        if (i == 1) {
            s0d = s0d + e0(1);
            s2d = s2d + e2(1);
        } else if (i == nsize) {
            s0d = s0d + e0(4 * nl);
            s2d = s2d + e2(4 * nl);
        } else {
            s0d = s0d + e0(4 * i - 4) + e0(4 * i - 3);
            s2d = s2d + e2(4 * i - 4) + e2(4 * i - 3);
        }
        if (i >= 2) {
            s0o = s0o + e0(4 * i - 6);
            s2o = s2o + e2(4 * i - 6);
        }
    }
    size_t base = ((size_t)w * (d.nn + 1) + jj) * 2;
    a0[base + 0] = s0o;
    a0[base + 1] = s0d;
    a2[base + 0] = s2o;
    a2[base + 1] = s2d;
}

// One thread per (omega, l) system.  Basis right-hand sides: e_s, e_{s+1}
// (the two rows the source excitation g2 occupies, calg2) and e_nn (the
// surface row of the back-propagated source).
__global__ void __launch_bounds__(128) k_sh_solve(ShDev d, const cd* __restrict__ a0,
                                                  const cd* __restrict__ a2, WorkList wl, int nsys,
                                                  int jmin, const int* __restrict__ capmap,
                                                  cd* __restrict__ Lst, cd* __restrict__ Zst,
                                                  cd* __restrict__ Xcap) {
    int sys = blockIdx.x * blockDim.x + threadIdx.x;
    if (sys >= nsys) return;
    int w, l;
    wl_map(wl, sys, w, l);
    const int nn = d.nn, s = d.srow;
    const cd* A0 = a0 + (size_t)w * (nn + 1) * 2;
    const cd* A2 = a2 + (size_t)w * (nn + 1) * 2;
    const double xl2 = (double)l * (double)(l + 1);
    // row 1
    cd dg = A0[3] + mk(xl2) * A2[3];
    cd dr = mk(1.0) / dg;
    cd z0 = mk(s == 1 ? 1.0 : 0.0), z1 = mk(0.0);
    if (s == 1) {
        Zst[((size_t)0 * 2 + 0) * nsys + sys] = z0 * dr;
        Zst[((size_t)0 * 2 + 1) * nsys + sys] = z1 * dr;
    }
    for (int j = 2; j <= nn; ++j) {
        cd off = A0[2 * j] + mk(xl2) * A2[2 * j];
        cd dgj = A0[2 * j + 1] + mk(xl2) * A2[2 * j + 1];
        cd L = off * dr;               // a(1,j) <- a(1,j) dr(j-1)
        cd sv = dgj - off * L;         // s = a(2,j) - xx a(1,j)
        dr = mk(1.0) / sv;
        if (j > jmin) Lst[(size_t)j * nsys + sys] = L;
        z0 = mk(j == s ? 1.0 : 0.0) - L * z0;      // z(j) = b(j) - a(1,j) z(j-1)
        z1 = mk(j == s + 1 ? 1.0 : 0.0) - L * z1;
        if (j >= s) {  // rows below the source have zero scaled forward vectors
            Zst[((size_t)(j - s) * 2 + 0) * nsys + sys] = z0 * dr;
            Zst[((size_t)(j - s) * 2 + 1) * nsys + sys] = z1 * dr;
        }
    }
    // upward substitution b(j) = z(j) - a(1,j+1) b(j+1), from the surface down
    cd x0 = z0 * dr, x1 = z1 * dr, xb = dr;  // e_nn: z(nn) = 1
    int c = capmap[nn];
    if (c >= 0) {
        Xcap[((size_t)c * 3 + 0) * nsys + sys] = x0;
        Xcap[((size_t)c * 3 + 1) * nsys + sys] = x1;
        Xcap[((size_t)c * 3 + 2) * nsys + sys] = xb;
    }
    for (int j = nn - 1; j >= jmin; --j) {
        cd L = Lst[(size_t)(j + 1) * nsys + sys];
        cd zh0 = mk(0.0), zh1 = mk(0.0);
        if (j >= s) {
            zh0 = Zst[((size_t)(j - s) * 2 + 0) * nsys + sys];
            zh1 = Zst[((size_t)(j - s) * 2 + 1) * nsys + sys];
        }
        x0 = zh0 - L * x0;
        x1 = zh1 - L * x1;
        xb = mk(0.0) - L * xb;
        c = capmap[j];
        if (c >= 0) {
            Xcap[((size_t)c * 3 + 0) * nsys + sys] = x0;
            Xcap[((size_t)c * 3 + 1) * nsys + sys] = x1;
            Xcap[((size_t)c * 3 + 2) * nsys + sys] = xb;
        }
    }
}

// calga for one element set (nl elements, 4 entries each), calmat.f90:329-353
__device__ void calga(int nl, cd comega2, double xl2m2, const double* t, const double* h1,
                      const double* h2, const double* h3, const double* h4, cd coef, cd* a) {
    for (int i = 0; i < 4 * nl; ++i) {
        double h = h1[i] - h2[i] + h3[i] + xl2m2 * h4[i];
        a[i] = comega2 * mk(t[i]) - coef * mk(h);
    }
}

// rvec of calbveczero for |m| = 1 (src/SGTsh/trial.f90:120-157)
__device__ cd sh_rvec(int l, int icomp, int m) {
    double xl2 = (double)l * (double)(l + 1);
    double fact = (double)l * (double)(l + 1);
    double coef = sqrt((double)(2 * l + 1) / (4.0 * kPi) / fact);
    cd v;
    if (icomp == 2) v = mk(0.0, 1.0) * xl2 * coef / 2.0;
    else v = -(mk(1.0, 0.0) * xl2 * coef / 2.0);
    if (m < 0) v = -conj(v);
    return v;
}

// Per (omega, l): source coefficients of every slot, receiver fields and
// the cutoff probe.  blockIdx.y selects a group of 32 receivers (group 0
// also writes the surface pseudo-receiver and the probe).
__global__ void __launch_bounds__(128) k_sh_fields(ShDev d, const int* __restrict__ freqs, WorkList wl,
                                                   int nsys, const cd* __restrict__ Xcap,
                                                   double* __restrict__ A1, double* __restrict__ A2f,
                                                   int Lcap, double* __restrict__ amps) {
    int sys = blockIdx.x * blockDim.x + threadIdx.x;
    if (sys >= nsys) return;
    int w, l;
    wl_map(wl, sys, w, l);
    const int R = d.R;
    const int rows1 = SH_NSLOT1 * (R + 1) * SH_NF * 2, rows2 = SH_NSLOT2 * (R + 1) * SH_NF * 2;
    double* A1w = A1 + (size_t)w * rows1 * Lcap + l;
    double* A2w = A2f + (size_t)w * rows2 * Lcap + l;
    int rlo = blockIdx.y * 32, rhi = min(rlo + 32, R);
    bool g0 = blockIdx.y == 0;
    auto X = [&](int cap, int k) { return Xcap[((size_t)cap * 3 + k) * nsys + sys]; };
    auto put = [&](double* Aw, int q, int r, int f, cd v) {
        // rows ordered (slot, field, re/im, receiver): receivers contiguous
        const size_t row = ((size_t)(q * SH_NF + f) * 2) * (R + 1) + r;
        Aw[row * Lcap] = v.re;
        Aw[(row + (R + 1)) * Lcap] = v.im;
    };
    if (l == 0) {  // the SH m loop is empty at l = 0
        for (int r = rlo; r < rhi; ++r)
            for (int f = 0; f < SH_NF; ++f) {
                for (int q = 0; q < SH_NSLOT1; ++q) put(A1w, q, r, f, mk(0.0));
                for (int q = 0; q < SH_NSLOT2; ++q) put(A2w, q, r, f, mk(0.0));
            }
        if (g0) {
            for (int f = 0; f < SH_NF; ++f) {
                for (int q = 0; q < SH_NSLOT1; ++q) put(A1w, q, R, f, mk(0.0));
                for (int q = 0; q < SH_NSLOT2; ++q) put(A2w, q, R, f, mk(0.0));
            }
            for (int k = 0; k < 4; ++k) amps[((size_t)w * Lcap + l) * 4 + k] = 0.0;
        }
        return;
    }
    const double omega = 2.0 * kPi * (double)freqs[w] / d.tlen;
    const cd comega2 = mk(omega, -d.omegai) * mk(omega, -d.omegai);
    const cd coef = calcoef1(omega, d.qmu[d.spn - 1]);
    const double lsq = sqrt((double)l * (double)(l + 1));
    const double xl2 = (double)l * (double)(l + 1);
    // source element matrices (calga) and the 3x3 band of the split element
    cd aa[4], ga[8];
    calga(1, comega2, xl2 - 2.0, d.t + d.ins - 1, d.h1 + d.ins - 1, d.h2 + d.ins - 1,
          d.h3 + d.ins - 1, d.h4 + d.ins - 1, coef, aa);
    calga(2, comega2, xl2 - 2.0, d.g, d.g + 8, d.g + 16, d.g + 24, d.g + 32, coef, ga);
    // overlap(2, ga, ga2): ga2(1,j) off-diagonal, ga2(2,j) diagonal, j = 1..3
    cd o2 = ga[1], o3 = ga[5];
    cd d1 = ga[0], d2 = mk(0.0) + ga[3] + ga[4], d3 = ga[7];
    // dclisb0 on the 3x3 band (nud = 1)
    cd dr1 = mk(1.0) / d1;
    cd L2 = o2 * dr1;
    cd dr2 = mk(1.0) / (d2 - o2 * L2);
    cd L3 = o3 * dr2;
    cd dr3 = mk(1.0) / (d3 - o3 * L3);
    const double b1a = sqrt((double)(2 * l + 1) / (16.0 * kPi));
    const double b1b = (l >= 2) ? sqrt((double)(2 * l + 1) * (double)(l - 1) * (double)(l + 2) / (64.0 * kPi)) : 0.0;
    // slot coefficients (c_s, c_{s+1}) of the forward slots: g2(itmp+1),
    // g2(itmp+2) of calg2 for a unit right-hand side weight
    cd cs1[4][2], cs2[6][2];
    for (int ma = 1; ma <= 2; ++ma) {
        for (int sg = 0; sg < 2; ++sg) {
            int m = sg == 0 ? -ma : ma;
            double sgn = (m >= 0) ? 1.0 : -1.0;
            int nq = (ma == 1) ? 2 : 3;
            for (int k = 0; k < nq; ++k) {
                int imt = (ma == 1) ? (k == 0 ? 4 : 5) : (k == 0 ? 2 : (k == 1 ? 3 : 6));
                double mt12 = imt == 4, mt13 = imt == 5, mt22 = imt == 2, mt33 = imt == 3, mt23 = imt == 6;
                cd c1 = mk(0.0), c2 = mk(0.0), c3 = mk(0.0), dd = mk(0.0);
                if (ma == 1 && l >= 1) {
                    dd = mk(b1a) * mk(sgn * mt13, mt12) / (mk(d.r0 * d.r0 * d.mu0) * coef);
                    c2 = -dd * (ga[4] + ga[5]);
                    c3 = -dd * (ga[6] + ga[7]);
                } else if (ma == 2 && l >= 2) {
                    c2 = mk(b1b / d.r0) * mk(2.0 * mt23, sgn * (mt22 - mt33));
                }
                // dcsbsub0 on the factored 3x3 band
                cd y1 = c1, y2 = c2 - L2 * y1, y3 = c3 - L3 * y2;
                y1 = y1 * dr1; y2 = y2 * dr2; y3 = y3 * dr3;
                cd x3 = y3, x2 = y2 - L3 * x3, x1 = y1 - L2 * x2;
                x3 = x3 + dd;
                cd gs = aa[0] * x1 + aa[1] * x3;
                cd gs1 = aa[2] * x1 + aa[3] * x3;
                if (ma == 1) { cs1[sg * 2 + k][0] = gs; cs1[sg * 2 + k][1] = gs1; }
                else { cs2[sg * 3 + k][0] = gs; cs2[sg * 3 + k][1] = gs1; }
            }
        }
    }
    // probe for the cutoff: |g0(nn)| of imt = 3 for m = -2, -1, 1, 2
    if (g0) {
        double* ap = amps + ((size_t)w * Lcap + l) * 4;
        cd xn0 = X(d.cap_nn, 0), xn1 = X(d.cap_nn, 1);
        for (int mi = 0; mi < 4; ++mi) {
            int m = (mi == 0) ? -2 : (mi == 1 ? -1 : (mi == 2 ? 1 : 2));
            double a = 0.0;
            if (abs(m) == 2 && l >= 2) {
                int sg = m < 0 ? 0 : 1;
                cd gn = cs2[sg * 3 + 1][0] * xn0 + cs2[sg * 3 + 1][1] * xn1;
                a = cabs_(gn);
            }
            ap[mi] = a;
        }
    }
    // receiver and surface fields
    for (int pass = 0; pass < 2; ++pass) {
        int r_lo = pass == 0 ? rlo : R, r_hi = pass == 0 ? rhi : (g0 ? R + 1 : R);
        for (int r = r_lo; r < r_hi; ++r) {
            bool surf = r == R;
            // basis values interpolated at the receiver (value, derivative)
            cd bv[3], bd[3];
            if (surf) {
                for (int k = 0; k < 3; ++k) { bv[k] = X(d.cap_nn, k); bd[k] = mk(0.0); }
            } else {
                for (int k = 0; k < 3; ++k) { bv[k] = mk(0.0); bd[k] = mk(0.0); }
                for (int i = 0; i < 3; ++i) {
                    int c = d.rcap[3 * r + i];
                    double wvi = d.wv[3 * r + i], wdi = d.wd[3 * r + i];
                    for (int k = 0; k < 3; ++k) {
                        cd xv = X(c, k);
                        bv[k] = bv[k] + wvi * xv;
                        bd[k] = bd[k] + wdi * xv;
                    }
                }
            }
            // |m| = 1
            for (int sg = 0; sg < 2; ++sg) {
                int m = sg == 0 ? -1 : 1;
                for (int k = 0; k < 4; ++k) {
                    int q = sg * 4 + k;
                    cd W, Wd;
                    if (k < 2) {
                        cd c0 = cs1[sg * 2 + k][0], c1 = cs1[sg * 2 + k][1];
                        W = c0 * bv[0] + c1 * bv[1];
                        Wd = c0 * bd[0] + c1 * bd[1];
                    } else {
                        cd cb = -conj(sh_rvec(l, k == 2 ? 2 : 3, m)) / mk(lsq);
                        W = cb * bv[2];
                        Wd = cb * bd[2];
                        if (surf) { W = mk(0.0); }  // SYNN takes forward sources only
                    }
                    cd Wh = W / lsq, Wdh = Wd / lsq;
                    double* Aw = A1w;
                    put(Aw, q, r, 0, Wh);
                    put(Aw, q, r, 1, surf ? mk(0.0) : Wdh);
                    put(Aw, q, r, 2, surf ? mk(0.0) : xl2 * Wh);
                }
            }
            // |m| = 2
            for (int sg = 0; sg < 2; ++sg) {
                for (int k = 0; k < 3; ++k) {
                    int q = sg * 3 + k;
                    cd W = mk(0.0), Wd = mk(0.0);
                    if (l >= 2) {
                        cd c0 = cs2[q][0], c1 = cs2[q][1];
                        W = c0 * bv[0] + c1 * bv[1];
                        Wd = c0 * bd[0] + c1 * bd[1];
                    }
                    cd Wh = W / lsq, Wdh = Wd / lsq;
                    put(A2w, q, r, 0, Wh);
                    put(A2w, q, r, 1, surf ? mk(0.0) : Wdh);
                    put(A2w, q, r, 2, surf ? mk(0.0) : xl2 * Wh);
                }
            }
        }
    }
}

// cutoff scan: one thread per frequency
__global__ void k_sh_scan(int nf, WorkList wl, int Lcap, int maxlmax, double ratl, double tlen,
                          double vtop, double rtop, const int* __restrict__ freqs,
                          const double* __restrict__ amps, CutState* __restrict__ cut,
                          int* __restrict__ status) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nf) return;
    CutState c = cut[w];
    if (c.done) return;
    double omega = 2.0 * kPi * (double)freqs[w] / tlen;
    int lsuf = (int)(omega * rtop / vtop - 0.5) + 1;  // callsuf
    const int l0 = wl.lb[w], l1 = l0 + wl.off[w + 1] - wl.off[w];
    for (int l = l0; l < l1; ++l) {
        if (c.ismall > 20) {
            if (c.llog > l) c.llog = l;
            c.done = 1;
            c.norders = l;
            break;
        }
        if (l == 0) continue;
        const double* ap = amps + ((size_t)w * Lcap + l) * 4;
        for (int mi = 0; mi < 4; ++mi) {
            int m = (mi == 0) ? -2 : (mi == 1 ? -1 : (mi == 2 ? 1 : 2));
            if (abs(m) > l) continue;
            double amp = ap[mi], ampratio = 0.0;
            if (!isfinite(amp)) {  // the solves broke down: stop and report (llog -1)
                flag_nonfinite(status, true);
                c.done = 1;
                c.norders = l1;
                c.llog = -1;
                cut[w] = c;
                return;
            }
            if (amp > c.maxamp) c.maxamp = amp;
            if (amp != 0.0 && c.maxamp != 0.0) ampratio = amp / c.maxamp;
            if (ampratio < ratl && l > lsuf) c.ismall++;
            else c.ismall = 0;
        }
        if (l == maxlmax) { c.done = 1; c.norders = maxlmax + 1; }
    }
    cut[w] = c;
}

// Epilogue of one frequency: thread per (itheta, receiver); receiver R is
// the surface (SYNN).
// TC: double (FP64 contraction) or float (tensor-core contraction)
template <class TC>
__global__ void k_sh_epi(ShDev d, int w, int Th, const double* __restrict__ thx,
                         const double* __restrict__ ths, const int* __restrict__ pole,
                         const double* __restrict__ rr, const TC* __restrict__ C1,
                         const TC* __restrict__ C2, double* __restrict__ tsgt,
                         double* __restrict__ rsgt, double* __restrict__ synn, int* __restrict__ status) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int R = d.R;
    if (idx >= Th * (R + 1)) return;
    int it = idx / (R + 1), r = idx % (R + 1);
    bool surf = r == R;
    const int M1 = SH_NSLOT1 * (R + 1) * SH_NF * 2, M2 = SH_NSLOT2 * (R + 1) * SH_NF * 2;
    cd T[10], Rg[5], S[5];
    for (auto& v : T) v = mk(0.0);
    for (auto& v : Rg) v = mk(0.0);
    for (auto& v : S) v = mk(0.0);
    if (!pole[it]) {  // at the poles every SH vector harmonic is zero
        const double x = thx[it], s = ths[it];
        const double tc = x / s;  // thetacot = cos/sin
        const double ri = surf ? 1.0 : rr[r];
        for (int ma = 1; ma <= 2; ++ma) {
            const TC* C = ma == 1 ? C1 : C2;
            const int M = ma == 1 ? M1 : M2;
            const int nslot = ma == 1 ? SH_NSLOT1 : SH_NSLOT2;
            for (int q = 0; q < nslot; ++q) {
                int per = ma == 1 ? 4 : 3;
                int sg = q / per, k = q % per;
                int m = sg == 0 ? -ma : ma;
                double sigma = (m < 0 && (ma & 1)) ? -1.0 : 1.0;
                auto G = [&](int f, int b) {
                    size_t row = ((size_t)(q * SH_NF + f) * 2) * (R + 1) + r;
                    size_t col = (size_t)b * Th + it;
                    return mk((double)C[row + (size_t)M * col], (double)C[row + (R + 1) + (size_t)M * col]);
                };
                cd P = G(0, 0), D = G(0, 1);
                double mm = (double)m, m2 = mm * mm;
                // u = W bvec / lsq with bvec(2,m) = i m/sin Pbar, bvec(3,m) = -Dbar
                cd u2 = sigma * cmul_i(mm / s, P);
                cd u3 = sigma * (-D);
                if (surf) {
                    if ((ma == 1 && k >= 2)) continue;  // back slots: no SYNN
                    int imt = ma == 1 ? (k == 0 ? 4 : 5) : (k == 0 ? 2 : (k == 1 ? 3 : 6));
                    if (imt == 2) { S[0] = S[0] - 5.e-1 * u2; S[1] = S[1] - 5.e-1 * u2; }
                    if (imt == 3) { S[0] = S[0] - 5.e-1 * u2; S[1] = S[1] + 5.e-1 * u2; }
                    if (imt == 4) { S[3] = S[3] + u2; }
                    if (imt == 5) { S[4] = S[4] + u3; }
                    if (imt == 6) { S[2] = S[2] - u3; }
                    continue;
                }
                cd Pd = G(1, 0), Dd = G(1, 1), LP = G(2, 0);
                cd udr2 = sigma * cmul_i(mm / s, Pd);
                cd udr3 = sigma * (-Dd);
                cd udt2 = sigma * cmul_i(mm, D / s - (x / (1 - x * x)) * P);
                cd udt3 = sigma * ((x / s) * D - (m2 / (1 - x * x)) * P + LP);
                cd udp2 = sigma * ((-m2 / s) * P);
                cd udp3 = sigma * cmul_i(-mm, D);
                // locallyCartesianDerivatives (u(1) = 0 for SH)
                cd d12 = (mk(0.0) - u2) / ri;
                cd d13 = (mk(0.0) - u3) / ri;
                cd d21 = udr2;
                cd d22 = udt2 / ri;
                cd d23 = (udp2 / s - u3 * tc) / ri;
                cd d31 = udr3;
                cd d32 = udt3 / ri;
                cd d33 = (udp3 / s + u2 * tc) / ri;
                if (ma == 1 && k >= 2) {
                    int icomp = k == 2 ? 2 : 3;
                    if (icomp == 2) {
                        Rg[0] = Rg[0] - 5.e-1 * d22 - 5.e-1 * d33;
                        Rg[1] = Rg[1] - 5.e-1 * d22 + 5.e-1 * d33;
                        Rg[3] = Rg[3] - 5.e-1 * d12 - 5.e-1 * d21;
                    } else {
                        Rg[2] = Rg[2] - 5.e-1 * d23 - 5.e-1 * d32;
                        Rg[4] = Rg[4] + 5.e-1 * d13 + 5.e-1 * d31;
                    }
                    continue;
                }
                int imt = ma == 1 ? (k == 0 ? 4 : 5) : (k == 0 ? 2 : (k == 1 ? 3 : 6));
                if (imt == 2) {
                    T[1] = T[1] - 2.5e-1 * d22 - 2.5e-1 * d33;
                    T[6] = T[6] - 1.25e-1 * d12 - 1.25e-1 * d21;
                    T[7] = T[7] + 1.25e-1 * d12 + 1.25e-1 * d21;
                    T[8] = T[8] + 1.25e-1 * d22 - 1.25e-1 * d33;
                    T[9] = T[9] + 1.25e-1 * d22 - 1.25e-1 * d33;
                } else if (imt == 3) {
                    T[1] = T[1] + 2.5e-1 * d22 + 2.5e-1 * d33;
                    T[6] = T[6] - 1.25e-1 * d12 - 1.25e-1 * d21;
                    T[7] = T[7] + 1.25e-1 * d12 + 1.25e-1 * d21;
                    T[8] = T[8] - 1.25e-1 * d22 + 1.25e-1 * d33;
                    T[9] = T[9] - 1.25e-1 * d22 + 1.25e-1 * d33;
                } else if (imt == 4) {
                    T[0] = T[0] - 5.e-1 * d22 - 5.e-1 * d33;
                    T[2] = T[2] - 2.5e-1 * d12 - 2.5e-1 * d21;
                    T[3] = T[3] + 2.5e-1 * d12 + 2.5e-1 * d21;
                    T[4] = T[4] + 2.5e-1 * d22 - 2.5e-1 * d33;
                    T[5] = T[5] - 2.5e-1 * d22 + 2.5e-1 * d33;
                } else if (imt == 5) {
                    T[2] = T[2] + 2.5e-1 * d13 + 2.5e-1 * d31;
                    T[3] = T[3] + 2.5e-1 * d13 + 2.5e-1 * d31;
                    T[4] = T[4] - 2.5e-1 * d23 - 2.5e-1 * d32;
                    T[5] = T[5] - 2.5e-1 * d23 - 2.5e-1 * d32;
                } else if (imt == 6) {
                    T[6] = T[6] + 2.5e-1 * d13 + 2.5e-1 * d31;
                    T[7] = T[7] + 2.5e-1 * d13 + 2.5e-1 * d31;
                    T[8] = T[8] - 2.5e-1 * d23 - 2.5e-1 * d32;
                    T[9] = T[9] + 2.5e-1 * d23 + 2.5e-1 * d32;
                }
            }
        }
    }
    {
        bool bad = false;
        for (int c = 0; c < 5; ++c) bad |= surf && nonfinite2(S[c].re, S[c].im);
        for (int c = 0; c < 10; ++c) bad |= !surf && nonfinite2(T[c].re, T[c].im);
        for (int c = 0; c < 5; ++c) bad |= !surf && rsgt && nonfinite2(Rg[c].re, Rg[c].im);
        flag_nonfinite(status, bad);
    }
    if (surf) {
        if (synn)
            for (int c = 0; c < 5; ++c) {
                size_t o = ((size_t)w * Th + it) * 5 + c;
                synn[2 * o] = S[c].re;
                synn[2 * o + 1] = S[c].im;
            }
        return;
    }
    size_t pt = ((size_t)w * Th + it) * R + r;
    for (int c = 0; c < 10; ++c) {
        tsgt[2 * (pt * 10 + c)] = T[c].re;
        tsgt[2 * (pt * 10 + c) + 1] = T[c].im;
    }
    if (rsgt)
        for (int c = 0; c < 5; ++c) {
            rsgt[2 * (pt * 5 + c)] = Rg[c].re;
            rsgt[2 * (pt * 5 + c) + 1] = Rg[c].im;
        }
}

class ShEngine : public Engine {
  public:
    ShDev d{};
    std::vector<int> h_isp, h_nlayer;
    DBuf<int> nlayer, isp, jsp, capmap, rcap;
    DBuf<double> qmu, t, h1, h2, h3, h4, g, r, rrsta;
    DBuf<cd> a0, a2, Lst, Zst, Xcap;
    int jmin = 1, ncap = 0;
    double vtop = 0, rtop = 0;

    ShEngine(const dsm_sh_setup_t* s, const dsm_options_t* o) {
        mode = 0;
        opt = *o;
        init_common(opt.device);
        m_lo = 1;
        R = s->r_n;
        Th = s->theta_n;
        num_t = DSM_SH_NUM_TSGT; num_r = DSM_SH_NUM_RSGT; num_s = DSM_SH_NUM_SYNN;
        tlen = s->tlen; omegai = s->omegai; ratl = s->ratl; maxlmax = s->maxlmax;
        imin = s->imin; imax = s->imax;
        rsgt_sw = 1;  // the SH back-propagation runs unconditionally (SGTsh-MPI.f90:517)
        synn_sw = s->synn_switch == 1;
        if (R <= 0 || Th <= 0 || s->nzone <= 0 || s->nnlayer <= 0) throw Error(DSM_ERR_INVALID, "empty SH set-up");
        const int nn = s->nnlayer + 1;
        d.nn = nn; d.nzone = s->nzone; d.R = R;
        d.ins = s->ins; d.spn = s->spn; d.spo = s->spo; d.r0 = s->r0; d.mu0 = s->mu0;
        d.tlen = tlen; d.omegai = omegai;
        d.srow = s->isp[s->spn - 1] + (int)std::trunc(s->spo);
        if (d.srow < 1 || d.srow + 1 > nn) throw Error(DSM_ERR_INVALID, "source row outside the system");
        nlayer.upload(s->nlayer, s->nzone, st); isp.upload(s->isp, s->nzone, st); jsp.upload(s->jsp, s->nzone, st);
        qmu.upload(s->qmu, s->nzone, st);
        size_t ne = 4 * (size_t)s->nnlayer;
        t.upload(s->t, ne, st); h1.upload(s->h1, ne, st); h2.upload(s->h2, ne, st);
        h3.upload(s->h3, ne, st); h4.upload(s->h4, ne, st);
        std::vector<double> gg(40);
        for (int k = 0; k < 8; ++k) {
            gg[k] = s->gt[k]; gg[8 + k] = s->gh1[k]; gg[16 + k] = s->gh2[k];
            gg[24 + k] = s->gh3[k]; gg[32 + k] = s->gh4[k];
        }
        g.upload(gg, st);
        r.upload(s->r, R, st);
        rrsta.upload(s->rrsta, 3 * (size_t)R, st);
        // callsuf uses the top zone's summed Vsv coefficients and vrmax
        vtop = 0.0;
        for (int i = 0; i < 4; ++i) vtop = vtop + s->vsv[4 * (s->nzone - 1) + i] * 1.0;
        rtop = s->vrmax[s->nzone - 1];
        vtop_ = vtop;
        rtop_ = rtop;
        set_summaries(0, s->nzone, s->vrmin, s->vrmax, s->vsv, s->qmu, s->r0, s->vrmax[s->nzone - 1]);
        // capture rows: receiver stencils and the surface
        std::vector<int> cm(nn + 1, -1), rc(3 * (size_t)R);
        jmin = nn;
        for (int ir = 0; ir < R; ++ir)
            for (int k = 0; k < 3; ++k) {
                int j = s->iista[3 * ir + k];
                if (j < 1 || j > nn) throw Error(DSM_ERR_INVALID, "receiver node outside the system");
                if (cm[j] < 0) cm[j] = ncap++;
                rc[3 * ir + k] = cm[j];
                jmin = std::min(jmin, j);
            }
        if (cm[nn] < 0) cm[nn] = ncap++;
        d.cap_nn = cm[nn];
        d.ncap = ncap;
        capmap.upload(cm, st);
        rcap.upload(rc, st);
        // theta tables
        th.th_n = Th;
        th.h_x.resize(Th); th.h_s.resize(Th); th.h_pole.resize(Th);
        for (int i = 0; i < Th; ++i) {
            double tr = s->theta[i] / 180.0 * kPi;
            th.h_x[i] = std::cos(tr);
            th.h_s[i] = std::sin(tr);
            th.h_pole[i] = (tr == 0.0) ? 1 : (tr == kPi ? 2 : 0);
        }
        th.x.upload(th.h_x, st); th.s.upload(th.h_s, st); th.pole.upload(th.h_pole, st);
        build_weights(r.p, rrsta.p);
        d.nlayer = nlayer.p; d.isp = isp.p; d.jsp = jsp.p; d.qmu = qmu.p;
        d.t = t.p; d.h1 = h1.p; d.h2 = h2.p; d.h3 = h3.p; d.h4 = h4.p; d.g = g.p;
        d.rcap = rcap.p; d.wv = wv.p; d.wd = wd.p;
        // batch geometry
        F = opt.freq_batch > 0 ? opt.freq_batch : 16;
        Lc = opt.l_chunk > 0 ? ((opt.l_chunk + 31) / 32) * 32 : 256;
        Lcap = std::min(maxlmax + 1 + Lc, 2048);
        amp_k = 4;
        rows_m[1] = SH_NSLOT1 * (R + 1) * SH_NF * 2;
        rows_m[2] = SH_NSLOT2 * (R + 1) * SH_NF * 2;
        alloc_batch();
        build_basis(std::min(maxlmax + 1, 2048));
        DSM_CUDA(cudaStreamSynchronize(st));
    }

    void alloc_batch() {
        size_t nn = d.nn;
        size_t per = (nn + 1) * 16 + (nn - d.srow + 2) * 2 * 16 + (size_t)ncap * 3 * 16;
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        nsys_max = (int)std::max<size_t>(1024, std::min<size_t>(65536, (fr / 3) / per));
        // no more than a round of a batch can launch (F ranges of at most
        // max(4096, the first range of the top frequency)): contexts that
        // share a device leave each other room
        nsys_max = std::min(nsys_max, std::max(1024, F * std::max(4096, first_span(imax))));
        // DSM_MAX_SYSTEMS caps the systems per solve launch (and so the
        // factor scratch) below that, e.g. for small profiling captures
        if (const char* e = std::getenv("DSM_MAX_SYSTEMS")) nsys_max = std::max(1024, std::min(nsys_max, std::atoi(e)));
        size_t nsys = nsys_max;
        a0.reserve((size_t)F * (nn + 1) * 2);
        a2.reserve((size_t)F * (nn + 1) * 2);
        Lst.reserve((nn + 1) * nsys);
        Zst.reserve((nn - d.srow + 2) * 2 * nsys);
        Xcap.reserve((size_t)ncap * 3 * nsys);
        Afld[1].reserve((size_t)F * rows_m[1] * Lcap);
        Afld[2].reserve((size_t)F * rows_m[2] * Lcap);
        Cgemm.reserve(c_total());
        cut.reserve(F);
        amps.reserve((size_t)F * Lcap * 4);
        size_t pt, pr, ps;
        out_sizes(&pt, &pr, &ps);
        out_t.reserve(2 * pt * F);
        out_r.reserve(2 * pr * F);
        out_s.reserve(2 * ps * F);
    }

    size_t out_sizes(size_t* nt, size_t* nr, size_t* ns) const override {
        *nt = (size_t)num_t * R * Th;
        *nr = (size_t)num_r * R * Th;
        *ns = (size_t)num_s * Th;
        return *nt;
    }

    void omega_pieces(const int* fr, int nf) override {
        dim3 grid((d.nn + 127) / 128, nf);
        k_sh_omega<<<grid, 128, 0, st>>>(d, fr, a0.p, a2.p);
        DSM_LAUNCH(*this);
    }

    void solve_chunk(const int* fr, int nf, const WorkList& wl, int nsys) override {
        (void)nf;
        const double alg = 2.0 * 2.0 * d.nn * 16.0 + 14.0 * R * 2 * 2 * 16.0;
        int id = kid("sh_band_solve");
        kbegin(id);
        k_sh_solve<<<(nsys + 127) / 128, 128, 0, st>>>(d, a0.p, a2.p, wl, nsys, jmin, capmap.p,
                                                       Lst.p, Zst.p, Xcap.p);
        kend(id, alg * nsys, 0.0);
        DSM_LAUNCH(*this);
        dim3 grid((nsys + 127) / 128, (R + 31) / 32);
        k_sh_fields<<<grid, 128, 0, st>>>(d, fr, wl, nsys, Xcap.p, Afld[1].p, Afld[2].p, Lcap,
                                          amps.p);
        DSM_LAUNCH(*this);
        stats.solve_bytes += (double)nsys * d.nn * 2 * 16.0 * 2;
    }

    void scan_chunk(int nf, const WorkList& wl) override {
        k_sh_scan<<<(nf + 31) / 32, 32, 0, st>>>(nf, wl, Lcap, maxlmax, ratl, tlen, vtop, rtop,
                                                 d_freqs.p, amps.p, cut.p, dstatus());
        DSM_LAUNCH(*this);
    }

    void epilogue(const int* fr, int w, int nf, cudaStream_t s) override {
        (void)fr; (void)nf;
        int n = Th * (R + 1);
        int id = kid("sh_epilogue");
        kbegin(id, s);
        if (mixed()) {
            k_sh_epi<float><<<(n + 127) / 128, 128, 0, s>>>(d, w, Th, th.x.p, th.s.p, th.pole.p, r.p, c32(w, 1),
                                                         c32(w, 2), out_t.p, out_r.p,
                                                         synn_sw ? out_s.p : nullptr, dstatus());
        } else
            k_sh_epi<double><<<(n + 127) / 128, 128, 0, s>>>(d, w, Th, th.x.p, th.s.p, th.pole.p, r.p, c64(1),
                                                          c64(2), out_t.p, out_r.p,
                                                          synn_sw ? out_s.p : nullptr, dstatus());
        kend(id, 0.0, 0.0, s);
        DSM_LAUNCH(*this);
    }
};

}  // namespace

Engine* make_sh_engine(const dsm_sh_setup_t* s, const dsm_options_t* o) { return new ShEngine(s, o); }

}  // namespace dsm
