// P-SV engine: replaces src/SGTpsv/SGTpsv-MPI.f90:551-1095.
//
// Kernels (plain FP64 path; compiled without fused multiply-add):
//   k_psv_omega  per-omega, per-zone band blocks A0, A1, A2 (cala0, cala1,
//                cala2, calhml, overlapa, calb0, calb2, overlapb,
//                src/SGTpsv/calmat.f90:452-742; calcoef :409-447)
//   k_psv_solve  one thread per (omega, l >= 1): assembly a = A0 + l(l+1) A2
//                (rows 2,4) + sqrt(l(l+1)) A1 (rows 1,3), fluid rows 3,4,
//                fluid-solid boundary rows (cala, calbc, :747-809) streamed
//                into the unpivoted complex-symmetric band LDL^T of
//                half-width 3 (dcsymbdl0, src/SGTpsv/dcsymbdl.f90:2-88,
//                including its different update order in the last two
//                steps) and the substitutions (dcsbdlv0, :93-166;
//                mydcsbdlv3 is the same arithmetic) of six basis
//                right-hand sides: the four source rows jtmp..jtmp+3 and the
//                surface rows nn-1, nn.  The forward substitution of the
//                source bases runs inside the factorisation; the multipliers
//                stay in HBM for the upward sweep (k_psv_up, one lane per
//                system and six bases).
//   k_psv_l0     l = 0: the tridiagonal compaction (rea2 / rea2_back,
//                calmat.f90:1247-1389) and its solves (dcsymbdl0/dcsbdlv0
//                with half-width 1), one thread per frequency.
//   k_psv_fields source terms (calabnum, calya + rk3, calg, glu,
//                calmat.f90:815-1171), back-propagation sources
//                (caldveczero, trial.f90:326-364), receiver interpolation
//                (interpolate, others.f90:1170-1212); writes the per-order
//                receiver fields of every active slot and the probe of
//                calamp (imt = 1, m = 0).
//   k_psv_scan   the cutoff test (calamp, others.f90:1246-1264, the
//                ismall > 20 exit, SGTpsv-MPI.f90:606-609, 902-905).
// The epilogue (TSGT / RSGT / SYNN from the l-contractions) is psv_epi.cu.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "engine.cuh"
#include "psv_epi.cuh"

namespace dsm {
namespace {

using psvk::NS0;
using psvk::NS1;
using psvk::NS2;
using psvk::NFLD;  // U, U', V/lsq, V'/lsq, l(l+1) V/lsq
constexpr int NB = 6;                     // basis right-hand sides of a solve

struct PsvDev {
    int nzone, nn, itmp, R, Th, jsrc, spn;
    int n_sel, n_fel, n_hm;
    const int *iphase, *nlayer, *kkdr, *elem, *hmoff;
    const int* blkoff;      // [nzone] first block column of each zone
    int ncol_tot;
    const double *qmu, *qkappa;
    const double *sel, *fel, *hm;
    // assembly map per global column (1-based, [nn+1])
    const int *amz, *amc;   // [nn+1][2] zone (or -1) and zone-local column
    const int* bcrow;       // 0, 2 or 3
    const double* bcval;
    const int4* rowasm;     // [nn+1] per row: element offsets of the two zones
                            // (x4, -1 none), phase bits (1: zone 0 solid,
                            // 2: zone 1 solid), bcrow
    double tlen, omegai, rmax, r0, ecC0, ecF0, ecL0, ra0, ra1;
    const double* poly;     // [24]
    // receivers
    const int* rcap;        // [R][6] capture index of g0(ksta-1 .. ksta+4)
    const int* stop_row;    // [R] highest local row of each receiver's stencil (ksta+4)
    int cap_n1, cap_n;      // capture index of rows nn-1, nn
    int cap_p0, cap_p1;     // capture index of the probe rows ksta(r_n)-1, ksta(r_n)
    const double *wv, *wd;
    const int* fluid;       // [R]
    int Rs1, Rf;            // receiver rows of the solid class (incl. the surface), fluid receivers
    const int* rrow;        // [R+1] class index of each receiver row (psvk::fld_row)
    const double *lam, *qkp, *fr;  // [R]  lambda, Qkappa, float(r)
    // l = 0 compaction
    int nn0, itmp0, kc0;    // compact size, first row kept, compact row of jtmp
    const int* comp_src;    // global row -> compact row (or 0 when dropped), [nn+1]
    const int* jsta;        // [R]
};

__device__ __forceinline__ cd coefq(double omega, double q) {
    if (q <= 0.0) return mk(1.0);
    double aa = (omega == 0.0) ? 1.0 : 1.0 + log(omega / (2.0 * kPi)) / (kPi * q);
    double bb = 1.0 / (2.0 * q);
    return mk(aa, bb) * mk(aa, bb);
}

// ----------------------------------------------------------- omega pieces
struct ZoneCtx {
    const PsvDev* d;
    int z, off;
    cd c1, c2, comega2;
    __device__ double E(int k, int nnn) const {
        return d->sel[(size_t)k * d->n_sel + (off - 1) + (nnn - 1)];
    }
    // cala0 entry n (1-based, cwork)
    __device__ cd cw0(int n) const {
        if (n % 4 == 1) {
            int nnn = (n + 3) / 4;
            if (nnn % 4 == 3) return mk(0.0);
            cd hh0 = c2 * mk(4.0 * E(DSM_PSV_H1X, nnn)) + c1 * mk(16.0 / 3.0 * E(DSM_PSV_H2N, nnn)) +
                     c1 * mk(-4.0 * E(DSM_PSV_H2N, nnn)) +
                     c2 * mk(2.0 * (E(DSM_PSV_H3AY, nnn) + E(DSM_PSV_H5AY, nnn))) -
                     c1 * mk(4.0 / 3.0 * (E(DSM_PSV_H4AN, nnn) + E(DSM_PSV_H6AN, nnn))) +
                     c2 * mk(3.0 * E(DSM_PSV_H7Z, nnn) - 2.0 * E(DSM_PSV_H7Y, nnn)) +
                     c1 * mk(4.0 / 3.0 * E(DSM_PSV_H8N, nnn));
            return comega2 * mk(E(DSM_PSV_T, nnn)) - hh0;
        }
        if (n % 4 == 0) {
            int nnn = n / 4;
            if (nnn % 4 == 3) return mk(0.0);
            cd hh0 = c1 * mk(E(DSM_PSV_H2L, nnn)) + c1 * mk(-2.0 * E(DSM_PSV_H2N, nnn)) -
                     c1 * mk(E(DSM_PSV_H4AL, nnn) + E(DSM_PSV_H6AL, nnn)) + c1 * mk(E(DSM_PSV_H8L, nnn));
            return comega2 * mk(E(DSM_PSV_T, nnn)) - hh0;
        }
        return mk(0.0);
    }
    // cala1 entry n
    __device__ cd cw1(int n) const {
        if (n % 4 == 2) {
            int nnn = (n + 2) / 4;
            if (nnn % 4 == 3) return mk(0.0);
            cd hh1 = -c2 * mk(2.0 * E(DSM_PSV_H1X, nnn)) - c1 * mk(8.0 / 3.0 * E(DSM_PSV_H2N, nnn)) -
                     c1 * mk(E(DSM_PSV_H2L, nnn)) - c1 * mk(-2.0 * E(DSM_PSV_H2N, nnn)) -
                     c2 * mk(E(DSM_PSV_H3Y, nnn)) - c1 * mk(-2.0 / 3.0 * E(DSM_PSV_H4N, nnn)) +
                     c1 * mk(E(DSM_PSV_H6L, nnn));
            return -hh1;
        }
        if (n % 4 == 3) {
            int nnn = (n + 1) / 4;
            if (nnn % 4 != 2) return mk(0.0);
            cd hh1 = -c2 * mk(2.0 * E(DSM_PSV_H1X, nnn)) - c1 * mk(8.0 / 3.0 * E(DSM_PSV_H2N, nnn)) -
                     c1 * mk(-2.0 * E(DSM_PSV_H2N, nnn)) - c1 * mk(E(DSM_PSV_H2L, nnn)) +
                     c1 * mk(E(DSM_PSV_H4L, nnn)) - c2 * mk(E(DSM_PSV_H5Y, nnn)) +
                     c1 * mk(2.0 / 3.0 * E(DSM_PSV_H6N, nnn));
            return -hh1;
        }
        return mk(0.0);
    }
    // cala2 entry n
    __device__ cd cw2(int n) const {
        if (n % 4 == 1) {
            int nnn = (n + 3) / 4;
            if (nnn % 4 == 3) return mk(0.0);
            return -(c1 * mk(E(DSM_PSV_H2L, nnn)));
        }
        if (n % 4 == 0) {
            int nnn = n / 4;
            if (nnn % 4 == 3) return mk(0.0);
            return -(c2 * mk(E(DSM_PSV_H1X, nnn)) + c1 * mk(4.0 / 3.0 * E(DSM_PSV_H2N, nnn)));
        }
        return mk(0.0);
    }
};

// overlapa (calmat.f90:670-714): band entry (ii, i) of a zone block from the
// element array entries cw(n)
template <class F>
__device__ cd overlapa_entry(int nl, int ii, int i, F cw) {
    int nsize = 2 * (nl + 1), msize = 16 * nl;
    if (i == 1) return ii == 4 ? cw(1) : mk(0.0);
    if (i == 2) return ii == 3 ? cw(2) : (ii == 4 ? cw(4) : mk(0.0));
    if (i % 2 == 1) {  // 3 .. nsize-1
        int n1 = 16 * (i - 3) / 2 + 5;
        if (ii == 2) return cw(n1);
        if (ii == 3) return cw(n1 + 2);
        if (ii == 4) return (i != nsize - 1) ? cw(n1 + 8) + cw(n1 + 12) : cw(msize - 3);
        return mk(0.0);
    }
    int n1 = 16 * (i - 4) / 2 + 6;  // even, 4 .. nsize
    if (ii == 1) return cw(n1);
    if (ii == 2) return cw(n1 + 2);
    if (i != nsize) {
        if (ii == 3) return cw(n1 + 8) + cw(n1 + 12);
        return cw(n1 + 10) + cw(n1 + 14);
    }
    if (ii == 3) return cw(msize - 2);
    return cw(msize);
}

__global__ void k_psv_omega(PsvDev d, const int* __restrict__ freqs, cd* __restrict__ B0,
                            cd* __restrict__ B1, cd* __restrict__ B2) {
    int w = blockIdx.y;
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol_tot) return;
    int z = 0;
    while (z + 1 < d.nzone && d.blkoff[z + 1] <= col) ++z;
    int c = col - d.blkoff[z] + 1;
    double omega = 2.0 * kPi * (double)freqs[w] / d.tlen;
    cd comega2 = mk(omega, -d.omegai) * mk(omega, -d.omegai);
    cd c1 = coefq(omega, d.qmu[z]);
    cd c2 = coefq(omega, d.qkappa[z]);
    int nl = d.nlayer[z];
    size_t o = ((size_t)w * d.ncol_tot + col) * 4;
    if (d.iphase[z] == 1) {
        ZoneCtx zc{&d, z, d.elem[z], c1, c2, comega2};
        for (int ii = 1; ii <= 4; ++ii) {
            B0[o + ii - 1] = overlapa_entry(nl, ii, c, [&](int n) { return zc.cw0(n); });
            B2[o + ii - 1] = overlapa_entry(nl, ii, c, [&](int n) { return zc.cw2(n); });
            cd a1 = overlapa_entry(nl, ii, c, [&](int n) { return zc.cw1(n); });
            // calhml (calmat.f90:629-664)
            if (ii == 1 || ii == 3) {
                auto H = [&](int k, int lo, int m, int n) {
                    return d.hm[(size_t)k * 4 * d.n_hm + 4 * (size_t)(d.hmoff[z] - 1 + n - 1) + (m - lo)];
                };
                if (c % 2 == 0 && !(ii == 1 && c == 2)) {
                    int m = (-ii + 3) / 2, n = (ii + c - 3) / 2;
                    a1 = a1 - (-(c2 * mk(H(DSM_PSV_H3MY, -2, m, n))) +
                               c1 * mk(2.0 / 3.0 * H(DSM_PSV_H4M2N, -2, m, n)) +
                               c1 * mk(H(DSM_PSV_H6M2L, -2, m, n)));
                } else if (c % 2 == 1 && c >= 3 && c <= 2 * nl + 1 && !(ii == 1 && c == 3)) {
                    int m = (-ii + 5) / 2, n = (ii + c - 4) / 2;
                    a1 = a1 - (c1 * mk(H(DSM_PSV_H4M1L, -1, m, n)) -
                               c2 * mk(H(DSM_PSV_H5MY, -1, m, n)) +
                               c1 * mk(2.0 / 3.0 * H(DSM_PSV_H6M1N, -1, m, n)));
                }
            }
            B1[o + ii - 1] = a1;
        }
    } else {
        cd coef = mk(1.0) / c2;
        const double* p1 = d.fel + (d.elem[z] - 1);
        const double* p2 = d.fel + d.n_fel + (d.elem[z] - 1);
        const double* p3 = d.fel + 2 * (size_t)d.n_fel + (d.elem[z] - 1);
        auto b0 = [&](int n) {
            if (n % 4 == 3) return mk(0.0);
            return -(mk(p1[n - 1]) / comega2) + coef * mk(p3[n - 1]);
        };
        auto b2 = [&](int n) {
            if (n % 4 == 3) return mk(0.0);
            return -(mk(p2[n - 1]) / comega2);
        };
        // overlapb (calmat.f90:720-742)
        auto ovb = [&](int ii, auto f) -> cd {
            if (ii == 4) {
                if (c == 1) return f(1);
                if (c == nl + 1) return f(4 * nl);
                return f(4 * (c - 1)) + f(4 * (c - 1) + 1);
            }
            if (ii == 3 && c >= 2) return f(4 * (c - 2) + 2);
            return mk(0.0);
        };
        for (int ii = 1; ii <= 4; ++ii) {
            B0[o + ii - 1] = ovb(ii, b0);
            B2[o + ii - 1] = ovb(ii, b2);
            B1[o + ii - 1] = mk(0.0);
        }
    }
}

// band entries a(1..4, jj) of one global column for order l (cala + calbc)
__device__ __forceinline__ void assemble(const PsvDev& d, int jj, const cd* __restrict__ B0,
                                         const cd* __restrict__ B1, const cd* __restrict__ B2,
                                         double l2, double lsq, cd a[4]) {
    a[0] = a[1] = a[2] = a[3] = mk(0.0);
    const int4 ra = d.rowasm[jj];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int off = e == 0 ? ra.x : ra.y;
        if (off < 0) break;
        const size_t o = (size_t)off;
        if (ra.z & (1 << e)) {
            for (int ii = 2; ii <= 4; ii += 2) {
                cd x0 = B0[o + ii - 1], x2 = B2[o + ii - 1];
                a[ii - 1] = a[ii - 1] + mk(x0.re + l2 * x2.re, x0.im + l2 * x2.im);
            }
            for (int ii = 1; ii <= 3; ii += 2) {
                cd x1 = B1[o + ii - 1];
                a[ii - 1] = a[ii - 1] + mk(lsq * x1.re, lsq * x1.im);
            }
        } else {
            for (int ii = 3; ii <= 4; ++ii) {
                cd x0 = B0[o + ii - 1], x2 = B2[o + ii - 1];
                a[ii - 1] = a[ii - 1] + mk(x0.re + l2 * x2.re, x0.im + l2 * x2.im);
            }
        }
    }
    if (ra.w == 2) a[1] = mk(d.bcval[jj]);
    else if (ra.w == 3) a[2] = -mk(d.bcval[jj]);
}

// ---------------------------------------------------------------- solve
// Streaming LDL^T of the band system rows itmp..nn (local rows 1..n).
// Window W[p][q] holds the current values of A(k+p, k+q), q <= p <= 3.
// Per-omega band pieces by row: for row jj and band entry q, the l-free
// parts of a(q) = A[q] + l(l+1) B[q] + sqrt(l(l+1)) C[q] (cala), summed over
// the zones that share the row, with the calbc boundary value in A.  Rows
// of a single zone assemble to exactly what assemble() gives; rows where two
// zones meet add the two zones' sums before the l terms (a rounding-level
// difference).  Layout [omega][row][A0..3, B0..3, C0..3].
__global__ void k_psv_rows(PsvDev d, const cd* __restrict__ B0all, const cd* __restrict__ B1all,
                           const cd* __restrict__ B2all, cd* __restrict__ Prow) {
    const int w = blockIdx.y;
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj > d.nn) return;
    const size_t bo = (size_t)w * d.ncol_tot * 4;
    const cd *B0 = B0all + bo, *B1 = B1all + bo, *B2 = B2all + bo;
    cd A[4], B[4], C[4];
    for (int q = 0; q < 4; ++q) A[q] = B[q] = C[q] = mk(0.0);
    if (jj >= 1) {
        const int4 ra = d.rowasm[jj];
        for (int e = 0; e < 2; ++e) {
            const int off = e == 0 ? ra.x : ra.y;
            if (off < 0) break;
            const size_t o = (size_t)off;
            if (ra.z & (1 << e)) {
                for (int ii = 2; ii <= 4; ii += 2) {
                    A[ii - 1] = A[ii - 1] + B0[o + ii - 1];
                    B[ii - 1] = B[ii - 1] + B2[o + ii - 1];
                }
                for (int ii = 1; ii <= 3; ii += 2) C[ii - 1] = C[ii - 1] + B1[o + ii - 1];
            } else {
                for (int ii = 3; ii <= 4; ++ii) {
                    A[ii - 1] = A[ii - 1] + B0[o + ii - 1];
                    B[ii - 1] = B[ii - 1] + B2[o + ii - 1];
                }
            }
        }
        if (ra.w == 2) { A[1] = mk(d.bcval[jj]); B[1] = C[1] = mk(0.0); }
        else if (ra.w == 3) { A[2] = -mk(d.bcval[jj]); B[2] = C[2] = mk(0.0); }
    }
    cd* out = Prow + ((size_t)w * (d.nn + 1) + jj) * 12;
    for (int q = 0; q < 4; ++q) {
        out[q] = A[q];
        out[4 + q] = B[q];
        out[8 + q] = C[q];
    }
}

// raw pieces of one row (loaded ahead of use) and their assembly at order l
struct RowPieces {
    cd v[12];
};
__device__ __forceinline__ void load_row(const cd* __restrict__ P, RowPieces& r) {
#pragma unroll
    for (int i = 0; i < 12; ++i) r.v[i] = P[i];
}
// FAST = false: the plain path's arithmetic (separate multiply and add,
// Smith's complex reciprocal), the reference's rounding.  FAST = true (mixed
// precision): fused multiply-adds and a one-division reciprocal
// conj(D) / |D|^2, still in FP64.
template <bool FAST>
__device__ __forceinline__ void assemble_row(const RowPieces& r, double l2, double lsq, cd a[4]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const cd A = r.v[q], B = r.v[4 + q], C = r.v[8 + q];
        if (FAST) {
            a[q] = mk(fma(lsq, C.re, fma(l2, B.re, A.re)), fma(lsq, C.im, fma(l2, B.im, A.im)));
        } else {
            a[q] = mk(A.re + l2 * B.re, A.im + l2 * B.im);
            a[q] = mk(a[q].re + lsq * C.re, a[q].im + lsq * C.im);
        }
    }
}
// Depth cut-off (mixed path): rows below the system's first kept row kc
// leave the system.  Row j < kc becomes an identity row and the couplings of
// rows j >= kc to rows below kc vanish, so the factorisation of those rows
// yields pivot 1 and multipliers 0, and rows >= kc are factored exactly as a
// band that starts at kc (a zero-displacement boundary there).
__device__ __forceinline__ void cut_row(int j, int kc, cd a[4]) {
    // selects, no branches: the factorisation's step groups stay one block
#pragma unroll
    for (int p = 0; p < 3; ++p) a[p] = (j - 3 + p < kc) ? mk(0.0) : a[p];
    a[3] = (j < kc) ? mk(1.0) : a[3];
}
template <bool FAST>
__device__ __forceinline__ cd cmulT(cd a, cd b) {
    if (FAST) return mk(fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re));
    return a * b;
}
template <bool FAST>
__device__ __forceinline__ cd caddmulT(cd c, cd a, cd b) {  // c + a b
    if (FAST) return mk(fma(a.re, b.re, fma(-a.im, b.im, c.re)), fma(a.re, b.im, fma(a.im, b.re, c.im)));
    return c + a * b;
}
// 1/x for the fast path: the hardware's approximate reciprocal refined by
// two Newton-Raphson steps y <- y + y (1 - x y) (each roughly doubles the
// correct bits), a few ulp from the correctly rounded quotient.
__device__ __forceinline__ double rcp_newton(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    y = fma(y, fma(-x, y, 1.0), y);
    y = fma(y, fma(-x, y, 1.0), y);
    return y;
}
// 1/x with one Newton-Raphson step (about 2^-40 relative): enough for the
// mixed path, whose tolerance is far above it
__device__ __forceinline__ double rcp_newton1(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return fma(y, fma(-x, y, 1.0), y);
}
// the band multipliers w = m / D of a step.  FAST: w = (m conj(D)) / |D|^2,
// whose products with conj(D) run beside the reciprocal, so only one
// multiply follows it on the pivot chain; otherwise 1/D (Smith) times m, the
// reference's operations.
template <bool FAST>
__device__ __forceinline__ cd mult_of(cd m, cd D, double r, cd piv) {
    if (FAST) return mk(fma(m.re, D.re, m.im * D.im) * r, fma(m.im, D.re, -(m.re * D.im)) * r);
    return m * piv;
}
template <bool FAST>
__device__ __forceinline__ cd crecipT(cd D) {
    if (FAST) {
        const double r = rcp_newton(fma(D.re, D.re, D.im * D.im));
        return mk(D.re * r, -D.im * r);
    }
    return mk(1.0) / D;
}

// asynchronous global -> shared copies (16 B) and their groups
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// last pivots and multiplier of a factorisation, for the substitution pass
struct SysTail {
    cd Dn, Dm1, Lnn1, a22raw;
};

struct FactorCtx {
    const PsvDev* d;
    const cd* P;  // this frequency's row pieces, [row][12]
    double l2, lsq;
    int it, n, ls, lmin, nsys, sys;
    bool store;  // false for threads that only repeat another system
    cd* Lst;
    cd* Dst;     // pivots D(k) of rows k >= dmin, for the forward substitution
    int dmin;
};

// what a step hands to the forward substitution: the pivot D(k) and the
// multipliers L(k+1,k), L(k+2,k), L(k+3,k)
struct StepOut {
    cd D, w0, w1, w2;
};

// Step k of dcsymbdl0 (half-width 3), P = k % 4.  The 4x4 window of the
// band is a ring: entry (r, c) of local rows r-3 <= c <= r lives in
// M[r % 4][c % 4], so a step writes the entering row into the slot of the
// row it eliminated and moves nothing.  Same operations, in the same order,
// as the reference's band loop (main update for k <= n-3, the last two
// steps' order otherwise).
template <int P, bool FAST>
__device__ __forceinline__ bool factor_step(int k, cd (&M)[4][4], const cd (&anew)[4], SysTail& T,
                                            const FactorCtx& c, StepOut& so) {
    constexpr int S0 = P, S1 = (P + 1) & 3, S2 = (P + 2) & 3, S3 = (P + 3) & 3;
    const cd D = M[S0][S0];
    so.D = D;
    if (k == c.n) return true;
    if (k == c.n - 1) T.Dm1 = D;
    const double r = FAST ? rcp_newton1(fma(D.re, D.re, D.im * D.im)) : 0.0;
    const cd piv = FAST ? mk(0.0) : crecipT<false>(D);
    const int nw = min(3, c.n - k);
    cd wv0, wv1 = mk(0.0), wv2 = mk(0.0), zv0, zv1 = mk(0.0), zv2 = mk(0.0);
    zv0 = -M[S1][S0];
    wv0 = mult_of<FAST>(M[S1][S0], D, r, piv);
    if (nw >= 2) {
        zv1 = -M[S2][S0];
        wv1 = mult_of<FAST>(M[S2][S0], D, r, piv);
    }
    if (nw >= 3) {
        zv2 = -M[S3][S0];
        wv2 = mult_of<FAST>(M[S3][S0], D, r, piv);
    }
    so.w0 = wv0;
    so.w1 = wv1;
    so.w2 = wv2;
    if (c.store && k >= c.lmin) {
        cd* L = c.Lst + (size_t)k * 3 * c.nsys + c.sys;
        L[0] = wv0;
        L[c.nsys] = wv1;
        L[2 * (size_t)c.nsys] = wv2;
    }
    if (k == c.n - 1) T.Lnn1 = wv0;
    if (k <= c.n - 3) {  // main loop of dcsymbdl0: A(k+p,k+q) += w_q z_p
        M[S1][S1] = caddmulT<FAST>(M[S1][S1], wv0, zv0);
        M[S2][S2] = caddmulT<FAST>(M[S2][S2], wv1, zv1);
        M[S3][S3] = caddmulT<FAST>(M[S3][S3], wv2, zv2);
        M[S2][S1] = caddmulT<FAST>(M[S2][S1], wv0, zv1);
        M[S3][S2] = caddmulT<FAST>(M[S3][S2], wv1, zv2);
        M[S3][S1] = caddmulT<FAST>(M[S3][S1], wv0, zv2);
    } else {  // last two steps: A(k+p,k+q) += w_p z_q
        M[S1][S1] = caddmulT<FAST>(M[S1][S1], wv0, zv0);
        if (nw >= 2) {
            M[S2][S1] = caddmulT<FAST>(M[S2][S1], wv1, zv0);
            M[S2][S2] = caddmulT<FAST>(M[S2][S2], wv1, zv1);
        }
    }
    // row k+4 enters the slot of row k (columns k+1 .. k+4)
    if (k + 4 <= c.n) {
        M[S0][S1] = anew[0];
        M[S0][S2] = anew[1];
        M[S0][S3] = anew[2];
        M[S0][S0] = anew[3];
    } else {
        M[S0][S1] = M[S0][S2] = M[S0][S3] = M[S0][S0] = mk(0.0);
    }
    return false;
}

// Step k of the band loop away from its end (k <= n - 4: three
// multipliers, the main update, a row entering): factor_step without the
// end-of-band cases.
template <int P, bool FAST>
__device__ __forceinline__ void factor_step_main(int k, cd (&M)[4][4], const cd (&anew)[4], const FactorCtx& c,
                                                 StepOut& so) {
    constexpr int S0 = P, S1 = (P + 1) & 3, S2 = (P + 2) & 3, S3 = (P + 3) & 3;
    const cd D = M[S0][S0];
    const double r = FAST ? rcp_newton1(fma(D.re, D.re, D.im * D.im)) : 0.0;
    const cd piv = FAST ? mk(0.0) : crecipT<false>(D);
    const cd zv0 = -M[S1][S0], zv1 = -M[S2][S0], zv2 = -M[S3][S0];
    const cd wv0 = mult_of<FAST>(M[S1][S0], D, r, piv);
    const cd wv1 = mult_of<FAST>(M[S2][S0], D, r, piv);
    const cd wv2 = mult_of<FAST>(M[S3][S0], D, r, piv);
    so.D = D;
    so.w0 = wv0;
    so.w1 = wv1;
    so.w2 = wv2;
    if (c.store && k >= c.lmin) {
        cd* L = c.Lst + (size_t)k * 3 * c.nsys + c.sys;
        L[0] = wv0;
        L[c.nsys] = wv1;
        L[2 * (size_t)c.nsys] = wv2;
    }
    M[S1][S1] = caddmulT<FAST>(M[S1][S1], wv0, zv0);
    M[S2][S2] = caddmulT<FAST>(M[S2][S2], wv1, zv1);
    M[S3][S3] = caddmulT<FAST>(M[S3][S3], wv2, zv2);
    M[S2][S1] = caddmulT<FAST>(M[S2][S1], wv0, zv1);
    M[S3][S2] = caddmulT<FAST>(M[S3][S2], wv1, zv2);
    M[S3][S1] = caddmulT<FAST>(M[S3][S1], wv0, zv2);
    M[S0][S1] = anew[0];
    M[S0][S2] = anew[1];
    M[S0][S3] = anew[2];
    M[S0][S0] = anew[3];
}

// One thread per (omega, l) system: band assembly row by row and the
// unpivoted complex-symmetric LDL^T (dcsymbdl0) streamed through the ring
// window.  Multipliers of the rows the substitutions read go to Lst, the
// pivots of the rows the source bases' forward substitution reads (k >=
// dmin) to Dst, the last pivots to tail.  The row pieces stream through
// shared memory: a block (128 consecutive systems: consecutive orders of at
// most a few frequencies) copies CH rows of each of its frequencies
// with cp.async one chunk ahead, so the recurrence waits on shared-memory
// latency only.  Systems of frequencies beyond the first FAC_NW of a block
// read their rows from global memory.  All threads of a block take the same
// steps (the same n), so the block-wide barriers at chunk boundaries are
// uniform; threads past nsys repeat the last system's work without storing
// it.  The forward substitution of the source bases runs afterwards
// (k_psv_fwd) from the stored multipliers and pivots, so this kernel keeps
// only the 4x4 window and the entering row in registers (two thirds of the
// registers of a pass that carries the substitution too: more resident
// warps to hide the recurrence's latency), and one factorisation can serve
// several sources.
constexpr int FAC_THREADS = 128;
// rows per staged chunk (CH, a multiple of 4): 8 or 16, chosen per context
// (dsm_set_tuning / dsm_autotune)
constexpr int FAC_NW = 4;   // frequencies staged per block

template <bool FAST, int CH, bool MERGE>
__global__ void __launch_bounds__(FAC_THREADS, MERGE ? 2 : 3) k_psv_solve(PsvDev d, const cd* __restrict__ Prow, WorkList wl,
                                                              int nsys, int lmin, cd* __restrict__ Lst,
                                                              SysTail* __restrict__ tail, cd* __restrict__ Dst,
                                                              int dmin, const int* __restrict__ kcut,
                                                              const int* __restrict__ bperm, int lsf,
                                                              cd* __restrict__ Zst) {
    __shared__ __align__(16) cd sP[2][FAC_NW][CH][12];
    __shared__ int kb_sh;
    // bperm: blocks of the lowest orders of every frequency (the longest
    // recurrences) first, so that they start in the first wave
    const int sys0 = (bperm ? bperm[blockIdx.x] : (int)blockIdx.x) * FAC_THREADS;
    const int sysv = sys0 + threadIdx.x;
    const bool valid = sysv < nsys;
    const int sys = valid ? sysv : nsys - 1;
    int w, l, w0, w1, ltmp;
    wl_map(wl, sys, w, l);
    wl_map(wl, sys0, w0, ltmp);
    wl_map(wl, min(sys0 + FAC_THREADS, nsys) - 1, w1, ltmp);
    const int nws = min(FAC_NW, w1 - w0 + 1);
    const int ws = w - w0;
    const bool staged = ws < nws;
    FactorCtx c;
    c.d = &d;
    c.P = Prow + (size_t)w * (d.nn + 1) * 12;
    c.l2 = (double)l * (double)(l + 1);
    c.lsq = sqrt(c.l2);
    c.it = d.itmp;
    c.n = d.nn - c.it + 1;
    c.ls = d.jsrc - c.it + 1;  // local row of the first source row
    c.lmin = lmin;
    c.nsys = nsys;
    c.sys = sys;
    c.store = valid;
    c.Lst = Lst;
    c.Dst = Dst;
    c.dmin = dmin;
    const int n = c.n;
    // First kept row of the system (depth cut-off; 1 without), of its warp
    // (a step group boundary: all lanes of a warp take the same steps) and
    // of the block (the first staged chunk).  Warps start at their own row.
    const int kc = kcut ? kcut[sys] : 1;
    const int kw = ((__reduce_min_sync(0xffffffffu, kc) - 1) & ~3) + 1;
    if (threadIdx.x == 0) kb_sh = kw;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicMin(&kb_sh, kw);
    __syncthreads();
    const int q0 = (kb_sh - 1) / CH;
    // local rows 5 .. n in chunks: chunk q = rows 5 + q CH .. (global it + r - 1)
    auto stage = [&](int q, int buf) {
        const int r0 = 5 + q * CH;
        const int cnt = min(CH, n - r0 + 1);
        if (cnt <= 0) return;
        const int per = cnt * 12;
        for (int e = threadIdx.x; e < nws * per; e += FAC_THREADS) {
            const int wi = e / per, rem = e - wi * per, i = rem / 12, v = rem - i * 12;
            cp_async16(&sP[buf][wi][i][v], Prow + ((size_t)(w0 + wi) * (d.nn + 1) + c.it + r0 + i - 1) * 12 + v);
        }
    };
    stage(q0, q0 & 1);
    cp_async_commit();
    cd M[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) M[p][q] = mk(0.0);
    cd a[4];
    RowPieces rp;
    // local rows kw .. kw+3 go to slots 1, 2, 3, 0 (kw = 1 mod 4)
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        if (kw + p > n) break;
        load_row(c.P + (size_t)(c.it + kw - 1 + p) * 12, rp);
        assemble_row<FAST>(rp, c.l2, c.lsq, a);
        if (kcut) cut_row(kw + p, kc, a);
#pragma unroll
        for (int q = 0; q <= p; ++q) M[(1 + p) & 3][(1 + q) & 3] = a[4 - (p - q) - 1];
    }
    SysTail T;
    // dcsbdlv0 reads a(m-1,2) = a(2,2) of the unfactored band at row 2: it
    // goes to tail now, so nothing of it stays live through the band
    load_row(c.P + (size_t)(c.it + 1) * 12, rp);
    assemble_row<FAST>(rp, c.l2, c.lsq, a);
    if (valid) tail[sys].a22raw = a[1];
    T.Dm1 = mk(1.0);
    T.Lnn1 = mk(0.0);
    // row entering at step k: local row k+4, chunk (k-1)/CH, index (k-1)%CH
    auto entering = [&](int k, cd (&an)[4]) {
        if (k + 4 > n) return;
        const int i = (k - 1) % CH, buf = ((k - 1) / CH) & 1;
        if (staged) {
#pragma unroll
            for (int v = 0; v < 12; ++v) rp.v[v] = sP[buf][ws][i][v];
        } else {
            load_row(c.P + (size_t)(c.it + k + 3) * 12, rp);
        }
        assemble_row<FAST>(rp, c.l2, c.lsq, an);
        if (kcut) cut_row(k + 4, kc, an);
    };
    // the same away from the end of the band (row k+4 exists): the row comes
    // from shared memory or, for a frequency not staged, global memory,
    // through one generic pointer, so a step group has no branches
    // MASK: some lane's cut row is still within reach of the entering row
    auto entering_main = [&](int k, cd (&an)[4], auto MASK) {
        const int i = (k - 1) % CH, buf = ((k - 1) / CH) & 1;
        const cd* src = staged ? &sP[buf][staged ? ws : 0][i][0] : c.P + (size_t)(c.it + k + 3) * 12;
#pragma unroll
        for (int v = 0; v < 12; ++v) rp.v[v] = src[v];
        assemble_row<FAST>(rp, c.l2, c.lsq, an);
        if constexpr (decltype(MASK)::value) cut_row(k + 4, kc, an);
    };
    // entering rows j need the cut's selects while j < kc + 3 for some lane
    const int kc_max = __reduce_max_sync(0xffffffffu, kc);
    // chunk boundary at k (k - 1 a multiple of CH): the next chunk's copies go out
    auto boundary = [&](int k) {
        if ((k - 1) % CH == 0) {
            const int q = (k - 1) / CH;
            stage(q + 1, (q + 1) & 1);
            cp_async_commit();
            cp_async_wait<1>();
            __syncthreads();
        }
    };
    cd an[4];
    StepOut so{};
    auto keepD = [&](int k) {
        if (c.store && k >= c.dmin) c.Dst[(size_t)(k - c.dmin) * c.nsys + c.sys] = so.D;
    };
    // four main steps (rows k .. k+3, away from the end of the band); fwd
    // runs after each step (the forward pass below, or nothing)
    auto group = [&](int k, auto MASK, auto& fwd) {
        entering_main(k, an, MASK);
        factor_step_main<1, FAST>(k, M, an, c, so);
        keepD(k);
        fwd(k);
        entering_main(k + 1, an, MASK);
        factor_step_main<2, FAST>(k + 1, M, an, c, so);
        keepD(k + 1);
        fwd(k + 1);
        entering_main(k + 2, an, MASK);
        factor_step_main<3, FAST>(k + 2, M, an, c, so);
        keepD(k + 2);
        fwd(k + 2);
        entering_main(k + 3, an, MASK);
        factor_step_main<0, FAST>(k + 3, M, an, c, so);
        keepD(k + 3);
        fwd(k + 3);
    };
    auto nofwd = [](int) {};
    auto masked = [&](int k) { return kcut && k + 4 < kc_max + 3; };  // warp-uniform
    // Loop A: groups below the forward pass.  A cut row never reaches the
    // end of the band (it stays below the source), so warps wait for their
    // first row here only.
    int k = q0 * CH + 1;
    for (;; k += 4) {
        if (k + 3 > n - 4 || (MERGE && lsf > 3 && k + 6 >= lsf)) break;
        boundary(k);
        if (k < kw) {  // this warp's band starts further up
            if ((k + 3) % CH == 0) __syncthreads();
            continue;
        }
        if (masked(k)) group(k, std::true_type{}, nofwd);
        else group(k, std::false_type{}, nofwd);
        if ((k + 3) % CH == 0) __syncthreads();  // chunk fully used before its buffer refills
    }
    // Loop B: the rest, with the forward substitution of one source's four
    // bases (lsf > 3: its first source row; k_psv_fwd's operations, in the
    // same order) riding along: row k takes the pivot of step k and the
    // multipliers L(k,k-1), L(k,k-2), L(k,k-3) of the three steps before, so
    // from three steps below the source those are kept: h0 = w0 of the last
    // step, h1a/h1b = w1 of the last two, h2a/h2b/h2c = w2 of the last
    // three.  Its state lives in this loop only.
    {
        cd fz[4][3], h0 = mk(0.0), h1a = mk(0.0), h1b = mk(0.0), h2a = mk(0.0), h2b = mk(0.0), h2c = mk(0.0);
#pragma unroll
        for (int b = 0; b < 4; ++b) fz[b][0] = fz[b][1] = fz[b][2] = mk(0.0);
        auto fwd_step = [&](int k) {
            if (k >= lsf) {
                const cd D = so.D, l1 = h0, l2 = h1b, l3 = h2c;
                cd rcp = mk(0.0);
                if (FAST) rcp = crecipT<true>(D);
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const cd rhs = mk(lsf + b == k ? 1.0 : 0.0);
                    const cd z0 = fz[b][0], z1 = fz[b][1], z2 = fz[b][2];
                    cd zc;
                    if (FAST) {
                        cd sum = cmulT<true>(l3, z0);
                        sum = caddmulT<true>(sum, l2, z1);
                        sum = caddmulT<true>(sum, l1, z2);
                        zc = rhs - sum;
                    } else {
                        cd sum = mk(0.0) + l3 * z0 + l2 * z1 + l1 * z2;
                        zc = rhs - sum;
                    }
                    if (c.store)
                        Zst[((size_t)(k - lsf) * 4 + b) * nsys + sys] = FAST ? cmulT<true>(zc, rcp) : zc / D;
                    fz[b][0] = z1;
                    fz[b][1] = z2;
                    fz[b][2] = zc;
                }
            }
            h2c = h2b;
            h2b = h2a;
            h2a = so.w2;
            h1b = h1a;
            h1a = so.w1;
            h0 = so.w0;
        };
        const bool fw = MERGE && lsf > 3;
        for (;; k += 4) {
            boundary(k);
            if (k < kw) {
                if ((k + 3) % CH == 0) __syncthreads();
                continue;
            }
            if (k + 3 <= n - 4) {  // four steps away from the end of the band (same n block-wide)
                if (fw) group(k, std::false_type{}, fwd_step);  // the cut lies eight rows below the source
                else if (masked(k)) group(k, std::true_type{}, nofwd);
                else group(k, std::false_type{}, nofwd);
                if ((k + 3) % CH == 0) __syncthreads();  // chunk fully used before its buffer refills
                continue;
            }
            bool last;
            entering(k, an);
            last = factor_step<1, FAST>(k, M, an, T, c, so);
            keepD(k);
            if (fw) fwd_step(k);
            if (last) { T.Dn = M[1][1]; break; }
            entering(k + 1, an);
            last = factor_step<2, FAST>(k + 1, M, an, T, c, so);
            keepD(k + 1);
            if (fw) fwd_step(k + 1);
            if (last) { T.Dn = M[2][2]; break; }
            entering(k + 2, an);
            last = factor_step<3, FAST>(k + 2, M, an, T, c, so);
            keepD(k + 2);
            if (fw) fwd_step(k + 2);
            if (last) { T.Dn = M[3][3]; break; }
            entering(k + 3, an);
            last = factor_step<0, FAST>(k + 3, M, an, T, c, so);
            keepD(k + 3);
            if (fw) fwd_step(k + 3);
            if (last) { T.Dn = M[0][0]; break; }
            if ((k + 3) % CH == 0) __syncthreads();  // chunk fully used before its buffer refills
        }
    }
    cp_async_wait<0>();  // no copy outlives the block
    if (valid) {
        tail[sys].Dn = T.Dn;
        tail[sys].Dm1 = T.Dm1;
        tail[sys].Lnn1 = T.Lnn1;
    }
}

// Forward substitution of the four source bases (dcsbdlv0, m = 3) of one
// source from its first row ls up, one thread per system, from the stored
// multipliers L(k,k-1), L(k,k-2), L(k,k-3) and pivots D(k): below ls every
// z is zero.  zh = z / D goes to Zst.  The same operations as the
// reference's forward loop; a factorisation serves any number of sources.
template <bool FAST>
__global__ void __launch_bounds__(128) k_psv_fwd(PsvDev d, int nsys, int ls, const cd* __restrict__ Lst,
                                                 const cd* __restrict__ Dst, int dmin,
                                                 const SysTail* __restrict__ tail, cd* __restrict__ Zst,
                                                 const int* __restrict__ bperm) {
    const int sys = (bperm ? bperm[blockIdx.x] : (int)blockIdx.x) * blockDim.x + threadIdx.x;
    if (sys >= nsys) return;
    const int n = d.nn - d.itmp + 1;
    const cd a22raw = tail[sys].a22raw;
    auto L = [&](int row, int p) {  // multiplier p of step row (0 for rows before the band)
        return row >= 1 ? Lst[((size_t)row * 3 + p) * nsys + sys] : mk(0.0);
    };
    cd z[4][3];
#pragma unroll
    for (int b = 0; b < 4; ++b) z[b][0] = z[b][1] = z[b][2] = mk(0.0);
    for (int k = ls; k <= n; ++k) {
        const cd D = Dst[(size_t)(k - dmin) * nsys + sys];
        const cd l3 = L(k - 3, 2), l2 = L(k - 2, 1), l1 = L(k - 1, 0);  // L(k,k-3), L(k,k-2), L(k,k-1)
        cd rcp = mk(0.0);
        if (FAST) rcp = crecipT<true>(D);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const cd rhs = mk(ls + b == k ? 1.0 : 0.0);
            const cd z0 = z[b][0], z1 = z[b][1], z2 = z[b][2];
            cd zc;
            if (k == 1) {
                zc = rhs;
            } else if (k == 2) {
                zc = rhs - a22raw * z2;
            } else if (FAST) {
                cd sum = cmulT<true>(l3, z0);
                sum = caddmulT<true>(sum, l2, z1);
                sum = caddmulT<true>(sum, l1, z2);
                zc = rhs - sum;
            } else if (k == 3) {  // a(2,3) z(1) + a(3,3) z(2)
                cd sum = mk(0.0) + l2 * z1 + l1 * z2;
                zc = rhs - sum;
            } else {  // a(1,j) z(j-3) + a(2,j) z(j-2) + a(3,j) z(j-1)
                cd sum = mk(0.0) + l3 * z0 + l2 * z1 + l1 * z2;
                zc = rhs - sum;
            }
            Zst[((size_t)(k - ls) * 4 + b) * nsys + sys] = FAST ? cmulT<true>(zc, rcp) : zc / D;
            z[b][0] = z1;
            z[b][1] = z2;
            z[b][2] = zc;
        }
    }
}

// Upward substitution of the six basis right-hand sides (dcsbdlv0, m = 3):
// x(n) = zh(n); x(n-1) = zh(n-1) - L(n,n-1) x(n); x(j) = zh(j) - [L(j+3,j)
// x(j+3) + L(j+2,j) x(j+2) + L(j+1,j) x(j+1)], down to the deepest captured
// row; zh of the source bases comes from the factorisation's forward pass
// (zero below the source), bases 4 and 5 are the surface unit vectors
// e_{n-1}, e_n, and the values at receiver stencil rows go to Xcap.  One
// lane per system with all six bases in the lane: six independent
// recurrences, each multiplier read once.  FAST (mixed precision) uses fused
// multiply-adds; otherwise the reference's operation order.  Each lane stages its own
// multipliers (and, above the source, its zh) with cp.async into a private
// ring of UP_NBUF chunks in shared memory, UP_NBUF - 1 chunks ahead of use,
// and waits only for its own copies, so no barrier couples the lanes.  The
// captured rows come from a list in descending row order ({row, slot},
// ended by row -1).
constexpr int UP_WARPS = 4;
constexpr int UP_THREADS = 32 * UP_WARPS;
constexpr int UP_NBUF = 4;
constexpr int UP_CH1 = 2, UP_E1 = 7;  // at and above the source: rows per chunk, entries (3 L + 4 zh)
constexpr int UP_CH2 = 4, UP_E2 = 3;  // below it: rows per chunk, entries (3 L)
constexpr int UP_ROW_CD = 14;         // complex per lane and chunk, the larger of CH1 E1 and CH2 E2
constexpr int UP_WARP_CD = UP_NBUF * UP_ROW_CD * 32;
constexpr size_t UP_SMEM = sizeof(cd) * UP_WARP_CD * UP_WARPS;
static_assert(UP_CH1 * UP_E1 <= UP_ROW_CD && UP_CH2 * UP_E2 <= UP_ROW_CD, "ring too small");

template <bool FAST>
__global__ void __launch_bounds__(UP_THREADS, 2) k_psv_up(PsvDev d, int nsys, int jmin_loc,
                                                          const int* __restrict__ capmap,
                                                          const int2* __restrict__ caplist,
                                                          const cd* __restrict__ Lst, const cd* __restrict__ Zst,
                                                          const SysTail* __restrict__ tail, cd* __restrict__ Xcap,
                                                          const int* __restrict__ kcut, const int* __restrict__ bperm,
                                                          cd* __restrict__ Xprobe) {
    extern __shared__ __align__(16) unsigned char up_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int blk = bperm ? bperm[blockIdx.x] : (int)blockIdx.x;  // longest recurrences first
    const int sys = (blk * UP_WARPS + warp) * 32 + lane;
    // the warp's first factored row (the factorisation's warps are the same
    // 32 systems): rows below it hold no multipliers and no solution
    const int kw = kcut ? ((__reduce_min_sync(0xffffffffu, kcut[min(sys, nsys - 1)]) - 1) & ~3) + 1 : 1;
    if (sys >= nsys) return;  // nothing below synchronises across lanes
    jmin_loc = max(jmin_loc, kw);
    cd* ring = reinterpret_cast<cd*>(up_smem) + (size_t)warp * UP_WARP_CD + lane;
    const int it = d.itmp, n = d.nn - it + 1, ls = d.jsrc - it + 1;
    // captured values; the cutoff probe's two rows also go to Xprobe (the
    // amplitude test is formed by k_psv_coef)
    auto store = [&](int c, int b, cd v) {
        Xcap[((size_t)c * NB + b) * nsys + sys] = v;
        if (b < 4 && (c == d.cap_p0 || c == d.cap_p1)) Xprobe[((size_t)(c == d.cap_p0 ? 0 : 1) * 4 + b) * nsys + sys] = v;
    };
    cd x[NB][3];  // x(j+1), x(j+2), x(j+3) of each basis
    {
        const SysTail tl = tail[sys];
        const int cn = capmap[n + it - 1], cn1 = n - 1 >= jmin_loc ? capmap[n - 1 + it - 1] : -1;
        const cd Ln = n - 1 >= jmin_loc ? Lst[((size_t)(n - 1) * 3) * nsys + sys] : mk(0.0);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            cd xn;
            if (b < 4) xn = (n >= ls) ? Zst[((size_t)(n - ls) * 4 + b) * nsys + sys] : mk(0.0);
            // surface basis: e_{n-1}: z(n-1) = 1, z(n) = -L(n,n-1); e_n: z(n) = 1
            else if (b == 4) xn = (mk(0.0) - tl.Lnn1 * mk(1.0)) / tl.Dn;
            else xn = mk(1.0) / tl.Dn;
            if (cn >= 0) store(cn, b, xn);
            x[b][0] = xn;
            x[b][1] = mk(0.0);
            x[b][2] = mk(0.0);
            if (n - 1 >= jmin_loc) {
                cd zh = mk(0.0);
                if (b < 4 && n - 1 >= ls) zh = Zst[((size_t)(n - 1 - ls) * 4 + b) * nsys + sys];
                if (b == 4) zh = mk(1.0) / tl.Dm1;
                const cd v = zh - Ln * x[b][0];
                if (cn1 >= 0) store(cn1, b, v);
                x[b][1] = x[b][0];
                x[b][0] = v;
            }
        }
    }
    const int top = n - 2;
    if (top < jmin_loc) return;
    int2 cap = caplist[0];
    int ci = 0;
    // rows j0, j0 - 1, .. (cnt of them) with E staged entries per row, CH rows per chunk
    auto phase = [&](auto Etag, auto CHtag, int j0, int cnt) {
        constexpr int E = decltype(Etag)::value, CH = decltype(CHtag)::value, RING = UP_NBUF * CH;
        if (cnt <= 0) return;
        const int nq = (cnt + CH - 1) / CH;
        auto stage = [&](int q) {
            if (q >= nq) return;
            for (int i = 0; i < CH; ++i) {
                const int t = q * CH + i;
                if (t >= cnt) break;
                const int j = j0 - t;
                cd* dst = ring + (size_t)((t % RING) * E) * 32;
#pragma unroll
                for (int p = 0; p < 3; ++p) cp_async16(dst + p * 32, &Lst[((size_t)j * 3 + p) * nsys + sys]);
                if (E == 7) {
#pragma unroll
                    for (int b = 0; b < 4; ++b)
                        cp_async16(dst + (3 + b) * 32, &Zst[((size_t)(j - ls) * 4 + b) * nsys + sys]);
                }
            }
        };
#pragma unroll
        for (int q = 0; q < UP_NBUF - 1; ++q) {
            stage(q);
            cp_async_commit();
        }
        // row t (j = j0 - t) with roles (xa, xb, xc) = x[b][A], x[b][B], x[b][C]; x(j) replaces xc
        auto one = [&](int t, auto Atag, auto Btag, auto Ctag) {
            constexpr int A = decltype(Atag)::value, B = decltype(Btag)::value, C = decltype(Ctag)::value;
            if (t % CH == 0) {  // a chunk starts: the one UP_NBUF - 1 ahead goes out, this one is waited for
                stage(t / CH + UP_NBUF - 1);
                cp_async_commit();
                cp_async_wait<UP_NBUF - 1>();
            }
            const int j = j0 - t;
            const cd* src = ring + (size_t)((t % RING) * E) * 32;
            const cd L1 = src[0], L2 = src[32], L3 = src[64];
            const bool cap_here = j == cap.x;
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const cd zh = (E == 7 && b < 4) ? src[(3 + b) * 32] : mk(0.0);
                const cd xa = x[b][A], xb = x[b][B], xc = x[b][C];
                cd v;
                if (FAST) {
                    cd sum = cmulT<true>(L3, xc);
                    sum = caddmulT<true>(sum, L2, xb);
                    sum = caddmulT<true>(sum, L1, xa);
                    v = zh - sum;
                } else if (j == n - 2) {
                    cd sum = mk(0.0) + L2 * xb + L1 * xa;
                    v = zh - sum;
                } else {
                    cd sum = mk(0.0) + L3 * xc + L2 * xb + L1 * xa;
                    v = zh - sum;
                }
                if (cap_here) store(cap.y, b, v);
                x[b][C] = v;
            }
            if (cap_here) cap = caplist[++ci];
        };
        using I0 = std::integral_constant<int, 0>;
        using I1 = std::integral_constant<int, 1>;
        using I2 = std::integral_constant<int, 2>;
        int t = 0;
        for (; t + 3 <= cnt; t += 3) {
            one(t, I0{}, I1{}, I2{});      // x[.][2] <- x(j)
            one(t + 1, I2{}, I0{}, I1{});  // x[.][1] <- x(j-1)
            one(t + 2, I1{}, I2{}, I0{});  // x[.][0] <- x(j-2)
        }
        if (t < cnt) {  // one or two rows left: run them, then restore the roles
            one(t, I0{}, I1{}, I2{});
            if (t + 1 < cnt) {
                one(t + 1, I2{}, I0{}, I1{});
#pragma unroll
                for (int b = 0; b < NB; ++b) {  // (x0, x1, x2) = (x(j+1), x(j+2), x(j+3)) again
                    const cd a0 = x[b][0];
                    x[b][0] = x[b][1];
                    x[b][1] = x[b][2];
                    x[b][2] = a0;
                }
            } else {
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    const cd a2 = x[b][2];
                    x[b][2] = x[b][1];
                    x[b][1] = x[b][0];
                    x[b][0] = a2;
                }
            }
        }
        cp_async_wait<0>();  // the ring is reused by the next phase
    };
    const int lo1 = max(ls, jmin_loc);
    const int n1 = top >= lo1 ? top - lo1 + 1 : 0;  // rows at and above the source
    phase(std::integral_constant<int, UP_E1>{}, std::integral_constant<int, UP_CH1>{}, top, n1);
    phase(std::integral_constant<int, UP_E2>{}, std::integral_constant<int, UP_CH2>{}, top - n1,
          top - n1 - jmin_loc + 1);
    // captured rows below the cut: zero displacement
    for (; cap.x >= 1; cap = caplist[++ci])
#pragma unroll
        for (int b = 0; b < NB; ++b) store(cap.y, b, mk(0.0));
}

// ------------------------------------------------------------ l = 0 path
// One thread per frequency: compacted tridiagonal (rea2), its LDL^T and the
// solves of the three m = 0 sources (imt 1..3) and the back-propagated
// vertical force.  Writes the fields of column l = 0.
__device__ void calabnum_dev(const PsvDev& d, double omega, cd c1, cd c2, cd* anum, cd* bnum);
__device__ void calya_dev(const cd* anum, const cd* bnum, double l2, double ra0, double ra1, double r0,
                          cd* ya, cd* yb, cd* yc, cd* yd);
__device__ void calg_dev(const PsvDev& d, int l, int m, cd c1, cd c2, double lsq, const cd* ya,
                         const cd* yb, const cd* yc, const cd* yd, int imt, cd* g);

// (1) compaction, one thread per compact row: c(1,i), c(2,i) of rea2 from the
// assembled l = 0 band (l0col: global column, l0e1: band row of c(1,i), 0 for none)
__global__ void k_psv_l0_build(PsvDev d, const cd* __restrict__ B0all, const cd* __restrict__ B1all,
                               const cd* __restrict__ B2all, const int* __restrict__ l0col,
                               const int* __restrict__ l0e1, cd* __restrict__ Cc) {
    int w = blockIdx.y;
    int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > d.nn0) return;
    const size_t bo = (size_t)w * d.ncol_tot * 4;
    cd a[4];
    assemble(d, l0col[i], B0all + bo, B1all + bo, B2all + bo, 0.0, 0.0, a);
    int e1 = l0e1[i];
    cd* C = Cc + (size_t)w * (d.nn0 + 1) * 2;
    C[2 * i] = e1 == 2 ? a[1] : (e1 == 3 ? a[2] : mk(0.0));
    C[2 * i + 1] = a[3];
}

// (2) one CTA per frequency: right-hand sides (calg at l = 0 for imt 1..3,
// the back-propagated vertical force), dcsymbdl0 with half-width 1 fused
// with the forward substitution of dcsbdlv0, then the upward substitution,
// for the four right-hand sides.  Solutions in Dv[w][i][4].
// The recurrences are sequential in the row; the CTA streams the compact
// tridiagonal through shared memory in chunks (coalesced loads and stores
// by all threads) so that the chains run on shared-memory latency: thread 0
// factors a chunk, threads 0..3 then carry one right-hand side each.
constexpr int L0_CH = 256;  // rows per chunk (3 x 8 KB factor stages + 16 KB solution)

template <bool FAST>
__global__ void __launch_bounds__(128) k_psv_l0_solve(PsvDev d, const int* __restrict__ freqs, int nf,
                                                      const cd* __restrict__ ab, cd* __restrict__ Cc,
                                                      cd* __restrict__ Dv, int back) {
    const int w = blockIdx.x;
    if (w >= nf) return;
    const int n0 = d.nn0, it0 = d.itmp0, tid = threadIdx.x;
    cd* C = Cc + (size_t)w * (n0 + 1) * 2;
    cd* D = Dv + (size_t)w * (n0 + 1) * 4;
    __shared__ cd sC[3][L0_CH][2];
    __shared__ cd sD[L0_CH][4];
    __shared__ int srr[5];
    __shared__ cd srv[5][4];
    __shared__ int snr;
    if (tid == 0) {
        const double omega = 2.0 * kPi * (double)freqs[w] / d.tlen;
        const cd c1 = coefq(omega, d.qmu[d.spn - 1]), c2 = coefq(omega, d.qkappa[d.spn - 1]);
        cd ya[4], yb[4], yc[4], yd[4];
        calya_dev(ab + (size_t)w * 320, ab + (size_t)w * 320 + 160, 0.0, d.ra0, d.ra1, d.r0, ya, yb, yc, yd);
        // sparse right-hand sides: rea2 keeps the U rows of g0(jtmp..jtmp+3)
        int nr = 0;
        for (int k = 0; k < 4; ++k) {
            int cr = d.comp_src[d.jsrc + k];
            if (cr <= 0) continue;
            srr[nr] = cr;
            for (int b = 0; b < 4; ++b) srv[nr][b] = mk(0.0);
            ++nr;
        }
        for (int imt = 1; imt <= 3; ++imt) {
            cd g[4];
            calg_dev(d, 0, 0, c1, c2, 0.0, ya, yb, yc, yd, imt, g);
            int q = 0;
            for (int k = 0; k < 4; ++k)
                if (d.comp_src[d.jsrc + k] > 0) srv[q++][imt - 1] = g[k];
        }
        // caldveczero at l = 0: bvec(1,0) = cmplx(coef), single precision
        double coef = sqrt((double)1 / (4.0 * kPi) / 1.0);
        int cr = d.comp_src[d.nn - 1];
        srr[nr] = cr > 0 ? cr : -1;
        for (int b = 0; b < 4; ++b) srv[nr][b] = mk(0.0);
        if (back) srv[nr][3] = -conj(mk((double)(float)coef));
        snr = nr + 1;
    }
    __syncthreads();
    const int nr = snr;
    auto rhs = [&](int row, int b) {
        cd v = mk(0.0);
        for (int k = 0; k < nr; ++k)
            if (srr[k] == row) v = srv[k][b];
        return v;
    };
    // forward: factor step k = g-1 (piv = 1/c(2,k); w2 = c(1,k+1) piv;
    // c(2,k+1) += w2 (-c(1,k+1))), then z(k) = z(k)/c(2,k) and
    // z(g) = b(g) - c(1,g) z(g-1) for each right-hand side.  Three-stage
    // pipeline over chunks: in phase p warps 2-3 store chunk p-3 and load
    // chunk p, thread 0 (warp 0) factors chunk p-1 and threads 32..35
    // (warp 1) carry the right-hand sides through chunk p-2.
    cd dfac = C[2 * it0 + 1];      // thread 0: running pivot
    cd zb = mk(0.0), db = dfac;    // threads 32..35: z and pivot of the previous row
    const int rt = tid - 32;       // right-hand side of threads 32..35
    if (rt >= 0 && rt < 4) zb = rhs(it0, rt);
    const int nch = (n0 - it0 + L0_CH - 1) / L0_CH;  // chunks of rows it0+1 .. n0
    auto chunk_g0 = [&](int c) { return it0 + 1 + c * L0_CH; };
    auto chunk_cnt = [&](int c) { return min(L0_CH, n0 + 1 - chunk_g0(c)); };
    for (int p = 0; p < nch + 3; ++p) {
        if (tid >= 64) {
            const int lt = tid - 64, nl = blockDim.x - 64;
            if (p - 3 >= 0 && p - 3 < nch) {  // chunk p-3 is final: back to global
                const int c = p - 3, g0 = chunk_g0(c), cnt = chunk_cnt(c);
                for (int i = lt; i < 2 * cnt; i += nl) C[2 * g0 + i] = sC[c % 3][i >> 1][i & 1];
            }
            if (p < nch) {
                const int g0 = chunk_g0(p), cnt = chunk_cnt(p);
                for (int i = lt; i < 2 * cnt; i += nl) sC[p % 3][i >> 1][i & 1] = C[2 * g0 + i];
            }
        } else if (tid == 0) {
            if (p - 1 >= 0 && p - 1 < nch) {
                const int c = p - 1, cnt = chunk_cnt(c);
                cd(*sc)[2] = sC[c % 3];
                for (int i = 0; i < cnt; ++i) {
                    cd piv = crecipT<FAST>(dfac);
                    cd off = sc[i][0];
                    cd z2 = -off;
                    cd w2 = cmulT<FAST>(off, piv);
                    cd dg = caddmulT<FAST>(sc[i][1], w2, z2);
                    sc[i][0] = w2;
                    sc[i][1] = dg;
                    dfac = dg;
                }
            }
        } else if (rt >= 0 && rt < 4) {
            if (p - 2 >= 0 && p - 2 < nch) {
                const int c = p - 2, g0 = chunk_g0(c), cnt = chunk_cnt(c);
                cd(*sc)[2] = sC[c % 3];
                for (int i = 0; i < cnt; ++i) {
                    const int g = g0 + i;
                    D[4 * (g - 1) + rt] = FAST ? cmulT<true>(zb, crecipT<true>(db)) : zb / db;
                    zb = FAST ? caddmulT<true>(rhs(g, rt), -sc[i][0], zb) : rhs(g, rt) - sc[i][0] * zb;
                    db = sc[i][1];
                }
            }
        }
        __syncthreads();
    }
    if (rt >= 0 && rt < 4) D[4 * n0 + rt] = zb / db;
    __syncthreads();
    // upward substitution x(g) = z(g) - c(1,g+1) x(g+1), g = n0-1 .. it0
    cd x = mk(0.0);
    if (tid < 4) x = D[4 * n0 + tid];
    for (int ghi = n0 - 1; ghi >= it0; ghi -= L0_CH) {
        const int glo = max(it0, ghi - L0_CH + 1), cnt = ghi - glo + 1;
        for (int i = tid; i < cnt; i += blockDim.x) sC[0][i][0] = C[2 * (glo + i + 1)];
        for (int i = tid; i < 4 * cnt; i += blockDim.x) sD[i >> 2][i & 3] = D[4 * glo + i];
        __syncthreads();
        if (tid < 4) {
            for (int i = cnt - 1; i >= 0; --i) {
                x = sD[i][tid] - sC[0][i][0] * x;
                sD[i][tid] = x;
            }
        }
        __syncthreads();
        for (int i = tid; i < 4 * cnt; i += blockDim.x) D[4 * glo + i] = sD[i >> 2][i & 3];
        __syncthreads();
    }
}

// (3) fields of order 0, one thread per (frequency, receiver): m = 0 slots
// q = 0..2 (imt 1..3) and 3 (back), U and dU/dr (calup0 uses u(1) only)
// rows ordered (field group, slot, field, re/im, receiver): receivers
// contiguous, so the epilogue's threads (consecutive receivers) read
// consecutive rows; fields a fluid receiver does not need have no row
template <class T>
__device__ __forceinline__ void put_field(T* Aw, int Lcap, int nq, const PsvDev& d, int rr, int q, int f, cd v) {
    int im;
    const long long row = psvk::fld_row(nq, d.Rs1, d.Rf, q, f, rr, &im);
    if (row < 0) return;
    Aw[(size_t)row * Lcap] = (T)v.re;
    Aw[((size_t)row + im) * Lcap] = (T)v.im;
}

template <class T>
__global__ void k_psv_l0_fields(PsvDev d, const cd* __restrict__ Dv, T* __restrict__ A0f, T* __restrict__ A1f,
                                T* __restrict__ A2f, int Lcap, int back) {
    int w = blockIdx.y;
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int R = d.R;
    if (r > R) return;
    const int n0 = d.nn0;
    const cd* D = Dv + (size_t)w * (n0 + 1) * 4;
    const size_t rows0 = psvk::fld_rows(NS0, d.Rs1, d.Rf), rows1 = psvk::fld_rows(NS1, d.Rs1, d.Rf),
                 rows2 = psvk::fld_rows(NS2, d.Rs1, d.Rf);
    T* A0w = A0f + (size_t)w * rows0 * Lcap;
    T* A1w = A1f + (size_t)w * rows1 * Lcap;
    T* A2w = A2f + (size_t)w * rows2 * Lcap;
    const int rr = d.rrow[r];
    for (int q = 0; q < NS0; ++q) {
        cd U = mk(0.0), Ud = mk(0.0);
        if (q < 3 || back) {
            if (r < R) {
                for (int i = 0; i < 3; ++i) {
                    cd v = D[4 * (d.jsta[r] + i) + q];
                    U = U + d.wv[3 * r + i] * v;
                    Ud = Ud + d.wd[3 * r + i] * v;
                }
            } else if (q < 3) {
                U = D[4 * n0 + q];
            }
        }
        put_field(A0w, Lcap, NS0, d, rr, q, 0, U);
        put_field(A0w, Lcap, NS0, d, rr, q, 1, Ud);
        for (int f = 2; f < NFLD; ++f) put_field(A0w, Lcap, NS0, d, rr, q, f, mk(0.0));
    }
    for (int q = 0; q < NS1; ++q)
        for (int f = 0; f < NFLD; ++f) put_field(A1w, Lcap, NS1, d, rr, q, f, mk(0.0));
    for (int q = 0; q < NS2; ++q)
        for (int f = 0; f < NFLD; ++f) put_field(A2w, Lcap, NS2, d, rr, q, f, mk(0.0));
}

// ------------------------------------------------------- source terms
__device__ void calabnum_dev(const PsvDev& d, double omega, cd coef1, cd coef2, cd* anum, cd* bnum) {
    for (int k = 0; k < 160; ++k) anum[k] = bnum[k] = mk(0.0);
    auto AN = [&](int i, int j, int k) -> cd& { return anum[(k - 1) * 16 + (j - 1) * 4 + (i - 1)]; };
    auto BN = [&](int i, int j, int k) -> cd& { return bnum[(k - 1) * 16 + (j - 1) * 4 + (i - 1)]; };
    const double* P = d.poly;
    for (int i = 1; i <= 10; ++i) {
        double r;
        if (i <= 5) r = d.ra0 + (double)(i - 1) / 4.0 * (d.r0 - d.ra0);
        else r = d.ra1 - (double)(10 - i) / 4.0 * (d.ra1 - d.r0);
        double trho = 0, tvpv = 0, tvph = 0, tvsv = 0, tvsh = 0, teta = 0, coef = 1.0;
        for (int j = 1; j <= 4; ++j) {
            if (j == 1) coef = 1.0;
            else coef = coef * (r / d.rmax);
            trho = trho + P[0 + j - 1] * coef;
            tvpv = tvpv + P[4 + j - 1] * coef;
            tvph = tvph + P[8 + j - 1] * coef;
            tvsv = tvsv + P[12 + j - 1] * coef;
            tvsh = tvsh + P[16 + j - 1] * coef;
            teta = teta + P[20 + j - 1] * coef;
        }
        double tecA = trho * tvph * tvph, tecC = trho * tvpv * tvpv;
        double tecL = trho * tvsv * tvsv, tecN = trho * tvsh * tvsh, tmu = trho * tvsv * tvsv;
        double tAkappa = tecA - tmu * 4.0 / 3.0, tCkappa = tecC - tmu * 4.0 / 3.0;
        cd xAkappa = mk(tAkappa) * coef2, xCkappa = mk(tCkappa) * coef2;
        cd xrho = mk(trho), xmu = mk(tmu) * coef1, xecL = mk(tecL) * coef1, xecN = mk(tecN) * coef1;
        cd xecA = xAkappa + xmu * mk(4.0 / 3.0);
        cd xecC = xCkappa + xmu * mk(4.0 / 3.0);
        cd xecF = mk(teta) * (xecA - mk(2.0) * xecL);
        cd xFdC = xecF / xecC;
        cd xAmF2dC = xecA - xecF * xFdC;
        double r2 = r * r;
        cd comega2 = mk(omega, -d.omegai) * mk(omega, -d.omegai);
        AN(1, 1, i) = -(mk(2.0 / r) * xFdC);
        AN(1, 2, i) = mk(1.0) / xecC;
        AN(2, 1, i) = -(xrho * comega2) + mk(4.0 / r2) * (xAmF2dC - xecN);
        AN(2, 2, i) = mk(2.0 / r) * (xFdC - mk(1.0));
        AN(3, 1, i) = -mk(1.0 / r);
        AN(3, 3, i) = mk(1.0 / r);
        AN(3, 4, i) = mk(1.0) / xecL;
        AN(4, 1, i) = -(mk(2.0 / r2) * (xAmF2dC - xecN));
        AN(4, 2, i) = -(mk(1.0 / r) * xFdC);
        AN(4, 3, i) = -(xrho * comega2) - mk(2.0 / r2) * xecN;
        AN(4, 4, i) = -mk(3.0 / r);
        BN(1, 3, i) = mk(1.0 / r) * xFdC;
        BN(2, 3, i) = -(mk(2.0 / r2) * (xAmF2dC - xecN));
        BN(2, 4, i) = mk(1.0 / r);
        BN(4, 3, i) = xAmF2dC / mk(r2);
    }
}

__device__ void eqm(const cd* anum, const cd* bnum, int blk, double l2, const cd* y, cd* f) {
    int mt = 16 * (blk - 1);
    for (int i = 0; i < 4; ++i) f[i] = mk(0.0);
    cd c[4][4];
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i) {
            cd b = bnum[mt];
            c[i][j] = anum[mt] + mk(l2 * b.re, l2 * b.im);
            mt++;
        }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) f[i] = f[i] + c[i][j] * y[j];
}

// rk3 with one rkstep (src/SGTpsv/rk3.f90); x0 becomes xe
__device__ void rk1(const cd* anum, const cd* bnum, const int* blk, double l2, double& x0, double xe,
                    cd* y0) {
    const double c1 = 1.0 / 6.0, c2 = 1.0 / 3.0, c3 = c2, c4 = c1, b2 = 0.5, b3 = b2;
    double h = (xe - x0) / 1.0;
    cd ak[4], yn[4], w[4];
    eqm(anum, bnum, blk[0], l2, y0, ak);
    for (int i = 0; i < 4; ++i) yn[i] = y0[i] + mk(h * c1) * ak[i];
    for (int i = 0; i < 4; ++i) w[i] = y0[i] + mk(h * b2) * ak[i];
    eqm(anum, bnum, blk[1], l2, w, ak);
    for (int i = 0; i < 4; ++i) yn[i] = yn[i] + mk(h * c2) * ak[i];
    for (int i = 0; i < 4; ++i) w[i] = y0[i] + mk(h * b3) * ak[i];
    eqm(anum, bnum, blk[2], l2, w, ak);
    for (int i = 0; i < 4; ++i) yn[i] = yn[i] + mk(h * c3) * ak[i];
    for (int i = 0; i < 4; ++i) w[i] = y0[i] + mk(h) * ak[i];
    eqm(anum, bnum, blk[3], l2, w, ak);
    for (int i = 0; i < 4; ++i) yn[i] = yn[i] + mk(h * c4) * ak[i];
    for (int i = 0; i < 4; ++i) y0[i] = yn[i];
    x0 = xe;
}

__device__ void calya_dev(const cd* anum, const cd* bnum, double l2, double ra0, double ra1, double r0,
                          cd* ya, cd* yb, cd* yc, cd* yd) {
    for (int i = 0; i < 4; ++i) ya[i] = yb[i] = yc[i] = yd[i] = mk(0.0);
    ya[1] = mk(1.0);
    yb[3] = mk(1.0);
    double dr = (r0 - ra0) / 2.0;
    if (dr > 0.0) {
        double xs = ra0;
        const int blk[2][4] = {{1, 2, 2, 3}, {3, 4, 4, 5}};
        for (int k = 0; k < 2; ++k) {
            double xe = xs + dr;
            rk1(anum, bnum, blk[k], l2, xs, xe, ya);
            xs = xe - dr;
            rk1(anum, bnum, blk[k], l2, xs, xe, yb);
        }
    }
    yc[1] = mk(1.0);
    yd[3] = mk(1.0);
    dr = (ra1 - r0) / 2.0;
    if (dr > 0.0) {
        double xs = ra1;
        const int blk[2][4] = {{10, 9, 9, 8}, {8, 7, 7, 6}};
        for (int k = 0; k < 2; ++k) {
            double xe = xs - dr;
            rk1(anum, bnum, blk[k], l2, xs, xe, yc);
            xs = xe + dr;
            rk1(anum, bnum, blk[k], l2, xs, xe, yd);
        }
    }
}

// glu (src/SGTpsv/glu2.f90) on an n x n complex matrix, leading dim 4
__device__ void glu_dev(cd* a, int n, cd* b) {
    const double eps = 3.52e-15;
    auto A = [&](int i, int j) -> cd& { return a[(i - 1) + 4 * (j - 1)]; };
    int ip[4];
    cd wk[5];
    for (int k = 1; k <= n; ++k) {
        double amax = cabs_(A(k, k));
        int ipk = k;
        for (int i = k + 1; i <= n; ++i) {
            double aik = cabs_(A(i, k));
            if (aik > amax) { ipk = i; amax = aik; }
        }
        ip[k - 1] = ipk;
        if (!(amax > eps)) return;
        if (ipk != k) { cd t = A(ipk, k); A(ipk, k) = A(k, k); A(k, k) = t; }
        for (int i = k + 1; i <= n; ++i) {
            A(i, k) = -A(i, k) / A(k, k);
            wk[i] = A(i, k);
        }
        for (int j = k + 1; j <= n; ++j) {
            if (ipk != k) { cd t = A(ipk, j); A(ipk, j) = A(k, j); A(k, j) = t; }
            cd t = A(k, j);
            for (int i = k + 1; i <= n; ++i) A(i, j) = A(i, j) + wk[i] * t;
        }
    }
    for (int k = 1; k <= n; ++k) {
        if (ip[k - 1] != k) { cd t = b[ip[k - 1] - 1]; b[ip[k - 1] - 1] = b[k - 1]; b[k - 1] = t; }
        cd t = b[k - 1];
        for (int i = k + 1; i <= n; ++i) b[i - 1] = b[i - 1] + A(i, k) * t;
    }
    b[n - 1] = b[n - 1] / A(n, n);
    for (int k = n - 1; k >= 1; --k) {
        cd t = b[k];
        for (int i = 1; i <= k; ++i) b[i - 1] = b[i - 1] - A(i, k + 1) * t;
        b[k - 1] = b[k - 1] / A(k, k);
    }
}

// calg (calmat.f90:1075-1171) for the unit moment tensor imt
__device__ void calg_dev(const PsvDev& d, int l, int m, cd coef1, cd coef2, double lsq, const cd* ya,
                         const cd* yb, const cd* yc, const cd* yd, int imt, cd* g) {
    double mt11 = imt == 1, mt22 = imt == 2, mt33 = imt == 3, mt12 = imt == 4, mt13 = imt == 5,
           mt23 = imt == 6;
    double sgn = (m >= 0) ? 1.0 : -1.0;
    double b1 = sqrt((double)(2 * l + 1) / (16.0 * kPi));
    double b2 = 0.0;
    if (l != 0) b2 = sqrt((double)(2 * l + 1) * (double)(l - 1) * (double)(l + 2) / (64.0 * kPi));
    const double r0 = d.r0, ecC0 = d.ecC0, ecF0 = d.ecF0, ecL0 = d.ecL0;
    cd dd = mk(0.0), ee = mk(0.0), s1 = mk(0.0), s2 = mk(0.0);
    int am = abs(m);
    if (am == 1) ee = mk(-b1 * sgn * mt12, b1 * mt13) / (mk(r0 * r0 * ecL0) * coef1);
    if (am == 0) {
        dd = mk(2.0 * b1 * mt11 / (r0 * r0)) /
             (mk(ecC0 - 4.0 / 3.0 * ecL0) * coef2 + mk(4.0 / 3.0 * ecL0) * coef1);
        double r03 = r0 * r0 * r0;
        cd xtmp = ((ecF0 + 2.0 / 3.0 * ecL0) * coef2 - 2.0 / 3.0 * ecL0 * coef1) /
                  ((ecC0 - 4.0 / 3.0 * ecL0) * coef2 + 4.0 / 3.0 * ecL0 * coef1);
        s1 = mk(-2.0 * b1 * (mt22 + mt33) / r03) + mk(4.0 * b1 * mt11 / r03) * xtmp;
        s2 = mk(b1 * lsq * (mt22 + mt33) / r03) - mk(2.0 * b1 * lsq * mt11 / r03) * xtmp;
    }
    if (am == 2) {
        double r03 = r0 * r0 * r0;
        s2 = mk(-b2 * (mt22 - mt33) / r03, sgn * 2.0 * b2 * mt23 / r03);
    }
    cd sv[4];
    sv[0] = dd;
    sv[1] = s1;
    if (l != 0) {
        sv[2] = mk(ee.re / lsq, ee.im / lsq);
        sv[3] = mk(s2.re / lsq, s2.im / lsq);
    } else {
        sv[2] = sv[3] = mk(0.0);
    }
    cd a[16], b[4];
    if (l != 0) {
        for (int i = 0; i < 4; ++i) {
            a[i] = -ya[i]; a[i + 4] = -yb[i]; a[i + 8] = yc[i]; a[i + 12] = yd[i];
            b[i] = sv[i];
        }
        glu_dev(a, 4, b);
    } else {
        for (int i = 0; i < 2; ++i) {
            a[i] = -ya[i]; a[i + 4] = yc[i];
            b[i] = sv[i];
        }
        glu_dev(a, 2, b);
        b[2] = b[1];
        b[1] = mk(0.0);
        b[3] = mk(0.0);
    }
    double dt[4];
    dt[0] = -d.ra0 * d.ra0;
    dt[1] = dt[0] * lsq;
    dt[2] = d.ra1 * d.ra1;
    dt[3] = dt[2] * lsq;
    for (int i = 0; i < 4; ++i) g[i] = mk(b[i].re * dt[i], b[i].im * dt[i]);
}

// ----------------------------------------------------------------- fields
// Flat slot order (18 slots): 0..2 m = 0, imt 1..3; 3 m = 0 back-propagated
// vertical force; 4..11 |m| = 1: 4 + 4 sg + k (k: imt 4, imt 5, back 2,
// back 3; sg 0: m = -1, 1: m = +1); 12..17 |m| = 2: 12 + 3 sg + k (imt 2, 3, 6).
constexpr int NSLOT = 18;

__device__ __forceinline__ int slot_mi(int s) { return s < 4 ? 0 : (s < 12 ? 1 : 2); }
__device__ __forceinline__ int slot_q(int s) { return s < 4 ? s : (s < 12 ? s - 4 : s - 12); }

// calabnum of every frequency (once per omega)
__global__ void k_psv_abnum(PsvDev d, const int* __restrict__ freqs, int nf, cd* __restrict__ ab) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nf) return;
    const double omega = 2.0 * kPi * (double)freqs[w] / d.tlen;
    cd c1 = coefq(omega, d.qmu[d.spn - 1]), c2 = coefq(omega, d.qkappa[d.spn - 1]);
    calabnum_dev(d, omega, c1, c2, ab + (size_t)w * 320, ab + (size_t)w * 320 + 160);
}

// Per (omega, l >= 1): weights of the six basis solutions for every slot
// (calya + calg for the 13 forward sources, caldveczero for the back ones).
// Layout co[(slot * NB + b) * nsys + sys].
// The cutoff probe of the system (calamp on
// g0(ksta(r_n)-1), g0(ksta(r_n)) of imt = 1, m = 0) is formed here from the
// FP64 slot-0 coefficients and the FP64 probe captures, in every mode.
__global__ void __launch_bounds__(128) k_psv_coef(PsvDev d, const int* __restrict__ freqs, WorkList wl,
                                                  int nsys, const cd* __restrict__ ab,
                                                  cd* __restrict__ co, int back,
                                                  const cd* __restrict__ Xprobe, double* __restrict__ amps,
                                                  int Lcap, const int* __restrict__ bperm) {
    int sys = (bperm ? bperm[blockIdx.x] : (int)blockIdx.x) * blockDim.x + threadIdx.x;
    if (sys >= nsys) return;
    int w, l;
    wl_map(wl, sys, w, l);
    auto put = [&](int slot, const cd* g) {
        for (int b = 0; b < NB; ++b) co[((size_t)slot * NB + b) * nsys + sys] = g[b];
        if (slot == 0) {
            cd p0 = mk(0.0), p1 = mk(0.0);
            for (int b = 0; b < 4; ++b) {
                const cd cb = g[b];
                p0 = p0 + cb * Xprobe[(size_t)b * nsys + sys];
                p1 = p1 + cb * Xprobe[(size_t)(4 + b) * nsys + sys];
            }
            const double a1 = cabs_(p0), a2 = cabs_(p1);
            amps[(size_t)w * Lcap + l] = sqrt(a1 * a1 + a2 * a2);
        }
    };
    cd g[NB];
    for (int b = 0; b < NB; ++b) g[b] = mk(0.0);
    if (l == 0) {  // the order-0 kernels write this order's fields and probe
        for (int s = 0; s < NSLOT; ++s)
            for (int b = 0; b < NB; ++b) co[((size_t)s * NB + b) * nsys + sys] = g[b];
        return;
    }
    const double omega = 2.0 * kPi * (double)freqs[w] / d.tlen;
    const cd c1 = coefq(omega, d.qmu[d.spn - 1]), c2 = coefq(omega, d.qkappa[d.spn - 1]);
    const double l2 = (double)l * (double)(l + 1), lsq = sqrt(l2);
    const cd* anum = ab + (size_t)w * 320;
    const cd* bnum = anum + 160;
    cd ya[4], yb[4], yc[4], yd[4];
    calya_dev(anum, bnum, l2, d.ra0, d.ra1, d.r0, ya, yb, yc, yd);
    for (int s = 0; s < NSLOT; ++s) {
        for (int b = 0; b < NB; ++b) g[b] = mk(0.0);
        int mi = slot_mi(s), q = slot_q(s);
        if (mi == 0) {
            if (q < 3) {
                calg_dev(d, l, 0, c1, c2, lsq, ya, yb, yc, yd, q + 1, g);
            } else if (back) {
                double coef = sqrt((double)(2 * l + 1) / (4.0 * kPi) / 1.0);
                g[4] = -conj(mk((double)(float)coef));  // g0(nn-1) = -conjg(rdvec(1,0))
            }
        } else if (mi == 1) {
            int sg = q / 4, k = q % 4, m = sg == 0 ? -1 : 1;
            if (k < 2) {
                calg_dev(d, l, m, c1, c2, lsq, ya, yb, yc, yd, 4 + k, g);
            } else if (back) {
                // caldveczero, m = 1: bvec(2,1) = -xl2 coef/2, bvec(3,1) = i xl2 coef/2;
                // m = -1: conjugated and negated (odd m).  g0(nn) = conjg(rdvec)/lsq
                double fact = (double)l * (double)(l + 1);
                double coef = sqrt((double)(2 * l + 1) / (4.0 * kPi) / fact);
                cd v = (k == 2) ? mk(-1.0, 0.0) * l2 * coef / 2.0 : mk(0.0, 1.0) * l2 * coef / 2.0;
                if (m < 0) v = -conj(v);
                g[5] = conj(v) / mk(lsq);
            }
        } else if (l >= 2) {
            int sg = q / 3, k = q % 3, m = sg == 0 ? -2 : 2;
            calg_dev(d, l, m, c1, c2, lsq, ya, yb, yc, yd, k == 0 ? 2 : (k == 1 ? 3 : 6), g);
        }
        put(s, g);
    }
}

// Per (omega, l >= 1, receiver group): receiver fields of every slot and the
// cutoff probe (group 0).
// Fields of every slot at the receivers, one thread per (system, receiver):
// a warp holds FS consecutive systems (orders) x 32/FS receivers, so
// each coefficient load serves 32/FS receivers and each field store writes
// FS consecutive orders of one row (32 x 1 measured fastest of 4 x 8,
// 8 x 4, 16 x 2 and 32 x 1 on the benchmark; the results do not depend on
// it).  Values and radial derivatives of the six
// basis solutions come from the three-node weights (interpolate, calup),
// then U, V and derivatives of each slot are their combinations with the
// source coefficients.  Block row 0 also writes the cutoff probe (calamp of
// imt = 1, m = 0 at the top receiver's stencil); the last block row holds
// the surface (rows n-1, n).
// FS systems x 32/FS receivers per warp: 32 (default) or 16, chosen per
// context (dsm_set_tuning / dsm_autotune)


// Arithmetic of the field kernel: the reference's operations on the plain
// path, fused multiply-adds and one reciprocal of sqrt(l(l+1)) on the mixed
// path (whose rows are stored in FP32), both in FP64.  Measured on the
// 2048-frequency grid, FP32 slot combinations (FP64 interpolation) raised the
// mixed path's error to 9e-7 and FP32 interpolation to 5e-6: the derivative
// weights difference neighbouring nodes and the bases cancel.
template <bool FAST>
struct FieldMath {
    using V = cd;
    using R = double;
    __device__ static V coef(const cd* p, size_t i) { return p[i]; }
    __device__ static V from(cd v) { return v; }
    __device__ static V zero() { return mk(0.0); }
    __device__ static cd interp(cd acc, double r, cd x) {  // acc + r x
        if (FAST) return mk(fma(r, x.re, acc.re), fma(r, x.im, acc.im));
        return acc + r * x;
    }
    __device__ static V addmul(V acc, V a, V b) { return caddmulT<FAST>(acc, a, b); }  // acc + a b
    __device__ static V divl(V v, R lsq, R ilsq) { return FAST ? v * ilsq : v / lsq; }
};
template <class T, class V>
__device__ __forceinline__ void put_fieldv(T* Aw, int Lcap, int nq, const PsvDev& d, int rr, int q, int f, V v) {
    int im;
    const long long row = psvk::fld_row(nq, d.Rs1, d.Rf, q, f, rr, &im);
    if (row < 0) return;
    Aw[(size_t)row * Lcap] = (T)v.re;
    Aw[((size_t)row + im) * Lcap] = (T)v.im;
}

// Field rows of every (order, receiver): 3-node interpolation of the
// captured solutions (value and radial derivative), combined with the
// source coefficients of each slot (calup*, locallyCartesianDerivatives
// inputs); fluid receivers store U only.  The cutoff probe is formed by
// k_psv_coef.
template <bool MIXED, int FS>
__global__ void __launch_bounds__(128) k_psv_fields(PsvDev d, WorkList wl, int nsys,
                                                    const cd* __restrict__ Xcap, const cd* __restrict__ co,
                                                    typename std::conditional<MIXED, float, double>::type* __restrict__ A0f,
                                                    typename std::conditional<MIXED, float, double>::type* __restrict__ A1f,
                                                    typename std::conditional<MIXED, float, double>::type* __restrict__ A2f,
                                                    int Lcap, const int* __restrict__ bperm,
                                                    const int* __restrict__ kcut, int* __restrict__ zfirst) {
    using T = typename std::conditional<MIXED, float, double>::type;
    using FM = FieldMath<MIXED>;
    using V = typename FM::V;
    using RT = typename FM::R;
    // the four warps of a block take the same FS orders at 4 x 32/FS
    // neighbouring receivers: the coefficient and capture loads of the
    // orders are shared through L1
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int GPB = 128 / FS;  // order groups per 128-system block (bperm's unit)
    const int sb = bperm ? bperm[blockIdx.x / GPB] : (int)(blockIdx.x / GPB);
    const int sys = sb * 128 + (blockIdx.x % GPB) * FS + lane % FS;
    const int r = (blockIdx.y * 4 + warp) * (32 / FS) + lane / FS;
    const int R = d.R;
    if (sys >= nsys || r > R) return;
    int w, l;
    wl_map(wl, sys, w, l);
    if (l == 0) return;  // written by the order-0 kernels
    const size_t rows[3] = {psvk::fld_rows(NS0, d.Rs1, d.Rf), psvk::fld_rows(NS1, d.Rs1, d.Rf),
                            psvk::fld_rows(NS2, d.Rs1, d.Rf)};
    const int rr = d.rrow[r];
    T* Aw[3] = {A0f + (size_t)w * rows[0] * Lcap + l, A1f + (size_t)w * rows[1] * Lcap + l,
                A2f + (size_t)w * rows[2] * Lcap + l};
    const double l2d = (double)l * (double)(l + 1), lsqd = sqrt(l2d);
    const RT l2 = (RT)l2d, lsq = (RT)lsqd, ilsq = (RT)(1.0 / lsqd);
    auto X = [&](int cap, int b) { return Xcap[((size_t)cap * NB + b) * nsys + sys]; };
    auto C = [&](int s, int b) { return FM::coef(co, ((size_t)s * NB + b) * nsys + sys); };
    // With the depth cut-off, a receiver whose stencil lies below the
    // system's cut row (the same for the warp's 32 orders: a factorisation
    // warp) has zero captures, so every field is zero: written without the
    // loads of the coefficients and captures.
    if (kcut && r < R && d.stop_row[r] < kcut[sys]) {
        // the cut row grows with the order, so this receiver's fields are
        // zero from here on: its lowest order in the warp records that
        if (zfirst && lane % FS == 0) atomicMin(zfirst + (size_t)w * (R + 1) + r, l);
        for (int s = 0; s < NSLOT; ++s) {
            const int mi = slot_mi(s), q = slot_q(s), nqm = mi == 0 ? NS0 : (mi == 1 ? NS1 : NS2);
            const V z = FM::zero();
            if (rr < 0) {
                put_fieldv<T>(Aw[mi], Lcap, nqm, d, rr, q, 0, z);
                continue;
            }
            for (int f = 0; f < 5; ++f) put_fieldv<T>(Aw[mi], Lcap, nqm, d, rr, q, f, z);
        }
        return;
    }
    if (rr < 0) {  // fluid receiver: only U is stored
        V bU[NB];
        for (int b = 0; b < NB; ++b) {
            cd u = mk(0.0);
            for (int i = 0; i < 3; ++i) u = FM::interp(u, d.wv[3 * r + i], X(d.rcap[6 * r + 2 * i], b));
            bU[b] = FM::from(u);
        }
        for (int s = 0; s < NSLOT; ++s) {
            const int mi = slot_mi(s), q = slot_q(s);
            V U = FM::zero();
            for (int b = 0; b < NB; ++b) U = FM::addmul(U, C(s, b), bU[b]);
            put_fieldv<T>(Aw[mi], Lcap, mi == 0 ? NS0 : (mi == 1 ? NS1 : NS2), d, rr, q, 0, U);
        }
        return;
    }
    const bool surf = r == R;
    V bU[NB], bV[NB], bUd[NB], bVd[NB];
    for (int b = 0; b < NB; ++b) {
        cd u = mk(0.0), v = mk(0.0), ud = mk(0.0), vd = mk(0.0);
        if (surf) {
            u = X(d.cap_n1, b);
            v = X(d.cap_n, b);
        } else {
            for (int i = 0; i < 3; ++i) {
                const double wvi = d.wv[3 * r + i], wdi = d.wd[3 * r + i];
                const cd xu = X(d.rcap[6 * r + 2 * i], b), xv = X(d.rcap[6 * r + 2 * i + 1], b);
                u = FM::interp(u, wvi, xu);
                v = FM::interp(v, wvi, xv);
                ud = FM::interp(ud, wdi, xu);
                vd = FM::interp(vd, wdi, xv);
            }
        }
        bU[b] = FM::from(u);
        bV[b] = FM::from(v);
        bUd[b] = FM::from(ud);
        bVd[b] = FM::from(vd);
    }
    for (int s = 0; s < NSLOT; ++s) {
        const int mi = slot_mi(s), q = slot_q(s);
        const bool isback = (s == 3) || (mi == 1 && (q % 4) >= 2);
        V U = FM::zero(), Vv = FM::zero(), Ud = FM::zero(), Vd = FM::zero();
        if (!(surf && isback)) {
            for (int b = 0; b < NB; ++b) {
                const V cb = C(s, b);
                U = FM::addmul(U, cb, bU[b]);
                Vv = FM::addmul(Vv, cb, bV[b]);
                Ud = FM::addmul(Ud, cb, bUd[b]);
                Vd = FM::addmul(Vd, cb, bVd[b]);
            }
        }
        const V Vh = FM::divl(Vv, lsq, ilsq), Vdh = FM::divl(Vd, lsq, ilsq);
        const int nqm = mi == 0 ? NS0 : (mi == 1 ? NS1 : NS2);
        put_fieldv<T>(Aw[mi], Lcap, nqm, d, rr, q, 0, U);
        put_fieldv<T>(Aw[mi], Lcap, nqm, d, rr, q, 1, Ud);
        put_fieldv<T>(Aw[mi], Lcap, nqm, d, rr, q, 2, Vh);
        put_fieldv<T>(Aw[mi], Lcap, nqm, d, rr, q, 3, Vdh);
        put_fieldv<T>(Aw[mi], Lcap, nqm, d, rr, q, 4, l2 * Vh);
    }
}

// The cutoff test of one frequency is a sequential state machine over
// (l, m); here one warp runs it 32 orders at a time with the same results.
// Per order l >= 1 the updates are m = -2 (l >= 2), -1, 0, 1, 2 (l >= 2);
// only m = 0 has a nonzero amplitude, so
//   maxamp at the m = 0 update = max(carry, 0, amplitudes of orders <= l),
//   ismall after l = 0 when l < lsuf, else ismall + nm (m = 0 small) or the
//   count of updates after m = 0 (not small),
// a prefix maximum and a prefix composition of v -> a v + b (a in {0, 1}),
// both exact.  The exit fires at the first order whose incoming ismall
// exceeds 20.
__device__ __forceinline__ double warp_prefix_max(double x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x = fmax(x, y);
    }
    return x;
}
__global__ void k_psv_scan(int nf, WorkList wl, int Lcap, int maxlmax, double ratl, double tlen,
                           double vtop, double rtop, const int* __restrict__ freqs,
                           const double* __restrict__ amps, CutState* __restrict__ cut,
                           int* __restrict__ status) {
    const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= nf) return;
    CutState c = cut[w];
    if (c.done) return;
    const double omega = 2.0 * kPi * (double)freqs[w] / tlen;
    const int lsuf = (int)(omega * rtop / vtop - 0.5) + 1;
    const int l0 = wl.lb[w], l1 = l0 + wl.off[w + 1] - wl.off[w];
    double mx = c.maxamp;
    int v = c.ismall;
    for (int base = l0; base < l1; base += 32) {
        const int l = base + lane;
        const bool in = l < l1, act = in && l >= 1;
        const double amp = act ? amps[(size_t)w * Lcap + l] : 0.0;
        // an Inf/NaN probe means the solves broke down: stop this frequency
        // and report it (llog -1 marks it) instead of running to maxlmax
        if (__ballot_sync(0xffffffffu, !isfinite(amp))) {
            if (lane == 0) {
                flag_nonfinite(status, true);
                c.done = 1;
                c.norders = l1;
                c.llog = -1;
                cut[w] = c;
            }
            return;
        }
        // maxamp at this order's m = 0 update (the m = -1 update contributes 0)
        const double pm = warp_prefix_max(act ? amp : -1.0, lane);
        const double mxl = fmax(fmax(mx, pm), 0.0);
        double ratio = 0.0;
        if (amp != 0.0 && mxl != 0.0) ratio = amp / mxl;
        const bool small0 = ratio < ratl && l >= lsuf;
        int ra = 1, rb = 0;  // this order's map v -> ra v + rb
        if (act) {
            const int nm = l >= 2 ? 5 : 3, after = l >= 2 ? 2 : 1;
            if (l < lsuf) { ra = 0; rb = 0; }
            else if (small0) { ra = 1; rb = nm; }
            else { ra = 0; rb = after; }
        }
        // inclusive composition over lanes <= this one
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int pa = __shfl_up_sync(0xffffffffu, ra, o), pb = __shfl_up_sync(0xffffffffu, rb, o);
            if (lane >= o) { rb = ra * pb + rb; ra = ra * pa; }
        }
        const int vafter = ra * v + rb;
        int vbefore = __shfl_up_sync(0xffffffffu, vafter, 1);
        if (lane == 0) vbefore = v;
        const unsigned ex = __ballot_sync(0xffffffffu, in && vbefore > 20);
        if (ex) {
            const int e = __ffs(ex) - 1, le = base + e;
            const int ve = __shfl_sync(0xffffffffu, vbefore, e);
            // maxamp after the orders before le (those of this chunk are all active
            // unless one is order 0)
            const double pe = __shfl_sync(0xffffffffu, pm, e > 0 ? e - 1 : 0);
            double me = e > 0 ? fmax(mx, pe) : mx;
            if (e > 0 && base + e - 1 >= 1) me = fmax(me, 0.0);
            if (c.llog > le) c.llog = le;
            c.done = 1;
            c.norders = le;
            c.ismall = ve;
            c.maxamp = me;
            if (lane == 0) cut[w] = c;
            return;
        }
        // carry past the chunk
        const int last = min(31, l1 - 1 - base);
        const double plast = __shfl_sync(0xffffffffu, pm, last);
        const bool any_act = __ballot_sync(0xffffffffu, act) != 0;
        mx = fmax(mx, plast);
        if (any_act) mx = fmax(mx, 0.0);
        v = __shfl_sync(0xffffffffu, vafter, last);
        if (base <= maxlmax && maxlmax < base + 32 && maxlmax < l1) {
            c.done = 1;
            c.norders = maxlmax + 1;
        }
    }
    c.maxamp = mx;
    c.ismall = v;
    if (lane == 0) cut[w] = c;
}

// Depth cut-off of an (omega, l) system.  Below the turning depth of the
// slowest wave the displacement decays like exp(-E(r)),
//   E(r) = int_r^{r_s} kappa dr',  kappa^2 = ((l + 1/2) / r')^2 - (omega / v(r'))^2,
// counting only the evanescent parts (kappa^2 > 0); v is the SV speed in
// solid zones, and fluid zones count as never evanescent (kappa = 0), which
// only keeps more rows.  Starting at the deepest source r_s, the first node
// where E reaches X bounds the amplitude there by exp(-X) of the source's,
// and a zero-displacement boundary there perturbs what reaches the source
// and receivers above by about exp(-2X).  FP32 (a bound, not a result);
// nodes: x = r, y = 1 / v^2 (huge in fluid), z = local row of the node's
// first unknown.  kcut = that row less a margin of four, at most kmax
// (below the source rows).
// kappa grows with l at every node, and so does E: a frequency's lowest
// order in a warp has the lowest cut row of its orders there.  The warp
// computes the cut rows of those systems only (one per frequency it holds),
// each walk spread over the lanes: lane j takes the interval below node
// base - j, a prefix sum over the lanes gives E at each of the 32 nodes, and
// the first lane where E reaches X ends the walk.  Every lane takes the
// warp's lowest cut row, where the factorisation of its 32 systems starts
// anyway: lanes above it keep a few more rows than their own bound needs.
__global__ void k_psv_cutrow(const float4* __restrict__ nodes, int ks, float X, double tlen,
                             const int* __restrict__ freqs, WorkList wl, int nsys, int kmax, int* __restrict__ kcut,
                             int* __restrict__ blkmin) {
    const int sysv = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
    const bool valid = sysv < nsys;
    const int sys = valid ? sysv : nsys - 1;
    int w, l;
    wl_map(wl, sys, w, l);
    const int wprev = __shfl_up_sync(0xffffffffu, w, 1);
    unsigned lead = __ballot_sync(0xffffffffu, valid && (lane == 0 || wprev != w));
    int kc = INT_MAX;
    while (lead) {
        const int src = __ffs(lead) - 1;
        lead &= lead - 1;
        const int ws = __shfl_sync(0xffffffffu, w, src), ls = __shfl_sync(0xffffffffu, l, src);
        const float om = (float)(2.0 * kPi * (double)freqs[ws] / tlen);
        const float lam2 = ((float)ls + 0.5f) * ((float)ls + 0.5f), om2 = om * om;
        auto kappa = [&](float4 v) { return sqrtf(fmaxf(0.0f, lam2 / (v.x * v.x) - om2 * v.y)); };
        float E = 0.0f;
        int row = 1;
        // node max(k, 0) of this pass, and of the next pass (in flight
        // while this one runs); node k - 1 is the next lane's node, or for
        // lane 31 lane 0's node of the next pass
        float4 an = nodes[max(ks - lane, 0)];
        for (int base = ks; base >= 1; base -= 32) {
            const int k = base - lane;  // this lane's interval: node k down to node k - 1
            const bool in = k >= 1;
            const float4 a = an;
            an = nodes[max(base - 32 - lane, 0)];
            const float ka = kappa(a);
            float bx = __shfl_down_sync(0xffffffffu, a.x, 1), bz = __shfl_down_sync(0xffffffffu, a.z, 1);
            float kb = __shfl_down_sync(0xffffffffu, ka, 1);
            const float nx = __shfl_sync(0xffffffffu, an.x, 0), ny = __shfl_sync(0xffffffffu, an.y, 0),
                        nz = __shfl_sync(0xffffffffu, an.z, 0);
            if (lane == 31) {
                bx = nx;
                bz = nz;
                kb = kappa(make_float4(nx, ny, nz, 0.0f));
            }
            const float4 b = make_float4(bx, 0.0f, bz, 0.0f);
            float inc = in ? 0.5f * (ka + kb) * (a.x - b.x) : 0.0f;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            const unsigned hit = __ballot_sync(0xffffffffu, in && E + inc >= X);
            if (hit) {
                const int f = __ffs(hit) - 1;
                row = (int)__shfl_sync(0xffffffffu, b.z, f);
                break;
            }
            E += __shfl_sync(0xffffffffu, inc, 31);
        }
        kc = min(kc, max(1, min(row - 4, kmax)));
    }
    if (!valid) return;
    kcut[sys] = kc;
    if (lane == 0) atomicMin(&blkmin[sys / 128], kc);  // per 128-system block (a factorisation block)
}

// ---------------------------------------------------------------- engine
class PsvEngine : public Engine {
  public:
    PsvDev d{};
    DBuf<int> iphase, nlayer, kkdr, elem, hmoff, blkoff, amz, amc, bcrow, rcap, stoprow, fluid, rrow, comp_src, jsta,
        capmap, l0col, l0e1;
    DBuf<int2> caplist;
    DBuf<double> qmu, qkappa, sel, fel, hm, bcval, poly, lam, qkp, fr, r, rrsta;
    DBuf<cd> B0, B1, B2, Prow, Lst, Zst, Dst, Xcap, Xprobe, l0scr, l0d, ab, co;
    DBuf<int4> rowasm;
    DBuf<SysTail> tails;
    int jmin_loc = 1, ncap = 0;
    // depth cut-off: nodes (radius, 1/v^2, local row) from the centre up,
    // the node at the deepest source, the first kept row per system
    DBuf<float4> cnodes;
    int cnode_src = 0;
    DBuf<int> kcut;
    // launch order of the 128-system blocks of a solve round, the lowest
    // cut row per block, and the stream of the long recurrences
    DBuf<int> bperm, blkmin;
    cudaStream_t st3 = nullptr;
    cudaEvent_t ev_s3a = nullptr, ev_s3b = nullptr;
    // one parameter set per source depth (the source fields differ), and
    // the source polynomials they point to
    std::vector<PsvDev> dsrc;
    DBuf<double> polys;
    int ls_min = 1;  // local first source row of the deepest source
    // source s's slot of the field matrices (element type T)
    template <class T>
    T* afld_of(int m, int s) {
        return reinterpret_cast<T*>(reinterpret_cast<char*>(Afld[m].p) +
                                    (size_t)s * F * rows_m[m] * Lcap * afld_bytes);
    }
    double vtop = 0, rtop = 0;

    PsvEngine(const dsm_psv_setup_t* const* ss, int ns, const dsm_options_t* o) {
        if (!ss || ns < 1 || !ss[0]) throw Error(DSM_ERR_INVALID, "no PSV set-up");
        const dsm_psv_setup_t* s = ss[0];
        for (int k = 1; k < ns; ++k) check_same_grid(s, ss[k]);
        nsrc = ns;
        mode = 1;
        opt = *o;
        init_common(opt.device);
        {  // the long recurrences' stream: its blocks go first when SMs free up
            int lo = 0, hi = 0;
            DSM_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            DSM_CUDA(cudaStreamCreateWithPriority(&st3, cudaStreamNonBlocking, hi));
            DSM_CUDA(cudaEventCreateWithFlags(&ev_s3a, cudaEventDisableTiming));
            DSM_CUDA(cudaEventCreateWithFlags(&ev_s3b, cudaEventDisableTiming));
        }
        // the mixed path splits the fields into 11-bit pieces: FP32 storage
        // (24 bits) loses nothing it keeps and halves their traffic
        afld_bytes = mixed() ? 4 : 8;
        // the substitution's staging rings exceed the default 48 KB
        DSM_CUDA(cudaFuncSetAttribute(k_psv_up<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UP_SMEM));
        DSM_CUDA(cudaFuncSetAttribute(k_psv_up<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UP_SMEM));
        m_lo = 0;
        R = s->r_n;
        Th = s->theta_n;
        num_t = DSM_PSV_NUM_TSGT; num_r = DSM_PSV_NUM_RSGT; num_s = DSM_PSV_NUM_SYNN;
        tlen = s->tlen; omegai = s->omegai; ratl = s->ratl; maxlmax = s->maxlmax;
        imin = s->imin; imax = s->imax;
        rsgt_sw = s->rsgt_switch == 1;
        synn_sw = s->synn_switch == 1;
        const int nz = s->nzone, nn = s->nn;
        if (R <= 0 || Th <= 0 || nz <= 0 || nn <= 4) throw Error(DSM_ERR_INVALID, "empty PSV set-up");
        d.nzone = nz; d.nn = nn; d.R = R; d.Th = Th;
        d.itmp = (s->rmin == 0.0) ? 3 : 1;
        d.jsrc = s->jsrc; d.spn = s->spn;
        if (d.jsrc < d.itmp || d.jsrc + 3 > nn) throw Error(DSM_ERR_INVALID, "source rows outside the system");
        d.n_sel = s->n_sel; d.n_fel = s->n_fel; d.n_hm = s->n_hm;
        d.tlen = tlen; d.omegai = omegai; d.rmax = s->rmax; d.r0 = s->r0;
        d.ecC0 = s->ecC0; d.ecF0 = s->ecF0; d.ecL0 = s->ecL0; d.ra0 = s->ra_src[0]; d.ra1 = s->ra_src[1];
        iphase.upload(s->iphase, nz, st); nlayer.upload(s->nlayer, nz, st); kkdr.upload(s->kkdr, nz, st);
        elem.upload(s->elem, nz, st); hmoff.upload(s->hmoff, nz, st);
        qmu.upload(s->qmu, nz, st); qkappa.upload(s->qkappa, nz, st);
        sel.upload(s->solid_el, (size_t)DSM_PSV_NSOLID * s->n_sel, st);
        fel.upload(s->fluid_el, (size_t)3 * s->n_fel, st);
        hm.upload(s->hm_el, (size_t)DSM_PSV_NHM * 4 * s->n_hm, st);
        poly.upload(s->src_poly, 24, st);
        // zone blocks and the column assembly map
        std::vector<int> bo(nz);
        int tot = 0;
        for (int z = 0; z < nz; ++z) {
            bo[z] = tot;
            tot += (s->iphase[z] == 1) ? 2 * (s->nlayer[z] + 1) : s->nlayer[z] + 1;
        }
        d.ncol_tot = tot;
        blkoff.upload(bo, st);
        std::vector<int> az(2 * (nn + 1), -1), ac(2 * (nn + 1), 0), br(nn + 1, 0);
        std::vector<double> bv(nn + 1, 0.0);
        for (int z = 0; z < nz; ++z) {
            int kk = s->kkdr[z];
            int hi = (s->iphase[z] == 1) ? kk + 2 * s->nlayer[z] + 1 : kk + s->nlayer[z];
            for (int jj = kk; jj <= hi && jj <= nn; ++jj) {
                int e = (az[2 * jj] < 0) ? 0 : 1;
                if (e == 1 && az[2 * jj + 1] >= 0) throw Error(DSM_ERR_INVALID, "three zones overlap a column");
                az[2 * jj + e] = z;
                ac[2 * jj + e] = jj - kk + 1;
            }
        }
        for (int i = 1; i <= nz - 1; ++i) {
            double rv = s->vrmax[i - 1] * s->vrmax[i - 1];
            if (s->iphase[i - 1] == 1 && s->iphase[i] == 2) { br[s->kkdr[i]] = 2; bv[s->kkdr[i]] = rv; }
            if (s->iphase[i - 1] == 2 && s->iphase[i] == 1) { br[s->kkdr[i]] = 3; bv[s->kkdr[i]] = rv; }
        }
        amz.upload(az, st); amc.upload(ac, st); bcrow.upload(br, st); bcval.upload(bv, st);
        {
            std::vector<int4> ra(nn + 1);
            for (int jj = 0; jj <= nn; ++jj) {
                int4 v = make_int4(-1, -1, 0, br[jj]);
                for (int e = 0; e < 2; ++e) {
                    const int z = az[2 * jj + e];
                    if (z < 0) break;
                    const int o = (bo[z] + ac[2 * jj + e] - 1) * 4;
                    if (e == 0) v.x = o; else v.y = o;
                    if (s->iphase[z] == 1) v.z |= 1 << e;
                }
                ra[jj] = v;
            }
            rowasm.upload(ra, st);
        }
        // receivers
        r.upload(s->r, R, st);
        rrsta.upload(s->rrsta, 3 * (size_t)R, st);
        std::vector<int> ks(R), fl(R), cm(nn + 1, -1), rc(6 * (size_t)R);
        std::vector<double> frv(R);
        int jmin = nn;
        auto addcap = [&](int j) {
            if (j < d.itmp || j > nn) throw Error(DSM_ERR_INVALID, "receiver stencil outside the system");
            if (cm[j] < 0) cm[j] = ncap++;
            jmin = std::min(jmin, j);
            return cm[j];
        };
        for (int ir = 0; ir < R; ++ir) {
            int z = s->istazone[ir] - 1;
            ks[ir] = s->kkdr[z] + 2 * s->iista[3 * ir] - 1;
            fl[ir] = s->iphase[z] == 2;
            frv[ir] = (double)(float)s->r[ir];
            for (int k = 0; k < 6; ++k) rc[6 * ir + k] = addcap(ks[ir] - 1 + k);
        }
        d.cap_n1 = addcap(nn - 1);
        d.cap_n = addcap(nn);
        d.cap_p0 = cm[ks[R - 1] - 1];
        d.cap_p1 = cm[ks[R - 1]];

        jmin_loc = jmin - d.itmp + 1;
        capmap.upload(cm, st); rcap.upload(rc, st); fluid.upload(fl, st);
        {
            std::vector<int> rt(R);
            for (int ir = 0; ir < R; ++ir) rt[ir] = ks[ir] + 4 - d.itmp + 1;
            stoprow.upload(rt, st);
        }
        {  // receiver rows of the field matrices: solid class (with the surface) and fluid
            std::vector<int> rw(R + 1);
            int ns = 0, nf = 0;
            for (int ir = 0; ir < R; ++ir) rw[ir] = fl[ir] ? -(++nf) : ns++;
            rw[R] = ns++;
            d.Rs1 = ns;
            d.Rf = nf;
            rrow.upload(rw, st);
            d.rrow = rrow.p;
        }
        {  // captured rows below n - 1 in descending order, for the upward substitution
            std::vector<int2> cl;
            const int nloc = nn - d.itmp + 1;
            for (int j = nloc - 2; j >= jmin_loc; --j)
                if (cm[j + d.itmp - 1] >= 0) cl.push_back(make_int2(j, cm[j + d.itmp - 1]));
            cl.push_back(make_int2(-1, -1));
            caplist.upload(cl, st);
        }
        lam.upload(s->lambda, R, st); qkp.upload(s->qkp, R, st); fr.upload(frv, st);
        // l = 0 compaction (rea2): jsta, compact row of every kept global row
        {
            std::vector<int> js(R, 0), cs(nn + 1, 0), lc(nn + 2, 0), le(nn + 2, 0);
            int itmp = 0;
            for (int iz = 0; iz < nz; ++iz) {
                for (int ir = 0; ir < R; ++ir)
                    if (iz + 1 == s->istazone[ir]) js[ir] = itmp + s->iista[3 * ir];
                int kk = s->kkdr[iz], i1 = itmp + 1, i2;
                if (s->iphase[iz] == 1) {
                    i2 = (iz != nz - 1) ? i1 + (s->kkdr[iz + 1] - kk) / 2 - 1 : i1 + (nn + 1 - kk) / 2 - 1;
                    for (int i = i1; i <= i2; ++i) {
                        cs[kk + 2 * (i - i1)] = i;
                        lc[i] = kk + 2 * (i - i1);
                        le[i] = (i == i1) ? (iz == 0 ? 0 : (s->iphase[iz - 1] == 2 ? 3 : 2)) : 2;
                    }
                } else {
                    i2 = i1 + (s->kkdr[iz + 1] - kk) - 1;
                    for (int i = i1; i <= i2; ++i) {
                        cs[kk + (i - i1)] = i;
                        lc[i] = kk + (i - i1);
                        le[i] = (i == i1) ? (iz == 0 ? 0 : (s->iphase[iz - 1] == 1 ? 2 : 3)) : 3;
                    }
                }
                itmp = i2;
            }
            lc.resize(itmp + 1);
            le.resize(itmp + 1);
            l0col.upload(lc, st);
            l0e1.upload(le, st);
            d.nn0 = itmp;
            d.itmp0 = (s->rmin == 0.0) ? 2 : 1;
            jsta.upload(js, st);
            comp_src.upload(cs, st);
            for (int ir = 0; ir < R; ++ir)
                if (js[ir] < 1 || js[ir] + 2 > d.nn0) throw Error(DSM_ERR_INVALID, "receiver outside the l=0 system");
        }
        vtop = 0.0;
        for (int i = 0; i < 4; ++i) vtop = vtop + s->vsv[4 * (nz - 1) + i] * 1.0;
        rtop = s->vrmax[nz - 1];
        vtop_ = vtop;
        rtop_ = rtop;
        set_summaries(1, nz, s->vrmin, s->vrmax, s->vsv, s->qmu, s->r0, s->r[R - 1]);
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
        d.iphase = iphase.p; d.nlayer = nlayer.p; d.kkdr = kkdr.p; d.elem = elem.p; d.hmoff = hmoff.p;
        d.blkoff = blkoff.p; d.qmu = qmu.p; d.qkappa = qkappa.p; d.sel = sel.p; d.fel = fel.p; d.hm = hm.p;
        d.amz = amz.p; d.amc = amc.p; d.bcrow = bcrow.p; d.bcval = bcval.p; d.poly = poly.p;
        d.rowasm = rowasm.p;
        d.rcap = rcap.p; d.stop_row = stoprow.p; d.wv = wv.p; d.wd = wd.p; d.fluid = fluid.p; d.lam = lam.p; d.qkp = qkp.p;
        d.fr = fr.p; d.comp_src = comp_src.p; d.jsta = jsta.p;
        // per-source parameter sets: the fields set by the source position
        {
            std::vector<double> pl(24 * (size_t)nsrc);
            for (int k = 0; k < nsrc; ++k)
                for (int i = 0; i < 24; ++i) pl[24 * (size_t)k + i] = ss[k]->src_poly[i];
            polys.upload(pl, st);
            dsrc.assign(nsrc, d);
            ls_min = d.nn;
            for (int k = 0; k < nsrc; ++k) {
                const dsm_psv_setup_t* q = ss[k];
                PsvDev& e = dsrc[k];
                e.jsrc = q->jsrc;
                e.spn = q->spn;
                if (e.jsrc < e.itmp || e.jsrc + 3 > nn) throw Error(DSM_ERR_INVALID, "source rows outside the system");
                e.r0 = q->r0;
                e.ecC0 = q->ecC0; e.ecF0 = q->ecF0; e.ecL0 = q->ecL0;
                e.ra0 = q->ra_src[0]; e.ra1 = q->ra_src[1];
                e.poly = polys.p + 24 * (size_t)k;
                ls_min = std::min(ls_min, e.jsrc - e.itmp + 1);
            }
            d = dsrc[0];
        }
        {  // nodes of the depth cut-off (the grid of calra2_psv, its unknowns of calspdr)
            std::vector<float4> nd;
            double r0min = s->r0;
            for (int k = 1; k < nsrc; ++k) r0min = std::min(r0min, ss[k]->r0);
            auto inv_v2 = [&](int z, double rr) {
                if (s->iphase[z] != 1) return 1e30;
                double v = 0.0, x = 1.0;
                for (int j = 0; j < 4; ++j, x *= rr / s->rmax) v += s->vsv[4 * z + j] * x;
                return v > 0.0 ? 1.0 / (v * v) : 1e30;
            };
            nd.push_back(make_float4((float)s->vrmin[0], (float)inv_v2(0, s->vrmin[0]),
                                     (float)(s->kkdr[0] - d.itmp + 1), 0.0f));
            for (int z = 0; z < nz; ++z) {
                const int nl = s->nlayer[z];
                for (int i = 1; i <= nl; ++i) {
                    const double rr = s->vrmin[z] + (s->vrmax[z] - s->vrmin[z]) * (double)i / (double)nl;
                    double iv = inv_v2(z, rr);
                    if (i == nl && z + 1 < nz) iv = std::max(iv, inv_v2(z + 1, rr));  // the slower side
                    const int row = s->kkdr[z] + (s->iphase[z] == 1 ? 2 * i : i);
                    nd.push_back(make_float4((float)rr, (float)iv, (float)(row - d.itmp + 1), 0.0f));
                }
            }
            cnode_src = 0;
            for (int k = 0; k < (int)nd.size(); ++k)
                if ((double)nd[k].x <= r0min) cnode_src = k;
            cnodes.upload(nd, st);
        }
        depth_bound = mixed() ? 1e-20 : 0.0;
        F = opt.freq_batch > 0 ? opt.freq_batch : 8;
        Lc = opt.l_chunk > 0 ? ((opt.l_chunk + 31) / 32) * 32 : 256;
        Lcap = std::min(maxlmax + 1 + Lc, 2048);
        amp_k = 1;
        rows_m[0] = (int)psvk::fld_rows(NS0, d.Rs1, d.Rf);
        rows_m[1] = (int)psvk::fld_rows(NS1, d.Rs1, d.Rf);
        rows_m[2] = (int)psvk::fld_rows(NS2, d.Rs1, d.Rf);
        rows_full[0] = (int)psvk::fld_rows_full(NS0, d.Rs1);
        rows_full[1] = (int)psvk::fld_rows_full(NS1, d.Rs1);
        rows_full[2] = (int)psvk::fld_rows_full(NS2, d.Rs1);
        // contraction outputs row-major: the epilogue's lanes take
        // consecutive distances of one row (the rows of a receiver are
        // adjacent, psvk::fld_row)
        c_rowmajor = true;
        c_ld = (2 * Th + 3) / 4 * 4;
        {  // receiver row (0..R) of each field row, for the split's zero orders
            std::vector<int> solid_r(d.Rs1, R), fluid_r(std::max(d.Rf, 1), 0);
            std::vector<int> rw(R + 1);
            DSM_CUDA(cudaStreamSynchronize(st));  // rrow was uploaded on st
            DSM_CUDA(cudaMemcpy(rw.data(), rrow.p, sizeof(int) * (R + 1), cudaMemcpyDeviceToHost));
            for (int ir = 0; ir < R; ++ir) {
                if (rw[ir] >= 0) solid_r[rw[ir]] = ir;
                else fluid_r[-rw[ir] - 1] = ir;
            }
            const int nqs[3] = {NS0, NS1, NS2};
            for (int m = 0; m < 3; ++m) {
                std::vector<int> rr_of(rows_m[m], R);
                for (int rr = 0; rr < d.Rs1; ++rr)
                    for (int q = 0; q < nqs[m]; ++q)
                        for (int f = 0; f < 5; ++f) {
                            int im;
                            const long long row = psvk::fld_row(nqs[m], d.Rs1, d.Rf, q, f, rr, &im);
                            rr_of[row] = rr_of[row + im] = solid_r[rr];
                        }
                for (int fi = 0; fi < d.Rf; ++fi)
                    for (int q = 0; q < nqs[m]; ++q) {
                        int im;
                        const long long row = psvk::fld_row(nqs[m], d.Rs1, d.Rf, q, 0, -fi - 1, &im);
                        rr_of[row] = rr_of[row + im] = fluid_r[fi];
                    }
                rowrec[m].upload(rr_of, st);
            }
            zfirst.reserve((size_t)nsrc * F * (R + 1));
            use_zfirst = mixed();
        }
        alloc_batch();
        build_basis(std::min(maxlmax + 1, 2048));
        DSM_CUDA(cudaStreamSynchronize(st));
    }

    ~PsvEngine() override {
        if (st3) {
            cudaStreamSynchronize(st3);
            cudaStreamDestroy(st3);
        }
        if (ev_s3a) cudaEventDestroy(ev_s3a);
        if (ev_s3b) cudaEventDestroy(ev_s3b);
    }

    // every source of a context shares the model, grid, receivers and
    // distances; only the source fields may differ
    static void check_same_grid(const dsm_psv_setup_t* a, const dsm_psv_setup_t* b) {
        if (!b) throw Error(DSM_ERR_INVALID, "null PSV set-up");
        auto same = [](const void* x, const void* y, size_t bytes) {
            return bytes == 0 || (x && y && std::memcmp(x, y, bytes) == 0);
        };
        const bool ok =
            a->nzone == b->nzone && a->nn == b->nn && a->r_n == b->r_n && a->theta_n == b->theta_n &&
            a->n_sel == b->n_sel && a->n_fel == b->n_fel && a->n_hm == b->n_hm && a->rmin == b->rmin &&
            a->rmax == b->rmax && a->tlen == b->tlen && a->omegai == b->omegai && a->ratl == b->ratl &&
            a->maxlmax == b->maxlmax && a->rsgt_switch == b->rsgt_switch && a->synn_switch == b->synn_switch &&
            same(a->iphase, b->iphase, sizeof(int) * a->nzone) && same(a->nlayer, b->nlayer, sizeof(int) * a->nzone) &&
            same(a->kkdr, b->kkdr, sizeof(int) * a->nzone) && same(a->elem, b->elem, sizeof(int) * a->nzone) &&
            same(a->hmoff, b->hmoff, sizeof(int) * a->nzone) && same(a->qmu, b->qmu, sizeof(double) * a->nzone) &&
            same(a->qkappa, b->qkappa, sizeof(double) * a->nzone) &&
            same(a->solid_el, b->solid_el, sizeof(double) * DSM_PSV_NSOLID * a->n_sel) &&
            same(a->fluid_el, b->fluid_el, sizeof(double) * 3 * a->n_fel) &&
            same(a->hm_el, b->hm_el, sizeof(double) * DSM_PSV_NHM * 4 * a->n_hm) &&
            same(a->r, b->r, sizeof(double) * a->r_n) && same(a->rrsta, b->rrsta, sizeof(double) * 3 * a->r_n) &&
            same(a->iista, b->iista, sizeof(int) * 3 * a->r_n) &&
            same(a->istazone, b->istazone, sizeof(int) * a->r_n) &&
            same(a->theta, b->theta, sizeof(double) * a->theta_n);
        if (!ok)
            throw Error(DSM_ERR_INVALID,
                        "the sources of a context must share the model, grid, receivers and distances");
    }

    // first local row whose multipliers a substitution reads: the deepest
    // captured row or three rows below the deepest source
    int lst_min() const { return std::max(1, std::min(jmin_loc, ls_min - 3)); }

    void alloc_batch() {
        size_t n = (size_t)d.nn - d.itmp + 1;
        const size_t ls = (size_t)ls_min;  // scratch of the deepest source's forward substitution
        const size_t lrows = n - (size_t)lst_min() + 2;  // multiplier rows held (from lst_min up)
        size_t per = lrows * 3 * 16 + (n - ls + 2) * 5 * 16 + (size_t)ncap * NB * 16 + NSLOT * NB * 16;
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        // What the rest of a run allocates later, at the order capacity the
        // top frequency's first range needs: the field matrices (while they
        // grow, old and new copies), the split pieces and contraction output
        // of the mixed path, the batch outputs, and a margin.  The solve
        // scratch takes what is left, so that a batch's first ranges fit one
        // launch (one long low-order recurrence per batch, not one per round).
        size_t lfut = (size_t)Lcap;
        while (lfut < (size_t)first_span(imax) + 64 && lfut < (size_t)maxlmax + 1 + Lc) lfut *= 2;
        lfut = std::min(lfut, (size_t)maxlmax + 1 + Lc);
        size_t rows_all = 0;
        for (int m = 0; m < 3; ++m) rows_all += (size_t)rows_m[m];
        size_t pt, pr, ps;
        out_sizes(&pt, &pr, &ps);
        const size_t later = rows_all * lfut * (size_t)nsrc * F * afld_bytes * 3 / 2 +
                             (mixed() ? rows_all * lfut * F * 4 + c_total() * F * 4 : c_total() * 8) +
                             2 * (pt + pr + ps) * F * nsrc * 8 + ((size_t)4 << 30);
        const size_t avail = fr > later ? fr - later : 0;
        nsys_max = (int)std::max<size_t>(1024, std::min<size_t>(131072, avail / per));
        // no more than a round of a batch can launch (F ranges of at most
        // max(4096, the first range of the top frequency)): contexts that
        // share a device leave each other room
        nsys_max = std::min(nsys_max, std::max(1024, F * std::max(4096, first_span(imax))));
        // DSM_MAX_SYSTEMS caps the systems per solve launch (and so the
        // factor scratch) below that, e.g. for small profiling captures
        if (const char* e = std::getenv("DSM_MAX_SYSTEMS")) nsys_max = std::max(1024, std::min(nsys_max, std::atoi(e)));
        size_t nsys = nsys_max;
        B0.reserve((size_t)F * d.ncol_tot * 4);
        B1.reserve((size_t)F * d.ncol_tot * 4);
        B2.reserve((size_t)F * d.ncol_tot * 4);
        Prow.reserve((size_t)F * (d.nn + 1) * 12);
        Lst.reserve(lrows * 3 * nsys);
        Zst.reserve((n - ls + 2) * 4 * nsys);
        Dst.reserve((n - ls + 2) * nsys);
        Xcap.reserve((size_t)ncap * NB * nsys);
        Xprobe.reserve((size_t)8 * nsys);
        tails.reserve(nsys);
        kcut.reserve(nsys);
        l0scr.reserve((size_t)F * (d.nn0 + 1) * 2);
        l0d.reserve((size_t)F * (d.nn0 + 1) * 4);
        ab.reserve((size_t)nsrc * F * 320);
        co.reserve((size_t)NSLOT * NB * nsys);
        for (int m = 0; m < 3; ++m) Afld[m].reserve(((size_t)nsrc * F * rows_m[m] * Lcap * afld_bytes + 7) / 8);
        Cgemm.reserve(c_total());
        cut.reserve((size_t)nsrc * F);
        amps.reserve((size_t)nsrc * F * Lcap);
        out_t.reserve(2 * pt * F * nsrc);
        out_r.reserve(2 * pr * F * nsrc);
        out_s.reserve(2 * ps * F * nsrc);
    }

    size_t out_sizes(size_t* nt, size_t* nr, size_t* ns) const override {
        *nt = (size_t)num_t * R * Th;
        *nr = (size_t)num_r * R * Th;
        *ns = (size_t)num_s * Th;
        return *nt;
    }

    bool l0_done = false;
    void omega_pieces(const int* fr_, int nf) override {
        l0_done = false;
        // first zero order per receiver row: none yet (0x7f7f7f7f)
        if (use_zfirst) DSM_CUDA(cudaMemsetAsync(zfirst.p, 0x7f, sizeof(int) * (size_t)nsrc * F * (R + 1), st));
        dim3 grid((d.ncol_tot + 127) / 128, nf);
        int id = kid("psv_omega_blocks");
        kbegin(id);
        k_psv_omega<<<grid, 128, 0, st>>>(d, fr_, B0.p, B1.p, B2.p);
        DSM_LAUNCH(*this);
        k_psv_rows<<<dim3((d.nn + 1 + 127) / 128, nf), 128, 0, st>>>(d, B0.p, B1.p, B2.p, Prow.p);
        kend(id, 0.0, 0.0);
        DSM_LAUNCH(*this);
        for (int k = 0; k < nsrc; ++k) {
            k_psv_abnum<<<(nf + 31) / 32, 32, 0, st>>>(dsrc[k], fr_, nf, ab.p + (size_t)k * F * 320);
            DSM_LAUNCH(*this);
        }
    }

    void solve_chunk(const int* fr_, int nf, const WorkList& wl, int nsys) override {
        if (!l0_done) {  // order 0 once per batch (its own tridiagonal system)
            // order 0 is independent of the other orders: it runs on the side
            // stream while the band solves run, and joins before the l-sum.
            // Its solve factors the compact band in place: every source
            // rebuilds it first.
            fork_side();
            int id0 = kid("psv_order0");
            kbegin(id0, st2);
            for (int k = 0; k < nsrc; ++k) {
                const PsvDev& e = dsrc[k];
                const cd* abk = ab.p + (size_t)k * F * 320;
                k_psv_l0_build<<<dim3((d.nn0 + 127) / 128, nf), 128, 0, st2>>>(e, B0.p, B1.p, B2.p, l0col.p,
                                                                                l0e1.p, l0scr.p);
                if (mixed()) k_psv_l0_solve<true><<<nf, 128, 0, st2>>>(e, fr_, nf, abk, l0scr.p, l0d.p, rsgt_sw);
                else k_psv_l0_solve<false><<<nf, 128, 0, st2>>>(e, fr_, nf, abk, l0scr.p, l0d.p, rsgt_sw);
                if (afld_bytes == 4)
                    k_psv_l0_fields<float><<<dim3((R + 1 + 127) / 128, nf), 128, 0, st2>>>(
                        e, l0d.p, afld_of<float>(0, k), afld_of<float>(1, k), afld_of<float>(2, k), Lcap, rsgt_sw);
                else
                    k_psv_l0_fields<double><<<dim3((R + 1 + 127) / 128, nf), 128, 0, st2>>>(
                        e, l0d.p, afld_of<double>(0, k), afld_of<double>(1, k), afld_of<double>(2, k), Lcap,
                        rsgt_sw);
                DSM_LAUNCH(*this);
            }
            kend(id0, 0.0, 0.0, st2);
            l0_done = true;
        }
        // algorithmic bytes per system: the factorisation writes the three
        // multipliers of every row the substitutions read (rows lmin .. n)
        // and the pivots above the deepest source; per source, the forward
        // substitution writes zh of its four bases above its source, and
        // the upward substitution reads the multipliers and zh back and
        // stores six solutions at the captured rows
        const int n = d.nn - d.itmp + 1;
        const int lmin = lst_min();
        // Lst holds rows lmin .. n: kernels index rows from 0 off this base
        cd* const Lb = Lst.p - (size_t)lmin * 3 * nsys;
        const int nblk = (nsys + FAC_THREADS - 1) / FAC_THREADS;
        const int dmin = ls_min;  // pivots from the deepest source row up
        const int* kc = nullptr;
        // Block order and split.  With the depth cut, each 128-system block's
        // lowest first row comes back to the host: blocks go longest
        // recurrence first, and those whose recurrence spans more than 60 %
        // of the band run their whole solve chain (factorisation,
        // substitutions, coefficients, fields) on a second stream beside the
        // rest, so the short systems' substitutions and fields overlap the
        // long factorisations.  Without the cut every recurrence is the
        // whole band: blocks go by their rank inside their frequency's order
        // range, one stream.
        std::vector<int> order(nblk);
        std::vector<int> brow(nblk, 1);  // first factored row of each block (the cut's block minimum)
        int nlong = 0;
        if (depth_bound > 0.0 && ls_min > 9) {
            blkmin.reserve(nblk);
            DSM_CUDA(cudaMemsetAsync(blkmin.p, 0x7f, sizeof(int) * nblk, st));
            k_psv_cutrow<<<(nsys + 127) / 128, 128, 0, st>>>(cnodes.p, cnode_src, (float)-std::log(depth_bound),
                                                             d.tlen, fr_, wl, nsys, ls_min - 8, kcut.p, blkmin.p);
            DSM_LAUNCH(*this);
            kc = kcut.p;
            std::vector<int> bm(nblk);
            DSM_CUDA(cudaMemcpyAsync(bm.data(), blkmin.p, sizeof(int) * nblk, cudaMemcpyDeviceToHost, st));
            DSM_CUDA(cudaStreamSynchronize(st));
            for (int b = 0; b < nblk; ++b) {
                order[b] = b;
                brow[b] = std::max(1, std::min(bm[b], n));
            }
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return bm[a] < bm[b]; });
            const int lim = (int)(0.4 * n);
            for (int b = 0; b < nblk; ++b) nlong += bm[b] < lim ? 1 : 0;
            if (nlong == nblk) nlong = 0;
        } else {
            std::vector<int> rank(nblk);
            for (int b = 0; b < nblk; ++b) {
                const int s0 = b * FAC_THREADS, s1 = std::min(nsys, s0 + FAC_THREADS);
                int r = INT32_MAX;
                for (int w = 0; w < nf; ++w) {
                    const int lo = std::max(s0, wl_host_off[w]), hi = std::min(s1, wl_host_off[w + 1]);
                    if (lo < hi) r = std::min(r, (lo - wl_host_off[w]) / FAC_THREADS);
                }
                rank[b] = r;
                order[b] = b;
            }
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rank[a] < rank[b]; });
        }
        bperm.upload(order, st);
        // source 0's forward pass rides along the factorisation (its first
        // source row must lie above the band's first rows)
        const int ls0 = dsrc[0].jsrc - dsrc[0].itmp + 1;
        const int lsf = tune.fwd_merge && ls0 > 3 && ls0 + 8 <= n ? ls0 : -1;
        const int fs = tune.fld_orders == 16 ? 16 : 32, frec = 32 / fs;
        // the solve chain of blocks bp[0 .. nb) on stream s
        // the long recurrences' chain reports its kernels under their own
        // names (..._long): its length bounds the solve phase
        auto chain = [&](cudaStream_t s, const int* bp, int nb) {
            const std::string sfx = s == st3 ? "_long" : "";
            // algorithmic bytes count the rows each block factors and reads
            // (from its first factored row, or the deepest row read, up)
            const int* ob = order.data() + (bp - bperm.p);
            double rows_fac = 0.0, rows_sub = 0.0;
            for (int i = 0; i < nb; ++i) {
                const int b = ob[i], nsb_b = std::min(FAC_THREADS, nsys - b * FAC_THREADS);
                rows_fac += (double)(n - std::max(lmin, brow[b]) + 1) * nsb_b;
                rows_sub += (double)(n - std::max(jmin_loc, brow[b]) + 1) * nsb_b;
            }
            auto kname = [&](const char* base) { return kid((std::string(base) + sfx).c_str()); };
            int id = kname("psv_factor");
            kbegin(id, s);
            auto factor = [&](auto kern) {
                kern<<<nb, FAC_THREADS, 0, s>>>(d, Prow.p, wl, nsys, lmin, Lb, tails.p, Dst.p, dmin, kc, bp, lsf,
                                                Zst.p);
            };
            if (lsf > 0) {
                if (mixed()) {
                    if (tune.fac_rows == 8) factor(k_psv_solve<true, 8, true>);
                    else factor(k_psv_solve<true, 16, true>);
                } else {
                    if (tune.fac_rows == 8) factor(k_psv_solve<false, 8, true>);
                    else factor(k_psv_solve<false, 16, true>);
                }
            } else {
                if (mixed()) {
                    if (tune.fac_rows == 8) factor(k_psv_solve<true, 8, false>);
                    else factor(k_psv_solve<true, 16, false>);
                } else {
                    if (tune.fac_rows == 8) factor(k_psv_solve<false, 8, false>);
                    else factor(k_psv_solve<false, 16, false>);
                }
            }
            kend(id, rows_fac * 3 * 16.0 + (double)(n - ls_min + 1) * 16.0 * std::min(nsys, nb * FAC_THREADS), 0.0,
                 s);
            DSM_LAUNCH(*this);
            for (int k = 0; k < nsrc; ++k) {
                const PsvDev& e = dsrc[k];
                const int ls = e.jsrc - e.itmp + 1;
                const double nsb = std::min(nsys, nb * FAC_THREADS);
                const double fwd_bytes = (double)(n - ls + 1) * (4 * 16.0 + 3 * 16.0 + 16.0);
                const double sub_bytes = (double)(n - ls + 1) * 4 * 16.0 + (double)ncap * NB * 16.0;
                if (!(k == 0 && lsf > 0)) {  // otherwise done by the factorisation
                    id = kname("psv_forward");
                    kbegin(id, s);
                    if (mixed())
                        k_psv_fwd<true><<<nb, FAC_THREADS, 0, s>>>(e, nsys, ls, Lb, Dst.p, dmin, tails.p, Zst.p, bp);
                    else
                        k_psv_fwd<false><<<nb, FAC_THREADS, 0, s>>>(e, nsys, ls, Lb, Dst.p, dmin, tails.p, Zst.p, bp);
                    kend(id, fwd_bytes * nsb, 0.0, s);
                    DSM_LAUNCH(*this);
                }
                id = kname("psv_substitution");
                kbegin(id, s);
                if (mixed())
                    k_psv_up<true><<<nb, UP_THREADS, UP_SMEM, s>>>(e, nsys, jmin_loc, capmap.p, caplist.p, Lb, Zst.p,
                                                                  tails.p, Xcap.p, kc, bp, Xprobe.p);
                else
                    k_psv_up<false><<<nb, UP_THREADS, UP_SMEM, s>>>(e, nsys, jmin_loc, capmap.p, caplist.p, Lb,
                                                                   Zst.p, tails.p, Xcap.p, kc, bp, Xprobe.p);
                kend(id, rows_sub * 3 * 16.0 + sub_bytes * nsb, 0.0, s);
                DSM_LAUNCH(*this);
                id = kname("psv_source_coef");
                kbegin(id, s);
                double* amk = amps.p + (size_t)k * F * Lcap;
                k_psv_coef<<<nb, 128, 0, s>>>(e, fr_, wl, nsys, ab.p + (size_t)k * F * 320, co.p, rsgt_sw,
                                               Xprobe.p, amk, Lcap, bp);
                kend(id, 0.0, 0.0, s);
                DSM_LAUNCH(*this);
                dim3 grid((unsigned)(nb * (128 / fs)), (R + 1 + 4 * frec - 1) / (4 * frec));
                id = kname("psv_fields");
                kbegin(id, s);
                if (afld_bytes == 4) {
                    auto kern = fs == 16 ? k_psv_fields<true, 16> : k_psv_fields<true, 32>;
                    kern<<<grid, 128, 0, s>>>(e, wl, nsys, Xcap.p, co.p, afld_of<float>(0, k), afld_of<float>(1, k),
                                              afld_of<float>(2, k), Lcap, bp, kc,
                                              use_zfirst && kc ? zfirst.p + (size_t)k * F * (R + 1) : nullptr);
                } else {
                    auto kern = fs == 16 ? k_psv_fields<false, 16> : k_psv_fields<false, 32>;
                    kern<<<grid, 128, 0, s>>>(e, wl, nsys, Xcap.p, co.p, afld_of<double>(0, k), afld_of<double>(1, k),
                                              afld_of<double>(2, k), Lcap, bp, kc, nullptr);
                }
                kend(id, 0.0, 0.0, s);
                DSM_LAUNCH(*this);
                stats.solve_bytes += (k == 0 ? rows_fac * 3 * 16.0 + (double)(n - ls_min + 1) * 16.0 * nsb : 0.0) +
                                     rows_sub * 3 * 16.0 + (fwd_bytes + sub_bytes) * nsb;
            }
        };
        if (nlong > 0) {
            DSM_CUDA(cudaEventRecord(ev_s3a, st));
            DSM_CUDA(cudaStreamWaitEvent(st3, ev_s3a, 0));
            chain(st3, bperm.p, nlong);                 // the long recurrences
            chain(st, bperm.p + nlong, nblk - nlong);   // the rest
            DSM_CUDA(cudaEventRecord(ev_s3b, st3));
            DSM_CUDA(cudaStreamWaitEvent(st, ev_s3b, 0));
        } else {
            chain(st, bperm.p, nblk);
        }
    }

    void scan_chunk(int nf, const WorkList& wl) override {
        int id = kid("psv_cutoff_scan");
        kbegin(id);
        for (int k = 0; k < nsrc; ++k) {
            k_psv_scan<<<(nf + 3) / 4, 128, 0, st>>>(nf, wl, Lcap, maxlmax, ratl, tlen, vtop, rtop, d_freqs.p,
                                                      amps.p + (size_t)k * F * Lcap, cut.p + (size_t)k * F,
                                                      dstatus());
            DSM_LAUNCH(*this);
        }
        kend(id, 0.0, 0.0);
    }

    void epilogue(const int* fr_, int w, int nf, cudaStream_t s) override {
        (void)nf;
        psvk::EpiDev e{};
        e.R = R;
        e.Th = Th;
        e.tlen = d.tlen;
        e.omegai = d.omegai;
        e.fluid = d.fluid;
        e.Rs1 = d.Rs1;
        e.Rf = d.Rf;
        e.rrow = d.rrow;
        e.lam = d.lam;
        e.qkp = d.qkp;
        e.fr = d.fr;
        e.status = dstatus();
        e.c_ld = c_ld;
        int id = kid("psv_epilogue");
        kbegin(id, s);
        const bool tc = mixed();
        const void* c0 = tc ? (const void*)c32(w, 0) : (const void*)c64(0);
        const void* c1 = tc ? (const void*)c32(w, 1) : (const void*)c64(1);
        const void* c2 = tc ? (const void*)c32(w, 2) : (const void*)c64(2);
        psvk::launch_epilogue(e, w, th.x.p, th.s.p, th.pole.p, fr_, c0, c1, c2, tc, out_t_src(),
                              rsgt_sw ? out_r_src() : nullptr, synn_sw ? out_s_src() : nullptr, s);
        kend(id, 0.0, 0.0, s);
        DSM_LAUNCH(*this);
    }
};

}  // namespace

Engine* make_psv_engine(const dsm_psv_setup_t* const* s, int nsrc, const dsm_options_t* o) {
    return new PsvEngine(s, nsrc, o);
}

}  // namespace dsm
