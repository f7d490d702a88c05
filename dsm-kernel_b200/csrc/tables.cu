// Omega-independent tables of the engine and the output packing kernel.
//
// * Vector-harmonic basis tables.  The reference recomputes the associated
//   Legendre recurrence for every (omega, l, theta) (calplm +
//   caldvecphi0_withplm, src/SGTpsv/trial.f90:97-323; calbvecphi0,
//   src/SGTsh/trial.f90:1-118).  The values do not depend on omega, so they
//   are built once per context, for m = 0..2, as the two real functions
//   every vector harmonic is made of:
//       Pbar(l,m,theta) = c_lm P_l^m(cos theta)
//       Dbar(l,m,theta) = c_lm (m cos/sin P_l^m + P_l^{m+1})
//   with c_lm = sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!).  The recurrence runs with
//   round-to-nearest intrinsics (no fused multiply-add) in the reference's
//   operation order, so it reproduces the Fortran values.
// * Three-node interpolation weights of the receivers (interpolate +
//   glu, src/SGTpsv/others.f90:1170-1212, src/SGTpsv/glu2.f90).
// * complex128 -> complex64 packing in catalogue record order (the cast of
//   src/SGTpsv/SGTpsv-MPI.f90:1115-1116).
#include "engine.cuh"

namespace dsm {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// calplm (src/SGTsh/trial.f90:85-118) for one (l, m) step
__device__ void plm_step(int l, int m, double x, double* p) {
    if (l == m) {
        double pmm = 1.0;
        if (m > 0) {
            double somx2 = __dsqrt_rn(mul(sub(1.0, x), add(1.0, x)));
            double fact = 1.0;
            for (int i = 1; i <= m; ++i) {
                pmm = mul(mul(-pmm, fact), somx2);
                fact = add(fact, 2.0);
            }
        }
        p[2] = 0.0;
        p[1] = 0.0;
        p[0] = pmm;
    } else {
        p[2] = p[1];
        p[1] = p[0];
        if (l == m + 1) p[0] = mul(mul(x, (double)(2 * m + 1)), p[1]);
        else
            p[0] = dvd(sub(mul(mul(x, (double)(2 * l - 1)), p[1]), mul((double)(l + m - 1), p[2])),
                       (double)(l - m));
    }
}

__global__ void k_basis(int th_n, const double* __restrict__ xs, const double* __restrict__ ss,
                        const int* __restrict__ pole, int m_lo, int lcap, int psv,
                        double* __restrict__ B0, double* __restrict__ B1, double* __restrict__ B2) {
    int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= th_n) return;
    double* B[3] = {B0, B1, B2};
    if (pole[it]) {
        // caldvecphi0_withplm sets only bvec(1,0) at the poles, through the
        // single-precision cmplx() (src/SGTpsv/trial.f90:121-131); SH sets
        // every vector to zero (src/SGTsh/trial.f90:492-505).
        for (int l = 0; l < lcap; ++l) {
            for (int m = m_lo; m <= 2; ++m) {
                double P = 0.0;
                if (psv && m == 0) {
                    double coeff = __dsqrt_rn(dvd((double)(2 * l + 1), mul(4.0, kPi)));
                    double sign1 = (pole[it] == 2 && (l & 1)) ? -1.0 : 1.0;
                    P = (double)(float)coeff * sign1;
                }
                B[m][(size_t)(0 * th_n + it) * lcap + l] = P;
                B[m][(size_t)(1 * th_n + it) * lcap + l] = 0.0;
            }
        }
        return;
    }
    double x = xs[it], s = ss[it];
    double plm[4][3];
    for (int m = 0; m < 4; ++m) plm[m][0] = plm[m][1] = plm[m][2] = 0.0;
    for (int l = 0; l < lcap; ++l) {
        int mm = l < 3 ? l : 3;
        for (int m = 0; m <= mm; ++m) plm_step(l, m, x, plm[m]);
        for (int m = m_lo; m <= 2; ++m) {
            double P = 0.0, D = 0.0;
            if (m <= l) {
                double fact = 1.0;
                for (int i = l - m + 1; i <= l + m; ++i) fact = mul(fact, (double)i);
                double coef = __dsqrt_rn(dvd(dvd((double)(2 * l + 1), mul(4.0, kPi)), fact));
                double p = plm[m][0], pn = plm[m + 1][0];
                double plmdt = add(mul(dvd(mul((double)m, x), s), p), pn);
                P = mul(coef, p);
                D = mul(coef, plmdt);
            }
            B[m][(size_t)(0 * th_n + it) * lcap + l] = P;
            B[m][(size_t)(1 * th_n + it) * lcap + l] = D;
        }
    }
}

// glu (src/SGTsh/glu2.f90:140-281) restricted to the real 3x3 Vandermonde
// matrix of interpolate; returns the value (b = e1) and derivative (b = e2)
// weights.  Imaginary parts are zero throughout, so real arithmetic gives
// the same numbers as the complex routine.
__device__ void glu3(const double a0[3][3], const double rhs[3], double out[3]) {
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = a0[i][j];
    int ip[3];
    double wk[3];
    const double eps = 3.52e-15;
    for (int k = 0; k < 3; ++k) {
        double amax = fabs(a[k][k]);
        int ipk = k;
        for (int i = k + 1; i < 3; ++i) {
            double aik = fabs(a[i][k]);
            if (aik > amax) { ipk = i; amax = aik; }
        }
        ip[k] = ipk;
        if (!(amax > eps)) { ip[k] = k; continue; }
        if (ipk != k) { double w = a[ipk][k]; a[ipk][k] = a[k][k]; a[k][k] = w; }
        for (int i = k + 1; i < 3; ++i) {
            a[i][k] = dvd(-a[i][k], a[k][k]);
            wk[i] = a[i][k];
        }
        for (int j = k + 1; j < 3; ++j) {
            if (ipk != k) { double w = a[ipk][j]; a[ipk][j] = a[k][j]; a[k][j] = w; }
            double t = a[k][j];
            for (int i = k + 1; i < 3; ++i) a[i][j] = add(a[i][j], mul(wk[i], t));
        }
    }
    double b[3] = {rhs[0], rhs[1], rhs[2]};
    for (int k = 0; k < 3; ++k) {
        if (ip[k] != k) { double w = b[ip[k]]; b[ip[k]] = b[k]; b[k] = w; }
        double t = b[k];
        for (int i = k + 1; i < 3; ++i) b[i] = add(b[i], mul(a[i][k], t));
    }
    b[2] = dvd(b[2], a[2][2]);
    for (int k = 1; k >= 0; --k) {
        double t = b[k + 1];
        for (int i = 0; i <= k; ++i) b[i] = sub(b[i], mul(a[i][k + 1], t));
        b[k] = dvd(b[k], a[k][k]);
    }
    for (int i = 0; i < 3; ++i) out[i] = b[i];
}

__global__ void k_weights(int R, const double* __restrict__ r, const double* __restrict__ rrsta,
                          double* __restrict__ wv, double* __restrict__ wd) {
    int ir = blockIdx.x * blockDim.x + threadIdx.x;
    if (ir >= R) return;
    double dh[3];
    for (int i = 0; i < 3; ++i) dh[i] = sub(rrsta[3 * ir + i], r[ir]);
    double a[3][3];
    for (int i = 0; i < 3; ++i) {
        a[0][i] = 1.0;
        a[1][i] = dh[i];
        a[2][i] = dvd(mul(dh[i], dh[i]), 2.0);
    }
    double e1[3] = {1.0, 0.0, 0.0}, e2[3] = {0.0, 1.0, 0.0}, o[3];
    if (dh[1] == 0.0) {  // interpolate returns g(2) directly for the value
        wv[3 * ir + 0] = 0.0; wv[3 * ir + 1] = 1.0; wv[3 * ir + 2] = 0.0;
    } else {
        glu3(a, e1, o);
        for (int i = 0; i < 3; ++i) wv[3 * ir + i] = o[i];
    }
    glu3(a, e2, o);
    for (int i = 0; i < 3; ++i) wd[3 * ir + i] = o[i];
}

// complex128 (num, R, Th) column-major -> complex64 [R][Th][num] (catalogue
// record of each receiver); SYNN (num, Th) keeps its order.
__global__ void k_pack(int nf, int num, int R, int Th, const double* __restrict__ in,
                       float* __restrict__ out) {
    size_t per = (size_t)num * R * Th;
    size_t tot = per * nf;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < tot;
         k += (size_t)gridDim.x * blockDim.x) {
        size_t w = k / per, rem = k % per;
        int comp = (int)(rem % num);
        size_t t2 = rem / num;
        int ir = (int)(t2 % R);
        int it = (int)(t2 / R);
        size_t o = w * per + ((size_t)ir * Th + it) * num + comp;
        out[2 * o] = (float)in[2 * k];
        out[2 * o + 1] = (float)in[2 * k + 1];
    }
}

}  // namespace

void launch_basis_tables(Engine& e, int lcap) {
    for (int m = e.m_lo; m <= 2; ++m) e.basis[m].reserve((size_t)2 * e.Th * lcap);
    double* B[3];
    for (int m = 0; m < 3; ++m) B[m] = (m >= e.m_lo) ? e.basis[m].p : nullptr;
    k_basis<<<(e.Th + 63) / 64, 64, 0, e.st>>>(e.Th, e.th.x.p, e.th.s.p, e.th.pole.p, e.m_lo, lcap,
                                               e.mode == 1, B[0], B[1], B[2]);
    DSM_LAUNCH(e);
    e.lcapB = lcap;
}

void launch_interp_weights(Engine& e, const double* d_r, const double* d_rrsta) {
    e.wv.reserve(3 * (size_t)e.R);
    e.wd.reserve(3 * (size_t)e.R);
    k_weights<<<(e.R + 127) / 128, 128, 0, e.st>>>(e.R, d_r, d_rrsta, e.wv.p, e.wd.p);
    DSM_LAUNCH(e);
}

void launch_pack32(Engine& e, int nf, int w0, int w1, size_t per_t, size_t per_r, size_t per_s, cudaStream_t s) {
    float* o = e.out32.p;
    const int n = w1 - w0;
    if (n <= 0) return;
    int grid = e.nsm * 8;
    k_pack<<<grid, 256, 0, s>>>(n, e.num_t, e.R, e.Th, e.out_t_src() + 2 * per_t * w0, o + 2 * per_t * w0);
    DSM_LAUNCH(e);
    if (e.rsgt_sw) {
        k_pack<<<grid, 256, 0, s>>>(n, e.num_r, e.R, e.Th, e.out_r_src() + 2 * per_r * w0,
                                       o + 2 * per_t * nf + 2 * per_r * w0);
        DSM_LAUNCH(e);
    }
    if (e.synn_sw) {
        k_pack<<<grid, 256, 0, s>>>(n, e.num_s, 1, e.Th, e.out_s_src() + 2 * per_s * w0,
                                       o + 2 * (per_t + per_r) * nf + 2 * per_s * w0);
        DSM_LAUNCH(e);
    }
}

}  // namespace dsm
