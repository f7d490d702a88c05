// P-SV epilogue: the strain Green's tensors of one frequency from the
// l-contractions of its displacement fields (calup, calupfluid,
// locallyCartesianDerivatives, udertotsgt, udertorsgt, utosynn,
// src/SGTpsv/others.f90:161-344, 983-1031).
//
// One thread per (distance, receiver); a second kernel handles the surface
// row (SYNN).  The divisions by the receiver radius, sin(theta) and
// 1 - cos^2(theta) are taken once per thread as reciprocals.  The tensor-
// core path computes in FP32 (its contraction outputs are FP32 already);
// the plain path in FP64.  This file is compiled with fused multiply-add.
#include <cmath>

#include "psv_epi.cuh"

namespace dsm {
namespace psvk {
namespace {

// threads per block, both paths
template <class TC>
constexpr int epi_threads() { return 128; }

template <class RL>
struct PointConst {
    RL fr_inv, fs_inv, s_inv, xs, x_1mx2, inv_1mx2, fc;
};

template <class RL>
__device__ __forceinline__ PointConst<RL> point_const(double x, double s, double fr) {
    PointConst<RL> p;
    const double fs = (double)(float)s;
    p.fr_inv = (RL)(1.0 / fr);
    p.fs_inv = (RL)(1.0 / fs);
    p.s_inv = (RL)(1.0 / s);
    p.xs = (RL)(x / s);
    p.x_1mx2 = (RL)(x / (1.0 - x * x));
    p.inv_1mx2 = (RL)(1.0 / (1.0 - x * x));
    p.fc = (RL)(double)(float)(x / s);
    return p;
}

// slot q of |m| = mi: order m, moment-tensor index imt (1..6) or back
// component icomp (1..3), and whether it is a back (receiver-side) slot
struct Slot {
    int m, imt, icomp;
    bool isback;
};
__device__ __forceinline__ Slot slot_of(int mi, int q) {
    const int per = mi == 2 ? 3 : 4;
    const int sg = q / per, k = q % per;
    Slot t;
    t.m = mi == 0 ? 0 : (sg == 0 ? -mi : mi);
    t.isback = (mi == 0 && k == 3) || (mi == 1 && k >= 2);
    t.imt = 0;
    t.icomp = 0;
    if (mi == 0) {
        if (k < 3) t.imt = k + 1;
        else t.icomp = 1;
    } else if (mi == 1) {
        if (k < 2) t.imt = 4 + k;
        else t.icomp = k;
    } else {
        t.imt = k == 0 ? 2 : (k == 1 ? 3 : 6);
    }
    return t;
}

template <class TC, class RL>
struct Fields {
    const TC* C;
    size_t LD;  // row stride (row-major contraction outputs)
    int nq, Rs1, Rf, Th, it, rr, q;
    // complex entry of field f against basis column b (b = 1 only for the
    // fields 0, 2, 3; fluid receivers have field 0 against P only)
    __device__ __forceinline__ cx<RL> operator()(int f, int b) const {
        int im;
        const size_t row = (size_t)fld_row(nq, Rs1, Rf, q, f, rr, &im);
        const size_t col = (size_t)b * Th + it;
        return {(RL)C[row * LD + col], (RL)C[(row + im) * LD + col]};
    }
};

// displacement fields of the receivers below the surface
template <class TC, class RL, bool BACK>
__global__ void __launch_bounds__(epi_threads<TC>()) k_psv_epi(EpiDev d, int w, const double* __restrict__ thx,
                                                         const double* __restrict__ ths,
                                                         const int* __restrict__ pole,
                                                         const int* __restrict__ freqs,
                                                         const TC* __restrict__ C0, const TC* __restrict__ C1,
                                                         const TC* __restrict__ C2, double* __restrict__ tsgt,
                                                         double* __restrict__ rsgt) {
    using C = cx<RL>;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int R = d.R, Th = d.Th;
    if (idx >= Th * R) return;
    const int it = idx % Th, r = idx / Th;  // consecutive lanes: consecutive distances of one receiver
    const bool isp = pole[it] != 0;
    const TC* Cm[3] = {C0, C1, C2};
    const int rr = d.rrow[r];
    const double x = thx[it], s = ths[it];
    const PointConst<RL> pc = point_const<RL>(x, s, d.fr[r]);
    const bool fluid = d.fluid[r] != 0;
    C efl = {RL(0), RL(0)};
    if (fluid) {  // calupfluid factor omega / 3 / lambda(omega)
        const double omega = 2.0 * kPi * (double)freqs[w] / d.tlen;
        const cd comega = mk(omega, -d.omegai);
        const double deuxsurpi = 0.63661977236, unsurdeuxpi = 0.15915494309,
                     unsurtrois = 0.33333333333333333333;
        const double lam = d.lam[r], qk = d.qkp[r];
        cd fl = mk(lam * 1.0, lam * (1.0 / qk));
        const double fac = 1 + deuxsurpi / qk * log(unsurdeuxpi * comega.re);
        fl = mk(fl.re * fac, fl.im * fac);
        const cd e = comega * unsurtrois / fl;
        efl = {(RL)e.re, (RL)e.im};
    }
    C T[20], Rg[BACK ? 10 : 1];
#pragma unroll
    for (int c = 0; c < 20; ++c) T[c] = {RL(0), RL(0)};
#pragma unroll
    for (int c = 0; c < (BACK ? 10 : 1); ++c) Rg[c] = {RL(0), RL(0)};
    const RL h = RL(0.5), qr = RL(0.25), e8 = RL(0.125);
    for (int mi = 0; mi < 3; ++mi) {
        if (isp && mi != 0) break;  // only bvec(1,0) survives at the poles
        const int nq = mi == 0 ? NS0 : (mi == 1 ? NS1 : NS2);
        for (int q = 0; q < nq; ++q) {
            const Slot sl = slot_of(mi, q);
            if (sl.isback && !BACK) continue;
            const Fields<TC, RL> G{Cm[mi], (size_t)d.c_ld, nq, d.Rs1, d.Rf, Th, it, rr, q};
            const RL sigma = (sl.m < 0 && (mi & 1)) ? RL(-1) : RL(1);
            const RL mm = (RL)sl.m, m2 = mm * mm;
            C d11 = {RL(0), RL(0)}, d12 = d11, d13 = d11, d21 = d11, d22 = d11, d23 = d11, d31 = d11,
              d32 = d11, d33 = d11;
            const C PU = G(0, 0);
            if (fluid) {
                const C e = efl * (isp ? PU : sigma * PU);
                d11 = e;
                d22 = e;
                d33 = e;
            } else if (isp) {
                d11 = G(1, 0);
                d22 = PU * pc.fr_inv;
                d33 = d22;
            } else {
                const C PV = G(2, 0), DV = G(2, 1);
                const RL ms = mm * pc.s_inv;
                const C u1 = sigma * PU, u2 = sigma * DV, u3 = sigma * cmul_i(ms, PV);
                const C udr1 = sigma * G(1, 0), udr2 = sigma * G(3, 1), udr3 = sigma * cmul_i(ms, G(3, 0));
                const C udt1 = (sl.m >= 0) ? G(0, 1) : C{RL(0), RL(0)};
                const C udt2 = sigma * ((-pc.xs) * DV + (m2 * pc.inv_1mx2) * PV - G(4, 0));
                const C udt3 = sigma * cmul_i(mm, (-pc.x_1mx2) * PV + pc.s_inv * DV);
                const C udp1 = sigma * cmul_i(mm, PU), udp2 = sigma * cmul_i(mm, DV);
                const C udp3 = sigma * ((-m2 * pc.s_inv) * PV);
                d11 = udr1;
                d12 = (udt1 - u2) * pc.fr_inv;
                d13 = (udp1 * pc.fs_inv - u3) * pc.fr_inv;
                d21 = udr2;
                d22 = (udt2 + u1) * pc.fr_inv;
                d23 = (udp2 * pc.fs_inv - u3 * pc.fc) * pc.fr_inv;
                d31 = udr3;
                d32 = udt3 * pc.fr_inv;
                d33 = (udp3 * pc.fs_inv + u1 + u2 * pc.fc) * pc.fr_inv;
            }
            if (sl.icomp) {  // udertorsgt
                if constexpr (BACK) {
                    if (sl.icomp == 1) {
                        Rg[0] = Rg[0] + d11;
                        Rg[1] = Rg[1] - h * d21 - h * d12;
                        Rg[2] = Rg[2] + h * d22 - h * d33;
                        Rg[3] = Rg[3] - h * d22 - h * d33;
                    } else if (sl.icomp == 2) {
                        Rg[4] = Rg[4] + d11;
                        Rg[5] = Rg[5] - h * d22 - h * d33;
                        Rg[6] = Rg[6] - h * d22 + h * d33;
                        Rg[8] = Rg[8] - h * d12 - h * d21;
                    } else {
                        Rg[7] = Rg[7] - h * d23 - h * d32;
                        Rg[9] = Rg[9] + h * d13 + h * d31;
                    }
                }
                continue;
            }
            // udertotsgt
            const int imt = sl.imt;
            if (imt == 1) {
                T[0] = T[0] + d11;
                T[2] = T[2] - h * d22 - h * d33;
                T[5] = T[5] - h * d12 - h * d21;
                T[9] = T[9] + h * d22 - h * d33;
            } else if (imt == 2 || imt == 3) {
                const RL sgn = imt == 2 ? RL(1) : RL(-1);
                T[1] = T[1] - h * d11;
                T[3] = T[3] + qr * d22 + qr * d33;
                T[7] = T[7] + (sgn * qr) * d12 + (sgn * qr) * d21;
                T[8] = T[8] + (sgn * h) * d11;
                T[10] = T[10] - qr * d22 + qr * d33;
                T[11] = T[11] - (sgn * qr) * d22 - (sgn * qr) * d33;
                T[16] = T[16] - e8 * d12 - e8 * d21;
                T[17] = T[17] + e8 * d12 + e8 * d21;
                T[18] = T[18] + (sgn * e8) * d22 - (sgn * e8) * d33;
                T[19] = T[19] + (sgn * e8) * d22 - (sgn * e8) * d33;
            } else if (imt == 4) {
                T[4] = T[4] + d11;
                T[6] = T[6] - h * d22 - h * d33;
                T[12] = T[12] - qr * d12 - qr * d21;
                T[13] = T[13] + qr * d12 + qr * d21;
                T[14] = T[14] + qr * d22 - qr * d33;
                T[15] = T[15] - qr * d22 + qr * d33;
            } else if (imt == 5) {
                T[12] = T[12] + qr * d13 + qr * d31;
                T[13] = T[13] + qr * d13 + qr * d31;
                T[14] = T[14] - qr * d23 - qr * d32;
                T[15] = T[15] - qr * d23 - qr * d32;
            } else if (imt == 6) {
                T[16] = T[16] + qr * d13 + qr * d31;
                T[17] = T[17] + qr * d13 + qr * d31;
                T[18] = T[18] - qr * d23 - qr * d32;
                T[19] = T[19] + qr * d23 + qr * d32;
            }
        }
    }
    bool bad = false;
#pragma unroll
    for (int c = 0; c < 20; ++c) bad |= !isfinite(T[c].re) || !isfinite(T[c].im);
    if constexpr (BACK) {
#pragma unroll
        for (int c = 0; c < 10; ++c) bad |= !isfinite(Rg[c].re) || !isfinite(Rg[c].im);
    }
    flag_nonfinite(d.status, bad);
    const size_t pt = ((size_t)w * Th + it) * R + r;
    double2* t2 = reinterpret_cast<double2*>(tsgt) + pt * 20;
#pragma unroll
    for (int c = 0; c < 20; ++c) t2[c] = make_double2((double)T[c].re, (double)T[c].im);
    if constexpr (BACK) {
        double2* r2 = reinterpret_cast<double2*>(rsgt) + pt * 10;
#pragma unroll
        for (int c = 0; c < 10; ++c) r2[c] = make_double2((double)Rg[c].re, (double)Rg[c].im);
    }
}

// surface displacement (utosynn): one thread per distance
template <class TC, class RL>
__global__ void __launch_bounds__(epi_threads<TC>()) k_psv_epi_surf(EpiDev d, int w, const double* __restrict__ thx,
                                                              const double* __restrict__ ths,
                                                              const int* __restrict__ pole,
                                                              const TC* __restrict__ C0, const TC* __restrict__ C1,
                                                              const TC* __restrict__ C2, double* __restrict__ synn) {
    using C = cx<RL>;
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    const int R = d.R, Th = d.Th;
    if (it >= Th) return;
    const bool isp = pole[it] != 0;
    const TC* Cm[3] = {C0, C1, C2};
    const int rr = d.rrow[R];
    const RL s_inv = (RL)(1.0 / ths[it]);
    (void)thx;
    C S[10];
#pragma unroll
    for (int c = 0; c < 10; ++c) S[c] = {RL(0), RL(0)};
    const RL h = RL(0.5);
    for (int mi = 0; mi < 3; ++mi) {
        if (isp && mi != 0) break;
        const int nq = mi == 0 ? NS0 : (mi == 1 ? NS1 : NS2);
        for (int q = 0; q < nq; ++q) {
            const Slot sl = slot_of(mi, q);
            if (sl.isback) continue;  // back slots have no surface term
            const Fields<TC, RL> G{Cm[mi], (size_t)d.c_ld, nq, d.Rs1, d.Rf, Th, it, rr, q};
            const RL sigma = (sl.m < 0 && (mi & 1)) ? RL(-1) : RL(1);
            const C PU = G(0, 0);
            C u1, u2 = {RL(0), RL(0)}, u3 = {RL(0), RL(0)};
            if (isp) {
                u1 = PU;
            } else {
                u1 = sigma * PU;
                u2 = sigma * G(2, 1);
                u3 = sigma * cmul_i((RL)sl.m * s_inv, G(2, 0));
            }
            const int imt = sl.imt;
            if (imt == 1) { S[0] = S[0] + u1; S[4] = S[4] + u2; }
            if (imt == 2) {
                S[2] = S[2] + h * u1; S[3] = S[3] - h * u1;
                S[5] = S[5] - h * u2; S[6] = S[6] - h * u2;
            }
            if (imt == 3) {
                S[2] = S[2] - h * u1; S[3] = S[3] - h * u1;
                S[5] = S[5] - h * u2; S[6] = S[6] + h * u2;
            }
            if (imt == 4) { S[1] = S[1] + u1; S[8] = S[8] + u2; }
            if (imt == 5) { S[9] = S[9] + u3; }
            if (imt == 6) { S[7] = S[7] - u3; }
        }
    }
    bool bad = false;
#pragma unroll
    for (int c = 0; c < 10; ++c) bad |= !isfinite(S[c].re) || !isfinite(S[c].im);
    flag_nonfinite(d.status, bad);
    double2* s2 = reinterpret_cast<double2*>(synn) + ((size_t)w * Th + it) * 10;
#pragma unroll
    for (int c = 0; c < 10; ++c) s2[c] = make_double2((double)S[c].re, (double)S[c].im);
}

template <class TC, class RL>
void launch_t(const EpiDev& d, int w, const double* thx, const double* ths, const int* pole, const int* freqs,
              const void* C0, const void* C1, const void* C2, double* tsgt, double* rsgt, double* synn,
              cudaStream_t st) {
    const TC *c0 = static_cast<const TC*>(C0), *c1 = static_cast<const TC*>(C1), *c2 = static_cast<const TC*>(C2);
    const int n = d.Th * d.R;
    constexpr int EPI_THREADS = epi_threads<TC>();
    const unsigned grid = (unsigned)((n + EPI_THREADS - 1) / EPI_THREADS);
    if (rsgt)
        k_psv_epi<TC, RL, true><<<grid, EPI_THREADS, 0, st>>>(d, w, thx, ths, pole, freqs, c0, c1, c2, tsgt, rsgt);
    else
        k_psv_epi<TC, RL, false><<<grid, EPI_THREADS, 0, st>>>(d, w, thx, ths, pole, freqs, c0, c1, c2, tsgt,
                                                               nullptr);
    if (synn)
        k_psv_epi_surf<TC, RL><<<(d.Th + EPI_THREADS - 1) / EPI_THREADS, EPI_THREADS, 0, st>>>(d, w, thx, ths,
                                                                                               pole, c0, c1, c2,
                                                                                               synn);
}

}  // namespace

void launch_epilogue(const EpiDev& d, int w, const double* thx, const double* ths, const int* pole,
                     const int* freqs, const void* C0, const void* C1, const void* C2, bool tc, double* tsgt,
                     double* rsgt, double* synn, cudaStream_t st) {
    if (tc) launch_t<float, float>(d, w, thx, ths, pole, freqs, C0, C1, C2, tsgt, rsgt, synn, st);
    else launch_t<double, double>(d, w, thx, ths, pole, freqs, C0, C1, C2, tsgt, rsgt, synn, st);
}

}  // namespace psvk
}  // namespace dsm
