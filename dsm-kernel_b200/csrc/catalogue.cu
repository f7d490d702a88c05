// Catalogue consumer: SGT records of one receiver radius (frequency indices
// fmin..fmax, all catalogue distances) -> windowed time series at arbitrary
// epicentral distances, on the device.
//
// Restates KernelMaker's
//   rdsgtomega        src/KernelMaker/fourier.f90:1-123   (scale, 1e-21, reduction phase)
//   clsgt             src/KernelMaker/fourier.f90:128-162 (normalised sinc in distance)
//   findIdeltaRegion  src/KernelMaker/fourier.f90:165-190
//   vectorFFT_double  src/KernelMaker/fourier.f90:418-450 (Hermitian extension,
//                     length-2 np1 inverse transform, exp(omegai t) / tlen * 1e3)
//
// The sinc interpolation is a banded product: for every frequency n,
// sgtF[p][d] = sum_kk W[p][kk] omega[n][kk][d] with W nonzero on a window of
// 2 nhregion + 1 catalogue distances around each point.  Points are sorted by
// distance and grouped in tiles of up to 32 whose windows overlap; a tile's
// union of windows is its band of catalogue distances.
//
// Device plan, per call:
//   k_cat_omega   rdsgtomega over the catalogue distances some window covers:
//                 records (complex64/128) widened, times scale, reduction
//                 phase and 1e-21, record sets summed, as the reference's
//                 frequency-domain SGT [n][distance][component] in FP64.
// and per batch of sorted points:
//   k_cat_interp  one 4-warp CTA per (point tile, 4 frequencies), one warp per
//                 frequency, four CTAs per SM.  The band is walked in chunks
//                 of 16 distances, double-buffered in shared memory by
//                 cp.async (the chunk's SGT rows of the 4 frequencies and the
//                 tile's dense weights, zero outside each point's window),
//                 and multiplied on the FP64 tensor cores (mma.m16n8k4.f64:
//                 32 points x all components per warp, accumulated in
//                 registers).  Epilogue: divide by the weight sum, clsgt
//                 phase, the per-point component combination, and the
//                 Hermitian projection H_n = (x_n + conj(x_{N-n})) / 2
//                 (n = 0..np1) of the reference's extended vector x:
//                 Re(IDFT(x)) = IDFT(H), so a real-output transform gives the
//                 reference's Re(cvec).
//   cuFFT Z2D     in place, length N = 2 np1, batch = points x outputs.
//   k_cat_window  samples iwin_start..iwin_end, times exp(omegai t / sHz) /
//                 tlen * 1e3, written in the caller's point order.
//
// Compiled without fused multiply-add so the rdsgtomega and normalisation
// arithmetic rounds like the Fortran; the weighted sums (tensor-core
// products) and the component combination round once per term.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <map>
#include <memory>
#include <numeric>

#include "common.cuh"

namespace dsm {
namespace cat {

constexpr int PT = 32;          // points per tile: 8 lane groups x 4 points
constexpr int KC = 16;          // catalogue distances per staged chunk (a multiple of 4)
constexpr int CAT_WARPS = 4;
constexpr int CAT_THREADS = 32 * CAT_WARPS;
constexpr int MAX_SETS = 4;
constexpr int MAX_NUM = 32;     // components of the frequency-domain SGT
constexpr int MAX_OUT = 64;     // outputs per point
constexpr int MAX_NW = 256;     // catalogue distances in one sinc window

struct SetDev {
    const void* rec;   // [nf][theta_n][ncomp]
    int cplx64;        // 1: complex64 records, 0: complex128
    int ncomp;
    int src[MAX_NUM];  // record component feeding destination d, or -1
    double scale[MAX_NUM];  // factor of that record component
};

struct Tile {
    int p0, np;        // sorted positions [p0, p0 + np) of the batch
    int u0, U;         // band: rows [u0, u0 + U) of the frequency-domain SGT
    long long woff;    // offset of the tile's dense weights [U][WS] in wt
};

struct InterpArgs {
    int num, nout, identity, ntile;
    int fmin, fmax, np1, ucov;   // ucov: rows of om per frequency
    double tlen, c_red_reci;
    const Tile* tiles;
    const cd* om;          // [nf][ucov][nump] frequency-domain SGT (k_cat_omega)
    const double* wt;      // dense tile weights (zero outside each point's window)
    // per sorted position of the batch
    const double* norm;    // sum of the weights
    const double* dist;    // distance (deg)
    const int* orig;       // the caller's index of the point
    const double* coef;    // [caller point][nout][num] or null (identity)
    cd* h;                 // [sorted position][nout][np1+1]
    cd* spec;              // spectra mode: [caller point][nout][fmax-fmin+1], else null
};

__device__ __forceinline__ cd load_rec(const SetDev& s, size_t idx) {
    if (s.cplx64) {
        float2 v = __ldg(reinterpret_cast<const float2*>(s.rec) + idx);
        return cd{(double)v.x, (double)v.y};
    }
    const double2 v = __ldg(reinterpret_cast<const double2*>(s.rec) + idx);
    return cd{v.x, v.y};
}

// exp(i arg) as Fortran's exp(cmplx(0, arg))
__device__ __forceinline__ cd expi(double arg) {
    double sn, cs;
    sincos(arg, &sn, &cs);
    return cd{cs, sn};
}

// H_n of the reference's extended vector x (vectorFFT_double, fourier.f90:430-439)
// from the spectrum value v at index n (zero outside fmin..fmax):
// x_n + conj(x_{N-n}) = 2 v where the extension mirrors n, v where it leaves
// zeros (n > np1 - fmin), and the real part at n = 0 and n = np1
__device__ __forceinline__ cd herm_proj(cd v, int n, int np1, int fmin) {
    if (n == 0 || n == np1) return cd{v.re, 0.0};
    if (n <= np1 - fmin) return v;
    return v * 0.5;
}

// rdsgtomega (fourier.f90:87-116) on catalogue distances [u0, u0 + Ucov):
// om[n - fmin][u - u0][d] = sum over record sets of ((rec * scale) * phase) * 1e-21,
// components padded to nump with zeros; index 0 is never read (zero)
struct OmegaArgs {
    SetDev set[MAX_SETS];
    int nset, num, nump, theta_n, fmin, nf, u0, ucov, urows;   // rows >= ucov are zero
    double theta_min, theta_delta, tlen, c_red_reci;
    cd* om;   // [nf][urows][nump]
};

// grid (ceil(urows * nump / 256), min(nf, 65535)): one thread per (distance,
// component), frequencies strided by the grid height.
// The per-component set tables are copied to shared memory first: threads of
// a warp index them by different components, which kernel-parameter memory
// would serve one address at a time.
__global__ void __launch_bounds__(256) k_cat_omega(const OmegaArgs a) {
    __shared__ int src_s[MAX_SETS][MAX_NUM];
    __shared__ double scale_s[MAX_SETS][MAX_NUM];
    for (int i = threadIdx.x; i < MAX_SETS * MAX_NUM; i += blockDim.x) {
        const int s = i / MAX_NUM, d = i % MAX_NUM;
        src_s[s][d] = s < a.nset ? a.set[s].src[d] : -1;
        scale_s[s][d] = s < a.nset ? a.set[s].scale[d] : 0.0;
    }
    __syncthreads();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.urows * a.nump) return;
    const int d = j % a.nump, u = j / a.nump;
    for (int k = blockIdx.y; k < a.nf; k += gridDim.y) {   // frequencies, strided by the grid height
        const int n = a.fmin + k;
        cd om = mk(0.0);
        if (d < a.num && n != 0 && u < a.ucov) {
            const size_t base = (size_t)k * a.theta_n + (a.u0 + u);
            cd ph = mk(1.0);
            const bool reduce = a.c_red_reci != 0.0;
            if (reduce) {
                const double th = a.theta_min + (double)(a.u0 + u) * a.theta_delta;
                const double redtime = -th * a.c_red_reci;
                ph = expi(-(2.0 * kPi * (double)n / a.tlen * redtime));
            }
            for (int s = 0; s < a.nset; ++s) {
                const SetDev& S = a.set[s];
                const int c = src_s[s][d];
                if (c < 0) continue;
                cd t = load_rec(S, base * S.ncomp + c) * scale_s[s][c];
                if (reduce) t = t * ph;
                t = t * 1.0e-21;
                om = om + t;   // the first set adds to an exact zero
            }
        }
        a.om[((size_t)k * a.urows + u) * a.nump + d] = om;
    }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// k_cat_interp<C>: the band product on the FP64 tensor cores.  Per
// frequency it is D[point][column] += W[point][distance] * B[distance][column]
// with the real columns (re, im of each of 4C components); one
// mma.m16n8k4.f64 takes 16 points x 4 distances of W and 4 distances x 8
// columns of B.  A warp owns one frequency of the CTA: all PT = 32 points
// (two m16 tiles) x 8C real columns (C n8 tiles), 2C accumulator tiles.
//
// Fragments of mma.m16n8k4 .f64 (g = lane / 4, t = lane % 4):
//   A 16x4: a0 = A[g][t], a1 = A[g + 8][t];   B 4x8: b0 = B[t][g];
//   C 16x8: c0, c1 = C[g][2t], C[g][2t + 1];  c2, c3 = same in row g + 8.
// Shared-memory rows are padded so the 16 lanes of a half-warp hit distinct
// banks: weights [KC][WS] with WS = 36, SGT rows of SS = 8C + 4 doubles
// (2 SS mod 32 is 8 or 24, and 2 WS mod 32 is 8).
constexpr int WS = 36;
__host__ __device__ constexpr int sgt_stride(int C) { return 8 * C + 4; }

// shared memory of k_cat_interp (bytes): two staged chunks [CAT_WARPS][KC][SS]
// doubles, reused by the epilogue as [CAT_WARPS][PT * 4C + 1] cd, and two
// weight chunks [KC][WS] doubles
__host__ __device__ inline size_t interp_smem_bytes(int C) {
    const size_t om = (size_t)2 * CAT_WARPS * KC * sgt_stride(C) * sizeof(double);
    const size_t ep = (size_t)CAT_WARPS * (PT * 4 * C + 1) * sizeof(cd);
    return (om > ep ? om : ep) + (size_t)2 * KC * WS * sizeof(double);
}

__device__ __forceinline__ void mma_f64_16x8x4(double (&d)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
        "{%0, %1, %2, %3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

template <int C>
__global__ void __launch_bounds__(CAT_THREADS, C <= 5 ? 4 : 2) k_cat_interp(const InterpArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int NUMP = 4 * C, SS = sgt_stride(C);
    constexpr size_t OM_D = (size_t)2 * CAT_WARPS * KC * SS, EP_D = (size_t)CAT_WARPS * (PT * NUMP + 1) * 2;
    double* Om = reinterpret_cast<double*>(smem);                            // [2][CAT_WARPS][KC][SS]
    double* Wc = Om + (OM_D > EP_D ? OM_D : EP_D);                            // [2][KC][WS]
    // one-dimensional grid, tiles fastest: block b = frequency block * ntile + tile
    const Tile tl = a.tiles[blockIdx.x % a.ntile];
    const int n0 = (int)(blockIdx.x / a.ntile) * CAT_WARPS;
    const int nh = a.np1 + 1;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const bool reduce = a.c_red_reci != 0.0;
    const int nlo = max(n0, max(a.fmin, 1)), nhi = min(n0 + CAT_WARPS - 1, a.fmax);
    const bool any = nlo <= nhi;
    const int n = n0 + warp;
    const bool mine = n >= nlo && n <= nhi;
    const int nchunk = (tl.U + KC - 1) / KC;   // U is a multiple of 4

    // chunk k: the SGT rows of distances u0 + k KC .. of the CTA's
    // frequencies and the tile's weights of those distances
    auto issue = [&](int k) {
        const int buf = k & 1, k0 = k * KC, kc = min(KC, tl.U - k0);
        double* ob = Om + (size_t)buf * CAT_WARPS * KC * SS;
        for (int i = tid; i < CAT_WARPS * KC * NUMP; i += CAT_THREADS) {
            const int nl = i / (KC * NUMP), e = i % (KC * NUMP);
            const int kk = e / NUMP, d = e % NUMP;
            const int nn = n0 + nl;
            if (kk >= kc || nn < nlo || nn > nhi) continue;
            cp_async16(ob + ((size_t)nl * KC + kk) * SS + 2 * d,
                       a.om + ((size_t)(nn - a.fmin) * a.ucov + tl.u0 + k0 + kk) * NUMP + d);
        }
        double* wb = Wc + buf * KC * WS;
        const double* wsrc = a.wt + (size_t)tl.woff + (size_t)k0 * WS;
        for (int i = tid; i < kc * WS / 2; i += CAT_THREADS) cp_async16(wb + 2 * i, wsrc + 2 * i);
        cp_async_commit();
    };

    double acc[2][C][4];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int q = 0; q < C; ++q)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[m][q][e] = 0.0;

    if (any) {
        issue(0);
        for (int k = 0; k < nchunk; ++k) {
            if (k + 1 < nchunk) {
                issue(k + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            if (mine) {
                const int kc = min(KC, tl.U - k * KC);
                const double* orow = Om + ((size_t)(k & 1) * CAT_WARPS + warp) * KC * SS + t * SS + g;
                const double* wrow = Wc + (k & 1) * KC * WS + t * WS + g;
                for (int k4 = 0; k4 < kc; k4 += 4) {
                    const double a00 = wrow[k4 * WS], a01 = wrow[k4 * WS + 8];
                    const double a10 = wrow[k4 * WS + 16], a11 = wrow[k4 * WS + 24];
#pragma unroll
                    for (int q = 0; q < C; ++q) {
                        const double b = orow[k4 * SS + 8 * q];
                        mma_f64_16x8x4(acc[0][q], a00, a01, b);
                        mma_f64_16x8x4(acc[1][q], a10, a11, b);
                    }
                }
            }
            __syncthreads();
        }
        // epilogue 1: normalise, clsgt phase; stage [CAT_WARPS][PT * NUMP + 1] cd
        cd* E = reinterpret_cast<cd*>(smem);
        const int es = PT * NUMP + 1;
        if (mine) {
#pragma unroll
            for (int m = 0; m < 2; ++m)
#pragma unroll
                for (int hr = 0; hr < 2; ++hr) {
                    const int pl = m * 16 + g + 8 * hr;
                    if (pl >= tl.np) continue;
                    const int ps = tl.p0 + pl;
                    const double nrm = a.norm[ps];
                    cd phs = mk(1.0);
                    if (reduce) phs = expi(-(2.0 * kPi) * (double)n / a.tlen * a.dist[ps] * a.c_red_reci);
#pragma unroll
                    for (int q = 0; q < C; ++q) {
                        cd v = cd{acc[m][q][2 * hr], acc[m][q][2 * hr + 1]} / nrm;
                        if (reduce) v = v * phs;
                        E[(size_t)warp * es + pl * NUMP + 4 * q + t] = v;
                    }
                }
        }
        __syncthreads();
    }
    // epilogue 2: combine, Hermitian projection, store CAT_WARPS consecutive n per row
    const cd* E = reinterpret_cast<const cd*>(smem);
    const int es = PT * NUMP + 1;
    for (int i = tid; i < tl.np * a.nout * CAT_WARPS; i += CAT_THREADS) {
        const int nl = i % CAT_WARPS, rest = i / CAT_WARPS;
        const int j = rest % a.nout, pl = rest / a.nout;
        const int nn = n0 + nl;
        if (nn >= nh) continue;
        cd v = mk(0.0);
        if (any && nn >= nlo && nn <= nhi) {
            const cd* e = E + (size_t)nl * es + pl * NUMP;
            if (a.identity) {
                v = e[j];
            } else {
                const double* m = a.coef + ((size_t)a.orig[tl.p0 + pl] * a.nout + j) * a.num;
                for (int d = 0; d < a.num; ++d) {
                    v.re = fma(m[d], e[d].re, v.re);
                    v.im = fma(m[d], e[d].im, v.im);
                }
            }
        }
        if (a.spec) {  // spectra mode: the combined spectrum itself, frequencies fmin..fmax
            if (nn >= a.fmin && nn <= a.fmax)
                a.spec[((size_t)a.orig[tl.p0 + pl] * a.nout + j) * (a.fmax - a.fmin + 1) + (nn - a.fmin)] = v;
            continue;
        }
        a.h[((size_t)(tl.p0 + pl) * a.nout + j) * nh + nn] = herm_proj(v, nn, a.np1, a.fmin);
    }
}

// Hermitian projection H_n (n = 0..np1) of arbitrary spectra x[b][n - fmin]
// (vectorFFT_double's input ccvec), rows of h np1 + 1 apart
__global__ void k_cat_herm(const cd* __restrict__ x, int nb, int fmin, int fmax, int np1, cd* __restrict__ h) {
    const int nh = np1 + 1;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nh) return;
    for (int b = blockIdx.y; b < nb; b += gridDim.y) {
        const cd v = (n >= fmin && n <= fmax) ? x[(size_t)b * (fmax - fmin + 1) + (n - fmin)] : mk(0.0);
        h[(size_t)b * nh + n] = herm_proj(v, n, np1, fmin);
    }
}

// out[orig point][j][t] = y[row][iws + t] * e[t] / tlen * 1e3; rows of y (sorted
// position x nout + j) are 2 (np1+1) reals apart
__global__ void k_cat_window(const double* __restrict__ y, int row, int iws, int nwin, int nb, int nout,
                             const int* __restrict__ orig, const double* __restrict__ e, double tlen,
                             double* __restrict__ out) {
    const size_t total = (size_t)nb * nwin;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t b = i / nwin;
        const int t = (int)(i - b * nwin);
        const int ps = (int)(b / nout), j = (int)(b - (size_t)ps * nout);
        out[((size_t)orig[ps] * nout + j) * nwin + t] = y[b * row + iws + t] * e[t] / tlen * 1.0e3;
    }
}

// ---- per-point isotropic kernels (calculateKernel, calculateK.f90:131-235) ----

constexpr int KER_MAXFL = 16;   // filters ift = 0..nfilter
constexpr int KER_MAXNP = 10;   // Butterworth sections (bwfilt.f90:135)

// Frequency products of isovpfreq (calculateK.f90:261-265) and isovsfreq
// (:367-374 du; :395-403 duq with jacobianFuji), each times 1e3, written as
// the Hermitian projection H_n (n = 0..np1) that vectorFFT_double
// transforms: rows (batch point, series) np1 + 1 apart, series in the order
// P du, S du, S duq of the types present.  The operation order is the
// reference's (sums left to right, complex products (ac - bd, ad + bc)).
struct KerSpecArgs {
    const cd *h3, *h4;   // [point][6][nf]
    const cd* jac;       // jacobianFuji [n - fmin][nr]
    const int* ir;       // [point], 0-based radius
    int p0, nb, nr, fmin, fmax, np1, types, ns;
    cd* h;
};

__global__ void __launch_bounds__(256) k_ker_spec(const KerSpecArgs a) {
    const int nh = a.np1 + 1, nf = a.fmax - a.fmin + 1;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nh) return;
    for (int b = blockIdx.y; b < a.nb; b += gridDim.y) {
        const int pt = a.p0 + b;
        cd up = mk(0.0), us = mk(0.0), uq = mk(0.0);
        if (n >= a.fmin && n <= a.fmax) {
            const cd* x = a.h3 + (size_t)pt * 6 * nf + (n - a.fmin);
            const cd* y = a.h4 + (size_t)pt * 6 * nf + (n - a.fmin);
            cd g[6], q[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                g[k] = x[(size_t)k * nf];
                q[k] = y[(size_t)k * nf];
            }
            if (a.types & DSM_KER_VP) up = -((g[0] + g[1] + g[2]) * (q[0] + q[1] + q[2])) * 1.0e3;
            if (a.types & DSM_KER_VS) {
                const cd p4 = g[3] * q[3], p5 = g[4] * q[4], p6 = g[5] * q[5];
                const cd c1 = g[0] * (q[1] + q[2]), c2 = g[1] * (q[0] + q[2]), c3 = g[2] * (q[0] + q[1]);
                us = (-(2.0 * (p4 + p5 + p6)) + c1 + c2 + c3) * 1.0e3;
                const cd d1 = g[0] * q[0], d2 = g[1] * q[1], d3 = g[2] * q[2];
                cd v = -(4.0 * (p4 + p5 + p6)) + (2.0 / 3.0) * (c1 + c2 + c3) - (4.0 / 3.0) * (d1 + d2 + d3);
                v = v * a.jac[(size_t)(n - a.fmin) * a.nr + a.ir[pt]];
                uq = v * 1.0e3;
            }
        }
        cd* row = a.h + (size_t)b * a.ns * nh + n;
        if (a.types & DSM_KER_VP) {
            *row = herm_proj(up, n, a.np1, a.fmin);
            row += nh;
        }
        if (a.types & DSM_KER_VS) {
            row[0] = herm_proj(us, n, a.np1, a.fmin);
            row[nh] = herm_proj(uq, n, a.np1, a.fmin);
        }
    }
}

// The filter and trapezoid stage runs per (batch point, series, filter)
// "item".  The forward Butterworth recursion of rekurs (bwfilt.f90:54-90) is
// linear in its state (the last two inputs and both delayed outputs of every
// section), so the samples 0..T-1 an item needs are cut into G segments of
// L samples: k_ker_seg_zs runs every segment but the last from a zero state
// and keeps its end state; k_ker_seg_chain walks the segments in order,
// start(g+1) = P start(g) + end_zero(g), with P the recursion's transfer
// over L samples without input (formed on the host); k_ker_time then runs
// each segment from its true start state, producing the filtered samples
// and the segment's part of the trapezoid sums of the series' kernel types
// over nt1..nt2 (half weights at both ends, calculateK.f90:302-321,
// :497-513); k_ker_seg_sum adds the parts in segment order.  The samples
// are vectorFFT_double's window (exp(omegai t) / tlen * 1e3, as
// k_cat_window forms them).
struct KerTimeArgs {
    const double* y;      // transform rows, 2 (np1 + 1) reals apart
    const double* e;      // exp(omegai t / samplingHz) over the window
    const double* coeff;  // coeff, sample-major: [ir][k - 1][filter][window sample]
    const double* fc;     // [filter][a | b1 | b2][KER_MAXNP]
    const double* P;      // [filter][D][D] transfer over L samples, D = 2 + 2 NP
    const int *nt1, *nt2; // window-relative, per filter
    const int* ir;
    int p0, nb, ns, nfl, nr, nktype, nwin, iws, row, types, gmax;
    int segL[KER_MAXFL], segG[KER_MAXFL];
    double tlen;
    double* zs;           // [item][gmax][D] zero-state end states
    double* st;           // [item][gmax][D] segment start states
    double* part;         // [item][gmax][3] trapezoid parts
    double* ker;          // [point][nfl][nktype + 1]
    double* filt;         // [point][ns][nfl][nwin] or null
};

constexpr int KER_TB = 32;   // one warp per block
constexpr int KER_CH = 8;    // samples (and their coefficients) loaded ahead of the recursion

// kernel types fed by series s: kind 0 P du (1, 3, 4), 1 S du (5, 7), 2 S duq (8)
__device__ __forceinline__ void ker_types(const KerTimeArgs& a, int s, int& kind, int& nk, int& k0, int& k1, int& k2) {
    kind = (a.types & DSM_KER_VP) ? s : s + 1;
    nk = kind == 0 ? 3 : kind == 1 ? 2 : 1;
    k0 = kind == 0 ? 1 : kind == 1 ? 5 : 8;
    k1 = kind == 0 ? 3 : kind == 1 ? 7 : k0;
    k2 = kind == 0 ? 4 : k1;
}

template <int NP>
struct Bw {
    double A[NP], B1[NP], B2[NP], z1[NP], z2[NP], x1, x2;
    __device__ __forceinline__ void load(const double* fc) {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            A[k] = fc[k];
            B1[k] = fc[KER_MAXNP + k];
            B2[k] = fc[2 * KER_MAXNP + k];
            z1[k] = 0.0;
            z2[k] = 0.0;
        }
        x1 = 0.0;
        x2 = 0.0;
    }
    // state order: x1, x2, z1[0..NP), z2[0..NP)
    __device__ __forceinline__ void set_state(const double* q) {
        x1 = q[0];
        x2 = q[1];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            z1[k] = q[2 + k];
            z2[k] = q[2 + NP + k];
        }
    }
    __device__ __forceinline__ void get_state(double* q) const {
        q[0] = x1;
        q[1] = x2;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            q[2 + k] = z1[k];
            q[2 + NP + k] = z2[k];
        }
    }
    // one sample of rekurs (bwfilt.f90:75-89)
    __device__ __forceinline__ double step(double x) {
        double z[NP];
        z[0] = A[0] * (x - x2) - B1[0] * z1[0] - B2[0] * z2[0];
#pragma unroll
        for (int k = 1; k < NP; ++k) z[k] = A[k] * (z[k - 1] - z2[k - 1]) - B1[k] * z1[k] - B2[k] * z2[k];
        x2 = x1;
        x1 = x;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            z2[k] = z1[k];
            z1[k] = z[k];
        }
        return z[NP - 1];
    }
};

struct KerItem {
    int it, g, f, s, b, G, L, tb, te;
};
__device__ __forceinline__ bool ker_item(const KerTimeArgs& a, KerItem& q, bool need_last) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.nb * a.ns * a.nfl * a.gmax) return false;
    q.g = i % a.gmax;
    q.it = i / a.gmax;
    q.f = q.it % a.nfl;
    q.s = (q.it / a.nfl) % a.ns;
    q.b = q.it / (a.nfl * a.ns);
    q.G = a.segG[q.f];
    q.L = a.segL[q.f];
    if (q.g >= (need_last ? q.G : q.G - 1)) return false;
    const int T = a.filt ? a.nwin : a.nt2[q.f] + 1;
    q.tb = q.g * q.L;
    q.te = min(q.tb + q.L, T);
    return true;
}

template <int NP>
__global__ void __launch_bounds__(KER_TB) k_ker_seg_zs(const KerTimeArgs a) {
    KerItem q;
    if (!ker_item(a, q, false)) return;
    Bw<NP> w;
    w.load(a.fc + (size_t)q.f * 3 * KER_MAXNP);
    const double* yr = a.y + ((size_t)q.b * a.ns + q.s) * a.row + a.iws;
    for (int t0 = q.tb; t0 < q.te; t0 += KER_CH) {
        double xs[KER_CH];
#pragma unroll
        for (int j = 0; j < KER_CH; ++j) {
            const int t = min(t0 + j, q.te - 1);
            xs[j] = yr[t] * a.e[t] / a.tlen * 1.0e3;
        }
#pragma unroll
        for (int j = 0; j < KER_CH; ++j)
            if (t0 + j < q.te) w.step(xs[j]);
    }
    w.get_state(a.zs + ((size_t)q.it * a.gmax + q.g) * (2 + 2 * NP));
}

// D lanes per item (32 / D items per warp): lane r keeps state component r
// and row r of P, and gathers the other components by shuffles; the sums
// run in the same order as a one-thread matrix-vector product
template <int NP>
__global__ void __launch_bounds__(KER_TB) k_ker_seg_chain(const KerTimeArgs a) {
    constexpr int D = 2 + 2 * NP;
    constexpr int IPW = 32 / D;
    const int lane = threadIdx.x & 31;
    const int slot = lane / D, r = lane - slot * D;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int it = warp * IPW + slot;
    const bool act = slot < IPW && it < a.nb * a.ns * a.nfl;
    const int itc = act ? it : 0;
    const int f = itc % a.nfl, G = act ? a.segG[f] : 1;
    double prow[D];
#pragma unroll
    for (int c = 0; c < D; ++c) prow[c] = a.P[((size_t)f * D + r) * D + c];
    int gw = G;   // the warp's longest chain: every lane takes part in every shuffle
#pragma unroll
    for (int o = 16; o; o >>= 1) gw = max(gw, __shfl_xor_sync(0xffffffffu, gw, o));
    const int base = slot * D;
    double S = 0.0;
    for (int g = 0; g + 1 < gw; ++g) {
        const bool live = act && g + 1 < G;
        double v = live ? a.zs[((size_t)itc * a.gmax + g) * D + r] : 0.0;
#pragma unroll
        for (int c = 0; c < D; ++c) v = v + prow[c] * __shfl_sync(0xffffffffu, S, (base + c) & 31);
        if (live) {
            S = v;
            a.st[((size_t)itc * a.gmax + g + 1) * D + r] = v;
        }
    }
}

template <int NP>
__global__ void __launch_bounds__(KER_TB) k_ker_time(const KerTimeArgs a) {
    KerItem q;
    if (!ker_item(a, q, true)) return;
    int kind, nk, kt0, kt1, kt2;
    ker_types(a, q.s, kind, nk, kt0, kt1, kt2);
    Bw<NP> w;
    w.load(a.fc + (size_t)q.f * 3 * KER_MAXNP);
    if (q.g > 0) w.set_state(a.st + ((size_t)q.it * a.gmax + q.g) * (2 + 2 * NP));
    const int pt = a.p0 + q.b;
    const int t1 = a.nt1[q.f], t2 = a.nt2[q.f];
    const double* yr = a.y + ((size_t)q.b * a.ns + q.s) * a.row + a.iws;
    const double* cb = a.coeff + ((size_t)a.ir[pt] * a.nktype * a.nfl + q.f) * a.nwin;
    const size_t ks = (size_t)a.nfl * a.nwin;
    const size_t o0 = (kt0 - 1) * ks, o1 = (kt1 - 1) * ks, o2 = (kt2 - 1) * ks;
    double* fo = a.filt ? a.filt + (((size_t)pt * a.ns + q.s) * a.nfl + q.f) * a.nwin : nullptr;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int t0 = q.tb; t0 < q.te; t0 += KER_CH) {
        // the chunk's samples and coefficients first (independent loads, all
        // in flight together); indices clamped into the segment and into
        // nt1..nt2, so every load stays inside the transform row and coeff
        double xs[KER_CH], c0[KER_CH], c1[KER_CH], c2[KER_CH];
#pragma unroll
        for (int j = 0; j < KER_CH; ++j) {
            const int t = min(t0 + j, q.te - 1);
            xs[j] = yr[t] * a.e[t] / a.tlen * 1.0e3;
        }
        const bool in = t0 + KER_CH > t1 && t0 <= t2;
        if (in) {
#pragma unroll
            for (int j = 0; j < KER_CH; ++j) {
                const double* c = cb + min(max(t0 + j, t1), t2);
                c0[j] = c[o0];
                c1[j] = c[o1];
                c2[j] = c[o2];
            }
        }
#pragma unroll
        for (int j = 0; j < KER_CH; ++j) {
            const int t = t0 + j;
            if (t >= q.te) break;
            const double v = w.step(xs[j]);
            if (fo) fo[t] = v;
            if (t < t1 || t > t2) continue;
            // isovpfreq halves as coeff * duf / 2, isovsfreq as 0.5 * coeff * duf
            const double h0 = kind == 0 ? c0[j] * v / 2.0 : 0.5 * c0[j] * v;
            const double h1 = kind == 0 ? c1[j] * v / 2.0 : 0.5 * c1[j] * v;
            const double h2 = c2[j] * v / 2.0;
            if (t == t1) {
                acc0 = acc0 + h0;
                acc1 = acc1 + h1;
                acc2 = acc2 + h2;
            }
            if (t > t1 && t < t2) {
                acc0 = acc0 + c0[j] * v;
                acc1 = acc1 + c1[j] * v;
                acc2 = acc2 + c2[j] * v;
            }
            if (t == t2) {
                acc0 = acc0 + h0;
                acc1 = acc1 + h1;
                acc2 = acc2 + h2;
            }
        }
    }
    double* pp = a.part + ((size_t)q.it * a.gmax + q.g) * 3;
    pp[0] = acc0;
    pp[1] = acc1;
    pp[2] = acc2;
}

// The filters alone on window series (calculateRSGT / calculateTSGT,
// calculateK.f90:1-130): one thread per (series, filter), the samples in
// order (rekurs, bwfilt.f90:75-89), the next 8 loaded ahead.
template <int NP>
__global__ void __launch_bounds__(KER_TB) k_cat_bwfilt(const double* __restrict__ in, int nseries, int nfl, int nwin,
                                                       const double* __restrict__ fc, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseries * nfl) return;
    const int f = i % nfl, sr = i / nfl;
    Bw<NP> w;
    w.load(fc + (size_t)f * 3 * KER_MAXNP);
    const double* x = in + (size_t)sr * nwin;
    double* y = out + ((size_t)sr * nfl + f) * nwin;
    for (int t0 = 0; t0 < nwin; t0 += KER_CH) {
        double xs[KER_CH];
#pragma unroll
        for (int j = 0; j < KER_CH; ++j) xs[j] = x[min(t0 + j, nwin - 1)];
#pragma unroll
        for (int j = 0; j < KER_CH; ++j)
            if (t0 + j < nwin) y[t0 + j] = w.step(xs[j]);
    }
}

__global__ void __launch_bounds__(128) k_ker_seg_sum(const KerTimeArgs a) {
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= a.nb * a.ns * a.nfl) return;
    const int f = it % a.nfl, s = (it / a.nfl) % a.ns, b = it / (a.nfl * a.ns);
    int kind, nk, kt0, kt1, kt2;
    ker_types(a, s, kind, nk, kt0, kt1, kt2);
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int g = 0; g < a.segG[f]; ++g) {
        const double* pp = a.part + ((size_t)it * a.gmax + g) * 3;
        acc0 = acc0 + pp[0];
        acc1 = acc1 + pp[1];
        acc2 = acc2 + pp[2];
    }
    double* ko = a.ker + ((size_t)(a.p0 + b) * a.nfl + f) * (a.nktype + 1);
    ko[kt0] = acc0;
    if (nk > 1) ko[kt1] = acc1;
    if (nk > 2) ko[kt2] = acc2;
}

}  // namespace cat

#define DSM_CUFFT(x)                                                                      \
    do {                                                                                    \
        cufftResult r_ = (x);                                                               \
        if (r_ != CUFFT_SUCCESS)                                                            \
            throw ::dsm::Error(DSM_ERR_CUDA, std::string(#x ": cufft status ") + std::to_string((int)r_)); \
    } while (0)

}  // namespace dsm

using namespace dsm;
using namespace dsm::cat;

struct dsm_cat {
    dsm_cat_params_t p{};
    int dev = 0;
    cudaStream_t st = nullptr;
    std::string err;
    std::vector<SetDev> sets;
    DBuf<unsigned char> own[MAX_SETS];   // device copies of host record sets, kept across clears
    DBuf<int> orig;
    DBuf<Tile> tiles;
    DBuf<double> wt, norm, dist, coef, e, out;
    DBuf<cd> om;     // frequency-domain SGT of the covered catalogue distances
    DBuf<cd> spec;   // spectra copied in or out (dsm_cat_spectra, dsm_cat_transform)
    DBuf<cd> h;
    std::vector<double> he;
    std::map<int, cufftHandle> plans;   // batch -> plan
    size_t max_batch_bytes = (size_t)2 << 30;
    bool profiling = false;
    dsm_stats_t stats{};
    cudaEvent_t ev[8]{};
    // per-point kernels (dsm_cat_set_kernel_params): filters, integration
    // windows, coeff and jacobianFuji resident on the device
    bool kset = false;
    int ktypes = 0, kns = 0, knfl = 0, knp = 0, knr = 0, knkt = 0;
    DBuf<double> kcoef, kfc, kker, kfilt, kzs, kst, kpart, kP, kfin;
    std::vector<double> kfc_h;   // host copies for the segment transfers
    std::vector<int> knt_h;
    DBuf<cd> kjac, kh3, kh4;
    DBuf<int> knt, kir;

    ~dsm_cat() {
        if (dev >= 0) cudaSetDevice(dev);
        for (auto& kv : plans) cufftDestroy(kv.second);
        for (auto& x : ev)
            if (x) cudaEventDestroy(x);
        if (st) cudaStreamDestroy(st);
    }
    int nwin() const { return p.iwin_end - p.iwin_start + 1; }
    cufftHandle plan(int batch) {
        auto it = plans.find(batch);
        if (it != plans.end()) return it->second;
        if (plans.size() >= 8) {
            DSM_CUDA(cudaStreamSynchronize(st));
            for (auto& kv : plans) cufftDestroy(kv.second);
            plans.clear();
        }
        cufftHandle h0;
        int N = 2 * p.np1, inembed = p.np1 + 1, onembed = 2 * (p.np1 + 1);
        DSM_CUFFT(cufftPlanMany(&h0, 1, &N, &inembed, 1, p.np1 + 1, &onembed, 1, 2 * (p.np1 + 1), CUFFT_Z2D, batch));
        DSM_CUFFT(cufftSetStream(h0, st));
        plans[batch] = h0;
        return h0;
    }
};

namespace {
thread_local std::string g_cat_err;

template <class F>
int cat_guard(dsm_cat_t* c, F f) {
    try {
        f();
        return DSM_OK;
    } catch (const Error& e) {
        (c ? c->err : g_cat_err) = e.what();
        return e.code;
    } catch (const std::exception& e) {
        (c ? c->err : g_cat_err) = e.what();
        return DSM_ERR_INVALID;
    }
}

void need(bool ok, const std::string& m) {
    if (!ok) throw Error(DSM_ERR_INVALID, m);
}

// findIdeltaRegion (fourier.f90:165-190), 1-based
void idelta_region(int ix, int nhalf, int nmax, int& is, int& ie) {
    is = ix - nhalf;
    ie = ix + nhalf;
    if (is < 1) {
        ie += 1 - is;
        is = 1;
    }
    if (ie > nmax) {
        is -= ie - nmax;
        ie = nmax;
    }
    if (is < 1) is = 1;
    if (ie > nmax) ie = nmax;
}
}  // namespace

extern "C" int dsm_cat_np1(double tlen, int fmax, double sampling_hz, double start, double end, int* np1,
                           double* sampling_hz_out, int* iwin_start, int* iwin_end) {
    return cat_guard(nullptr, [&] {
        need(tlen > 0 && fmax >= 0 && sampling_hz > 0 && np1, "dsm_cat_np1: bad argument");
        // lsmoothfinder (others.f90:288-308) and KernelMaker-1.0.0.f90:311-330
        long long np_ = 1;
        while (np_ < fmax) np_ *= 2;
        int lsmooth = (int)(0.5 * tlen * sampling_hz / (double)np_);
        int i = 1;
        while (i < lsmooth) i *= 2;
        lsmooth = i;
        long long n1 = 1;
        while (n1 < fmax) n1 *= 2;
        n1 *= lsmooth;
        need(n1 <= (1 << 26), "dsm_cat_np1: transform length too large");
        *np1 = (int)n1;
        const double shz = (double)(2 * n1) / tlen;
        if (sampling_hz_out) *sampling_hz_out = shz;
        if (iwin_start) *iwin_start = (int)(start * shz);
        if (iwin_end) *iwin_end = (int)(end * shz);
    });
}

extern "C" int dsm_cat_create(const dsm_cat_params_t* p, dsm_cat_t** out) {
    if (!out) return DSM_ERR_INVALID;
    *out = nullptr;
    auto c = std::make_unique<dsm_cat_t>();
    const int rc = cat_guard(nullptr, [&] {
        need(p != nullptr, "dsm_cat_create: null parameters");
        need(p->num >= 1 && p->num <= MAX_NUM, "dsm_cat_create: num must be in [1, 32]");
        need(p->theta_n >= 1 && p->theta_delta > 0, "dsm_cat_create: bad catalogue distance grid");
        need(p->fmin >= 0 && p->fmax >= p->fmin, "dsm_cat_create: bad frequency range");
        need(p->np1 >= 1 && (p->np1 & (p->np1 - 1)) == 0 && p->np1 >= p->fmax,
             "dsm_cat_create: np1 must be a power of two >= fmax");
        need(p->np1 <= (1 << 26), "dsm_cat_create: np1 too large");
        need(p->tlen > 0, "dsm_cat_create: tlen must be positive");
        need(p->iwin_start >= 0 && p->iwin_end >= p->iwin_start && p->iwin_end < 2 * p->np1,
             "dsm_cat_create: window must lie in [0, 2 np1)");
        need(p->ipdistance >= 0, "dsm_cat_create: negative ipdistance");
        need((int)(p->ipdistance / p->theta_delta / 2.0) <= (MAX_NW - 1) / 2,
             "dsm_cat_create: sinc window wider than 255 catalogue distances");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || p->device < 0 || p->device >= n)
            throw Error(DSM_ERR_NODEVICE, "dsm_cat_create: no CUDA device (or the ordinal is out of range)");
        c->p = *p;
        c->dev = p->device;
        DSM_CUDA(cudaSetDevice(c->dev));
        DSM_CUDA(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
        for (auto& x : c->ev) DSM_CUDA(cudaEventCreate(&x));
        // window factors exp(omegai i / samplingHz), samplingHz = 2 np1 / tlen
        const double shz = (double)(2 * p->np1) / p->tlen;
        c->he.resize(c->nwin());
        for (int t = 0; t < c->nwin(); ++t) c->he[t] = std::exp(p->omegai * (double)(p->iwin_start + t) / shz);
        c->e.upload(c->he, c->st);
        DSM_CUDA(cudaStreamSynchronize(c->st));
    });
    if (rc != DSM_OK) return rc;
    *out = c.release();
    return DSM_OK;
}

extern "C" int dsm_cat_clear(dsm_cat_t* c) {
    if (!c) return DSM_ERR_INVALID;
    return cat_guard(c, [&] { c->sets.clear(); });
}

extern "C" int dsm_cat_add(dsm_cat_t* c, const void* rec, int elem_bytes, int ncomp, const int* dst,
                           const double* scale, int on_device) {
    if (!c) return DSM_ERR_INVALID;
    return cat_guard(c, [&] {
        need(rec != nullptr, "dsm_cat_add: null records");
        need(elem_bytes == 8 || elem_bytes == 16, "dsm_cat_add: elem_bytes must be 8 (complex64) or 16 (complex128)");
        need(ncomp >= 1 && ncomp <= MAX_NUM, "dsm_cat_add: ncomp must be in [1, 32]");
        need((int)c->sets.size() < MAX_SETS, "dsm_cat_add: at most 4 record sets");
        SetDev s{};
        for (int d = 0; d < MAX_NUM; ++d) s.src[d] = -1;
        for (int k = 0; k < ncomp; ++k) {
            const int d = dst ? dst[k] : k;
            need(d >= 0 && d < c->p.num, "dsm_cat_add: destination component out of range");
            need(s.src[d] < 0, "dsm_cat_add: two record components map to one destination");
            s.src[d] = k;
            s.scale[k] = scale ? scale[k] : 1.0;
            need(std::isfinite(s.scale[k]), "dsm_cat_add: non-finite scale");
        }
        s.cplx64 = elem_bytes == 8;
        s.ncomp = ncomp;
        const size_t bytes = (size_t)(c->p.fmax - c->p.fmin + 1) * c->p.theta_n * ncomp * elem_bytes;
        DSM_CUDA(cudaSetDevice(c->dev));
        if (on_device) {
            need(((uintptr_t)rec % elem_bytes) == 0, "dsm_cat_add: misaligned device records");
            s.rec = rec;
        } else {
            auto& buf = c->own[c->sets.size()];
            buf.reserve(bytes);
            DSM_CUDA(cudaMemcpyAsync(buf.p, rec, bytes, cudaMemcpyHostToDevice, c->st));
            s.rec = buf.p;
        }
        c->sets.push_back(s);
    });
}

namespace {
template <int C>
void launch_interp(const InterpArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
    DSM_CUDA(cudaFuncSetAttribute(k_cat_interp<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_cat_interp<C><<<grid, CAT_THREADS, smem, st>>>(a);
}
void launch_interp_c(int C, const InterpArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
    switch (C) {
        case 1: launch_interp<1>(a, grid, smem, st); break;
        case 2: launch_interp<2>(a, grid, smem, st); break;
        case 3: launch_interp<3>(a, grid, smem, st); break;
        case 4: launch_interp<4>(a, grid, smem, st); break;
        case 5: launch_interp<5>(a, grid, smem, st); break;
        case 6: launch_interp<6>(a, grid, smem, st); break;
        case 7: launch_interp<7>(a, grid, smem, st); break;
        default: launch_interp<8>(a, grid, smem, st); break;
    }
    DSM_CUDA(cudaGetLastError());
}
}  // namespace

namespace {
// Points of dsm_cat_series (time series, spectra = false) and of
// dsm_cat_spectra (the combined spectra before the transform, spectra =
// true: out is complex128 [point][nout][fmax-fmin+1]).
int cat_points(dsm_cat_t* c, int npoint, const double* distance, int nout, const double* coef, void* out,
               int out_on_device, bool spectra) {
    if (!c) return DSM_ERR_INVALID;
    const std::string fn = spectra ? "dsm_cat_spectra" : "dsm_cat_series";
    return cat_guard(c, [&] {
        const dsm_cat_params_t& p = c->p;
        need(npoint >= 0 && (npoint == 0 || (distance && out)), fn + ": null argument");
        need(!c->sets.empty(), fn + ": no record set added");
        const bool identity = coef == nullptr;
        if (identity) nout = p.num;
        need(nout >= 1 && nout <= MAX_OUT, fn + ": nout must be in [1, 64]");
        // device outputs are written with 16-byte (complex128 spectra) or
        // 8-byte (series) stores
        if (out_on_device)
            need(((uintptr_t)out % (spectra ? 16 : 8)) == 0, fn + ": misaligned device output");
        if (npoint == 0) return;
        DSM_CUDA(cudaSetDevice(c->dev));
        const int nh = p.np1 + 1, nwin = c->nwin();
        // sinc windows and weights (clsgt, fourier.f90:136-155), on the host
        const int nhregion = (int)(p.ipdistance / p.theta_delta / 2.0);
        const int nwmax = std::min(2 * nhregion + 1, p.theta_n);
        std::vector<int> wid(npoint), wn(npoint);
        std::vector<double> ww((size_t)npoint * nwmax, 0.0), wnorm(npoint);
        for (int k = 0; k < npoint; ++k) {
            const double dk = distance[k];
            need(std::isfinite(dk), fn + ": non-finite distance");
            const double q = (dk - p.theta_min) / p.theta_delta;
            need(std::fabs(q) < 1e9, fn + ": distance far outside the catalogue");
            const int idelta = 1 + (int)q;   // Fortran int(): truncation toward zero
            int is, ie;
            idelta_region(idelta, nhregion, p.theta_n, is, ie);
            wid[k] = is - 1;
            wn[k] = ie - is + 1;
            const double th_s = p.theta_min + (double)(is - 1) * p.theta_delta;
            double nrm = 0.0;
            for (int kk = is; kk <= ie; ++kk) {
                const double t = kPi * ((dk - th_s) / p.theta_delta - (double)(kk - is));
                const double wv = t == 0.0 ? 1.0 : std::sin(t) / t;
                ww[(size_t)k * nwmax + (kk - is)] = wv;
                nrm = nrm + wv;
            }
            need(nrm != 0.0 && std::isfinite(nrm), fn + ": sinc weights sum to zero");
            wnorm[k] = nrm;
        }
        if (!identity)
            for (size_t i = 0; i < (size_t)npoint * nout * p.num; ++i)
                need(std::isfinite(coef[i]), fn + ": non-finite coefficient");
        // points sorted by window start (then distance); per-point arrays in that order
        std::vector<int> ord(npoint);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
            return wid[x] != wid[y] ? wid[x] < wid[y] : distance[x] < distance[y];
        });
        std::vector<int> hids(npoint), hnw(npoint);
        std::vector<double> hw((size_t)npoint * nwmax), hnorm(npoint), hdist(npoint);
        for (int s = 0; s < npoint; ++s) {
            const int k = ord[s];
            hids[s] = wid[k];
            hnw[s] = wn[k];
            hnorm[s] = wnorm[k];
            hdist[s] = distance[k];
            std::copy(ww.begin() + (size_t)k * nwmax, ww.begin() + (size_t)(k + 1) * nwmax, hw.begin() + (size_t)s * nwmax);
        }

        // points per batch: the in-place transform buffer stays under max_batch_bytes
        const size_t per_point = (size_t)nout * nh * sizeof(cd);
        int pc = (int)std::max<size_t>(1, c->max_batch_bytes / per_point);
        pc = std::min(pc, npoint);
        const int nump = (p.num + 3) / 4 * 4;
        // rows of the frequency-domain SGT: the catalogue distances some window covers
        int ubase = p.theta_n, uend = 0;
        for (int k = 0; k < npoint; ++k) {
            ubase = std::min(ubase, hids[k]);
            uend = std::max(uend, hids[k] + hnw[k]);
        }
        const int ucov = uend - ubase;
        // tiles: consecutive sorted points of one batch, at most PT, band at
        // most nwmax + 64 catalogue distances wide and rounded up to a
        // multiple of 4 (the product's k step); dense weights [U][WS], zero
        // outside each point's window.  The frequency-domain SGT has 4 zero
        // rows after the covered distances for the rounding.
        std::vector<Tile> tiles;
        std::vector<int> tile_begin;   // first tile of each batch
        std::vector<double> hwt;
        for (int b0 = 0; b0 < npoint; b0 += pc) {
            const int b1 = std::min(npoint, b0 + pc);
            tile_begin.push_back((int)tiles.size());
            int s = b0;
            while (s < b1) {
                int lo = hids[s], hi = hids[s] + hnw[s];
                int e = s + 1;
                while (e < b1 && e - s < PT) {
                    const int lo2 = std::min(lo, hids[e]), hi2 = std::max(hi, hids[e] + hnw[e]);
                    if (hi2 - lo2 > nwmax + 64) break;
                    lo = lo2;
                    hi = hi2;
                    ++e;
                }
                const int U = (hi - lo + 3) / 4 * 4;
                const long long woff = (long long)hwt.size();
                hwt.resize(hwt.size() + (size_t)U * WS, 0.0);
                for (int t = s; t < e; ++t)
                    for (int q = 0; q < hnw[t]; ++q)
                        hwt[woff + (size_t)(hids[t] + q - lo) * WS + (t - s)] = hw[(size_t)t * nwmax + q];
                tiles.push_back(Tile{s - b0, e - s, lo - ubase, U, woff});
                s = e;
            }
        }
        tile_begin.push_back((int)tiles.size());

        auto& S = c->stats;
        S = dsm_stats_t{};
        const bool prof = c->profiling;
        if (prof) DSM_CUDA(cudaEventRecord(c->ev[0], c->st));
        c->wt.upload(hwt.data(), hwt.size(), c->st);
        c->norm.upload(hnorm.data(), npoint, c->st);
        c->dist.upload(hdist.data(), npoint, c->st);
        c->orig.upload(ord.data(), npoint, c->st);
        c->tiles.upload(tiles.data(), tiles.size(), c->st);
        if (!identity) c->coef.upload(coef, (size_t)npoint * nout * p.num, c->st);
        const int nf = p.fmax - p.fmin + 1;
        double* dout = static_cast<double*>(out);
        cd* dspec = static_cast<cd*>(out);
        if (!out_on_device) {
            if (spectra) {
                c->spec.reserve((size_t)npoint * nout * nf);
                dspec = c->spec.p;
            } else {
                c->out.reserve((size_t)npoint * nout * nwin);
                dout = c->out.p;
            }
        }
        if (!spectra) c->h.reserve((size_t)pc * nout * nh);

        const int urows = ucov + 4;
        c->om.reserve((size_t)nf * urows * nump);
        OmegaArgs oa{};
        oa.nset = (int)c->sets.size();
        for (int s = 0; s < oa.nset; ++s) oa.set[s] = c->sets[s];
        oa.num = p.num;
        oa.nump = nump;
        oa.theta_n = p.theta_n;
        oa.fmin = p.fmin;
        oa.nf = nf;
        oa.u0 = ubase;
        oa.ucov = ucov;
        oa.urows = urows;
        oa.theta_min = p.theta_min;
        oa.theta_delta = p.theta_delta;
        oa.tlen = p.tlen;
        oa.c_red_reci = p.c_red_reci;
        oa.om = c->om.p;
        if (prof) DSM_CUDA(cudaEventRecord(c->ev[6], c->st));
        need((size_t)urows * nump < (1u << 30), fn + ": catalogue rows too large");
        k_cat_omega<<<dim3((urows * nump + 255) / 256, std::min(nf, 65535)), 256, 0, c->st>>>(oa);
        DSM_CUDA(cudaGetLastError());
        if (prof) DSM_CUDA(cudaEventRecord(c->ev[7], c->st));
        S.launches += 1;

        InterpArgs a{};
        a.num = p.num;
        a.nout = nout;
        a.identity = identity;
        a.fmin = p.fmin;
        a.fmax = p.fmax;
        a.np1 = p.np1;
        a.ucov = urows;
        a.tlen = p.tlen;
        a.c_red_reci = p.c_red_reci;
        a.om = c->om.p;
        a.wt = c->wt.p;
        a.coef = identity ? nullptr : c->coef.p;
        a.h = c->h.p;
        a.spec = spectra ? dspec : nullptr;
        const size_t smem = interp_smem_bytes(nump / 4);
        double ms_i = 0, ms_f = 0, ms_w = 0;
        int nbatch = 0;
        for (int b0 = 0, bi = 0; b0 < npoint; b0 += pc, ++bi) {
            const int np_ = std::min(pc, npoint - b0);
            a.tiles = c->tiles.p + tile_begin[bi];
            a.norm = c->norm.p + b0;
            a.dist = c->dist.p + b0;
            a.orig = c->orig.p + b0;
            if (prof) DSM_CUDA(cudaEventRecord(c->ev[1], c->st));
            a.ntile = tile_begin[bi + 1] - tile_begin[bi];
            const long long nblk = (long long)a.ntile * ((nh + CAT_WARPS - 1) / CAT_WARPS);
            need(nblk < (1LL << 31), fn + ": too many point tiles x frequency blocks in one batch");
            launch_interp_c(nump / 4, a, dim3((unsigned)nblk), smem, c->st);
            if (prof) DSM_CUDA(cudaEventRecord(c->ev[2], c->st));
            if (spectra) {
                S.launches += 1;
                ++nbatch;
                if (prof) {
                    DSM_CUDA(cudaEventSynchronize(c->ev[2]));
                    float t1;
                    cudaEventElapsedTime(&t1, c->ev[1], c->ev[2]);
                    ms_i += t1;
                }
                continue;
            }
            const int nb = np_ * nout;
            DSM_CUFFT(cufftExecZ2D(c->plan(nb), reinterpret_cast<cufftDoubleComplex*>(c->h.p),
                                   reinterpret_cast<cufftDoubleReal*>(c->h.p)));
            if (prof) DSM_CUDA(cudaEventRecord(c->ev[3], c->st));
            const size_t total = (size_t)nb * nwin;
            const int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)148 * 16);
            k_cat_window<<<blocks, 256, 0, c->st>>>(reinterpret_cast<const double*>(c->h.p), 2 * nh, p.iwin_start,
                                                    nwin, nb, nout, c->orig.p + b0, c->e.p, p.tlen, dout);
            DSM_CUDA(cudaGetLastError());
            S.launches += 2;   // interp + window (the transform is cuFFT's)
            ++nbatch;
            if (prof) {
                DSM_CUDA(cudaEventRecord(c->ev[4], c->st));
                DSM_CUDA(cudaEventSynchronize(c->ev[4]));
                float t1, t2, t3;
                cudaEventElapsedTime(&t1, c->ev[1], c->ev[2]);
                cudaEventElapsedTime(&t2, c->ev[2], c->ev[3]);
                cudaEventElapsedTime(&t3, c->ev[3], c->ev[4]);
                ms_i += t1;
                ms_f += t2;
                ms_w += t3;
            }
        }
        if (!out_on_device) {
            if (spectra)
                DSM_CUDA(cudaMemcpyAsync(out, dspec, (size_t)npoint * nout * nf * sizeof(cd), cudaMemcpyDeviceToHost,
                                         c->st));
            else
                DSM_CUDA(cudaMemcpyAsync(out, dout, (size_t)npoint * nout * nwin * sizeof(double),
                                         cudaMemcpyDeviceToHost, c->st));
        }
        if (prof) DSM_CUDA(cudaEventRecord(c->ev[5], c->st));
        DSM_CUDA(cudaStreamSynchronize(c->st));
        if (prof) {
            float tt;
            cudaEventElapsedTime(&tt, c->ev[0], c->ev[5]);
            S.ms_total = tt;
            // algorithmic bytes: the records of the covered catalogue
            // distances read once and the frequency-domain SGT written
            // (omega); that SGT read once and H written (interp); H read and
            // written (transform); window samples read and written.  Flops of
            // the interpolation: 4 per weight, frequency and component.
            float to;
            cudaEventElapsedTime(&to, c->ev[6], c->ev[7]);
            std::vector<char> cover(p.theta_n, 0);
            double wterms = 0;
            for (int k = 0; k < npoint; ++k) {
                for (int q = 0; q < hnw[k]; ++q) cover[hids[k] + q] = 1;
                wterms += hnw[k];
            }
            double ncov = 0;
            for (char x : cover) ncov += x;
            double rec_bytes = 0;
            for (auto& s : c->sets) rec_bytes += (double)nf * ncov * s.ncomp * (s.cplx64 ? 8.0 : 16.0);
            const double ob = (double)nf * ncov * p.num * sizeof(cd);
            const double hb = (double)npoint * nout * nh * sizeof(cd);
            const double wb = 2.0 * npoint * nout * nwin * sizeof(double);
            const char* nm[4] = {"cat_omega", "cat_interp", "cat_fft", "cat_window"};
            const double ms[4] = {to, ms_i, ms_f, ms_w};
            const double by[4] = {rec_bytes + ob, ob + hb, 2.0 * hb, wb};
            const double fl[4] = {0.0, 4.0 * wterms * nf * p.num, 0.0, 0.0};
            for (int k = 0; k < 4; ++k) {
                snprintf(S.kern[k].name, sizeof(S.kern[k].name), "%s", nm[k]);
                S.kern[k].ms = ms[k];
                S.kern[k].launches = k == 0 ? 1 : nbatch;
                S.kern[k].alg_bytes = by[k];
                S.kern[k].alg_flops = fl[k];
            }
            S.nk = 4;
        }
    });
}
}  // namespace

extern "C" int dsm_cat_series(dsm_cat_t* c, int npoint, const double* distance, int nout, const double* coef,
                              double* out, int out_on_device) {
    return cat_points(c, npoint, distance, nout, coef, out, out_on_device, false);
}

extern "C" int dsm_cat_spectra(dsm_cat_t* c, int npoint, const double* distance, int nout, const double* coef,
                               void* out, int out_on_device) {
    return cat_points(c, npoint, distance, nout, coef, out, out_on_device, true);
}

extern "C" int dsm_cat_transform(dsm_cat_t* c, int nseries, const void* spectra, int spectra_on_device,
                                 double* out, int out_on_device) {
    if (!c) return DSM_ERR_INVALID;
    return cat_guard(c, [&] {
        const dsm_cat_params_t& p = c->p;
        need(nseries >= 0 && (nseries == 0 || (spectra && out)), "dsm_cat_transform: null argument");
        if (nseries == 0) return;
        DSM_CUDA(cudaSetDevice(c->dev));
        const int nh = p.np1 + 1, nwin = c->nwin(), nf = p.fmax - p.fmin + 1;
        if (spectra_on_device)
            need(((uintptr_t)spectra % 16) == 0, "dsm_cat_transform: misaligned device spectra");
        if (out_on_device) need(((uintptr_t)out % 8) == 0, "dsm_cat_transform: misaligned device output");
        // series per batch: the in-place transform buffer stays under max_batch_bytes
        const int pc = (int)std::min<size_t>((size_t)nseries, std::max<size_t>(1, c->max_batch_bytes / (nh * sizeof(cd))));
        const cd* dx = static_cast<const cd*>(spectra);
        if (!spectra_on_device) {
            c->spec.upload(static_cast<const cd*>(spectra), (size_t)nseries * nf, c->st);
            dx = c->spec.p;
        }
        double* dout = out;
        if (!out_on_device) {
            c->out.reserve((size_t)nseries * nwin);
            dout = c->out.p;
        }
        c->h.reserve((size_t)pc * nh);
        std::vector<int> iota_h(pc);
        std::iota(iota_h.begin(), iota_h.end(), 0);
        c->orig.upload(iota_h.data(), pc, c->st);
        for (int b0 = 0; b0 < nseries; b0 += pc) {
            const int nb = std::min(pc, nseries - b0);
            k_cat_herm<<<dim3((nh + 255) / 256, std::min(nb, 65535)), 256, 0, c->st>>>(dx + (size_t)b0 * nf, nb, p.fmin,
                                                                                      p.fmax, p.np1, c->h.p);
            DSM_CUDA(cudaGetLastError());
            DSM_CUFFT(cufftExecZ2D(c->plan(nb), reinterpret_cast<cufftDoubleComplex*>(c->h.p),
                                   reinterpret_cast<cufftDoubleReal*>(c->h.p)));
            const size_t total = (size_t)nb * nwin;
            const int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)148 * 16);
            k_cat_window<<<blocks, 256, 0, c->st>>>(reinterpret_cast<const double*>(c->h.p), 2 * nh, p.iwin_start,
                                                    nwin, nb, 1, c->orig.p, c->e.p, p.tlen, dout + (size_t)b0 * nwin);
            DSM_CUDA(cudaGetLastError());
        }
        if (!out_on_device)
            DSM_CUDA(cudaMemcpyAsync(out, dout, (size_t)nseries * nwin * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        DSM_CUDA(cudaStreamSynchronize(c->st));
    });
}

namespace {
// bpcoeff (src/KernelMaker/bwfilt.f90:124-166): the npoles second-order
// sections a, b1, b2 of the recursive band-pass [f1, f2] (Hz) at step dt.
// The reference builds its poles from single-precision complex values:
// cexp(cmplx(0, phase)) is a single-precision exponential (cos and sin
// rounded to single here), cmplx(w0, 0) and cmplx(w1 w2, 0) round their
// real parts to single; only s(1..npoles) of the 2 npoles roots are used.
void bpcoeff(double f1, double f2, int npoles, double dt, double* a, double* b1, double* b2) {
    const double pi = 3.141592653589793;
    const double d2 = 2.0 / dt;
    const double w1 = d2 * std::tan(2.0 * pi * f1 / d2);
    const double w2 = d2 * std::tan(2.0 * pi * f2 / d2);
    const double w0 = 0.5 * (w2 - w1);
    auto cm = [](std::complex<double> x, std::complex<double> y) {
        return std::complex<double>(x.real() * y.real() - x.imag() * y.imag(),
                                    x.real() * y.imag() + x.imag() * y.real());
    };
    std::complex<double> s[2 * KER_MAXNP];
    for (int n = 1, i = 0; n <= npoles; ++n, i += 2) {
        const float ph = (float)((double)(2 * n - 1 + npoles) * pi / (double)(2 * npoles));
        const std::complex<double> p((double)(float)std::cos((double)ph), (double)(float)std::sin((double)ph));
        const std::complex<double> t1 = cm(p, std::complex<double>((double)(float)w0, 0.0));
        const std::complex<double> t2 = std::sqrt(cm(t1, t1) - std::complex<double>((double)(float)(w1 * w2), 0.0));
        s[i] = t1 + t2;
        s[i + 1] = t1 - t2;
    }
    for (int n = 0; n < npoles; ++n) {
        const double ssum = 2.0 * s[n].real();
        const double sprod = s[n].real() * s[n].real() - s[n].imag() * (-s[n].imag());
        const double fact1 = d2 * d2 - d2 * ssum + sprod;
        const double fact2 = 2.0 * (sprod - d2 * d2);
        const double fact3 = d2 * d2 + d2 * ssum + sprod;
        a[n] = 2.0 * d2 * w0 / fact1;
        b1[n] = fact2 / fact1;
        b2[n] = fact3 / fact1;
    }
}

template <int NP>
void launch_ker_time(const KerTimeArgs& a, cudaStream_t st) {
    const int nit = a.nb * a.ns * a.nfl, nthr = nit * a.gmax;
    if (a.gmax > 1) {
        k_ker_seg_zs<NP><<<(nthr + KER_TB - 1) / KER_TB, KER_TB, 0, st>>>(a);
        constexpr int ipw = 32 / (2 + 2 * NP);
        k_ker_seg_chain<NP><<<(nit + ipw - 1) / ipw, KER_TB, 0, st>>>(a);
    }
    k_ker_time<NP><<<(nthr + KER_TB - 1) / KER_TB, KER_TB, 0, st>>>(a);
    k_ker_seg_sum<<<(nit + 127) / 128, 128, 0, st>>>(a);
}

// transfer of the recursion over L samples without input, [D][D] row-major
// (column j: the state after L steps from unit state j), D = 2 + 2 npoles
void ker_transfer(const double* fc, int np, int L, double* P) {
    const int D = 2 + 2 * np;
    std::vector<double> q(D);
    for (int j = 0; j < D; ++j) {
        std::fill(q.begin(), q.end(), 0.0);
        q[j] = 1.0;
        double x1 = q[0], x2 = q[1], z1[KER_MAXNP], z2[KER_MAXNP], z[KER_MAXNP];
        for (int k = 0; k < np; ++k) {
            z1[k] = q[2 + k];
            z2[k] = q[2 + np + k];
        }
        for (int t = 0; t < L; ++t) {
            z[0] = fc[0] * (0.0 - x2) - fc[KER_MAXNP] * z1[0] - fc[2 * KER_MAXNP] * z2[0];
            for (int k = 1; k < np; ++k)
                z[k] = fc[k] * (z[k - 1] - z2[k - 1]) - fc[KER_MAXNP + k] * z1[k] - fc[2 * KER_MAXNP + k] * z2[k];
            x2 = x1;
            x1 = 0.0;
            for (int k = 0; k < np; ++k) {
                z2[k] = z1[k];
                z1[k] = z[k];
            }
        }
        P[0 * D + j] = x1;
        P[1 * D + j] = x2;
        for (int k = 0; k < np; ++k) {
            P[(2 + k) * D + j] = z1[k];
            P[(2 + np + k) * D + j] = z2[k];
        }
    }
}
void launch_ker_time_np(int np, const KerTimeArgs& a, cudaStream_t st) {
    switch (np) {
        case 1: launch_ker_time<1>(a, st); break;
        case 2: launch_ker_time<2>(a, st); break;
        case 3: launch_ker_time<3>(a, st); break;
        case 4: launch_ker_time<4>(a, st); break;
        case 5: launch_ker_time<5>(a, st); break;
        case 6: launch_ker_time<6>(a, st); break;
        case 7: launch_ker_time<7>(a, st); break;
        case 8: launch_ker_time<8>(a, st); break;
        case 9: launch_ker_time<9>(a, st); break;
        default: launch_ker_time<10>(a, st); break;
    }
    DSM_CUDA(cudaGetLastError());
}
}  // namespace

extern "C" int dsm_cat_set_kernel_params(dsm_cat_t* c, const dsm_cat_kernel_params_t* kp) {
    if (!c) return DSM_ERR_INVALID;
    return cat_guard(c, [&] {
        const char* fn = "dsm_cat_set_kernel_params";
        need(kp != nullptr, std::string(fn) + ": null parameters");
        const dsm_cat_params_t& p = c->p;
        const int nwin = c->nwin(), nf = p.fmax - p.fmin + 1;
        need(kp->types >= 1 && kp->types <= (DSM_KER_VP | DSM_KER_VS), std::string(fn) + ": types must be VP, VS or both");
        need(kp->nfilter >= 0 && kp->nfilter < KER_MAXFL, std::string(fn) + ": nfilter must be in [0, 15]");
        need(kp->npoles >= 1 && kp->npoles <= KER_MAXNP, std::string(fn) + ": npoles must be in [1, 10]");
        need(std::isfinite(kp->sampling_hz) && kp->sampling_hz > 0, std::string(fn) + ": sampling_hz must be positive");
        need(kp->nr >= 1 && kp->nktype >= 8, std::string(fn) + ": nr >= 1 and nktype >= 8 required");
        need(kp->fclp && kp->fchp && kp->nt1 && kp->nt2 && kp->coeff, std::string(fn) + ": null argument");
        need(!(kp->types & DSM_KER_VS) || kp->jacobian, std::string(fn) + ": VS kernels need jacobianFuji");
        const int nfl = kp->nfilter + 1;
        std::vector<double> fc((size_t)nfl * 3 * KER_MAXNP, 0.0);
        std::vector<int> nt(2 * nfl);
        for (int f = 0; f < nfl; ++f) {
            need(std::isfinite(kp->fclp[f]) && std::isfinite(kp->fchp[f]), std::string(fn) + ": non-finite corner frequency");
            need(kp->nt1[f] >= p.iwin_start && kp->nt1[f] <= kp->nt2[f] && kp->nt2[f] <= p.iwin_end,
                 std::string(fn) + ": nt1/nt2 must satisfy iwin_start <= nt1 <= nt2 <= iwin_end");
            double* q = fc.data() + (size_t)f * 3 * KER_MAXNP;
            bpcoeff(kp->fclp[f], kp->fchp[f], kp->npoles, 1.0 / kp->sampling_hz, q, q + KER_MAXNP, q + 2 * KER_MAXNP);
            for (int k = 0; k < 3 * KER_MAXNP; ++k)
                need(std::isfinite(q[k]), std::string(fn) + ": the filter's coefficients are not finite");
            nt[f] = kp->nt1[f] - p.iwin_start;
            nt[nfl + f] = kp->nt2[f] - p.iwin_start;
        }
        const size_t ncoef = (size_t)nwin * kp->nr * kp->nktype * nfl;
        for (size_t i = 0; i < ncoef; ++i) need(std::isfinite(kp->coeff[i]), std::string(fn) + ": non-finite coeff");
        // sample-major on the device, [ir][k - 1][filter][sample]: a thread's
        // coefficients of consecutive samples are adjacent
        std::vector<double> ct(ncoef);
        const size_t rows = (size_t)kp->nr * kp->nktype * nfl;
        for (int t = 0; t < nwin; ++t)
            for (size_t r = 0; r < rows; ++r) ct[r * nwin + t] = kp->coeff[(size_t)t * rows + r];
        DSM_CUDA(cudaSetDevice(c->dev));
        c->kset = false;
        c->kfc.upload(fc, c->st);
        c->knt.upload(nt, c->st);
        c->kfc_h = fc;
        c->knt_h = nt;
        c->kcoef.upload(ct, c->st);
        if (kp->types & DSM_KER_VS) {
            const cd* j = static_cast<const cd*>(kp->jacobian);
            for (size_t i = 0; i < (size_t)nf * kp->nr; ++i)
                need(std::isfinite(j[i].re) && std::isfinite(j[i].im), std::string(fn) + ": non-finite jacobian");
            c->kjac.upload(j, (size_t)nf * kp->nr, c->st);
        }
        DSM_CUDA(cudaStreamSynchronize(c->st));
        c->ktypes = kp->types;
        c->kns = ((kp->types & DSM_KER_VP) ? 1 : 0) + ((kp->types & DSM_KER_VS) ? 2 : 0);
        c->knfl = nfl;
        c->knp = kp->npoles;
        c->knr = kp->nr;
        c->knkt = kp->nktype;
        c->kset = true;
    });
}

extern "C" int dsm_cat_kernels(dsm_cat_t* c, int npoint, const int* ir, const void* h3, const void* h4,
                               int spectra_on_device, double* ker, double* filtered, int out_on_device) {
    if (!c) return DSM_ERR_INVALID;
    return cat_guard(c, [&] {
        const char* fn = "dsm_cat_kernels";
        need(c->kset, std::string(fn) + ": dsm_cat_set_kernel_params has not been called");
        need(npoint >= 0 && (npoint == 0 || (ir && h3 && h4 && ker)), std::string(fn) + ": null argument");
        if (spectra_on_device)
            need(((uintptr_t)h3 % 16) == 0 && ((uintptr_t)h4 % 16) == 0, std::string(fn) + ": misaligned device spectra");
        if (out_on_device)
            need(((uintptr_t)ker % 8) == 0 && ((uintptr_t)filtered % 8) == 0, std::string(fn) + ": misaligned device output");
        if (npoint == 0) return;
        for (int k = 0; k < npoint; ++k)
            need(ir[k] >= 0 && ir[k] < c->knr, std::string(fn) + ": radius index out of range");
        const dsm_cat_params_t& p = c->p;
        const int nh = p.np1 + 1, nf = p.fmax - p.fmin + 1, nwin = c->nwin();
        const int ns = c->kns, nfl = c->knfl, nkt1 = c->knkt + 1;
        DSM_CUDA(cudaSetDevice(c->dev));
        c->kir.upload(ir, npoint, c->st);
        const cd* d3 = static_cast<const cd*>(h3);
        const cd* d4 = static_cast<const cd*>(h4);
        if (!spectra_on_device) {
            c->kh3.upload(d3, (size_t)npoint * 6 * nf, c->st);
            c->kh4.upload(d4, (size_t)npoint * 6 * nf, c->st);
            d3 = c->kh3.p;
            d4 = c->kh4.p;
        }
        double* dker = ker;
        double* dfilt = filtered;
        if (!out_on_device) {
            c->kker.reserve((size_t)npoint * nfl * nkt1);
            dker = c->kker.p;
            if (filtered) {
                c->kfilt.reserve((size_t)npoint * ns * nfl * nwin);
                dfilt = c->kfilt.p;
            }
        }
        DSM_CUDA(cudaMemsetAsync(dker, 0, (size_t)npoint * nfl * nkt1 * sizeof(double), c->st));
        // segments of each filter's samples (at least 32 samples, at most 16
        // segments) and their transfers
        const int D = 2 + 2 * c->knp;
        std::vector<double> Ph((size_t)nfl * D * D);
        int gmax = 1;
        int segL[KER_MAXFL], segG[KER_MAXFL];
        for (int f = 0; f < nfl; ++f) {
            const int T = filtered ? nwin : c->knt_h[nfl + f] + 1;
            const int L = std::max(32, (T + 15) / 16);
            segL[f] = L;
            segG[f] = (T + L - 1) / L;
            gmax = std::max(gmax, segG[f]);
            ker_transfer(c->kfc_h.data() + (size_t)f * 3 * KER_MAXNP, c->knp, L, Ph.data() + (size_t)f * D * D);
        }
        // points per batch: the in-place transform rows and the segment
        // scratch (end and start states, trapezoid parts) stay under
        // max_batch_bytes, and the stage's threads fit an int
        const size_t per_point =
            (size_t)ns * nh * sizeof(cd) + (size_t)ns * nfl * gmax * (2 * D + 3) * sizeof(double);
        size_t pcs = std::min<size_t>((size_t)npoint, std::max<size_t>(1, c->max_batch_bytes / per_point));
        pcs = std::min<size_t>(pcs, ((size_t)1 << 30) / ((size_t)ns * nfl * gmax));
        const int pc = (int)std::max<size_t>(1, pcs);
        c->h.reserve((size_t)pc * ns * nh);
        KerSpecArgs sa{};
        sa.h3 = d3;
        sa.h4 = d4;
        sa.jac = c->kjac.p;
        sa.ir = c->kir.p;
        sa.nr = c->knr;
        sa.fmin = p.fmin;
        sa.fmax = p.fmax;
        sa.np1 = p.np1;
        sa.types = c->ktypes;
        sa.ns = ns;
        sa.h = c->h.p;
        KerTimeArgs ta{};
        ta.y = reinterpret_cast<const double*>(c->h.p);
        ta.e = c->e.p;
        ta.coeff = c->kcoef.p;
        ta.fc = c->kfc.p;
        ta.nt1 = c->knt.p;
        ta.nt2 = c->knt.p + nfl;
        ta.ir = c->kir.p;
        ta.ns = ns;
        ta.nfl = nfl;
        ta.nr = c->knr;
        ta.nktype = c->knkt;
        ta.nwin = nwin;
        ta.iws = p.iwin_start;
        ta.row = 2 * nh;
        ta.types = c->ktypes;
        ta.tlen = p.tlen;
        ta.ker = dker;
        ta.filt = dfilt;
        ta.gmax = gmax;
        for (int f = 0; f < nfl; ++f) {
            ta.segL[f] = segL[f];
            ta.segG[f] = segG[f];
        }
        c->kP.upload(Ph, c->st);
        ta.P = c->kP.p;
        c->kzs.reserve((size_t)pc * ns * nfl * gmax * D);
        c->kst.reserve((size_t)pc * ns * nfl * gmax * D);
        c->kpart.reserve((size_t)pc * ns * nfl * gmax * 3);
        ta.zs = c->kzs.p;
        ta.st = c->kst.p;
        ta.part = c->kpart.p;
        auto& S = c->stats;
        S = dsm_stats_t{};
        const bool prof = c->profiling;
        if (prof) DSM_CUDA(cudaEventRecord(c->ev[0], c->st));
        double ms_s = 0, ms_f = 0, ms_t = 0;
        int nbatch = 0;
        const int fl_launches = (ta.gmax > 1 ? 4 : 2);
        for (int b0 = 0; b0 < npoint; b0 += pc) {
            const int nb = std::min(pc, npoint - b0);
            sa.p0 = b0;
            sa.nb = nb;
            if (prof) DSM_CUDA(cudaEventRecord(c->ev[1], c->st));
            k_ker_spec<<<dim3((nh + 255) / 256, std::min(nb, 65535)), 256, 0, c->st>>>(sa);
            DSM_CUDA(cudaGetLastError());
            if (prof) DSM_CUDA(cudaEventRecord(c->ev[2], c->st));
            DSM_CUFFT(cufftExecZ2D(c->plan(nb * ns), reinterpret_cast<cufftDoubleComplex*>(c->h.p),
                                   reinterpret_cast<cufftDoubleReal*>(c->h.p)));
            if (prof) DSM_CUDA(cudaEventRecord(c->ev[3], c->st));
            ta.p0 = b0;
            ta.nb = nb;
            launch_ker_time_np(c->knp, ta, c->st);
            S.launches += 1 + fl_launches;
            ++nbatch;
            if (prof) {
                DSM_CUDA(cudaEventRecord(c->ev[4], c->st));
                DSM_CUDA(cudaEventSynchronize(c->ev[4]));
                float t1, t2, t3;
                cudaEventElapsedTime(&t1, c->ev[1], c->ev[2]);
                cudaEventElapsedTime(&t2, c->ev[2], c->ev[3]);
                cudaEventElapsedTime(&t3, c->ev[3], c->ev[4]);
                ms_s += t1;
                ms_f += t2;
                ms_t += t3;
            }
        }
        if (prof) DSM_CUDA(cudaEventRecord(c->ev[5], c->st));
        if (!out_on_device) {
            DSM_CUDA(cudaMemcpyAsync(ker, dker, (size_t)npoint * nfl * nkt1 * sizeof(double), cudaMemcpyDeviceToHost,
                                     c->st));
            if (filtered)
                DSM_CUDA(cudaMemcpyAsync(filtered, dfilt, (size_t)npoint * ns * nfl * nwin * sizeof(double),
                                         cudaMemcpyDeviceToHost, c->st));
        }
        DSM_CUDA(cudaStreamSynchronize(c->st));
        if (prof) {
            float tt;
            cudaEventElapsedTime(&tt, c->ev[0], c->ev[5]);
            S.ms_total = tt;
            // algorithmic bytes: h3 and h4 read once and the transform rows
            // written (products); the rows read and written (transform); the
            // samples each item integrates or writes read once, the filtered
            // series and the kernels written (filter stage)
            double samples = 0;
            for (int f = 0; f < nfl; ++f) samples += filtered ? nwin : c->knt_h[nfl + f] + 1;
            const double rows = (double)npoint * ns * nh * sizeof(cd);
            const double by[3] = {2.0 * npoint * 6 * nf * sizeof(cd) + rows, 2.0 * rows,
                                  (double)npoint * ns * samples * sizeof(double) * (filtered ? 2.0 : 1.0) +
                                      (double)npoint * nfl * nkt1 * sizeof(double)};
            const char* nm[3] = {"ker_spec", "ker_fft", "ker_filter"};
            const double ms[3] = {ms_s, ms_f, ms_t};
            const long long nl[3] = {nbatch, nbatch, (long long)nbatch * fl_launches};
            for (int k = 0; k < 3; ++k) {
                snprintf(S.kern[k].name, sizeof(S.kern[k].name), "%s", nm[k]);
                S.kern[k].ms = ms[k];
                S.kern[k].launches = nl[k];
                S.kern[k].alg_bytes = by[k];
                S.kern[k].alg_flops = 0.0;
            }
            S.nk = 3;
        }
    });
}

namespace {
template <int NP>
void launch_bwfilt(const double* in, int nseries, int nfl, int nwin, const double* fc, double* out, cudaStream_t st) {
    const int n = nseries * nfl;
    k_cat_bwfilt<NP><<<(n + KER_TB - 1) / KER_TB, KER_TB, 0, st>>>(in, nseries, nfl, nwin, fc, out);
}
}  // namespace

extern "C" int dsm_cat_filter(dsm_cat_t* c, int nseries, const double* in, double* out, int on_device) {
    if (!c) return DSM_ERR_INVALID;
    return cat_guard(c, [&] {
        const char* fn = "dsm_cat_filter";
        need(c->kset, std::string(fn) + ": dsm_cat_set_kernel_params has not been called");
        need(nseries >= 0 && (nseries == 0 || (in && out)), std::string(fn) + ": null argument");
        if (on_device)
            need(((uintptr_t)in % 8) == 0 && ((uintptr_t)out % 8) == 0, std::string(fn) + ": misaligned device pointer");
        if (nseries == 0) return;
        const int nwin = c->nwin(), nfl = c->knfl;
        need((long long)nseries * nfl < (1LL << 30), std::string(fn) + ": too many series");
        DSM_CUDA(cudaSetDevice(c->dev));
        const double* din = in;
        double* dout = out;
        if (!on_device) {
            c->kfin.upload(in, (size_t)nseries * nwin, c->st);
            din = c->kfin.p;
            c->kfilt.reserve((size_t)nseries * nfl * nwin);
            dout = c->kfilt.p;
        }
        switch (c->knp) {
            case 1: launch_bwfilt<1>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 2: launch_bwfilt<2>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 3: launch_bwfilt<3>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 4: launch_bwfilt<4>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 5: launch_bwfilt<5>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 6: launch_bwfilt<6>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 7: launch_bwfilt<7>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 8: launch_bwfilt<8>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            case 9: launch_bwfilt<9>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
            default: launch_bwfilt<10>(din, nseries, nfl, nwin, c->kfc.p, dout, c->st); break;
        }
        DSM_CUDA(cudaGetLastError());
        if (!on_device)
            DSM_CUDA(cudaMemcpyAsync(out, dout, (size_t)nseries * nfl * nwin * sizeof(double), cudaMemcpyDeviceToHost,
                                     c->st));
        DSM_CUDA(cudaStreamSynchronize(c->st));
    });
}

namespace {
// a real combination of the catalogue components (the coefficient row of one
// h3 / h4 entry), with the arithmetic the reference's formulas use
template <int N>
struct Comb {
    double c[N] = {};
    static Comb e(int k) {   // component k (1-based, as tsgtF(k) / rsgtF(k))
        Comb r;
        r.c[k - 1] = 1.0;
        return r;
    }
    friend Comb operator+(Comb a, const Comb& b) {
        for (int i = 0; i < N; ++i) a.c[i] += b.c[i];
        return a;
    }
    friend Comb operator-(Comb a, const Comb& b) {
        for (int i = 0; i < N; ++i) a.c[i] -= b.c[i];
        return a;
    }
    friend Comb operator-(Comb a) {
        for (int i = 0; i < N; ++i) a.c[i] = -a.c[i];
        return a;
    }
    friend Comb operator*(Comb a, double m) {
        for (int i = 0; i < N; ++i) a.c[i] *= m;
        return a;
    }
};
}  // namespace

extern "C" int dsm_cat_h3h4_coef(int npoint, const double* ang, char compo, const double* mt, double* coef3,
                                 double* coef4) {
    return cat_guard(nullptr, [&] {
        const char* fn = "dsm_cat_h3h4_coef";
        need(npoint >= 0 && (npoint == 0 || ang), std::string(fn) + ": null argument");
        need(!coef4 || mt, std::string(fn) + ": h4 needs the moment tensor");
        need(!coef3 || compo == 'Z' || compo == 'R' || compo == 'T', std::string(fn) + ": compo must be Z, R or T");
        using C10 = Comb<10>;
        using C20 = Comb<20>;
        for (int p = 0; p < npoint; ++p) {
            const double* a = ang + (size_t)p * 12;
            for (int k = 0; k < 12; ++k) need(std::isfinite(a[k]), std::string(fn) + ": non-finite angle factor");
            const double crq = a[0], srq = a[1], crq2 = a[2], srq2 = a[3];
            const double csq = a[4], ssq = a[5], csq2 = a[6], ssq2 = a[7];
            const double cqs = a[8], sqs = a[9], cqs2 = a[10], sqs2 = a[11];
            if (coef3) {
                // rsgt2h3freq (fourier.f90:278-320); order rr, tt, pp, rt, rp, tp
                C10 h[6];
                auto F = [](int k) { return C10::e(k); };
                if (compo == 'Z') {
                    h[0] = F(1);
                    h[1] = F(3) * crq2 - F(4);
                    h[2] = -F(3) * crq2 - F(4);
                    h[3] = F(2) * (2.0 * crq);
                    h[4] = F(2) * (2.0 * srq);
                    h[5] = F(3) * (2.0 * srq2);
                } else if (compo == 'R') {
                    h[0] = F(5);
                    h[1] = -F(7) * crq2 - F(6);
                    h[2] = F(7) * crq2 - F(6);
                    h[3] = F(9) * (4.0 * crq);
                    h[4] = F(9) * (4.0 * srq);
                    h[5] = F(7) * (-2.0 * srq2);
                } else {
                    // the reference writes h3(3) = -h3(3) (:314), negating the
                    // previous call's value; the transverse pp entry is -tt
                    h[1] = F(8) * srq2;
                    h[2] = -h[1];
                    h[3] = F(10) * (2.0 * srq);
                    h[4] = F(10) * (-2.0 * crq);
                    h[5] = F(8) * (-2.0 * crq2);
                }
                for (int j = 0; j < 6; ++j)
                    for (int k = 0; k < 10; ++k) coef3[((size_t)p * 6 + j) * 10 + k] = h[j].c[k];
            }
            if (coef4) {
                // tsgt2h4freq (fourier.f90:322-415): the 4th-order TSGT
                // double-dotted with the moment tensor mt(1..6)
                auto F = [](int k) { return C20::e(k); };
                const C20 t01 = F(7) * cqs, t02 = F(7) * sqs, t03 = F(8) * csq, t04 = F(8) * ssq;
                const C20 t05 = F(9) * cqs2, t06 = F(10) * csq2, t07 = F(11) * csq2, t08 = F(11) * ssq2;
                const C20 t09 = F(12) * cqs2, t10 = F(12) * sqs2;
                const C20 t11 = F(13) * (csq * cqs - ssq * sqs), t12 = F(13) * (ssq * cqs + csq * sqs);
                const C20 t13 = F(14) * (csq * cqs + ssq * sqs), t14 = F(14) * (ssq * cqs - csq * sqs);
                const C20 t15 = F(15) * (csq2 * cqs - ssq2 * sqs), t16 = F(15) * (ssq2 * cqs + csq2 * sqs);
                const C20 t17 = F(17) * (csq * cqs2 - ssq * sqs2), t18 = F(17) * (ssq * cqs2 + csq * sqs2);
                const C20 t19 = F(19) * (csq2 * cqs2 - ssq2 * sqs2), t20 = F(19) * (ssq2 * cqs2 + csq2 * sqs2);
                const C20 t21 = F(20) * (csq2 * cqs2 + ssq2 * sqs2), t22 = F(20) * (ssq2 * cqs2 - csq2 * sqs2);
                const C20 t23 = F(16) * (csq2 * cqs + ssq2 * sqs), t24 = F(16) * (ssq2 * cqs - csq2 * sqs);
                const C20 t25 = F(18) * (csq * cqs2 + ssq * sqs2), t26 = F(18) * (ssq * cqs2 - csq * sqs2);
                C20 h[6];
                h[0] = F(1) * mt[0] + (t05 - F(2)) * mt[1] + (-t05 - F(2)) * mt[2] -
                       F(5) * (cqs * mt[3] + sqs * mt[4]) + F(9) * (sqs2 * mt[5]);
                h[1] = (t06 - F(3)) * mt[0] + (t21 + t19 - t07 - t09 + F(4)) * mt[1] +
                       (-t21 - t19 - t07 + t09 + F(4)) * mt[2] + (t23 - t15 + t01) * mt[3] +
                       (-t24 - t16 + t02) * mt[4] + (-t22 + t20 - t10) * mt[5];
                h[2] = (-t06 - F(3)) * mt[0] + (-t21 - t19 + t07 - t09 + F(4)) * mt[1] +
                       (t21 + t19 + t07 + t09 + F(4)) * mt[2] + (-t23 + t15 + t01) * mt[3] +
                       (t24 + t16 + t02) * mt[4] + (t22 - t20 - t10) * mt[5];
                h[3] = -F(6) * (csq * mt[0]) + (t25 - t17 + t03) * mt[1] + (-t25 + t17 + t03) * mt[2] +
                       (-t13 + t11) * mt[3] + (t14 + t12) * mt[4] + (-t26 - t18) * mt[5];
                h[4] = -F(6) * (ssq * mt[0]) + (t26 - t18 + t04) * mt[1] + (-t26 + t18 + t04) * mt[2] +
                       (-t14 + t12) * mt[3] + (-t13 - t11) * mt[4] + (t25 + t17) * mt[5];
                h[5] = F(10) * (ssq2 * mt[0]) + (t22 + t20 - t08) * mt[1] + (-t22 - t20 - t08) * mt[2] +
                       (t24 - t16) * mt[3] + (t23 + t15) * mt[4] + (t21 - t19) * mt[5];
                for (int j = 0; j < 6; ++j)
                    for (int k = 0; k < 20; ++k) coef4[((size_t)p * 6 + j) * 20 + k] = h[j].c[k];
            }
        }
    });
}

extern "C" int dsm_cat_set_profiling(dsm_cat_t* c, int on) {
    if (!c) return DSM_ERR_INVALID;
    c->profiling = on != 0;
    return DSM_OK;
}

extern "C" int dsm_cat_get_stats(const dsm_cat_t* c, dsm_stats_t* s) {
    if (!c || !s) return DSM_ERR_INVALID;
    *s = c->stats;
    return DSM_OK;
}

extern "C" int dsm_cat_set_batch_bytes(dsm_cat_t* c, size_t bytes) {
    if (!c || bytes < ((size_t)1 << 20)) return DSM_ERR_INVALID;
    c->max_batch_bytes = bytes;
    return DSM_OK;
}

namespace {
// independent FP64 fused multiply-add chains, 8 per thread
__global__ void k_fp64_probe(double* out, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

namespace {
// independent FP64 tensor-core products, 8 accumulator tiles per warp
__global__ void k_fp64_mma_probe(double* out, int iters, double a) {
    double acc[8][4];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[k][e] = 0.0;
    const double a0 = a * threadIdx.x, a1 = a0 + 1.0, b = 1e-3 * (threadIdx.x & 7);
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int k = 0; k < 8; ++k) cat::mma_f64_16x8x4(acc[k], a0, a1, b);
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += acc[k][0] + acc[k][1] + acc[k][2] + acc[k][3];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

extern "C" int dsm_fp64_peak(int device, double* tflops) {
    return cat_guard(nullptr, [&] {
        need(tflops != nullptr, "dsm_fp64_peak: null output");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
            throw Error(DSM_ERR_NODEVICE, "dsm_fp64_peak: no CUDA device");
        DSM_CUDA(cudaSetDevice(device));
        int sms = 0;
        DSM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        const int blocks = sms * 8, threads = 256, iters = 1 << 14;
        DBuf<double> out;
        out.reserve((size_t)blocks * threads);
        cudaEvent_t e0, e1;
        DSM_CUDA(cudaEventCreate(&e0));
        DSM_CUDA(cudaEventCreate(&e1));
        k_fp64_probe<<<blocks, threads>>>(out.p, iters / 16, 0.999999, 1e-7);   // warm-up
        DSM_CUDA(cudaEventRecord(e0));
        k_fp64_probe<<<blocks, threads>>>(out.p, iters, 0.999999, 1e-7);
        DSM_CUDA(cudaEventRecord(e1));
        DSM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (ms * 1e-3) / 1e12;
    });
}

extern "C" int dsm_fp64_mma_peak(int device, double* tflops) {
    return cat_guard(nullptr, [&] {
        need(tflops != nullptr, "dsm_fp64_mma_peak: null output");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
            throw Error(DSM_ERR_NODEVICE, "dsm_fp64_mma_peak: no CUDA device");
        DSM_CUDA(cudaSetDevice(device));
        int sms = 0;
        DSM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        const int blocks = sms * 4, threads = 256, iters = 1 << 12;
        DBuf<double> out;
        out.reserve((size_t)blocks * threads);
        cudaEvent_t e0, e1;
        DSM_CUDA(cudaEventCreate(&e0));
        DSM_CUDA(cudaEventCreate(&e1));
        k_fp64_mma_probe<<<blocks, threads>>>(out.p, iters / 16, 1e-6);   // warm-up
        DSM_CUDA(cudaEventRecord(e0));
        k_fp64_mma_probe<<<blocks, threads>>>(out.p, iters, 1e-6);
        DSM_CUDA(cudaEventRecord(e1));
        DSM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        const double warps = (double)blocks * threads / 32;
        *tflops = 2.0 * 16 * 8 * 4 * 8.0 * iters * warps / (ms * 1e-3) / 1e12;
    });
}

extern "C" int dsm_cat_destroy(dsm_cat_t* c) {
    delete c;
    return DSM_OK;
}

extern "C" const char* dsm_cat_last_error(const dsm_cat_t* c) { return c ? c->err.c_str() : g_cat_err.c_str(); }
