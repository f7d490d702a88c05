// P-SV epilogue: TSGT / RSGT / SYNN of one frequency from its l-contractions.
#pragma once

#include "common.cuh"

namespace dsm {
namespace psvk {

constexpr int NS0 = 4, NS1 = 8, NS2 = 6;  // slots per |m|
constexpr int NFLD = 5;                   // U, U', V/lsq, V'/lsq, l(l+1) V/lsq

// Row layout of the per-order field matrix of one |m| (nq slots).  The
// receiver rows are split into the solid class (solid receivers and the
// surface row, Rs1 of them, index rr >= 0) and fluid receivers (Rf, index
// -rr - 1): a fluid receiver's strain needs only U against P.
//   group A (contracted with both basis columns P and dP/dtheta): fields
//     U, V/lsq, V'/lsq of the solid class, rows rr*6nq + (q*3 + fa)*2 + re/im;
//   group B (against P only): fields U', l(l+1)V/lsq of the solid class,
//     rows rr*4nq + (q*2 + fb)*2 + re/im, then U of the fluid receivers,
//     rows fluid index*2nq + q*2 + re/im.
// Receiver-major: the rows of a receiver are adjacent and receivers follow
// in radius order, so a 128-row tile of the contraction holds a few
// neighbouring receivers.  With the depth cut-off a receiver's fields are
// exactly zero above an order that grows with its radius, and a tile of
// deep receivers stops its order sum early (tc::Problem::kbt).
// Row of the real part of (q, f) for receiver class index rr, or -1 when the
// receiver has no row for f; *im is the offset of the imaginary part.
__host__ __device__ __forceinline__ size_t fld_rows_full(int nq, int Rs1) { return (size_t)nq * 6 * Rs1; }
__host__ __device__ __forceinline__ size_t fld_rows(int nq, int Rs1, int Rf) {
    return (size_t)nq * (10 * (size_t)Rs1 + 2 * (size_t)Rf);
}
__host__ __device__ __forceinline__ long long fld_row(int nq, int Rs1, int Rf, int q, int f, int rr, int* im) {
    *im = 1;
    if (rr >= 0) {
        if (f == 1 || f == 4)
            return (long long)fld_rows_full(nq, Rs1) + (long long)rr * 4 * nq + (q * 2 + (f == 4)) * 2;
        return (long long)rr * 6 * nq + (q * 3 + (f == 0 ? 0 : f - 1)) * 2;
    }
    if (f != 0) return -1;
    return (long long)nq * 10 * Rs1 + (long long)(-rr - 1) * 2 * nq + q * 2;
}

// receiver data the epilogue reads
struct EpiDev {
    int R, Th;
    int Rs1, Rf;                   // receiver rows of the solid class and fluid receivers
    double tlen, omegai;
    const int* fluid;              // [R]
    const int* rrow;               // [R+1] class index of each receiver row (fld_row)
    const double *lam, *qkp, *fr;  // [R]  lambda, Qkappa, float(r)
    int* status;                   // run status word: DEV_NONFINITE when an output is Inf/NaN
    int c_ld;                      // row stride of the row-major contraction outputs
};

// Contraction outputs C0..C2 (one per |m|, row-major with row stride
// c_ld, rows as fld_row, columns b*Th+it) are FP64 when tc is
// false and FP32 (tensor-core path, FP32 arithmetic) when it is true.
// Writes tsgt[w][Th][R][20], rsgt[w][Th][R][10] (when rsgt) and
// synn[w][Th][10] (when synn) as complex128.
void launch_epilogue(const EpiDev& d, int w, const double* thx, const double* ths, const int* pole,
                     const int* freqs, const void* C0, const void* C1, const void* C2, bool tc, double* tsgt,
                     double* rsgt, double* synn, cudaStream_t st);

}  // namespace psvk
}  // namespace dsm
