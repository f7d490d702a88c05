// P-SV epilogue: TSGT / RSGT / SYNN of one frequency from its l-contractions.
#pragma once

#include "common.cuh"

namespace dsm {
namespace psvk {

constexpr int NS0 = 4, NS1 = 8, NS2 = 6;  // slots per |m|
constexpr int NFLD = 5;                   // U, U', V/lsq, V'/lsq, l(l+1) V/lsq

// Row layout of the per-order field matrix of one |m| (nq slots, R + 1
// receiver rows r): fields 0, 2, 3 (U, V/lsq, V'/lsq), which the epilogue
// contracts with both basis columns (P and dP/dtheta), come first; fields 1
// and 4 (U', l(l+1) V/lsq), needed against P only, follow, so the l-sum of
// the second group runs over half the columns.  Row of the real part of
// (q, f) at r = 0; the imaginary part is R + 1 rows further.
__host__ __device__ __forceinline__ size_t fld_rows_full(int nq, int R) { return (size_t)nq * 3 * 2 * (R + 1); }
__host__ __device__ __forceinline__ size_t fld_row(int nq, int R, int q, int f) {
    if (f == 1 || f == 4) return fld_rows_full(nq, R) + ((size_t)(q * 2 + (f == 4)) * 2) * (R + 1);
    return ((size_t)(q * 3 + (f == 0 ? 0 : f - 1)) * 2) * (R + 1);
}

// receiver data the epilogue reads
struct EpiDev {
    int R, Th;
    double tlen, omegai;
    const int* fluid;              // [R]
    const double *lam, *qkp, *fr;  // [R]  lambda, Qkappa, float(r)
};

// Contraction outputs C0..C2 (one per |m|, column-major, rows
// ((q*NFLD+f)*2+{re,im})*(R+1)+r, columns b*Th+it) are FP64 when tc is
// false and FP32 (tensor-core path, FP32 arithmetic) when it is true.
// Writes tsgt[w][Th][R][20], rsgt[w][Th][R][10] (when rsgt) and
// synn[w][Th][10] (when synn) as complex128.
void launch_epilogue(const EpiDev& d, int w, const double* thx, const double* ths, const int* pole,
                     const int* freqs, const void* C0, const void* C1, const void* C2, bool tc, double* tsgt,
                     double* rsgt, double* synn, cudaStream_t st);

}  // namespace psvk
}  // namespace dsm
