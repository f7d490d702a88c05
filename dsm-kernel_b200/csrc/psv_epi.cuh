// P-SV epilogue: TSGT / RSGT / SYNN of one frequency from its l-contractions.
#pragma once

#include "common.cuh"

namespace dsm {
namespace psvk {

constexpr int NS0 = 4, NS1 = 8, NS2 = 6;  // slots per |m|
constexpr int NFLD = 5;                   // U, U', V/lsq, V'/lsq, l(l+1) V/lsq

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
