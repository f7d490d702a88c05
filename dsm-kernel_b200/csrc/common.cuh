// Internal definitions of the SGT engine (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "dsmsgt.h"

namespace dsm {

constexpr double kPi = 3.1415926535897932;

// ------------------------------------------------------------ complex
// 16-byte aligned, so a complex moves with one 128-bit load or store
struct __align__(16) cd {
    double re, im;
};
__host__ __device__ __forceinline__ cd mk(double r, double i = 0.0) { return cd{r, i}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cd operator-(cd a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cd operator*(double a, cd b) { return {a * b.re, a * b.im}; }
__host__ __device__ __forceinline__ cd operator*(cd a, double b) { return {a.re * b, a.im * b}; }
__host__ __device__ __forceinline__ cd operator/(cd a, double b) { return {a.re / b, a.im / b}; }
// Smith's division, the rule gfortran applies to complex division.
__host__ __device__ __forceinline__ cd operator/(cd a, cd b) {
    double c = b.re, d = b.im;
    if (fabs(c) < fabs(d)) {
        double ratio = c / d, div = c * ratio + d;
        return {(a.re * ratio + a.im) / div, (a.im * ratio - a.re) / div};
    }
    double ratio = d / c, div = d * ratio + c;
    return {(a.im * ratio + a.re) / div, (a.im - a.re * ratio) / div};
}
__host__ __device__ __forceinline__ cd conj(cd a) { return {a.re, -a.im}; }
__host__ __device__ __forceinline__ cd cmul_i(double m, cd a) { return {-m * a.im, m * a.re}; }  // (i m) a
__device__ __forceinline__ double cabs_(cd a) { return hypot(a.re, a.im); }

// complex of a chosen real type (float on the mixed path, double on the
// plain one); division by a real multiplies by its reciprocal
template <class RL>
struct alignas(2 * sizeof(RL)) cx {
    RL re, im;
    __host__ __device__ __forceinline__ friend cx operator+(cx a, cx b) { return {a.re + b.re, a.im + b.im}; }
    __host__ __device__ __forceinline__ friend cx operator-(cx a, cx b) { return {a.re - b.re, a.im - b.im}; }
    __host__ __device__ __forceinline__ friend cx operator-(cx a) { return {-a.re, -a.im}; }
    __host__ __device__ __forceinline__ friend cx operator*(cx a, cx b) {
        return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    }
    __host__ __device__ __forceinline__ friend cx operator*(RL a, cx b) { return {a * b.re, a * b.im}; }
    __host__ __device__ __forceinline__ friend cx operator*(cx a, RL b) { return {a.re * b, a.im * b}; }
};
template <class RL>
__host__ __device__ __forceinline__ cx<RL> cmul_i(RL m, cx<RL> a) { return {-m * a.im, m * a.re}; }  // (i m) a

// ------------------------------------------------------------ errors
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define DSM_CUDA(x)                                                                             \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess)                                                                  \
            throw ::dsm::Error(DSM_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_));     \
    } while (0)
#define DSM_CUBLAS(x)                                                                           \
    do {                                                                                        \
        cublasStatus_t s_ = (x);                                                                \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                        \
            throw ::dsm::Error(DSM_ERR_CUDA, std::string(#x ": cublas status ") +               \
                                                 std::to_string((int)s_));                      \
    } while (0)
#define DSM_LAUNCH(ctx)                                                                         \
    do {                                                                                        \
        (ctx).launches++;                                                                       \
        DSM_CUDA(cudaGetLastError());                                                           \
    } while (0)

// device buffer
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void reserve(size_t count) {  // grows only
        if (count <= n) return;
        release();
        if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
            p = nullptr;
            throw Error(DSM_ERR_NOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
        }
        n = count;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        reserve(count);
        DSM_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
};

// device-side status words of a run: set by kernels, read by the host at
// the synchronisations the run already has.  Word 0: a bounded wait of the
// tensor-core l-sum gave up.  Word 1: DevErr bits.
enum DevErr : int { DEV_OK = 0, DEV_NONFINITE = 1 };
constexpr int DEV_WORD_TC = 0, DEV_WORD_STATUS = 1;

#ifdef __CUDACC__
// sets DEV_NONFINITE in the status word when bad (rare: no warp traffic)
__device__ __forceinline__ void flag_nonfinite(int* status, bool bad) {
    if (bad) atomicOr(status, DEV_NONFINITE);
}
__device__ __forceinline__ bool nonfinite2(double a, double b) { return !isfinite(a) || !isfinite(b); }
#endif

}  // namespace dsm
