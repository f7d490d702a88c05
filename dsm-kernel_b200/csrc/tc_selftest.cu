// Self-check of the tensor-core contraction on seeded pieces: the kernel's
// output against a plain FP64 sum of the same three piece products.  An
// internal entry point for the test suite; not part of the C-ABI.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstring>
#include <vector>

#include "lsum_tc.cuh"

namespace dsm {
void set_global_error(const std::string& e);
namespace {

__device__ __forceinline__ float urand(uint32_t s) {  // [-1, 1)
    s ^= s >> 16;
    s *= 0x7feb352du;
    s ^= s >> 15;
    s *= 0x846ca68bu;
    s ^= s >> 16;
    return (float)(s >> 8) * (1.0f / 8388608.0f) - 1.0f;
}

template <class T>
__device__ __forceinline__ T from_f(float x);
template <>
__device__ __forceinline__ __half from_f<__half>(float x) { return __float2half_rn(x); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
__device__ __forceinline__ double to_d(__half x) { return (double)__half2float(x); }
__device__ __forceinline__ double to_d(__nv_bfloat16 x) { return (double)__bfloat162float(x); }

// pieces[2][n] : hi uniform in [-1,1), lo = small residual-like value
template <class T>
__global__ void k_fill(T* p, size_t n, uint32_t seed, float lo_scale) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    p[i] = from_f<T>(urand((uint32_t)i * 2654435761u + seed));
    p[n + i] = from_f<T>(lo_scale * urand((uint32_t)i * 2246822519u + seed * 7u + 1u));
}

template <class T>
__global__ void k_ref(const T* A, const T* B, const float* sa, const float* sb, int M, int N, int K, int kcap,
                      int nf, double* C) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= (size_t)nf * M * N) return;
    int z = (int)(i / ((size_t)M * N));
    int r = (int)(i % ((size_t)M * N));
    int n = r / M, m = r % M;
    const size_t An = (size_t)nf * M * kcap, Bn = (size_t)N * kcap;
    const T* ah = A + ((size_t)z * M + m) * kcap;
    const T* bh = B + (size_t)n * kcap;
    double s = 0.0;
    for (int k = 0; k < K; ++k)
        s += to_d(ah[k]) * to_d(bh[k]) + to_d(ah[k]) * to_d(bh[Bn + k]) + to_d(ah[An + k]) * to_d(bh[k]);
    C[i] = s * (double)sa[m] * (double)sb[n];
}

__global__ void k_cmp(const float* C, const double* R, size_t n, double* out) {
    __shared__ double e[256], a[256];
    double me = 0.0, ma = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        me = fmax(me, fabs((double)C[i] - R[i]));
        ma = fmax(ma, fabs(R[i]));
    }
    e[threadIdx.x] = me;
    a[threadIdx.x] = ma;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            e[threadIdx.x] = fmax(e[threadIdx.x], e[threadIdx.x + s]);
            a[threadIdx.x] = fmax(a[threadIdx.x], a[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // non-negative doubles order like their bit patterns
        atomicMax(reinterpret_cast<unsigned long long*>(out), (unsigned long long)__double_as_longlong(e[0]));
        atomicMax(reinterpret_cast<unsigned long long*>(out + 1), (unsigned long long)__double_as_longlong(a[0]));
    }
}

__global__ void k_scales(float* sa, int M, float* sb, int N) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < M) sa[i] = ldexpf(1.0f, (i % 5) - 2);
    if (i < N) sb[i] = ldexpf(1.0f, (i % 3) - 1);
}

template <class T>
int run(int M, int N, int K, int nf, int fmt, int bk, uint32_t flags, int chunk, int reps, int check, double* res) {
    const int kcap = K + bk;  // capacity beyond K holds nonzero values the kernel must not read
    const size_t An = (size_t)nf * M * kcap, Bn = (size_t)N * kcap;
    DBuf<T> A, B;
    DBuf<float> sa, sb, C;
    DBuf<double> R, out;
    DBuf<int> err;
    A.reserve(2 * An);
    B.reserve(2 * Bn);
    sa.reserve(M);
    sb.reserve(N);
    C.reserve((size_t)nf * M * N);
    if (check) R.reserve((size_t)nf * M * N);
    out.reserve(2);
    err.reserve(1);
    DSM_CUDA(cudaMemset(out.p, 0, 2 * sizeof(double)));
    DSM_CUDA(cudaMemset(err.p, 0, sizeof(int)));
    DSM_CUDA(cudaMemset(C.p, 0, sizeof(float) * (size_t)nf * M * N));
    k_fill<T><<<(unsigned)((An + 255) / 256), 256>>>(A.p, An, 11u, 1.0f / 2048.0f);
    k_fill<T><<<(unsigned)((Bn + 255) / 256), 256>>>(B.p, Bn, 23u, 1.0f / 2048.0f);
    k_scales<<<(std::max(M, N) + 255) / 256, 256>>>(sa.p, M, sb.p, N);
    DSM_CUDA(cudaGetLastError());

    tc::Maps maps;
    std::memset(&maps, 0, sizeof(maps));
    tc::encode_a(&maps.a[0], A.p, fmt, kcap, M, nf, bk);
    tc::encode_b(&maps.b[0], B.p, fmt, kcap, N, bk);
    std::vector<tc::Problem> hp(nf);
    int tiles = 0;
    const int tm = (M + tc::BM - 1) / tc::BM, tn = (N + tc::BN - 1) / tc::BN;
    for (int z = 0; z < nf; ++z) {
        tc::Problem& P = hp[z];
        P.amap = 0;
        P.z = z;
        P.bmap = 0;
        P.row0 = 0;
        P.kblocks = K / bk;
        P.M = M;
        P.N = N;
        P.tiles_n = tn;
        P.tile0 = tiles;
        P.C = C.p + (size_t)z * M * N;
        P.sa = sa.p;
        P.sb = sb.p;
        P.ldc = M;
        tiles += tm * tn;
    }
    DBuf<tc::Problem> dp;
    dp.reserve(nf);
    DSM_CUDA(cudaMemcpy(dp.p, hp.data(), sizeof(tc::Problem) * nf, cudaMemcpyHostToDevice));
    int dev = 0, nsm = 0;
    DSM_CUDA(cudaGetDevice(&dev));
    DSM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));

    tc::launch(maps, dp.p, nf, tiles, fmt, bk, flags, chunk, err.p, nsm, 0);
    DSM_CUDA(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    DSM_CUDA(cudaEventCreate(&e0));
    DSM_CUDA(cudaEventCreate(&e1));
    DSM_CUDA(cudaEventRecord(e0, 0));
    for (int r = 0; r < reps; ++r) tc::launch(maps, dp.p, nf, tiles, fmt, bk, flags, chunk, err.p, nsm, 0);
    DSM_CUDA(cudaEventRecord(e1, 0));
    DSM_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    DSM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);

    const size_t nc = (size_t)nf * M * N;
    if (check) {
        k_ref<T><<<(unsigned)((nc + 255) / 256), 256>>>(A.p, B.p, sa.p, sb.p, M, N, K, kcap, nf, R.p);
        k_cmp<<<256, 256>>>(C.p, R.p, nc, out.p);
    }
    DSM_CUDA(cudaGetLastError());
    DSM_CUDA(cudaDeviceSynchronize());
    int herr = 0;
    DSM_CUDA(cudaMemcpy(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    DSM_CUDA(cudaMemcpy(res, out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost));
    res[2] = reps > 0 ? ms / reps : 0.0;
    res[3] = 2.0 * 3.0 * (double)nf * M * N * K;  // tensor flops per launch
    if (herr) throw Error(DSM_ERR_TIMEOUT, "a bounded wait in the tensor-core contraction gave up");
    return DSM_OK;
}

}  // namespace
}  // namespace dsm

// res[0] max |C - ref|, res[1] max |ref| (both 0 unless check), res[2] ms per
// launch over reps timed launches, res[3] tensor flops per launch
extern "C" int dsm_tc_selftest(int M, int N, int K, int nfreq, int piece_fmt, int bk, int flags, int chunk,
                               int reps, int check, double* res) {
    try {
        if (M <= 0 || N <= 0 || K <= 0 || nfreq <= 0 || nfreq > dsm::tc::MAXP || (K % bk) != 0 || !res)
            return DSM_ERR_INVALID;
        if (piece_fmt == dsm::tc::PIECE_BF16)
            return dsm::run<__nv_bfloat16>(M, N, K, nfreq, piece_fmt, bk, (uint32_t)flags, chunk, reps, check, res);
        return dsm::run<__half>(M, N, K, nfreq, piece_fmt, bk, (uint32_t)flags, chunk, reps, check, res);
    } catch (const dsm::Error& e) {
        dsm::set_global_error(std::string("dsm_tc_selftest: ") + e.what());
        return e.code;
    }
}
