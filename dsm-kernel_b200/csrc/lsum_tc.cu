// Split-precision l-sum contraction on the sm_100a tensor cores.
//
// Persistent, warp-specialised kernel, one CTA per SM:
//   warp 0      TMA producer: per stage, the hi and lo pieces of a 128 x BK
//               A tile and of a 128 x BK B tile (four bulk tensor loads,
//               one mbarrier with the byte count)
//   warp 1      MMA issuer: per stage and 16-order step, three
//               tcgen05.mma (hi*hi, hi*lo, lo*hi) into the current chunk
//               accumulator; tcgen05.commit frees the stage and hands
//               finished chunk accumulators over
//   warps 2..9  epilogue: tcgen05.ld of the chunk accumulators (two warps
//               per 32-lane quarter, 64 columns each), FP64 sum of the
//               chunks, row x column scaling, column-major or row-major stores
// Accuracy: the tensor cores add each step into the FP32 accumulator with a
// rounding relative to the accumulator's magnitude, so a long order sum
// loses bits in proportion to its length.  The products therefore go into
// short chunks (chunk stages of BK orders) whose partial sums the epilogue
// adds in FP64.  The cross terms (2^-11 smaller than hi*hi) share the chunk
// accumulator: each stage issues them before its hi*hi products, so in a
// one-stage chunk they are summed while the accumulator is still small.  Tensor
// memory (512 columns): four chunk buffers of 128 columns, so the epilogue
// drains a pair while the MMAs fill the other pair, across tile boundaries
// too.  TC_REVERSE runs the orders from high to low.
// Every wait is bounded: after about a second a role raises the CTA's abort
// flag, all roles leave their loops, the issued copies and MMAs are waited
// for (again bounded), the tensor memory is freed and the error word is set.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <mutex>

#include "lsum_tc.cuh"

namespace dsm {
namespace tc {

namespace {

constexpr int EPI_THREADS = 256;                 // warps 2..9
constexpr int NTHREADS = 64 + EPI_THREADS;
constexpr uint32_t TMEM_COLS = 512;
constexpr int SMEM_STAGES = 192 * 1024;         // operand stages
constexpr int NHB = 4;                          // chunk buffers in tensor memory

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait.  Gives up when another role has aborted or after the limit
// (then it aborts the CTA itself).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag,
                                          unsigned long long limit_ns) {
    const unsigned long long t0 = gtimer();
    for (uint32_t n = 0;; ++n) {
        if (mbar_try(b, parity)) return true;
        if ((n & 63) == 63) {
            if (*abort_flag) return false;
            if (gtimer() - t0 > limit_ns) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}
// Bounded wait used while draining after an abort (ignores the flag).
__device__ __forceinline__ void mbar_drain(uint64_t* b, uint32_t parity, unsigned long long limit_ns) {
    const unsigned long long t0 = gtimer();
    while (!mbar_try(b, parity))
        if (gtimer() - t0 > limit_ns) return;
}

__device__ __forceinline__ void tma_a(const CUtensorMap* m, void* dst, uint64_t* bar, int x, int y, int z, int w) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
        : "memory");
}
__device__ __forceinline__ void tma_b(const CUtensorMap* m, void* dst, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(m)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of an order-major tile whose rows are
// BK*2 bytes, swizzled as the TMA wrote them (64B or 128B pattern), 8-row
// groups at 8*BK*2 bytes.
template <int BK>
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
    constexpr uint64_t layout = BK == 32 ? 4 : 2;   // SWIZZLE_64B : SWIZZLE_128B
    constexpr uint64_t sbo = (8 * BK * 2) >> 4;
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | (sbo << 32) | (1ull << 46) | (layout << 61);
}

__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
// Tile t of a launch: its problem p, row tile mt and column tile nt.  A CTA
// visits its tiles in increasing order, so p only moves forward from the
// previous tile's problem (the caller keeps it, starting at 0).
__device__ __forceinline__ void decode(const Problem* ps, int np, int t, int& p, int& mt, int& nt) {
    while (p + 1 < np && ps[p + 1].tile0 <= t) ++p;
    const int loc = t - ps[p].tile0;
    mt = loc / ps[p].tiles_n;
    nt = loc - mt * ps[p].tiles_n;
}

template <int BK>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_lsum_tc(const __grid_constant__ Maps maps, const Problem* __restrict__ probs, int np, int ntiles,
              uint32_t idesc, uint32_t flags, int chunk, int* __restrict__ err, unsigned long long wait_ns) {
    constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2;
    constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
    constexpr int STAGES = SMEM_STAGES / STAGE;
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], hfull[NHB], hempty[NHB], fin;
    __shared__ uint32_t tmem_sh;
    __shared__ int abort_sh;
    __shared__ Problem ps[MAXP];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool reverse = (flags & TC_REVERSE) != 0;
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    volatile int* abort_flag = &abort_sh;

    for (int i = threadIdx.x; i < np; i += NTHREADS) ps[i] = probs[i];
    if (threadIdx.x == 0) {
        abort_sh = 0;
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < NHB; ++b) {
            mbar_init(&hfull[b], 1);
            mbar_init(&hempty[b], EPI_THREADS);
        }
        mbar_init(&fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.a[0])) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.b[0])) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_sh;
    // tensor memory: chunk accumulators [0..NHB) at columns [0, NHB BN)

    if (warp == 0) {
        if (lane == 0) {  // ---------------------------------------- producer
            int it = 0, p = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int mt, nt;
                decode(ps, np, t, p, mt, nt);
                const Problem& P = ps[p];
                const int kbn = P.kb ? max(0, min(P.kb[mt], P.kblocks)) : P.kblocks;  // this row tile's order blocks
                for (int kb = 0; kb < kbn; ++kb, ++it) {
                    const int s = it % STAGES;
                    const uint32_t ph = (it / STAGES) & 1;
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag, wait_ns)) {
                        ok = false;
                        break;
                    }
                    // test hook: CTA 0 issues nothing for its first stage
                    if ((flags & TC_TEST_STALL) && blockIdx.x == 0 && it == 0) continue;
                    unsigned char* sp = base + s * STAGE;
                    const int x = (reverse ? kbn - 1 - kb : kb) * BK;
                    mbar_expect_tx(&full[s], STAGE);
                    tma_a(&maps.a[P.amap], sp, &full[s], x, P.row0 + mt * BM, P.z, 0);
                    tma_a(&maps.a[P.amap], sp + A_BYTES, &full[s], x, P.row0 + mt * BM, P.z, 1);
                    tma_b(&maps.b[P.bmap], sp + 2 * A_BYTES, &full[s], x, nt * BN, 0);
                    tma_b(&maps.b[P.bmap], sp + 2 * A_BYTES + B_BYTES, &full[s], x, nt * BN, 1);
                }
            }
            // every issued copy has landed before the CTA may exit
            for (int s = 0; s < STAGES && s < it; ++s) {
                const int last = s + ((it - 1 - s) / STAGES) * STAGES;
                mbar_drain(&full[s], (last / STAGES) & 1, wait_ns);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // ---------------------------------------- MMA issuer
            int it = 0, cc = 0, p = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int mt, nt;
                decode(ps, np, t, p, mt, nt);
                const int kbn = ps[p].kb ? max(0, min(ps[p].kb[mt], ps[p].kblocks)) : ps[p].kblocks;
                const int ch = chunk > 0 ? chunk : max(kbn, 1);
                // the last column tile of a contraction runs with N cut to
                // its columns (a multiple of 16): no MMA time on padding
                const int nrem = ps[p].N - nt * BN;
                const uint32_t ncols = (uint32_t)min(BN, (nrem + 15) & ~15);
                const uint32_t idt = (idesc & ~(0x3Fu << 17)) | ((ncols >> 3) << 17);
                uint32_t dh = tmem;
                int hb = 0;
                for (int kb = 0; kb < kbn; ++kb, ++it) {
                    const bool cfirst = kb % ch == 0;
                    if (cfirst) {
                        hb = cc % NHB;
                        if (!mbar_wait(&hempty[hb], ((cc / NHB) & 1) ^ 1, abort_flag, wait_ns)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        dh = tmem + (uint32_t)(hb * BN);
                    }
                    const int s = it % STAGES;
                    if (!mbar_wait(&full[s], (it / STAGES) & 1, abort_flag, wait_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t ah = smem_u32(base + s * STAGE), al = ah + A_BYTES;
                    const uint32_t bh = ah + 2 * A_BYTES, bl = bh + B_BYTES;
                    // the cross terms first: while the accumulator holds only
                    // them (2^-11 of hi*hi), their roundings are that much smaller
#pragma unroll
                    for (int j = 0; j < BK / 16; ++j) {
                        const uint32_t o = 32u * j;
                        mma_f16(dh, sdesc<BK>(ah + o), sdesc<BK>(bl + o), idt, (cfirst && j == 0) ? 0u : 1u);
                        mma_f16(dh, sdesc<BK>(al + o), sdesc<BK>(bh + o), idt, 1u);
                    }
#pragma unroll
                    for (int j = 0; j < BK / 16; ++j) {
                        const uint32_t o = 32u * j;
                        mma_f16(dh, sdesc<BK>(ah + o), sdesc<BK>(bh + o), idt, 1u);
                    }
                    mma_commit(&empty[s]);
                    if (kb % ch == ch - 1 || kb == kbn - 1) {
                        mma_commit(&hfull[hb]);
                        ++cc;
                    }
                }
            }
            // all issued MMAs complete before tensor memory is released
            mma_commit(&fin);
            mbar_drain(&fin, 0, wait_ns);
        }
    } else {  // ------------------------------------------------------ epilogue
        // two warps per tensor-memory lane quarter, each owning 64 columns;
        // the chunks are summed in FP64 registers
        const int q = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lanes = (uint32_t)(q * 32) << 16;
        int cc = 0, p = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            int mt, nt;
            decode(ps, np, t, p, mt, nt);
            const Problem& P = ps[p];
            const int kbn = P.kb ? max(0, min(P.kb[mt], P.kblocks)) : P.kblocks, ch = chunk > 0 ? chunk : max(kbn, 1);
            const int nch = (kbn + ch - 1) / ch;
            double acc[64];
#pragma unroll
            for (int j = 0; j < 64; ++j) acc[j] = 0.0;
            // chunks in pairs: the two FP32 chunk sums are added in FP32
            // (one rounding, unbiased) before the FP64 accumulation, which
            // halves the conversions and FP64 additions
            for (int c = 0; c + 1 < nch; c += 2, cc += 2) {
                const int hb0 = cc % NHB, hb1 = (cc + 1) % NHB;
                bool got = mbar_wait(&hfull[hb0], (cc / NHB) & 1, abort_flag, wait_ns);
                got = got && mbar_wait(&hfull[hb1], ((cc + 1) / NHB) & 1, abort_flag, wait_ns);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t ta0 = tmem + lanes + (uint32_t)(hb0 * BN + half * 64);
                const uint32_t ta1 = tmem + lanes + (uint32_t)(hb1 * BN + half * 64);
#pragma unroll
                for (int g = 0; g < 4; ++g) {
                    uint32_t r0[16], r1[16];
                    tmem_ld16(ta0 + 16 * g, r0);
                    tmem_ld16(ta1 + 16 * g, r1);
                    tmem_wait();
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        acc[g * 16 + j] += (double)(__uint_as_float(r0[j]) + __uint_as_float(r1[j]));
                }
                tc_fence_before();
                mbar_arrive(&hempty[hb0]);
                mbar_arrive(&hempty[hb1]);
            }
            if (ok && (nch & 1)) {  // the odd last chunk
                const int hb = cc % NHB;
                const bool got = mbar_wait(&hfull[hb], (cc / NHB) & 1, abort_flag, wait_ns);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t ta = tmem + lanes + (uint32_t)(hb * BN + half * 64);
#pragma unroll
                for (int g = 0; g < 4; ++g) {
                    uint32_t r0[16];
                    tmem_ld16(ta + 16 * g, r0);
                    tmem_wait();
#pragma unroll
                    for (int j = 0; j < 16; ++j) acc[g * 16 + j] += (double)__uint_as_float(r0[j]);
                }
                tc_fence_before();
                mbar_arrive(&hempty[hb]);
                ++cc;
            }
            if (!ok) break;
            const int m = mt * BM + q * 32 + lane;
            const bool mv = m < P.M;
            const double rs = mv ? (double)P.sa[m] : 0.0;
            if (P.rowmajor) {  // a row's 64 columns: 16-byte stores where a whole group of 32 lies within N
                float* Cr = P.C + (long long)m * P.ldc;
#pragma unroll
                for (int g = 0; g < 2; ++g) {
                    const int n0 = nt * BN + half * 64 + g * 32;
                    if (!mv) continue;
                    if (n0 + 32 <= P.N) {
#pragma unroll
                        for (int j = 0; j < 32; j += 4) {
                            float4 v;
                            v.x = (float)(acc[g * 32 + j] * rs * (double)P.sb[n0 + j]);
                            v.y = (float)(acc[g * 32 + j + 1] * rs * (double)P.sb[n0 + j + 1]);
                            v.z = (float)(acc[g * 32 + j + 2] * rs * (double)P.sb[n0 + j + 2]);
                            v.w = (float)(acc[g * 32 + j + 3] * rs * (double)P.sb[n0 + j + 3]);
                            *reinterpret_cast<float4*>(Cr + n0 + j) = v;
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (n0 + j < P.N) Cr[n0 + j] = (float)(acc[g * 32 + j] * rs * (double)P.sb[n0 + j]);
                    }
                }
            } else {
                float* Cm = P.C + m;
#pragma unroll
                for (int g = 0; g < 2; ++g) {
                    const int n0 = nt * BN + half * 64 + g * 32;
                    if (mv) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int n = n0 + j;
                            if (n < P.N)
                                Cm[(long long)n * P.ldc] =
                                    (float)(acc[g * 32 + j] * rs * (double)P.sb[n]);
                        }
                    }
                }
            }
        }
    }

    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
    if (threadIdx.x == 0 && abort_sh) atomicExch(err, 1);
}

// ------------------------------------------------------------ piece split
// x = s (hi + lo): s = 2^e with the row (column) maximum scaled into
// [2^14, 2^15), below the fp16 limit with a factor-two margin.  The scale is
// exact, so hi + lo carries ~22 (fp16) or ~16 (bf16) significant bits.
__device__ __forceinline__ int piece_exp(double mx) {
    if (!(mx > 0.0)) return 0;
    int e = ilogb(mx) - 14;
    return max(-126, min(127, e));
}
__device__ __forceinline__ void split2(double x, int fmt, uint16_t& hi, uint16_t& lo) {
    if (fmt == PIECE_BF16) {
        __nv_bfloat16 h = __double2bfloat16(x);
        __nv_bfloat16 l = __double2bfloat16(x - (double)__bfloat162float(h));
        hi = __bfloat16_as_ushort(h);
        lo = __bfloat16_as_ushort(l);
    } else {
        __half h = __double2half(x);
        __half l = __double2half(x - (double)__half2float(h));
        hi = __half_as_ushort(h);
        lo = __half_as_ushort(l);
    }
}

// the same split for an FP32 value already scaled by 2^-e: the residual
// x - hi has at most 13 (fp16) or 16 (bf16) significant bits, so it is exact
// in FP32 and each piece is one rounding of an exact value, as in split2
__device__ __forceinline__ void split2f(float x, int fmt, uint16_t& hi, uint16_t& lo) {
    if (fmt == PIECE_BF16) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        hi = __bfloat16_as_ushort(h);
        lo = __bfloat16_as_ushort(__float2bfloat16_rn(x - __bfloat162float(h)));
    } else {
        const __half h = __float2half_rn(x);
        hi = __half_as_ushort(h);
        lo = __half_as_ushort(__float2half_rn(x - __half2float(h)));
    }
}

// FP32 rows whose length is a multiple of four: one warp per row, four
// orders per lane and load (16-byte loads, 8-byte piece stores), SPLIT_U
// loads in flight per lane.
constexpr int SPLIT_THREADS = 128;
constexpr int SPLIT_U = 4;
__global__ void __launch_bounds__(SPLIT_THREADS) k_split_rows_f4(const float* __restrict__ A, int nrows, int per_w,
                                                                 int lcap, const int* __restrict__ nord, int kcap,
                                                                 int bk, uint16_t* __restrict__ P,
                                                                 size_t piece_stride, float* __restrict__ sa,
                                                                 int fmt, int* __restrict__ lnz,
                                                                 const int* __restrict__ zf,
                                                                 const int* __restrict__ rowrec, int R1) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= nrows) return;
    const int K = nord ? min(nord[row / per_w], lcap) : lcap;
    const int Kp = min(kcap, (K + bk - 1) / bk * bk);
    // orders at or above Kr are known to be zero: not read
    const int Kr = zf ? min(K, zf[(row / per_w) * R1 + rowrec[row % per_w]]) : K;
    const float4* a4 = reinterpret_cast<const float4*>(A + (size_t)row * lcap);
    float mx = 0.0f;
    int last = 0;  // one past the last nonzero order
    for (int i0 = lane; 4 * i0 < Kr; i0 += 32 * SPLIT_U) {
        float4 v[SPLIT_U];
#pragma unroll
        for (int u = 0; u < SPLIT_U; ++u) {
            const int i = i0 + 32 * u;
            v[u] = 4 * i < Kr ? a4[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
#pragma unroll
        for (int u = 0; u < SPLIT_U; ++u) {
            const int i = i0 + 32 * u;
            const float x[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (4 * i + c < Kr) {
                    mx = fmaxf(mx, fabsf(x[c]));
                    if (x[c] != 0.0f) last = 4 * i + c + 1;
                }
        }
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    last = __reduce_max_sync(0xffffffffu, last);
    const int e = piece_exp((double)mx);
    if (lane == 0) {
        sa[row] = __int_as_float((127 + e) << 23);
        if (lnz) lnz[row] = last;
    }
    uint2* ph = reinterpret_cast<uint2*>(P + (size_t)row * kcap);
    uint2* pl = reinterpret_cast<uint2*>(P + piece_stride + (size_t)row * kcap);
    for (int i0 = lane; 4 * i0 < Kp; i0 += 32 * SPLIT_U) {
        float4 v[SPLIT_U];
#pragma unroll
        for (int u = 0; u < SPLIT_U; ++u) {
            const int i = i0 + 32 * u;
            v[u] = 4 * i < Kr ? a4[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
#pragma unroll
        for (int u = 0; u < SPLIT_U; ++u) {
            const int i = i0 + 32 * u;
            if (4 * i >= Kp) break;
            const float x[4] = {v[u].x, v[u].y, v[u].z, v[u].w};
            uint16_t h[4], lo[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                h[c] = lo[c] = 0;
                if (4 * i + c < K) split2f(ldexpf(x[c], -e), fmt, h[c], lo[c]);
            }
            ph[i] = make_uint2((uint32_t)h[0] | ((uint32_t)h[1] << 16), (uint32_t)h[2] | ((uint32_t)h[3] << 16));
            pl[i] = make_uint2((uint32_t)lo[0] | ((uint32_t)lo[1] << 16), (uint32_t)lo[2] | ((uint32_t)lo[3] << 16));
        }
    }
}

// one warp per row: row maximum over the counted orders, then the pieces
template <class TIN>
__global__ void k_split_rows(const TIN* __restrict__ A, int nrows, int per_w, int lcap,
                             const int* __restrict__ nord, int kcap, int bk, uint16_t* __restrict__ P,
                             size_t piece_stride, float* __restrict__ sa, int fmt, int* __restrict__ lnz) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= nrows) return;
    const int K = nord ? min(nord[row / per_w], lcap) : lcap;
    const int Kp = min(kcap, (K + bk - 1) / bk * bk);
    const TIN* a = A + (size_t)row * lcap;
    double mx = 0.0;
    int last = 0;  // one past the last nonzero order
    for (int l = lane; l < K; l += 32) {
        const double x = (double)a[l];
        mx = fmax(mx, fabs(x));
        if (x != 0.0) last = l + 1;
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    last = __reduce_max_sync(0xffffffffu, last);
    const int e = piece_exp(mx);
    if (lane == 0) {
        sa[row] = __int_as_float((127 + e) << 23);
        if (lnz) lnz[row] = last;
    }
    uint16_t* ph = P + (size_t)row * kcap;
    uint16_t* pl = ph + piece_stride;
    for (int l = lane; l < Kp; l += 32) {
        uint16_t h = 0, lo = 0;
        if (l < K) split2(scalbn((double)a[l], -e), fmt, h, lo);
        ph[l] = h;
        pl[l] = lo;
    }
}

// One block per problem, one warp per row tile at a time.
__global__ void k_tile_orders(const Problem* __restrict__ probs, int bk) {
    const Problem& P = probs[blockIdx.x];
    if (!P.kb || !P.lz) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int mtiles = (P.M + BM - 1) / BM;
    for (int mt = warp; mt < mtiles; mt += nw) {
        int last = 0;
        for (int r = mt * BM + lane; r < min(P.M, (mt + 1) * BM); r += 32) last = max(last, P.lz[r]);
        last = __reduce_max_sync(0xffffffffu, last);
        if (lane == 0) P.kb[mt] = min(P.kblocks, (last + bk - 1) / bk);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) throw Error(DSM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

CUtensorMapDataType dtype(int piece_fmt) {
    return piece_fmt == PIECE_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
}

void check(CUresult r, const char* what) {
    if (r != CUDA_SUCCESS) throw Error(DSM_ERR_CUDA, std::string("tensor map for ") + what + " rejected (" +
                                                         std::to_string((int)r) + ")");
}

}  // namespace

void encode_a(CUtensorMap* m, const void* base, int piece_fmt, int kcap, int rows, int nfreq, int bk) {
    if (kcap % bk) throw Error(DSM_ERR_INVALID, "order capacity of the split fields is not a multiple of BK");
    cuuint64_t dims[4] = {(cuuint64_t)kcap, (cuuint64_t)rows, (cuuint64_t)nfreq, 2};
    cuuint64_t strides[3] = {(cuuint64_t)kcap * 2, (cuuint64_t)kcap * 2 * rows, (cuuint64_t)kcap * 2 * rows * nfreq};
    cuuint32_t box[4] = {(cuuint32_t)bk, BM, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    check(encoder()(m, dtype(piece_fmt), 4, const_cast<void*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE,
                    bk == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE),
          "the split fields");
}

void encode_b(CUtensorMap* m, const void* base, int piece_fmt, int kcap, int cols, int bk) {
    if (kcap % bk) throw Error(DSM_ERR_INVALID, "order capacity of the split bases is not a multiple of BK");
    cuuint64_t dims[3] = {(cuuint64_t)kcap, (cuuint64_t)cols, 2};
    cuuint64_t strides[2] = {(cuuint64_t)kcap * 2, (cuuint64_t)kcap * 2 * cols};
    cuuint32_t box[3] = {(cuuint32_t)bk, BN, 1};
    cuuint32_t es[3] = {1, 1, 1};
    check(encoder()(m, dtype(piece_fmt), 3, const_cast<void*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE,
                    bk == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE),
          "the split bases");
}

void split_fields(const void* A, int in_bytes, int nf, int rows, int lcap, const int* d_nord, uint16_t* P,
                  float* sa, int kcap, int F, int piece_fmt, int bk, cudaStream_t st, int* lnz, const int* zf,
                  const int* rowrec, int R1) {
    const int n = nf * rows;
    if (n <= 0) return;
    if (kcap % bk) throw Error(DSM_ERR_INVALID, "order capacity of the split fields is not a multiple of BK");
    if (in_bytes == 4 && lcap % 4 == 0 && kcap % 4 == 0) {
        k_split_rows_f4<<<(n + SPLIT_THREADS / 32 - 1) / (SPLIT_THREADS / 32), SPLIT_THREADS, 0, st>>>(
            static_cast<const float*>(A), n, rows, lcap, d_nord, kcap, bk, P, (size_t)F * rows * kcap, sa, piece_fmt,
            lnz, zf, rowrec, R1);
    } else if (in_bytes == 4)
        k_split_rows<float><<<(n + 7) / 8, 256, 0, st>>>(static_cast<const float*>(A), n, rows, lcap, d_nord, kcap,
                                                         bk, P, (size_t)F * rows * kcap, sa, piece_fmt, lnz);
    else
        k_split_rows<double><<<(n + 7) / 8, 256, 0, st>>>(static_cast<const double*>(A), n, rows, lcap, d_nord,
                                                          kcap, bk, P, (size_t)F * rows * kcap, sa, piece_fmt, lnz);
    DSM_CUDA(cudaGetLastError());
}

void split_bases(const double* B, int cols, int lcap, uint16_t* P, float* sb, int kcap, int piece_fmt,
                 cudaStream_t st) {
    if (cols <= 0) return;
    k_split_rows<double><<<(cols + 7) / 8, 256, 0, st>>>(B, cols, cols, lcap, nullptr, kcap, kcap, P,
                                                 (size_t)cols * kcap, sb, piece_fmt, nullptr);
    DSM_CUDA(cudaGetLastError());
}

void tile_orders(const Problem* d_probs, int np, int bk, cudaStream_t st) {
    if (np <= 0) return;
    k_tile_orders<<<np, 128, 0, st>>>(d_probs, bk);
    DSM_CUDA(cudaGetLastError());
}

void launch(const Maps& maps, const Problem* d_probs, int np, int ntiles, int piece_fmt, int bk, uint32_t flags,
            int chunk, int* d_err, int nsm, cudaStream_t st, unsigned long long wait_ns) {
    if (np <= 0 || ntiles <= 0) return;
    if (np > MAXP) throw Error(DSM_ERR_INVALID, "too many contractions in one launch");
    // kind::f16 instruction descriptor: FP32 accumulator, both operands of
    // the piece type and order-major, N = BN, M = BM
    const uint32_t fmt = piece_fmt == PIECE_BF16 ? 1u : 0u;
    const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
    const int grid = std::min(ntiles, nsm);
    const size_t smem = SMEM_STAGES + 1024;
    // the shared-memory attribute is set on every launch: it belongs to the
    // current device, and contexts of several devices or host threads
    // launch here (a host call of about a microsecond)
    if (bk == 32) {
        DSM_CUDA(cudaFuncSetAttribute(k_lsum_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_lsum_tc<32><<<grid, NTHREADS, smem, st>>>(maps, d_probs, np, ntiles, idesc, flags, chunk, d_err, wait_ns);
    } else if (bk == 64) {
        DSM_CUDA(cudaFuncSetAttribute(k_lsum_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_lsum_tc<64><<<grid, NTHREADS, smem, st>>>(maps, d_probs, np, ntiles, idesc, flags, chunk, d_err, wait_ns);
    } else {
        throw Error(DSM_ERR_INVALID, "BK must be 32 or 64");
    }
    DSM_CUDA(cudaGetLastError());
}

}  // namespace tc
}  // namespace dsm
