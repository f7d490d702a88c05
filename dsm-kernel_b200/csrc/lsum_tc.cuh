// Split-precision l-sum contraction on the sm_100a tensor cores (tcgen05).
//
// One launch contracts every (frequency, |m|) problem of a batch:
//     C[M x N] = sum_l A[M x l] * B[N x l]^T ,   both operands order-major,
// with A (the receiver fields) and B (the Legendre bases) each stored as two
// 16-bit pieces, x = s * (x_hi + x_lo) with a power-of-two scale s per row of
// A and per column of B.  The product runs as x_hi*y_hi + x_hi*y_lo +
// x_lo*y_hi on the tensor cores with FP32 accumulation in tensor memory;
// the epilogue applies s_row * s_col and writes C column-major (ld = M),
// the layout the FP64 contraction writes.  The hi*hi products are summed in
// chunks of `chunk` stages whose partial sums are added in FP64.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace dsm {
namespace tc {

constexpr int BM = 128;          // rows of a tile (tensor-memory lanes)
constexpr int BN = 128;          // columns of a tile (tensor-memory columns)
constexpr int MAXP = 96;         // problems per launch
constexpr int PIECE_F16 = 0;     // fp16 pieces (11-bit significand each)
constexpr int PIECE_BF16 = 1;    // bf16 pieces (8-bit significand each)
constexpr uint32_t TC_REVERSE = 1;    // orders summed from high to low
// test hook: CTA 0 withholds the copies of its first stage, so the MMA
// issuer's bounded wait runs out and the launch reports a timeout
constexpr uint32_t TC_TEST_STALL = 2;
constexpr unsigned long long WAIT_NS = 1000000000ull;  // limit of every bounded wait (1 s)

// One contraction of a launch: rows row0 .. row0 + M of the A map against
// the first N columns of the B map.  Rows beyond the map and columns beyond
// N are read as zeros (or are other rows' data) and never stored.
struct Problem {
    int amap, z, bmap, kblocks;  // A map (|m|), frequency slot, B map, orders / BK
    int row0;                    // first row of A (in the map) and of C
    int M, N, tiles_n, tile0;    // shape, column tiles, index of the first tile
    float* C;                    // M x N: column-major (ldc >= M) or row-major (rowmajor, ldc >= N)
    const float* sa;             // M row scales
    const float* sb;             // N column scales
    long long ldc;
    // Order blocks of each row tile (ceil(M / BM) entries, at most kblocks),
    // or null: kblocks for every tile.  Rows whose orders above some l are
    // exactly zero (the depth cut-off's deep receivers) let a tile stop its
    // order sum early.  Filled by tile_orders from lz.
    int* kb;
    const int* lz;               // M rows: one past the last nonzero order (or null)
    int rowmajor;                // C row-major (ldc a multiple of 4, C 16-byte aligned)
};

struct Maps {
    CUtensorMap a[3];  // [piece][frequency][row][order] fp16/bf16
    CUtensorMap b[3];  // [piece][column][order]
};

// Encodes the tensor maps of a launch.  BK selects the stage depth: 32
// orders (64-byte rows, 64B swizzle) or 64 orders (128B swizzle).
void encode_a(CUtensorMap* m, const void* base, int piece_fmt, int kcap, int rows, int nfreq, int bk);
void encode_b(CUtensorMap* m, const void* base, int piece_fmt, int kcap, int cols, int bk);

// Splits the field matrices of a batch, A[F][rows][lcap] (orders
// contiguous; FP64 or FP32 elements, in_bytes 8 or 4), into pieces
// P[2][F][rows][kcap] with one power-of-two scale per row (sa[F][rows]);
// orders at or beyond the frequency's count nord[w] become zeros up to the
// next multiple of bk (the contraction reads whole BK blocks).  lnz (or
// null) receives one past each row's last nonzero order.
// zf (or null): per frequency of the run, R1 entries; a row whose receiver
// row rowrec[row] has zf < K is zero from that order on and is read only up
// to it.
void split_fields(const void* A, int in_bytes, int nf, int rows, int lcap, const int* d_nord, uint16_t* P,
                  float* sa, int kcap, int F, int piece_fmt, int bk, cudaStream_t st, int* lnz = nullptr,
                  const int* zf = nullptr, const int* rowrec = nullptr, int R1 = 0);
// Splits the basis table B[cols][lcap] into P[2][cols][kcap] with one scale
// per column (sb[cols]); orders >= lcap become zeros.
void split_bases(const double* B, int cols, int lcap, uint16_t* P, float* sb, int kcap, int piece_fmt,
                 cudaStream_t st);

// Fills each problem's kb (where both kb and lz are set): the order blocks
// a row tile needs, ceil(max over its rows of lz / bk), at most kblocks.
void tile_orders(const Problem* d_probs, int np, int bk, cudaStream_t st);

// Launches the persistent contraction over all tiles of probs[0..np).
// err (device int) is set nonzero if a bounded wait inside gave up.
// wait_ns bounds every wait inside (WAIT_NS unless a test shortens it).
void launch(const Maps& maps, const Problem* d_probs, int np, int ntiles, int piece_fmt, int bk, uint32_t flags,
            int chunk, int* d_err, int nsm, cudaStream_t st, unsigned long long wait_ns = WAIT_NS);

}  // namespace tc
}  // namespace dsm
