// Learned angular-order cutoff (internal declarations).
#pragma once

#include "common.cuh"

namespace dsm {
namespace lmax {

constexpr int NF_ = DSM_LMAX_NFEAT, H_ = DSM_LMAX_WIDTH;
constexpr int OFF_XM = 0, OFF_XS = NF_, OFF_YM = 2 * NF_, OFF_YS = 2 * NF_ + 1;
constexpr int OFF_W1 = 2 * NF_ + 2;
constexpr int OFF_B1 = OFF_W1 + H_ * NF_;
constexpr int OFF_W2 = OFF_B1 + H_;
constexpr int OFF_B2 = OFF_W2 + H_ * H_;
constexpr int OFF_W3 = OFF_B2 + H_;
constexpr int OFF_B3 = OFF_W3 + H_ * H_;
constexpr int OFF_W4 = OFF_B3 + H_;
constexpr int OFF_B4 = OFF_W4 + H_;
static_assert(OFF_B4 + 1 == DSM_LMAX_NPARAM, "parameter block layout");

// standardisation from the data, He-initialised weights
void init_params(const float* X, const float* T, int n, unsigned seed, float* P);
// AdamW on the GPU (weight decay wd); P in/out; losses[epochs] (mean
// squared error of the standardised target per epoch)
void train(const float* X, const float* T, int n, int epochs, int batch, float lr, float wd, unsigned seed,
           float* P, float* losses, int device);
// loss and gradient of one batch (the first n rows), for checks
void grad(const float* P, const float* X, const float* T, int n, float* G, float* loss, int device);

// device-resident network of a context
struct Predictor {
    bool ready = false;
    DBuf<float> params, X, y, out;
    DBuf<__nv_bfloat16> pb;
    void load(const float* P, cudaStream_t st);
    void predict(const float* hX, int n, float* hout, cudaStream_t st);  // log lmax
};

}  // namespace lmax
}  // namespace dsm
