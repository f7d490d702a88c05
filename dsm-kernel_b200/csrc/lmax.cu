// Learned angular-order cutoff: a 4-layer MLP (width 128, GELU) from
// (omega, source radius, receiver radius, 8 model summaries) to log(lmax),
// with bf16 weights and FP32 accumulation; forward, backward and Adam are
// the kernels below.  The engine uses the prediction to size the first
// order range of each frequency; the plain DSM amplitude test still decides
// the cutoff on the device and extends any range that falls short, so the
// truncation is the plain method's (src/SGTpsv/SGTpsv-MPI.f90:606-609).
//
// Parameter block (float, DSM_LMAX_NPARAM entries):
//   x_mean[NF] x_std[NF] y_mean y_std | W1[H][NF] b1[H] | W2[H][H] b2[H] |
//   W3[H][H] b3[H] | W4[H] b4
// Inputs are standardised with (x_mean, x_std); the network output is the
// standardised log(lmax).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "common.cuh"
#include "lmax.cuh"

namespace dsm {
namespace lmax {

namespace {

constexpr int H = DSM_LMAX_WIDTH, NF = DSM_LMAX_NFEAT;
constexpr int S = 32;  // samples per forward / delta block

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float dgelu(float z) {
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    return cdf + z * pdf;
}

// bf16 working copy of the weights (biases and normalisation stay FP32)
__global__ void k_to_bf16(const float* __restrict__ P, __nv_bfloat16* __restrict__ Pb, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) Pb[i] = __float2bfloat16_rn(P[i]);
}
__device__ __forceinline__ float wt(const __nv_bfloat16* Pb, int i) { return __bfloat162float(Pb[i]); }

// Forward of S samples per block, thread j = neuron j.  Saves the
// pre-activations Z[l][n][H] (l = 0..2) and returns the standardised
// output y[n] (and, with denorm, log(lmax) in out[n]).
__global__ void __launch_bounds__(H) k_fwd(const float* __restrict__ P, const __nv_bfloat16* __restrict__ Pb,
                                           const float* __restrict__ X, const int* __restrict__ idx, int n,
                                           float* __restrict__ Xn, float* __restrict__ Z, float* __restrict__ y,
                                           float* __restrict__ out) {
    __shared__ float a[S][H + 1];
    __shared__ float xin[S][NF];
    const int j = threadIdx.x, s0 = blockIdx.x * S;
    for (int t = j; t < S * NF; t += H) {
        const int s = t / NF, i = t % NF;
        float v = 0.0f;
        if (s0 + s < n) {
            const int row = idx ? idx[s0 + s] : s0 + s;
            v = (X[(size_t)row * NF + i] - P[OFF_XM + i]) / P[OFF_XS + i];
            if (Xn) Xn[(size_t)(s0 + s) * NF + i] = v;
        }
        xin[s][i] = v;
    }
    __syncthreads();
    float acc[S];
    // layer 1
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = P[OFF_B1 + j];
    for (int i = 0; i < NF; ++i) {
        const float w = wt(Pb, OFF_W1 + j * NF + i);
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] += w * xin[s][i];
    }
    for (int layer = 0; layer < 3; ++layer) {
        if (layer > 0) {
            const int ow = layer == 1 ? OFF_W2 : OFF_W3, ob = layer == 1 ? OFF_B2 : OFF_B3;
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] = P[ob + j];
            for (int i = 0; i < H; ++i) {
                const float w = wt(Pb, ow + j * H + i);
#pragma unroll
                for (int s = 0; s < S; ++s) acc[s] += w * a[s][i];
            }
            __syncthreads();  // everyone has read a[] of the previous layer
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (Z && s0 + s < n) Z[((size_t)layer * n + s0 + s) * H + j] = acc[s];
            a[s][j] = gelu(acc[s]);
        }
        __syncthreads();
    }
    if (j < S && s0 + j < n) {
        float v = P[OFF_B4];
        for (int i = 0; i < H; ++i) v += wt(Pb, OFF_W4 + i) * a[j][i];
        y[s0 + j] = v;
        if (out) out[s0 + j] = v * P[OFF_YS] + P[OFF_YM];
    }
}

// loss = mean (y - t)^2 on standardised targets; dY = 2 (y - t) / n
__global__ void k_loss(const float* __restrict__ P, const float* __restrict__ y, const float* __restrict__ T,
                       const int* __restrict__ idx, int n, float* __restrict__ dY, float* __restrict__ loss) {
    __shared__ float red[256];
    float l = 0.0f;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const int row = idx ? idx[s] : s;
        const float t = (T[row] - P[OFF_YM]) / P[OFF_YS];
        const float d = y[s] - t;
        dY[s] = 2.0f * d / (float)n;
        l += d * d;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)n);
}

// activation of layer l (0..2) recomputed from its pre-activation
__device__ __forceinline__ float act(const float* Z, int layer, int n, int s, int i) {
    return gelu(Z[((size_t)layer * n + s) * H + i]);
}

// dZ of the last hidden layer: dZ3[s][i] = dY[s] W4[i] gelu'(Z3)
__global__ void k_delta_top(const __nv_bfloat16* __restrict__ Pb, const float* __restrict__ Z,
                            const float* __restrict__ dY, int n, float* __restrict__ dZ) {
    const int s = blockIdx.x, i = threadIdx.x;
    if (s >= n) return;
    dZ[((size_t)2 * n + s) * H + i] = dY[s] * wt(Pb, OFF_W4 + i) * dgelu(Z[((size_t)2 * n + s) * H + i]);
}

// dZ of layer l-1 from dZ of layer l (l = 2, 1): dA[s][i] = sum_j dZ[s][j] W[j][i]
__global__ void __launch_bounds__(H) k_delta(const __nv_bfloat16* __restrict__ Pb, int layer,
                                             const float* __restrict__ Z, int n, float* __restrict__ dZ) {
    __shared__ float d[S][H + 1];
    const int i = threadIdx.x, s0 = blockIdx.x * S;
    const int ow = layer == 2 ? OFF_W3 : OFF_W2;
    for (int s = 0; s < S; ++s) d[s][i] = (s0 + s < n) ? dZ[((size_t)layer * n + s0 + s) * H + i] : 0.0f;
    __syncthreads();
    float acc[S];
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = 0.0f;
    for (int j = 0; j < H; ++j) {
        const float w = wt(Pb, ow + j * H + i);
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] += d[s][j] * w;
    }
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (s0 + s < n) {
            const size_t o = ((size_t)(layer - 1) * n + s0 + s) * H + i;
            dZ[o] = acc[s] * dgelu(Z[o]);
        }
}

// weight gradients: block j (output neuron), thread i (input), summed over
// the batch.  layer 0 takes the standardised inputs.
__global__ void k_wgrad(int layer, const float* __restrict__ Xn, const float* __restrict__ Z,
                        const float* __restrict__ dZ, const float* __restrict__ dY, int n, float* __restrict__ G) {
    const int j = blockIdx.x, i = threadIdx.x;
    if (layer == 3) {  // W4[i], b4 (grid 1)
        float g = 0.0f, gb = 0.0f;
        for (int s = 0; s < n; ++s) {
            g += dY[s] * act(Z, 2, n, s, i);
            gb += dY[s];
        }
        G[OFF_W4 + i] = g;
        if (i == 0) G[OFF_B4] = gb;
        return;
    }
    const int nin = layer == 0 ? NF : H;
    const int ow = layer == 0 ? OFF_W1 : (layer == 1 ? OFF_W2 : OFF_W3);
    const int ob = layer == 0 ? OFF_B1 : (layer == 1 ? OFF_B2 : OFF_B3);
    float g = 0.0f, gb = 0.0f;
    for (int s = 0; s < n; ++s) {
        const float dz = dZ[((size_t)layer * n + s) * H + j];
        if (i < nin) g += dz * (layer == 0 ? Xn[(size_t)s * NF + i] : act(Z, layer - 1, n, s, i));
        gb += dz;
    }
    if (i < nin) G[ow + j * nin + i] = g;
    if (i == 0) G[ob + j] = gb;
}

// Adam on the weights and biases (the normalisation block is not trained)
__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ m1,
                       float* __restrict__ m2, int* __restrict__ step, float lr, float wd,
                       __nv_bfloat16* __restrict__ Pb) {
    const int i = OFF_W1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int t = *step + 1;
    if (i < DSM_LMAX_NPARAM) {
        const float b1 = 0.9f, b2 = 0.999f;
        const float g = G[i];
        const float a = b1 * m1[i] + (1.0f - b1) * g, b = b2 * m2[i] + (1.0f - b2) * g * g;
        m1[i] = a;
        m2[i] = b;
        const float ah = a / (1.0f - powf(b1, (float)t)), bh = b / (1.0f - powf(b2, (float)t));
        // decoupled weight decay (AdamW) keeps the network from leaning on
        // inputs that hardly vary between the training models
        P[i] -= lr * (ah / (sqrtf(bh) + 1e-8f) + wd * P[i]);
        Pb[i] = __float2bfloat16_rn(P[i]);
    }
}
// the step counter advances in its own launch, after every block of k_adam read it
__global__ void k_step(int* step) { *step += 1; }

struct Net {
    DBuf<float> P, G, m1, m2, Xn, Z, dZ, y, dY, loss, X, T, out;
    DBuf<__nv_bfloat16> Pb;
    DBuf<int> idx, step;
    int cap = 0;
    void reserve(int nb) {
        if (nb <= cap) return;
        Xn.reserve((size_t)nb * NF);
        Z.reserve((size_t)3 * nb * H);
        dZ.reserve((size_t)3 * nb * H);
        y.reserve(nb);
        dY.reserve(nb);
        out.reserve(nb);
        cap = nb;
    }
};

// forward + loss + backward of one batch (idx into X/T, or the first n rows)
void grad_step(Net& net, const int* d_idx, int n, float* loss, cudaStream_t st) {
    k_fwd<<<(n + S - 1) / S, H, 0, st>>>(net.P.p, net.Pb.p, net.X.p, d_idx, n, net.Xn.p, net.Z.p, net.y.p, nullptr);
    k_loss<<<1, 256, 0, st>>>(net.P.p, net.y.p, net.T.p, d_idx, n, net.dY.p, loss);
    k_delta_top<<<n, H, 0, st>>>(net.Pb.p, net.Z.p, net.dY.p, n, net.dZ.p);
    k_delta<<<(n + S - 1) / S, H, 0, st>>>(net.Pb.p, 2, net.Z.p, n, net.dZ.p);
    k_delta<<<(n + S - 1) / S, H, 0, st>>>(net.Pb.p, 1, net.Z.p, n, net.dZ.p);
    k_wgrad<<<1, H, 0, st>>>(3, net.Xn.p, net.Z.p, net.dZ.p, net.dY.p, n, net.G.p);
    for (int l = 0; l < 3; ++l) k_wgrad<<<H, H, 0, st>>>(l, net.Xn.p, net.Z.p, net.dZ.p, net.dY.p, n, net.G.p);
    DSM_CUDA(cudaGetLastError());
}

}  // namespace

void init_params(const float* X, const float* T, int n, unsigned seed, float* P) {
    std::memset(P, 0, sizeof(float) * DSM_LMAX_NPARAM);
    for (int i = 0; i < NF; ++i) {
        double m = 0.0, v = 0.0;
        for (int s = 0; s < n; ++s) m += X[(size_t)s * NF + i];
        m /= std::max(n, 1);
        for (int s = 0; s < n; ++s) v += (X[(size_t)s * NF + i] - m) * (X[(size_t)s * NF + i] - m);
        v = std::sqrt(v / std::max(n, 1));
        P[OFF_XM + i] = (float)m;
        P[OFF_XS + i] = (float)(v > 1e-6 ? v : 1.0);
    }
    double m = 0.0, v = 0.0;
    for (int s = 0; s < n; ++s) m += T[s];
    m /= std::max(n, 1);
    for (int s = 0; s < n; ++s) v += (T[s] - m) * (T[s] - m);
    v = std::sqrt(v / std::max(n, 1));
    P[OFF_YM] = (float)m;
    P[OFF_YS] = (float)(v > 1e-6 ? v : 1.0);
    std::mt19937 rng(seed);
    auto fill = [&](int off, int rows, int cols) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)cols));
        for (int k = 0; k < rows * cols; ++k) P[off + k] = nd(rng);
    };
    fill(OFF_W1, H, NF);
    fill(OFF_W2, H, H);
    fill(OFF_W3, H, H);
    fill(OFF_W4, 1, H);
}

void train(const float* X, const float* T, int n, int epochs, int batch, float lr, float wd, unsigned seed,
           float* P, float* losses, int device) {
    if (n <= 0 || batch <= 0 || epochs <= 0) throw Error(DSM_ERR_INVALID, "empty training set");
    DSM_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    DSM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    Net net;
    batch = std::min(batch, n);
    net.reserve(batch);
    net.P.upload(P, DSM_LMAX_NPARAM, st);
    net.G.reserve(DSM_LMAX_NPARAM);
    net.m1.reserve(DSM_LMAX_NPARAM);
    net.m2.reserve(DSM_LMAX_NPARAM);
    DSM_CUDA(cudaMemsetAsync(net.G.p, 0, sizeof(float) * DSM_LMAX_NPARAM, st));
    DSM_CUDA(cudaMemsetAsync(net.m1.p, 0, sizeof(float) * DSM_LMAX_NPARAM, st));
    DSM_CUDA(cudaMemsetAsync(net.m2.p, 0, sizeof(float) * DSM_LMAX_NPARAM, st));
    net.Pb.reserve(DSM_LMAX_NPARAM);
    k_to_bf16<<<(DSM_LMAX_NPARAM + 255) / 256, 256, 0, st>>>(net.P.p, net.Pb.p, DSM_LMAX_NPARAM);
    net.X.upload(X, (size_t)n * NF, st);
    net.T.upload(T, n, st);
    net.loss.reserve(epochs);
    DSM_CUDA(cudaMemsetAsync(net.loss.p, 0, sizeof(float) * epochs, st));
    net.step.reserve(1);
    DSM_CUDA(cudaMemsetAsync(net.step.p, 0, sizeof(int), st));
    net.idx.reserve(n);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    std::mt19937 rng(seed ^ 0x9e3779b9u);
    const int nb = n / batch;  // full batches per epoch
    const int nadam = (DSM_LMAX_NPARAM - OFF_W1 + 255) / 256;
    // one optimiser step, captured once and replayed: gather by index,
    // forward, loss, backward, Adam
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DBuf<int> cur;  // batch indices of the current step
    cur.reserve(batch);
    DBuf<float> lossacc;
    lossacc.reserve(1);
    DSM_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    {
        grad_step(net, cur.p, batch, lossacc.p, st);
        k_adam<<<nadam, 256, 0, st>>>(net.P.p, net.G.p, net.m1.p, net.m2.p, net.step.p, lr, wd, net.Pb.p);
        k_step<<<1, 1, 0, st>>>(net.step.p);
    }
    DSM_CUDA(cudaStreamEndCapture(st, &graph));
    DSM_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    for (int e = 0; e < epochs; ++e) {
        std::shuffle(perm.begin(), perm.end(), rng);
        net.idx.upload(perm, st);
        DSM_CUDA(cudaMemsetAsync(lossacc.p, 0, sizeof(float), st));
        for (int b = 0; b < nb; ++b) {
            DSM_CUDA(cudaMemcpyAsync(cur.p, net.idx.p + (size_t)b * batch, sizeof(int) * batch,
                                     cudaMemcpyDeviceToDevice, st));
            DSM_CUDA(cudaGraphLaunch(exec, st));
        }
        // epoch loss = mean of the batch losses
        DSM_CUDA(cudaMemcpyAsync(net.loss.p + e, lossacc.p, sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    std::vector<float> hl(epochs);
    DSM_CUDA(cudaMemcpyAsync(hl.data(), net.loss.p, sizeof(float) * epochs, cudaMemcpyDeviceToHost, st));
    DSM_CUDA(cudaMemcpyAsync(P, net.P.p, sizeof(float) * DSM_LMAX_NPARAM, cudaMemcpyDeviceToHost, st));
    DSM_CUDA(cudaStreamSynchronize(st));
    if (losses)
        for (int e = 0; e < epochs; ++e) losses[e] = hl[e] / (float)std::max(nb, 1);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    cudaStreamDestroy(st);
}

void grad(const float* P, const float* X, const float* T, int n, float* G, float* loss, int device) {
    DSM_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    DSM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    Net net;
    net.reserve(n);
    net.P.upload(P, DSM_LMAX_NPARAM, st);
    net.Pb.reserve(DSM_LMAX_NPARAM);
    k_to_bf16<<<(DSM_LMAX_NPARAM + 255) / 256, 256, 0, st>>>(net.P.p, net.Pb.p, DSM_LMAX_NPARAM);
    net.G.reserve(DSM_LMAX_NPARAM);
    DSM_CUDA(cudaMemsetAsync(net.G.p, 0, sizeof(float) * DSM_LMAX_NPARAM, st));
    net.X.upload(X, (size_t)n * NF, st);
    net.T.upload(T, n, st);
    net.loss.reserve(1);
    DSM_CUDA(cudaMemsetAsync(net.loss.p, 0, sizeof(float), st));
    grad_step(net, nullptr, n, net.loss.p, st);
    DSM_CUDA(cudaMemcpyAsync(G, net.G.p, sizeof(float) * DSM_LMAX_NPARAM, cudaMemcpyDeviceToHost, st));
    DSM_CUDA(cudaMemcpyAsync(loss, net.loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    DSM_CUDA(cudaStreamSynchronize(st));
    cudaStreamDestroy(st);
}

void Predictor::load(const float* P, cudaStream_t st) {
    params.upload(P, DSM_LMAX_NPARAM, st);
    pb.reserve(DSM_LMAX_NPARAM);
    k_to_bf16<<<(DSM_LMAX_NPARAM + 255) / 256, 256, 0, st>>>(params.p, pb.p, DSM_LMAX_NPARAM);
    DSM_CUDA(cudaGetLastError());
    ready = true;
}

void Predictor::predict(const float* hX, int n, float* hout, cudaStream_t st) {
    if (!ready) throw Error(DSM_ERR_INVALID, "no lmax model loaded");
    X.upload(hX, (size_t)n * NF, st);
    y.reserve(n);
    out.reserve(n);
    k_fwd<<<(n + S - 1) / S, H, 0, st>>>(params.p, pb.p, X.p, nullptr, n, nullptr, nullptr, y.p, out.p);
    DSM_CUDA(cudaGetLastError());
    DSM_CUDA(cudaMemcpyAsync(hout, out.p, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    DSM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace lmax
}  // namespace dsm
