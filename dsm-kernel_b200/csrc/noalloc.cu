// dsm_sh_cutoff_noalloc: the SH angular-order cutoff (the reference's llog)
// computed without allocating device memory.
//
// Who needs it: callers that decide batch sizes before the SGT run (the
// cutoff sets the work of a frequency) from a process whose GPU memory is
// already reserved by another framework's caching allocator, so a
// cudaMalloc there would fail or fragment that pool, and callers that must
// not trigger the implicit device-wide synchronisation of cudaMalloc /
// cudaFree while other streams of the same GPU are running.
//
// How: every device buffer of the computation (the staged set-up arrays,
// the per-order probe amplitudes, the cutoff state) lives in one
// file-scope __device__ array of kScratchBytes.  Each GPU that loads the
// library holds that array until the process exits.  Host code cannot use
// the array's name as a device address, so the first call on a device
// looks the address up with cudaGetSymbolAddress (with that device
// current) and caches it; make that first call before any stream capture.
// Every call reuses the same array and leaves its contents behind: calls
// that overlap on the GPU (two host threads, or one call while an earlier
// one is still running on another stream) race on it.
//
// The probe kernel is a variant of the SH band solve (sh.cu, k_sh_solve):
// the same complex-symmetric tridiagonal LDL^T (dclisb0,
// src/SGTsh/dclib.f90:1-89) of a = a0 + l(l+1) a2 (cala0, cala2, overlap,
// src/SGTsh/calmat.f90:267-304, 386-423), assembled on the fly from the
// element integrals, keeping only the surface row the cutoff test reads
// (calamp on g0(nn), src/SGTsh/SGTsh-MPI.f90:476-478).  This file is
// compiled without fused multiply-add, like sh.cu, so the cutoff matches.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

namespace dsm {
void set_global_error(const std::string& e);
namespace {

constexpr size_t kScratchBytes = 64ull << 20;  // 64 MiB per device
constexpr int kChunk = 256;                     // orders solved per launch
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

struct NaDev {
    int nn, nzone, srow, ins, spn, n;
    double spo, r0, mu0, tlen, omegai;
    const int *nlayer, *isp, *jsp, *freqs;
    const double *qmu, *t, *h1, *h2, *h3, *h4, *g;
};

__device__ __forceinline__ cd na_coef(double omega, double q) {
    if (q <= 0.0) return mk(1.0);
    double aa = (omega == 0.0) ? 1.0 : 1.0 + log(omega / (2.0 * kPi)) / (kPi * q);
    double bb = 1.0 / (2.0 * q);
    return mk(aa, bb) * mk(aa, bb);
}

// band entries (off-diagonal, diagonal) of a0 and a2 at column jj
__device__ void na_band(const NaDev& d, int jj, cd comega2, double omega, cd* a0o, cd* a0d, cd* a2o,
                        cd* a2d) {
    cd s0d = mk(0.0), s0o = mk(0.0), s2d = mk(0.0), s2o = mk(0.0);
    for (int z = 0; z < d.nzone; ++z) {
        int nl = d.nlayer[z], i = jj - d.isp[z] + 1;
        if (i < 1 || i > nl + 1) continue;
        cd coef = na_coef(omega, d.qmu[z]);
        const int o = d.jsp[z] - 2;
        auto e0 = [&](int n) {
            double h = d.h1[o + n] - d.h2[o + n] + d.h3[o + n] - 2.0 * d.h4[o + n];
            return comega2 * mk(d.t[o + n]) - coef * mk(h);
        };
        auto e2 = [&](int n) { return -coef * mk(d.h4[o + n]); };
        if (i == 1) {
            s0d = s0d + e0(1);
            s2d = s2d + e2(1);
        } else if (i == nl + 1) {
            s0d = s0d + e0(4 * nl);
            s2d = s2d + e2(4 * nl);
        } else {
            s0d = s0d + e0(4 * i - 4) + e0(4 * i - 3);
            s2d = s2d + e2(4 * i - 4) + e2(4 * i - 3);
        }
        if (i >= 2) {
            s0o = s0o + e0(4 * i - 6);
            s2o = s2o + e2(4 * i - 6);
        }
    }
    *a0o = s0o; *a0d = s0d; *a2o = s2o; *a2d = s2d;
}

// One thread per (frequency, order): surface values of the two source basis
// solutions, the imt = 3 (pp) excitation for m = -2, +2 (calga, calg2,
// src/SGTsh/calmat.f90:329-353, 427-479) and the four probe amplitudes of
// the order (m = -2, -1, 1, 2; the m = +-1 pp excitation is zero).
__global__ void __launch_bounds__(128) k_na_probe(NaDev d, int l0, int lc, double* __restrict__ amps) {
    int sys = blockIdx.x * blockDim.x + threadIdx.x;
    if (sys >= d.n * lc) return;
    int w = sys / lc, l = l0 + sys % lc;
    double* ap = amps + (size_t)sys * 4;
    ap[0] = ap[1] = ap[2] = ap[3] = 0.0;
    if (l < 2) return;
    const double omega = 2.0 * kPi * (double)d.freqs[w] / d.tlen;
    const cd comega2 = mk(omega, -d.omegai) * mk(omega, -d.omegai);
    const double xl2 = (double)l * (double)(l + 1);
    const int nn = d.nn, s = d.srow;
    cd a0o, a0d, a2o, a2d;
    na_band(d, 1, comega2, omega, &a0o, &a0d, &a2o, &a2d);
    cd dr = mk(1.0) / (a0d + mk(xl2) * a2d);
    cd z0 = mk(s == 1 ? 1.0 : 0.0), z1 = mk(0.0);
    for (int j = 2; j <= nn; ++j) {
        na_band(d, j, comega2, omega, &a0o, &a0d, &a2o, &a2d);
        cd off = a0o + mk(xl2) * a2o, dg = a0d + mk(xl2) * a2d;
        cd L = off * dr;
        dr = mk(1.0) / (dg - off * L);
        z0 = mk(j == s ? 1.0 : 0.0) - L * z0;
        z1 = mk(j == s + 1 ? 1.0 : 0.0) - L * z1;
    }
    const cd x0 = z0 * dr, x1 = z1 * dr;  // basis solutions at the surface row
    // source element of the split layer and its 3x3 band (calga, overlap, dclisb0)
    const cd coef = na_coef(omega, d.qmu[d.spn - 1]);
    const double xl2m2 = xl2 - 2.0;
    cd aa[4], ga[8];
    for (int i = 0; i < 4; ++i) {
        int k = d.ins - 1 + i;
        double h = d.h1[k] - d.h2[k] + d.h3[k] + xl2m2 * d.h4[k];
        aa[i] = comega2 * mk(d.t[k]) - coef * mk(h);
    }
    for (int i = 0; i < 8; ++i) {
        double h = d.g[8 + i] - d.g[16 + i] + d.g[24 + i] + xl2m2 * d.g[32 + i];
        ga[i] = comega2 * mk(d.g[i]) - coef * mk(h);
    }
    cd o2 = ga[1], o3 = ga[5], d1 = ga[0], d2 = mk(0.0) + ga[3] + ga[4], d3 = ga[7];
    cd dr1 = mk(1.0) / d1, L2 = o2 * dr1, dr2 = mk(1.0) / (d2 - o2 * L2), L3 = o3 * dr2;
    cd dr3 = mk(1.0) / (d3 - o3 * L3);
    const double b1 = sqrt((double)(2 * l + 1) * (double)(l - 1) * (double)(l + 2) / (64.0 * kPi));
    for (int sg = 0; sg < 2; ++sg) {
        double sgn = sg == 0 ? -1.0 : 1.0;
        cd c2 = mk(b1 / d.r0) * mk(0.0, sgn * (0.0 - 1.0));  // imt 3: mt22 - mt33 = -1
        cd y2 = c2 - L2 * mk(0.0), y3 = mk(0.0) - L3 * y2;
        cd y1 = mk(0.0) * dr1;
        y2 = y2 * dr2;
        y3 = y3 * dr3;
        cd xx3 = y3, xx2 = y2 - L3 * xx3, xx1 = y1 - L2 * xx2;
        cd gs = aa[0] * xx1 + aa[1] * xx3, gs1 = aa[2] * xx1 + aa[3] * xx3;
        cd gn = gs * x0 + gs1 * x1;
        ap[sg == 0 ? 0 : 3] = hypot(gn.re, gn.im);
    }
}

// cutoff test in the reference's order (calamp, src/SGTsh/others.f90:805-824;
// ismall > 20, SGTsh-MPI.f90:431-436)
__global__ void k_na_scan(int n, int l0, int lc, int maxlmax, double ratl, double tlen, double vtop,
                          double rtop, const int* __restrict__ freqs, const double* __restrict__ amps,
                          CutState* __restrict__ cut) {
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n) return;
    CutState c = cut[w];
    if (c.done) return;
    double omega = 2.0 * kPi * (double)freqs[w] / tlen;
    int lsuf = (int)(omega * rtop / vtop - 0.5) + 1;
    for (int l = l0; l < l0 + lc; ++l) {
        if (c.ismall > 20) {
            if (c.llog > l) c.llog = l;
            c.done = 1;
            break;
        }
        if (l >= 1) {
            const double* ap = amps + ((size_t)w * lc + (l - l0)) * 4;
            for (int mi = 0; mi < 4; ++mi) {
                int m = (mi == 0) ? -2 : (mi == 1 ? -1 : (mi == 2 ? 1 : 2));
                if (abs(m) > l) continue;
                double amp = ap[mi], ampratio = 0.0;
                if (amp > c.maxamp) c.maxamp = amp;
                if (amp != 0.0 && c.maxamp != 0.0) ampratio = amp / c.maxamp;
                if (ampratio < ratl && l > lsuf) c.ismall++;
                else c.ismall = 0;
            }
        }
        if (l == maxlmax) c.done = 1;
    }
    cut[w] = c;
}

void* scratch_address(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= kMaxDevices) throw Error(DSM_ERR_NODEVICE, "device ordinal out of range");
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            throw Error(DSM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

// bump allocator over the scratch array (offsets only; nothing is allocated)
struct Carve {
    unsigned char* base;
    size_t off = 0;
    template <class T>
    T* take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

}  // namespace
}  // namespace dsm

extern "C" int dsm_sh_cutoff_noalloc(const dsm_sh_setup_t* s, const int* ilist, int n, int* llog) {
    using namespace dsm;
    if (!s || !ilist || !llog || n <= 0) {
        set_global_error("dsm_sh_cutoff_noalloc: null argument or empty frequency list");
        return DSM_ERR_INVALID;
    }
    try {
        int dev = 0;
        DSM_CUDA(cudaGetDevice(&dev));
        unsigned char* base = static_cast<unsigned char*>(scratch_address(dev));
        for (int k = 0; k < n; ++k)
            if (ilist[k] <= 0) throw Error(DSM_ERR_INVALID, "dsm_sh_cutoff_noalloc: frequency index must be > 0");
        const int nz = s->nzone, nn = s->nnlayer + 1;
        const size_t ne = 4 * (size_t)s->nnlayer;
        // layout and size check before anything is written
        Carve cv{base};
        int* d_nl = cv.take<int>(nz);
        int* d_isp = cv.take<int>(nz);
        int* d_jsp = cv.take<int>(nz);
        int* d_fr = cv.take<int>(n);
        double* d_q = cv.take<double>(nz);
        double* d_e[5];
        for (auto& p : d_e) p = cv.take<double>(ne);
        double* d_g = cv.take<double>(40);
        double* d_amp = cv.take<double>((size_t)n * kChunk * 4);
        CutState* d_cut = cv.take<CutState>(n);
        if (cv.off > kScratchBytes)
            throw Error(DSM_ERR_INVALID, "dsm_sh_cutoff_noalloc: the set-up needs " + std::to_string(cv.off) +
                                             " bytes of device scratch, more than the fixed " +
                                             std::to_string(kScratchBytes) + " bytes");
        cudaStream_t st = cudaStreamPerThread;
        auto up = [&](void* dst, const void* src, size_t b) {
            DSM_CUDA(cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, st));
        };
        up(d_nl, s->nlayer, sizeof(int) * nz);
        up(d_isp, s->isp, sizeof(int) * nz);
        up(d_jsp, s->jsp, sizeof(int) * nz);
        up(d_fr, ilist, sizeof(int) * n);
        up(d_q, s->qmu, sizeof(double) * nz);
        const double* he[5] = {s->t, s->h1, s->h2, s->h3, s->h4};
        for (int k = 0; k < 5; ++k) up(d_e[k], he[k], sizeof(double) * ne);
        std::vector<double> gg(40);
        for (int k = 0; k < 8; ++k) {
            gg[k] = s->gt[k]; gg[8 + k] = s->gh1[k]; gg[16 + k] = s->gh2[k];
            gg[24 + k] = s->gh3[k]; gg[32 + k] = s->gh4[k];
        }
        up(d_g, gg.data(), sizeof(double) * 40);
        // the cutoff state must start from the reference's initial values
        std::vector<CutState> init(n);
        for (auto& c : init) { c.ismall = 0; c.done = 0; c.llog = s->maxlmax; c.norders = 0; c.maxamp = -1.0; }
        up(d_cut, init.data(), sizeof(CutState) * n);
        NaDev d{};
        d.nn = nn; d.nzone = nz; d.ins = s->ins; d.spn = s->spn; d.n = n;
        d.srow = s->isp[s->spn - 1] + (int)std::trunc(s->spo);
        d.spo = s->spo; d.r0 = s->r0; d.mu0 = s->mu0; d.tlen = s->tlen; d.omegai = s->omegai;
        d.nlayer = d_nl; d.isp = d_isp; d.jsp = d_jsp; d.freqs = d_fr; d.qmu = d_q;
        d.t = d_e[0]; d.h1 = d_e[1]; d.h2 = d_e[2]; d.h3 = d_e[3]; d.h4 = d_e[4]; d.g = d_g;
        double vtop = 0.0;
        for (int i = 0; i < 4; ++i) vtop = vtop + s->vsv[4 * (nz - 1) + i] * 1.0;
        const double rtop = s->vrmax[nz - 1];
        std::vector<CutState> hc(n);
        for (int l0 = 0; l0 <= s->maxlmax; l0 += kChunk) {
            int lc = std::min(kChunk, s->maxlmax + 1 - l0);
            k_na_probe<<<(n * lc + 127) / 128, 128, 0, st>>>(d, l0, lc, d_amp);
            DSM_CUDA(cudaGetLastError());
            k_na_scan<<<(n + 31) / 32, 32, 0, st>>>(n, l0, lc, s->maxlmax, s->ratl, s->tlen, vtop, rtop, d_fr,
                                                    d_amp, d_cut);
            DSM_CUDA(cudaGetLastError());
            DSM_CUDA(cudaMemcpyAsync(hc.data(), d_cut, sizeof(CutState) * n, cudaMemcpyDeviceToHost, st));
            DSM_CUDA(cudaStreamSynchronize(st));
            bool all = true;
            for (auto& c : hc) all = all && c.done;
            if (all) break;
        }
        for (int k = 0; k < n; ++k) llog[k] = hc[k].llog;
        return DSM_OK;
    } catch (const Error& e) {
        set_global_error(e.what());
        return e.code;
    }
}
