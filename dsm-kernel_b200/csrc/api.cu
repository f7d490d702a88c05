// C-ABI entry points (include/dsmsgt.h) and the batch driver shared by the
// SH and PSV engines.
//
// One call of dsm_run_freqs replaces, for every requested frequency index,
// one pass of the reference's omega loop (src/SGTsh/SGTsh-MPI.f90:389-613,
// src/SGTpsv/SGTpsv-MPI.f90:535-1152) minus the file writes.  Frequencies are
// processed in batches of F.  For a batch the driver
//   1. builds the per-omega operator pieces          (mode kernel)
//   2. solves chunks of Lc angular orders of every frequency of the batch at
//      once, then runs the reference's cutoff test on the device; chunks
//      continue until every frequency has met its cutoff (the test is the
//      reference's, evaluated in the same order, so the number of orders
//      summed is the reference's llog)
//   3. contracts the per-order receiver fields with the vector-harmonic
//      tables over l (one GEMM per frequency and |m|)
//   4. turns the contractions into TSGT/RSGT/SYNN (mode epilogue kernel)
//   5. packs complex64 catalogue records when asked.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <climits>
#include <cstdint>
#include <cstring>
#include <thread>

#include "engine.cuh"

namespace dsm {

void Engine::init_common(int dev) {
    DSM_CUDA(cudaSetDevice(dev));
    // the source-term kernels keep the 4x4x10 Runge-Kutta coefficient
    // tables of calabnum in thread-local memory
    size_t stack = 0;
    DSM_CUDA(cudaDeviceGetLimit(&stack, cudaLimitStackSize));
    if (stack < 16384) DSM_CUDA(cudaDeviceSetLimit(cudaLimitStackSize, 16384));
    DSM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    {  // the side stream carries latency-bound chains: give its blocks priority
        int lo = 0, hi = 0;
        DSM_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        DSM_CUDA(cudaStreamCreateWithPriority(&st2, cudaStreamNonBlocking, hi));
    }
    DSM_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    DSM_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    DSM_CUDA(cudaStreamCreateWithFlags(&stc, cudaStreamNonBlocking));
    for (auto& e : ev_grp) DSM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    {  // mixed l-sum pipeline: the contraction's stream has priority
        int lo = 0, hi = 0;
        DSM_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        DSM_CUDA(cudaStreamCreateWithPriority(&stt, cudaStreamNonBlocking, hi));

        DSM_CUDA(cudaEventCreateWithFlags(&ev_lp, cudaEventDisableTiming));
        DSM_CUDA(cudaEventCreateWithFlags(&ev_lj, cudaEventDisableTiming));
    }
    DSM_CUBLAS(cublasCreate(&cub));
    DSM_CUBLAS(cublasSetStream(cub, st));
    for (auto& e : ev) DSM_CUDA(cudaEventCreate(&e));
    DSM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (opt.precision != DSM_PREC_FP64 && !mixed())
        throw Error(DSM_ERR_INVALID, "unknown precision mode " + std::to_string(opt.precision));
    tc_fmt = opt.precision == DSM_PREC_MIXED_BF16 ? tc::PIECE_BF16 : tc::PIECE_F16;
    // tuning knobs of the tensor-core contraction (stage depth, accumulation
    // order and split), overridable for measurements
    if (const char* e = std::getenv("DSM_TC_FLAGS")) tc_flags = (uint32_t)std::atoi(e);
    if (const char* e = std::getenv("DSM_TC_BK")) tc_bk = std::atoi(e) == 64 ? 64 : 32;
    tune.tc_orders = tc_bk;
    if (const char* e = std::getenv("DSM_TC_CHUNK")) tc_chunk = std::max(0, std::atoi(e));
    if (const char* e = std::getenv("DSM_LSUM_GROUPS")) lsum_groups = std::max(1, std::atoi(e));
    dflags.reserve(2);
    DSM_CUDA(cudaMemset(dflags.p, 0, 2 * sizeof(int)));
}

Engine::~Engine() {
    if (st) cudaStreamSynchronize(st);
    for (auto& r : recs) { evpool.push_back(r.a); evpool.push_back(r.b); }
    for (auto e : evpool) cudaEventDestroy(e);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (cub) cublasDestroy(cub);
    if (st2) { cudaStreamSynchronize(st2); cudaStreamDestroy(st2); }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (stc) { cudaStreamSynchronize(stc); cudaStreamDestroy(stc); }
    for (auto& e : ev_grp)
        if (e) cudaEventDestroy(e);
    if (stt) { cudaStreamSynchronize(stt); cudaStreamDestroy(stt); }
    if (ev_lp) cudaEventDestroy(ev_lp);
    if (ev_lj) cudaEventDestroy(ev_lj);
    if (st) cudaStreamDestroy(st);
}

double* Engine::out_t_src() const {
    size_t pt, pr, ps;
    out_sizes(&pt, &pr, &ps);
    return out_t.p + 2 * pt * (size_t)F * src;
}
double* Engine::out_r_src() const {
    size_t pt, pr, ps;
    out_sizes(&pt, &pr, &ps);
    return out_r.p + 2 * pr * (size_t)F * src;
}
double* Engine::out_s_src() const {
    size_t pt, pr, ps;
    out_sizes(&pt, &pr, &ps);
    return out_s.p + 2 * ps * (size_t)F * src;
}

int Engine::kid(const char* name) {
    for (int i = 0; i < stats.nk; ++i)
        if (std::strncmp(stats.kern[i].name, name, 31) == 0) return i;
    if (stats.nk >= DSM_MAX_KSTATS) return -1;
    int i = stats.nk++;
    std::snprintf(stats.kern[i].name, sizeof(stats.kern[i].name), "%s", name);
    return i;
}

void Engine::fork_side() {
    DSM_CUDA(cudaEventRecord(ev_fork, st));
    DSM_CUDA(cudaStreamWaitEvent(st2, ev_fork, 0));
    side_pending = true;
}

void Engine::join_side() {
    if (!side_pending) return;
    DSM_CUDA(cudaEventRecord(ev_join, st2));
    DSM_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
    side_pending = false;
}

void Engine::kbegin(int id, cudaStream_t s) {
    if (!s) s = st;
    if (!prof || id < 0) return;
    if (evpool.size() < 2) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            DSM_CUDA(cudaEventCreate(&e));
            evpool.push_back(e);
        }
    }
    cudaEvent_t a = evpool.back();
    evpool.pop_back();
    cudaEvent_t b = evpool.back();
    evpool.pop_back();
    DSM_CUDA(cudaEventRecord(a, s));
    recs.push_back({id, a, b});
}

void Engine::kend(int id, double bytes, double flops, cudaStream_t s) {
    if (!s) s = st;
    if (id < 0) return;
    stats.kern[id].launches++;
    stats.kern[id].alg_bytes += bytes;
    stats.kern[id].alg_flops += flops;
    if (!prof) return;
    DSM_CUDA(cudaEventRecord(recs.back().b, s));
}

void Engine::kcollect() {
    if (recs.empty()) return;
    DSM_CUDA(cudaStreamSynchronize(st));
    DSM_CUDA(cudaStreamSynchronize(st2));
    for (auto& r : recs) {
        float ms = 0;
        cudaEventElapsedTime(&ms, r.a, r.b);
        stats.kern[r.id].ms += ms;
        evpool.push_back(r.a);
        evpool.push_back(r.b);
    }
    recs.clear();
}

void Engine::build_basis(int lneed) {
    if (lneed <= lcapB) return;
    int cap = std::max(lcapB, 1024);
    while (cap < lneed) cap *= 2;
    cap = std::min(cap, maxlmax + 1);
    if (cap < lneed) cap = lneed;
    launch_basis_tables(*this, cap);
    if (mixed()) {  // split the new tables once; every batch reuses them
        kcB = (lcapB + 63) / 64 * 64;
        for (int m = m_lo; m <= 2; ++m) {
            Bpc[m].reserve((size_t)2 * 2 * Th * kcB);
            sB[m].reserve((size_t)2 * Th);
            tc::split_bases(basis[m].p, 2 * Th, lcapB, Bpc[m].p, sB[m].p, kcB, tc_fmt, st);
            launches++;
        }
    }
}

// Mixed l-sum of a batch: split the field matrices, then persistent
// tensor-core launches over the (frequency, |m|) contractions (at most
// tc::MAXP per launch).  Outputs go to Cmix, one block per frequency.
void Engine::lsum_prepare(int nf, const std::vector<int>& nord) {
    (void)nf;
    kcA = (Lcap + 63) / 64 * 64;
    for (int m = m_lo; m <= 2; ++m) {
        if (!rows_m[m]) continue;
        Apc[m].reserve((size_t)2 * F * rows_m[m] * kcA);
        sA[m].reserve((size_t)F * rows_m[m]);
        lnzA[m].reserve((size_t)F * rows_m[m]);
    }
    Cmix.reserve((size_t)F * c_total());
    d_nord.upload(nord, st);
    std::memset(&tcmaps, 0, sizeof(tcmaps));
    for (int m = m_lo; m <= 2; ++m) {
        if (!rows_m[m]) continue;
        tc::encode_a(&tcmaps.a[m], Apc[m].p, tc_fmt, kcA, rows_m[m], F, tc_bk);
        tc::encode_b(&tcmaps.b[m], Bpc[m].p, tc_fmt, kcB, 2 * Th, tc_bk);
    }
    tcp.reserve((size_t)F * 6);  // at most two row groups per |m| and frequency
    tcp_next = 0;
}

// Problem lists of every frequency group of the batch, uploaded in one copy
// before the first group's launches (a pageable copy per group could hold
// the host until the stream has drained, between the groups' launches).
void Engine::lsum_plan(const std::vector<std::vector<int>>& groups, const std::vector<int>& nord) {
    tc_groups.clear();
    std::vector<tc::Problem> all;
    {  // row-tile entries of every problem (two row groups per |m| and frequency)
        size_t ntm = 0;
        for (const auto& slots : groups)
            for (size_t k = 0; k < slots.size(); ++k)
                for (int m = m_lo; m <= 2; ++m)
                    ntm += (size_t)(rows_m[m] + 2 * tc::BM) / tc::BM;
        tcKb.reserve(std::max<size_t>(ntm, 1));
    }
    size_t kboff = 0;
    for (const auto& slots : groups) {
        TcGroup G{slots, {}, 0.0, 0.0, 0.0};
        // per (frequency, |m|): the leading rows against all 2 Th basis
        // columns, the remaining rows against the first Th
        std::vector<tc::Problem> hp;
        for (int w : G.slots)
            for (int m = m_lo; m <= 2; ++m) {
                if (!rows_m[m]) continue;
                const double kp = (double)((nord[w] + tc_bk - 1) / tc_bk * tc_bk);
                G.split_bytes += (double)rows_m[m] * ((double)afld_bytes * nord[w] + 4.0 * kp);
                const int rf = full_rows(m);
                for (int h = 0; h < 2; ++h) {
                    const int row0 = h == 0 ? 0 : rf, M = h == 0 ? rf : rows_m[m] - rf, N = h == 0 ? 2 * Th : Th;
                    if (M <= 0) continue;
                    tc::Problem P{};
                    P.amap = m;
                    P.z = w;
                    P.bmap = m;
                    P.row0 = row0;
                    P.kblocks = (nord[w] + tc_bk - 1) / tc_bk;
                    P.M = M;
                    P.N = N;
                    P.tiles_n = (N + tc::BN - 1) / tc::BN;
                    P.C = Cmix.p + (size_t)w * c_total() + c_off(m) + (c_rowmajor ? (size_t)row0 * c_ld : row0);
                    P.sa = sA[m].p + (size_t)w * rows_m[m] + row0;
                    P.sb = sB[m].p;
                    P.ldc = c_rowmajor ? c_ld : rows_m[m];
                    P.rowmajor = c_rowmajor ? 1 : 0;
                    P.lz = lnzA[m].p + (size_t)w * rows_m[m] + row0;
                    P.kb = tcKb.p + kboff;
                    kboff += (size_t)(M + tc::BM - 1) / tc::BM;
                    hp.push_back(P);
                    // algorithmic: one real product per (row, column, order) up to
                    // the cutoff (the tensor cores run three piece products on
                    // orders padded to BK)
                    G.flops += 2.0 * P.M * (double)N * (double)nord[w];
                    G.bytes += 4.0 * ((double)P.M + N) * (double)P.kblocks * tc_bk + 4.0 * (double)P.M * N;
                }
            }
        // longest contractions first: a CTA takes tiles t, t + grid, ... in
        // list order, so the heavy tiles spread over the CTAs and the light
        // ones fill in at the end (instead of the top frequencies' tiles
        // trailing the launch)
        std::stable_sort(hp.begin(), hp.end(),
                         [](const tc::Problem& a, const tc::Problem& b) { return a.kblocks > b.kblocks; });
        for (size_t k = 0; k < hp.size(); k += tc::MAXP) {
            const int np = (int)std::min<size_t>(tc::MAXP, hp.size() - k);
            int tiles = 0;
            for (int i = 0; i < np; ++i) {
                hp[k + i].tile0 = tiles;
                tiles += ((hp[k + i].M + tc::BM - 1) / tc::BM) * hp[k + i].tiles_n;
            }
            G.launches.push_back({tcp_next + all.size(), np, tiles});
            all.insert(all.end(), hp.begin() + k, hp.begin() + k + np);
        }
        tc_groups.push_back(std::move(G));
    }
    tc_plan = all;
    tc_kbn = kboff;
    if (tcp_next + all.size() > tcp.n) throw Error(DSM_ERR_INVALID, "contraction list exceeds its buffer");
    // each source's lists take their own slots of tcp, so no copy overwrites
    // a list an earlier launch may still read
    if (!all.empty())
        DSM_CUDA(cudaMemcpyAsync(tcp.p + tcp_next, all.data(), sizeof(tc::Problem) * all.size(),
                                 cudaMemcpyHostToDevice, st));
    tcp_next += all.size();
}

// Flops the last plan's contraction executed: each row tile runs its own
// order blocks (tile_orders); read back when profiling, after the batch.
void Engine::count_exec_flops() {
    if (!prof || tc_plan.empty() || tc_kbn == 0) return;
    std::vector<int> kb(tc_kbn);
    DSM_CUDA(cudaMemcpy(kb.data(), tcKb.p, sizeof(int) * tc_kbn, cudaMemcpyDeviceToHost));
    for (const tc::Problem& P : tc_plan) {
        const size_t off = (size_t)(P.kb - tcKb.p);
        for (int mt = 0; mt * tc::BM < P.M; ++mt) {
            const int rows = std::min(tc::BM, P.M - mt * tc::BM);
            stats.lsum_flops_exec += 2.0 * rows * (double)P.N * (double)std::min(kb[off + mt], P.kblocks) * tc_bk;
        }
    }
}

// Split of group g of the mixed l-sum (field pieces, row scales, each row
// tile's order blocks) on stt.
void Engine::lsum_split(int g) {
    const TcGroup& G = tc_groups[(size_t)g];
    if (G.slots.empty()) return;
    int id = kid("lsum_split");
    kbegin(id, stt);
    // zero orders recorded by the field kernels of this batch (the cut on)
    const bool zf_ok = use_zfirst && depth_bound > 0.0 && afld_bytes == 4;
    // one split launch per |m| and run of consecutive slots
    std::vector<int> sl = G.slots;
    std::sort(sl.begin(), sl.end());
    for (size_t i = 0; i < sl.size();) {
        size_t j = i + 1;
        while (j < sl.size() && sl[j] == sl[j - 1] + 1) ++j;
        const int w0 = sl[i], n = (int)(j - i);
        for (int m = m_lo; m <= 2; ++m) {
            if (!rows_m[m]) continue;
            const size_t rw = (size_t)rows_m[m];
            const char* A =
                reinterpret_cast<const char*>(Afld[m].p) + ((size_t)src * F + w0) * rw * Lcap * afld_bytes;
            tc::split_fields(A, afld_bytes, n, rows_m[m], Lcap, d_nord.p + w0, Apc[m].p + (size_t)w0 * rw * kcA,
                             sA[m].p + (size_t)w0 * rw, kcA, F, tc_fmt, tc_bk, stt, lnzA[m].p + (size_t)w0 * rw,
                             zf_ok ? zfirst.p + ((size_t)src * F + w0) * (R + 1) : nullptr, rowrec[m].p, R + 1);
            launches++;
        }
        i = j;
    }
    // each row tile's order blocks from its rows' last nonzero orders
    for (const TcLaunch& L : G.launches) {
        tc::tile_orders(tcp.p + L.first, L.np, tc_bk, stt);
        launches++;
    }
    kend(id, G.split_bytes, 0.0, stt);
}

// Tensor-core contraction launches of group g on stt.
void Engine::lsum_contract(int g) {
    const TcGroup& G = tc_groups[(size_t)g];
    if (G.slots.empty()) return;
    const int id = kid("lsum_tc");
    kbegin(id, stt);
    const uint32_t fl = tc_flags | (test_tc_stall ? tc::TC_TEST_STALL : 0u);
    const unsigned long long wait_ns = test_tc_stall ? 20000000ull : tc::WAIT_NS;
    for (const TcLaunch& L : G.launches) {
        tc::launch(tcmaps, tcp.p + L.first, L.np, L.tiles, tc_fmt, tc_bk, fl, tc_chunk, tc_err(), nsm, stt, wait_ns);
        launches++;
    }
    kend(id, G.bytes, G.flops, stt);
}

// Reads the run's status words (the stream is synchronised here anyway);
// a set word is cleared and reported, leaving the context usable.
void Engine::check_device_flags() {
    int h[2] = {0, 0};
    DSM_CUDA(cudaMemcpyAsync(h, dflags.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    DSM_CUDA(cudaStreamSynchronize(st));
    if (h[DEV_WORD_TC] || h[DEV_WORD_STATUS]) {
        DSM_CUDA(cudaMemsetAsync(dflags.p, 0, sizeof(h), st));
        DSM_CUDA(cudaStreamSynchronize(st));
    }
    if (h[DEV_WORD_TC]) throw Error(DSM_ERR_TIMEOUT, "a bounded wait in the tensor-core l-sum gave up");
    if (h[DEV_WORD_STATUS] & DEV_NONFINITE)
        throw Error(DSM_ERR_NONFINITE, "an output (TSGT, RSGT or SYNN) became Inf or NaN");
}

// sums[c][0] += |a - b|^2, sums[c][1] += |b|^2 over npt points of num
// complex components (component fastest); a thread takes whole points
__global__ void __launch_bounds__(256) k_cmp_sums(const double2* __restrict__ a, const double2* __restrict__ b,
                                                  size_t npt, int num, double* __restrict__ sums) {
    constexpr int NMAX = DSM_PSV_NUM_TSGT;
    double dd[NMAX], rr[NMAX];
#pragma unroll
    for (int c = 0; c < NMAX; ++c) dd[c] = rr[c] = 0.0;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npt; p += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < NMAX; ++c) {
            if (c < num) {
                const double2 x = a[p * num + c], y = b[p * num + c];
                const double ex = x.x - y.x, ey = x.y - y.y;
                dd[c] += ex * ex + ey * ey;
                rr[c] += y.x * y.x + y.y * y.y;
            }
        }
    }
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < NMAX; ++c) {
        if (c >= num) break;
        double u = dd[c], v = rr[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            u += __shfl_down_sync(0xffffffffu, u, o);
            v += __shfl_down_sync(0xffffffffu, v, o);
        }
        if (lane == 0) {
            atomicAdd(&sums[2 * c], u);
            atomicAdd(&sums[2 * c + 1], v);
        }
    }
}

static void launch_cmp(const double* a, const double* b, size_t npt, int num, double* sums, int nsm,
                       cudaStream_t st) {
    if (npt == 0 || num <= 0) return;
    const unsigned grid = (unsigned)std::min<size_t>((npt + 255) / 256, (size_t)nsm * 4);
    k_cmp_sums<<<grid, 256, 0, st>>>(reinterpret_cast<const double2*>(a), reinterpret_cast<const double2*>(b),
                                     npt, num, sums);
    DSM_CUDA(cudaGetLastError());
}

void Engine::check_batch(const int* ilist, int b0, int nf, const std::vector<CutState>& hc) {
    if (!check_ref || check_stride <= 0) return;
    std::vector<int> sub, pos;
    for (int w = 0; w < nf; ++w)
        if ((b0 + w) % check_stride == 0) {
            sub.push_back(ilist[b0 + w]);
            pos.push_back(w);
        }
    if (sub.empty()) return;
    DSM_CUDA(cudaEventRecord(ev[6], st));
    size_t pt, pr, ps;
    out_sizes(&pt, &pr, &ps);
    double* sums = acc_sums.p;
    for (size_t k0 = 0; k0 < sub.size(); k0 += (size_t)check_ref->F) {
        const int m = (int)std::min<size_t>((size_t)check_ref->F, sub.size() - k0);
        const void *rt = nullptr, *rr = nullptr, *rs = nullptr;
        std::vector<int> ll(m);
        // the FP64 engine synchronises its own stream before it returns
        check_ref->run(sub.data() + k0, m, nullptr, &rt, &rr, &rs, ll.data());
        for (int k = 0; k < m; ++k) {
            const int w = pos[k0 + k];
            if (ll[k] != hc[w].llog) acc.llog_equal = 0;
            launch_cmp(out_t.p + 2 * pt * w, static_cast<const double*>(rt) + 2 * pt * k, pt / num_t, num_t, sums,
                       nsm, st);
            if (rsgt_sw)
                launch_cmp(out_r.p + 2 * pr * w, static_cast<const double*>(rr) + 2 * pr * k, pr / num_r, num_r,
                           sums + 2 * num_t, nsm, st);
            if (synn_sw)
                launch_cmp(out_s.p + 2 * ps * w, static_cast<const double*>(rs) + 2 * ps * k, ps / num_s, num_s,
                           sums + 2 * (num_t + num_r), nsm, st);
        }
        // the FP64 engine's next run reuses the buffers just read
        DSM_CUDA(cudaStreamSynchronize(st));
    }
    acc.nfreq += (int)sub.size();
    DSM_CUDA(cudaEventRecord(ev[7], st));
    DSM_CUDA(cudaEventSynchronize(ev[7]));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[6], ev[7]);
    ms_check += ms;
}

void Engine::finish_accuracy() {
    if (!check_ref || check_stride <= 0 || acc.nfreq == 0) return;
    const int ntot = num_t + num_r + num_s;
    std::vector<double> h(2 * (size_t)ntot);
    DSM_CUDA(cudaMemcpy(h.data(), acc_sums.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    auto kind = [&](int off, int num, double* out, double* mx) {
        double tot = 0.0;
        for (int c = 0; c < num; ++c) tot += h[2 * (off + c) + 1];
        *mx = 0.0;
        for (int c = 0; c < num; ++c) {
            const double d = h[2 * (off + c)], r = h[2 * (off + c) + 1];
            const double den = r >= 1e-20 * tot ? r : tot;  // (1e-10 of the norm)^2
            out[c] = den > 0.0 ? std::sqrt(d / den) : std::sqrt(d);
            *mx = std::max(*mx, out[c]);
        }
    };
    kind(0, num_t, acc.tsgt, &acc.tsgt_max);
    if (rsgt_sw) kind(num_t, num_r, acc.rsgt, &acc.rsgt_max);
    if (synn_sw) kind(num_t + num_r, num_s, acc.synn, &acc.synn_max);
}

void Engine::build_weights(const double* d_r, const double* d_rrsta) {
    launch_interp_weights(*this, d_r, d_rrsta);
}

// C[mi] (rows x 2Th, column-major) = A^T (A stored [row][l], ld Lcap) x
// B (stored [col][l], ld lcapB), summed over the K orders of frequency w.
// The leading full_rows(mi) rows take all 2 Th columns, the rest the first Th.
void Engine::gemm_fp64(int w, int mi, int K) {
    const int M = rows_m[mi], rf = full_rows(mi);
    if (M == 0) return;
    if (afld_bytes != 8) throw Error(DSM_ERR_INVALID, "FP64 l-sum of FP32 field matrices");
    const double one = 1.0, zero = 0.0;
    const double* A = Afld[mi].p + ((size_t)src * F + w) * M * Lcap;
    int id = kid("lsum_dgemm");
    kbegin(id);
    double bytes = 0.0, flops = 0.0;
    for (int g = 0; g < 2; ++g) {
        const int row0 = g == 0 ? 0 : rf, Mg = g == 0 ? rf : M - rf, N = g == 0 ? 2 * Th : Th;
        if (Mg <= 0) continue;
        if (c_rowmajor)  // C^T (N x Mg, column-major, ld c_ld) = B^T-view x A-view
            DSM_CUBLAS(cublasDgemm(cub, CUBLAS_OP_T, CUBLAS_OP_N, N, Mg, K, &one, basis[mi].p, lcapB,
                                   A + (size_t)row0 * Lcap, Lcap, &zero, Cgemm.p + c_off(mi) + (size_t)row0 * c_ld,
                                   c_ld));
        else
            DSM_CUBLAS(cublasDgemm(cub, CUBLAS_OP_T, CUBLAS_OP_N, Mg, N, K, &one, A + (size_t)row0 * Lcap, Lcap,
                                   basis[mi].p, lcapB, &zero, Cgemm.p + c_off(mi) + row0, M));
        bytes += 8.0 * ((double)Mg * K + (double)K * N + (double)Mg * N);
        flops += 2.0 * Mg * N * (double)K;
        launches++;
    }
    kend(id, bytes, flops);
}

// Grows the order capacity of the field matrices and of the probe table,
// keeping the columns already written (the cutoff of a frequency is not
// known before its orders are solved; the reference allows up to maxlmax).
void Engine::grow_orders(int need) {
    if (need <= Lcap) return;
    join_side();  // side-stream work may still write the old field buffers
    int cap = Lcap;
    while (cap < need) cap *= 2;
    cap = std::min(cap, maxlmax + 1 + Lc);
    if (cap < need) cap = need;
    for (int m = m_lo; m <= 2; ++m) {
        size_t h = (size_t)nsrc * F * rows_m[m];
        if (h == 0) continue;
        const size_t eb = (size_t)afld_bytes, bytes = (h * cap * eb + 7) / 8 * 8;
        double* np_ = nullptr;
        if (cudaMalloc(&np_, bytes) != cudaSuccess)
            throw Error(DSM_ERR_NOMEM, "cannot grow the field matrices to " + std::to_string(cap) + " orders");
        DSM_CUDA(cudaMemcpy2DAsync(np_, (size_t)cap * eb, Afld[m].p, (size_t)Lcap * eb, (size_t)Lcap * eb, h,
                                   cudaMemcpyDeviceToDevice, st));
        DSM_CUDA(cudaStreamSynchronize(st));
        Afld[m].release();
        Afld[m].p = np_;
        Afld[m].n = bytes / 8;
    }
    double* na = nullptr;
    if (cudaMalloc(&na, (size_t)nsrc * F * cap * amp_k * sizeof(double)) != cudaSuccess)
        throw Error(DSM_ERR_NOMEM, "cannot grow the probe table");
    DSM_CUDA(cudaMemcpy2DAsync(na, (size_t)cap * amp_k * sizeof(double), amps.p,
                               (size_t)Lcap * amp_k * sizeof(double), (size_t)Lcap * amp_k * sizeof(double),
                               (size_t)nsrc * F, cudaMemcpyDeviceToDevice, st));
    DSM_CUDA(cudaStreamSynchronize(st));
    amps.release();
    amps.p = na;
    amps.n = (size_t)nsrc * F * cap * amp_k;
    Lcap = cap;
}

// First order range of a frequency: past lsuf (callsuf), at least 512
// (or the fixed chunk the options ask for).
void Engine::set_summaries(int is_psv, int nzone, const double* vrmin, const double* vrmax, const double* vsv,
                           const double* qmu, double r0, double rrcv) {
    const double rmax = vrmax[nzone - 1];
    auto vs_at = [&](int z, double r) {
        const double x = r / rmax;
        return vsv[4 * z] + vsv[4 * z + 1] * x + vsv[4 * z + 2] * x * x + vsv[4 * z + 3] * x * x * x;
    };
    int zs = nzone - 1;
    for (int z = 0; z < nzone; ++z)
        if (r0 >= vrmin[z] && r0 <= vrmax[z]) { zs = z; break; }
    double vmin = 1e30, vmax = 0.0;
    for (int z = 0; z < nzone; ++z) {
        const double v = vs_at(z, 0.5 * (vrmin[z] + vrmax[z]));
        if (v <= 0.0) continue;  // fluid zone
        vmin = std::min(vmin, v);
        vmax = std::max(vmax, v);
    }
    if (vmax == 0.0) vmin = 0.0;
    summ[0] = (float)(r0 / rmax);
    summ[1] = (float)(rrcv / rmax);
    summ[2] = (float)(vtop_ / 10.0);
    summ[3] = (float)(vs_at(zs, r0) / 10.0);
    summ[4] = (float)(vmin / 10.0);
    summ[5] = (float)(vmax / 10.0);
    summ[6] = (float)((rmax - r0) / 1000.0);
    summ[7] = (float)((vrmax[nzone - 1] - vrmin[nzone - 1]) / 100.0);
    summ[8] = (float)is_psv;
    summ[9] = (float)(std::log10(std::max(1.0, std::fabs(qmu[zs]))) / 3.0);
}

void Engine::lmax_features(const int* ilist, int n, float* out) const {
    for (int k = 0; k < n; ++k) {
        const double omega = 2.0 * kPi * (double)ilist[k] / tlen;
        float* f = out + (size_t)k * DSM_LMAX_NFEAT;
        f[0] = (float)std::log1p(omega * rtop_ / vtop_);
        for (int i = 0; i < 10; ++i) f[1 + i] = summ[i];
    }
}

int Engine::first_span(int ifreq) const {
    if (opt.l_chunk > 0) return ((opt.l_chunk + 31) / 32) * 32;
    double omega = 2.0 * kPi * (double)ifreq / tlen;
    int lsuf = (int)(omega * rtop_ / vtop_ - 0.5) + 1;
    int s = std::max(512, lsuf + 64);
    return ((s + 31) / 32) * 32;
}

void Engine::run(const int* ilist, int n, dsm_out_t* ho, const void** dt, const void** dr,
                 const void** ds, int* llog_out) {
    if (n <= 0) throw Error(DSM_ERR_INVALID, "empty frequency list");
    for (int k = 0; k < n; ++k)
        if (ilist[k] <= 0) throw Error(DSM_ERR_INVALID, "frequency index must be > 0 (i = 0 is never computed)");
    if (dt && n > F) throw Error(DSM_ERR_INVALID, "device outputs hold at most one batch of frequencies");
    std::memset(&stats, 0, sizeof(stats));
    launches = 0;
    rounds = 0;
    recs.clear();
    // the test hook applies to this run only
    struct StallOnce {
        int& v;
        ~StallOnce() { v = 0; }
    } stall_once{test_tc_stall};
    DSM_CUDA(cudaMemsetAsync(dflags.p, 0, 2 * sizeof(int), st));
    std::memset(&acc, 0, sizeof(acc));
    acc.llog_equal = 1;
    ms_check = 0.0;
    if (check_ref && check_stride > 0) {
        acc_sums.reserve(2 * (size_t)(num_t + num_r + num_s));
        DSM_CUDA(cudaMemsetAsync(acc_sums.p, 0, acc_sums.n * sizeof(double), st));
    }
    cudaEvent_t e0 = ev[0], e1 = ev[1], es0 = ev[2], es1 = ev[3], eg0 = ev[4], eg1 = ev[5];
    DSM_CUDA(cudaEventRecord(e0, st));
    float ms_solve = 0, ms_lsum = 0;
    size_t pt, pr, ps;
    out_sizes(&pt, &pr, &ps);
    for (int b0 = 0; b0 < n; b0 += F) {
        int nf = std::min(F, n - b0);
        d_freqs.upload(ilist + b0, nf, st);
        // --- 1+2: per-omega pieces and chunked solves with the cutoff scan
        DSM_CUDA(cudaEventRecord(es0, st));
        omega_pieces(d_freqs.p, nf);
        // cutoff state of (source s, frequency w) at s F + w
        const size_t ncut = (size_t)nsrc * F;
        {
            std::vector<CutState> init(ncut);
            for (auto& c : init) { c.ismall = 0; c.done = 0; c.llog = maxlmax; c.norders = 0; c.maxamp = -1.0; }
            cut.upload(init, st);
        }
        std::vector<CutState> hcs(ncut);
        for (auto& c : hcs) c.done = 0;
        // a frequency is done when every source has met its cutoff
        std::vector<CutState> hc(nf);
        for (auto& c : hc) c.done = 0;
        auto all_sources_done = [&](int w) {
            for (int s = 0; s < nsrc; ++s)
                if (!hcs[(size_t)s * F + w].done) return 0;
            return 1;
        };
        // Rounds of ragged order ranges: every unfinished frequency continues
        // from where it stopped.  The first range of a frequency reaches past
        // lsuf (the cutoff is never below it); later ranges grow by half.
        std::vector<int> next(nf, 0), span(nf, 0);
        std::vector<int> hf(ilist + b0, ilist + b0 + nf);
        // first ranges: the lsuf rule scaled by what the context's earlier
        // batches needed (span_hint, 1 while the rule covers the cutoffs)
        std::vector<int> span_rule(nf);
        for (int w = 0; w < nf; ++w) {
            span_rule[w] = first_span(hf[w]);
            const double sp = std::min((double)maxlmax + 1.0, std::ceil(span_rule[w] * span_hint));
            span[w] = opt.l_chunk > 0 ? span_rule[w] : std::max(span_rule[w], ((int)sp + 31) / 32 * 32);
        }
        if (opt.use_lmax_predictor && pred.ready && opt.l_chunk <= 0) {
            // the network predicts log(lmax) - f0, f0 = log(1 + omega rtop /
            // vtop) (the lsuf scale); first range = lmax * 1.02 + 24, never
            // below lsuf + 8 (the amplitude test cannot stop before lsuf)
            std::vector<float> f((size_t)nf * DSM_LMAX_NFEAT), lp(nf);
            lmax_features(hf.data(), nf, f.data());
            pred.predict(f.data(), nf, lp.data(), st);
            for (int w = 0; w < nf; ++w) {
                const double omega = 2.0 * kPi * (double)hf[w] / tlen;
                const int lsuf = (int)(omega * rtop_ / vtop_ - 0.5) + 1;
                const double pl = std::exp((double)lp[w] + (double)f[(size_t)w * DSM_LMAX_NFEAT]);
                int sp = (int)std::ceil(std::min(pl * 1.02 + 24.0, (double)maxlmax + 1.0));
                sp = std::max(sp, lsuf + 8);
                span[w] = (sp + 31) / 32 * 32;
            }
        }
        const std::vector<int> span0 = span;  // first order range of each frequency
        // goal[w]: end of the order range a frequency has asked for so far.
        // A round that cannot hold every open range shares its capacity
        // evenly (water-filling, multiples of 32 orders) from each
        // frequency's lowest open order, so the long low-order systems of
        // all frequencies share a launch and later launches hold the short
        // high-order ones (a solve launch lasts as long as its longest
        // system's recurrence).
        std::vector<int> goal(nf);
        for (int w = 0; w < nf; ++w) goal[w] = std::min(maxlmax + 1, span[w]);
        int maxend = 0;
        for (;;) {
            std::vector<int> off(nf + 1, 0), lb(nf, 0), need(nf, 0);
            long long want = 0;
            for (int w = 0; w < nf; ++w) {
                if (!hc[w].done && next[w] <= maxlmax) need[w] = std::max(0, goal[w] - next[w]);
                want += need[w];
            }
            int share = INT32_MAX;  // every open range fits
            if (want > nsys_max) {
                std::vector<int> sorted;
                for (int w = 0; w < nf; ++w)
                    if (need[w] > 0) sorted.push_back(need[w]);
                std::sort(sorted.begin(), sorted.end());
                long long cap = nsys_max;
                int left = (int)sorted.size();
                for (int v : sorted) {
                    if ((long long)v * left > cap) break;
                    cap -= v;
                    --left;
                }
                share = left > 0 ? std::max(32, (int)(cap / left) / 32 * 32) : INT32_MAX;
            }
            int tot = 0;
            for (int w = 0; w < nf; ++w) {
                lb[w] = next[w];
                const int cnt = std::max(0, std::min({need[w], share, nsys_max - tot}));
                off[w] = tot;
                tot += cnt;
                next[w] += cnt;
                maxend = std::max(maxend, next[w]);
            }
            off[nf] = tot;
            if (tot == 0) break;
            if (maxend > Lcap) grow_orders(maxend);
            wl_off.upload(off, st);
            wl_host_off = off;
            wl_lb.upload(lb, st);
            WorkList wl{wl_off.p, wl_lb.p, nf};
            solve_chunk(d_freqs.p, nf, wl, tot);
            scan_chunk(nf, wl);
            stats.systems += tot;
            rounds++;
            DSM_CUDA(cudaMemcpyAsync(hcs.data(), cut.p, sizeof(CutState) * ncut, cudaMemcpyDeviceToHost, st));
            int hstat = 0;
            DSM_CUDA(cudaMemcpyAsync(&hstat, dstatus(), sizeof(int), cudaMemcpyDeviceToHost, st));
            DSM_CUDA(cudaStreamSynchronize(st));
            if (hstat & DEV_NONFINITE) {  // a cutoff probe is Inf/NaN: the solves broke down
                join_side();
                DSM_CUDA(cudaMemsetAsync(dflags.p, 0, 2 * sizeof(int), st));
                DSM_CUDA(cudaStreamSynchronize(st));
                int bad = hf[0];
                for (size_t k = 0; k < ncut; ++k)
                    if ((int)(k % F) < nf && hcs[k].llog < 0) { bad = hf[k % F]; break; }
                throw Error(DSM_ERR_NONFINITE, "a pivot of the banded solve or the cutoff probe became Inf or NaN "
                                               "(frequency index " + std::to_string(bad) + ")");
            }
            bool all = true;
            for (int w = 0; w < nf; ++w) {
                hc[w].done = all_sources_done(w);
                if (!hc[w].done && next[w] > maxlmax) { hc[w].done = 1; }
                all = all && hc[w].done;
                if (!hc[w].done && next[w] >= goal[w]) {  // its range is solved: the next one grows by half
                    if (opt.l_chunk <= 0) span[w] = std::min(4096, span[w] + span[w] / 2);
                    goal[w] = std::min(maxlmax + 1, next[w] + span[w]);
                }
            }
            if (all) break;
        }
        double need_ratio = 1.0;  // cutoff (+ a step group) over the lsuf rule, largest of the batch
        for (int s = 0; s < nsrc; ++s)
            for (int w = 0; w < nf; ++w) {
                CutState& c = hcs[(size_t)s * F + w];
                if (c.norders == 0) { c.norders = maxlmax + 1; c.llog = maxlmax; }
                stats.orders_padded += (long long)next[w] - c.norders;
                stats.freqs_extended += c.norders > span0[w] ? 1 : 0;
                need_ratio = std::max(need_ratio, (c.norders + 32.0) / span_rule[w]);
            }
        // the next batch's first ranges cover what this one needed (the
        // amplitude test still decides every cutoff; only the work split moves)
        if (!(opt.use_lmax_predictor && pred.ready)) span_hint = std::min(4.0, need_ratio);
        // source 0's states stand for the batch where one set is reported
        for (int w = 0; w < nf; ++w) hc[w] = hcs[w];
        join_side();
        DSM_CUDA(cudaEventRecord(es1, st));
        if (cutoffs_only) {  // the realised cutoffs (of source 0) are all that was asked for
            for (int w = 0; w < nf; ++w) {
                if (llog_out) llog_out[b0 + w] = hc[w].llog;
                stats.orders_used += hc[w].norders;
            }
            DSM_CUDA(cudaStreamSynchronize(st));
            kcollect();
            float a = 0;
            cudaEventElapsedTime(&a, es0, es1);
            ms_solve += a;
            continue;
        }
        // --- 3+4: contraction and epilogue per frequency, source by source
        int lneed = 1;
        for (auto& c : hcs) lneed = std::max(lneed, c.norders);
        {
            int id = kid("basis_tables");
            kbegin(id);
            build_basis(lneed);
            kend(id, 0.0, 0.0);
        }
        DSM_CUDA(cudaEventRecord(eg0, st));
        const bool rec32 = ho && (ho->tsgt32 || ho->rsgt32 || ho->synn32);
        for (src = 0; src < nsrc; ++src) {
            const CutState* hs = hcs.data() + (size_t)src * F;
            dsm_out_t* hos = ho ? ho + src : nullptr;
            std::vector<int> nord(nf);
            for (int w = 0; w < nf; ++w) nord[w] = hs[w].norders;
            if (mixed()) lsum_prepare(nf, nord);
            // complex64 records for the host leave per group of frequencies on
            // the copy stream while the next group's l-sum runs; the mixed
            // path groups its frequencies in any case (its pipeline below)
            const int ngrp = rec32 ? (nf >= 2 * MAX_OUT_GROUPS ? MAX_OUT_GROUPS : std::max(1, nf / 2))
                                   : (mixed() ? std::max(1, std::min({lsum_groups, nf, MAX_OUT_GROUPS})) : 1);
            if (rec32) out32.reserve(2 * (pt + pr + ps) * (size_t)nf);
            if (rec32 && src > 0) {  // this source's records reuse out32: the last source's copies first
                DSM_CUDA(cudaEventRecord(ev_grp[0], stc));
                DSM_CUDA(cudaStreamWaitEvent(st, ev_grp[0], 0));
            }
            // Groups of batch slots.  Plain path: consecutive slots.  Mixed
            // path, in order on stt: the first group's split, contraction and
            // epilogue, then the other groups' splits and each group's
            // contraction and epilogue, so that the complex64 records of a
            // group go to the host (stc) while later groups are contracted.
            // (Kernels beside the contraction's CTAs made almost no progress,
            // so nothing runs beside it.)
            std::vector<std::vector<int>> groups(ngrp);
            if (mixed()) {
                // the lightest frequencies first (a fifth of the batch: their
                // records start the host copies early and keep the copy
                // engine busy while the other groups' splits and the next
                // contraction run), the others dealt by their cutoff,
                // heaviest first, in serpentine order
                std::vector<int> byw(nf);
                for (int w = 0; w < nf; ++w) byw[w] = w;
                std::stable_sort(byw.begin(), byw.end(), [&](int a, int b) { return nord[a] > nord[b]; });
                const int nfirst = ngrp > 1 ? std::max(1, std::min(nf / 5, nf - (ngrp - 1))) : 0;
                const int gfirst = ngrp > 1 ? 1 : 0, rest = ngrp - gfirst;
                for (int k = 0; k < nfirst; ++k) groups[0].push_back(byw[nf - 1 - k]);
                for (int k = 0; k < nf - nfirst; ++k) {
                    const int r = k / rest, c = k % rest;
                    groups[gfirst + ((r & 1) ? rest - 1 - c : c)].push_back(byw[k]);
                }
            } else {
                for (int g = 0; g < ngrp; ++g)
                    for (int w = g * nf / ngrp; w < (g + 1) * nf / ngrp; ++w) groups[g].push_back(w);
            }
            cudaStream_t se = st;
            if (mixed()) {
                lsum_plan(groups, nord);
                DSM_CUDA(cudaEventRecord(ev_lp, st));
                DSM_CUDA(cudaStreamWaitEvent(stt, ev_lp, 0));
                lsum_split(0);
                se = stt;
            }
            for (int g = 0; g < ngrp; ++g) {
                // the other groups' splits once the first group's records are on their way
                if (mixed() && g == 1)
                    for (int h = 1; h < ngrp; ++h) lsum_split(h);
                if (mixed()) lsum_contract(g);
                for (int w : groups[g]) {
                    stats.orders_used += hs[w].norders;
                    if (!mixed())
                        for (int mi = m_lo; mi <= 2; ++mi) gemm_fp64(w, mi, hs[w].norders);
                    epilogue(d_freqs.p, w, nf, se);
                    for (int mi = m_lo; mi <= 2; ++mi)
                        stats.lsum_flops +=
                            2.0 * (2.0 * full_rows(mi) + (rows_m[mi] - full_rows(mi))) * Th * hs[w].norders;
                }
                if (rec32) {  // per run of consecutive slots of the group
                    std::vector<int> sl = groups[g];
                    std::sort(sl.begin(), sl.end());
                    std::vector<std::pair<int, int>> runs;
                    for (size_t i = 0; i < sl.size();) {
                        size_t j = i + 1;
                        while (j < sl.size() && sl[j] == sl[j - 1] + 1) ++j;
                        runs.push_back({sl[i], sl[j - 1] + 1});
                        i = j;
                    }
                    for (const auto& r : runs) launch_pack32(*this, nf, r.first, r.second, pt, pr, ps, se);
                    DSM_CUDA(cudaEventRecord(ev_grp[g], se));
                    DSM_CUDA(cudaStreamWaitEvent(stc, ev_grp[g], 0));
                    const float* o = out32.p;
                    for (const auto& r : runs) {
                        const int w0 = r.first;
                        const size_t n = (size_t)(r.second - r.first);
                        if (hos->tsgt32)
                            DSM_CUDA(cudaMemcpyAsync(hos->tsgt32 + 2 * pt * (b0 + w0), o + 2 * pt * w0, 8 * pt * n,
                                                     cudaMemcpyDeviceToHost, stc));
                        if (hos->rsgt32 && rsgt_sw)
                            DSM_CUDA(cudaMemcpyAsync(hos->rsgt32 + 2 * pr * (b0 + w0),
                                                     o + 2 * pt * nf + 2 * pr * w0, 8 * pr * n,
                                                     cudaMemcpyDeviceToHost, stc));
                        if (hos->synn32 && synn_sw)
                            DSM_CUDA(cudaMemcpyAsync(hos->synn32 + 2 * ps * (b0 + w0),
                                                     o + 2 * (pt + pr) * nf + 2 * ps * w0, 8 * ps * n,
                                                     cudaMemcpyDeviceToHost, stc));
                    }
                }
            }
            if (mixed()) {  // st continues after the last group's epilogue
                DSM_CUDA(cudaEventRecord(ev_lj, stt));
                DSM_CUDA(cudaStreamWaitEvent(st, ev_lj, 0));
                if (prof) {  // executed flops (row-tile order counts) before the next source reuses them
                    DSM_CUDA(cudaStreamSynchronize(stt));
                    count_exec_flops();
                }
            }
            // --- 5: outputs
            if (llog_out && src == 0)
                for (int w = 0; w < nf; ++w) llog_out[b0 + w] = hs[w].llog;
            if (hos) {
                if (hos->llog)
                    for (int w = 0; w < nf; ++w) hos->llog[b0 + w] = hs[w].llog;
                if (hos->tsgt)
                    DSM_CUDA(cudaMemcpyAsync(hos->tsgt + 2 * pt * b0, out_t_src(), 16 * pt * nf,
                                             cudaMemcpyDeviceToHost, st));
                if (hos->rsgt && rsgt_sw)
                    DSM_CUDA(cudaMemcpyAsync(hos->rsgt + 2 * pr * b0, out_r_src(), 16 * pr * nf,
                                             cudaMemcpyDeviceToHost, st));
                if (hos->synn && synn_sw)
                    DSM_CUDA(cudaMemcpyAsync(hos->synn + 2 * ps * b0, out_s_src(), 16 * ps * nf,
                                             cudaMemcpyDeviceToHost, st));
            }
        }
        src = 0;
        DSM_CUDA(cudaEventRecord(eg1, st));
        // the next batch overwrites out32 and the outputs: its records wait
        // for this batch's copies
        if (rec32) {
            DSM_CUDA(cudaEventRecord(ev_grp[0], stc));
            DSM_CUDA(cudaStreamWaitEvent(st, ev_grp[0], 0));
        }
        DSM_CUDA(cudaStreamSynchronize(st));
        check_device_flags();
        kcollect();
        if (nsrc == 1) check_batch(ilist, b0, nf, hc);
        float a = 0, g = 0;
        cudaEventElapsedTime(&a, es0, es1);
        cudaEventElapsedTime(&g, eg0, eg1);
        ms_solve += a;
        ms_lsum += g;
    }
    if (dt) *dt = out_t.p;
    if (dr) *dr = out_r.p;
    if (ds) *ds = out_s.p;
    DSM_CUDA(cudaEventRecord(e1, st));
    DSM_CUDA(cudaEventSynchronize(e1));
    float tot = 0;
    cudaEventElapsedTime(&tot, e0, e1);
    finish_accuracy();
    stats.ms_total = tot - ms_check;
    stats.solve_rounds = rounds;
    stats.ms_solve = ms_solve;
    stats.ms_lsum = ms_lsum;
    stats.launches = launches;
}

}  // namespace dsm

// ------------------------------------------------------------------ C-ABI
using dsm::Error;

namespace {
thread_local std::string g_create_err;
}  // namespace

namespace dsm {
// error text of context-free entry points, read back by dsm_last_error(NULL)
void set_global_error(const std::string& e) { g_create_err = e; }
}  // namespace dsm

namespace {

template <class F>
int guarded(dsm_ctx_t* ctx, F f) {
    try {
        f();
        return DSM_OK;
    } catch (const Error& e) {
        if (ctx) ctx->err = e.what();
        else g_create_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (ctx) ctx->err = e.what();
        else g_create_err = e.what();
        return DSM_ERR_INVALID;
    }
}
}  // namespace

extern "C" int dsm_abi_version(void) { return DSM_ABI_VERSION; }

extern "C" const char* dsm_strerror(int code) {
    switch (code) {
        case DSM_OK: return "ok";
        case DSM_ERR_INVALID: return "invalid argument";
        case DSM_ERR_CUDA: return "CUDA error";
        case DSM_ERR_NONFINITE: return "non-finite value";
        case DSM_ERR_LMAX: return "angular-order cutoff beyond the allowed maximum";
        case DSM_ERR_TIMEOUT: return "device wait timed out";
        case DSM_ERR_NOMEM: return "out of memory";
        case DSM_ERR_NODEVICE: return "no usable CUDA device";
        default: return "unknown error";
    }
}

extern "C" const char* dsm_last_error(const dsm_ctx_t* ctx) {
    return ctx ? ctx->err.c_str() : g_create_err.c_str();
}

static int check_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= dev || dev < 0) {
        g_create_err = "no CUDA device (or the requested ordinal is out of range)";
        return DSM_ERR_NODEVICE;
    }
    cudaDeviceProp p{};
    cudaGetDeviceProperties(&p, dev);
    if (p.major < 10) {
        g_create_err = "the engine is built for sm_100a (B200); device compute capability is too low";
        return DSM_ERR_NODEVICE;
    }
    return DSM_OK;
}

extern "C" int dsm_sh_create(const dsm_sh_setup_t* s, const dsm_options_t* o, dsm_ctx_t** out) {
    if (!s || !out) { g_create_err = "null argument"; return DSM_ERR_INVALID; }
    *out = nullptr;
    dsm_options_t opt{};
    if (o) opt = *o;
    int rc = check_device(opt.device);
    if (rc) return rc;
    return guarded(nullptr, [&] {
        DSM_CUDA(cudaSetDevice(opt.device));
        auto* c = new dsm_ctx;
        try {
            c->eng.reset(dsm::make_sh_engine(s, &opt));
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

extern "C" int dsm_psv_create(const dsm_psv_setup_t* s, const dsm_options_t* o, dsm_ctx_t** out) {
    if (!s || !out) { g_create_err = "null argument"; return DSM_ERR_INVALID; }
    *out = nullptr;
    dsm_options_t opt{};
    if (o) opt = *o;
    int rc = check_device(opt.device);
    if (rc) return rc;
    return guarded(nullptr, [&] {
        DSM_CUDA(cudaSetDevice(opt.device));
        auto* c = new dsm_ctx;
        try {
            c->eng.reset(dsm::make_psv_engine(&s, 1, &opt));
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

extern "C" int dsm_psv_create_multi(const dsm_psv_setup_t* const* setups, int nsrc, const dsm_options_t* o,
                                    dsm_ctx_t** out) {
    if (!setups || nsrc < 1 || !out) { g_create_err = "null argument or no source"; return DSM_ERR_INVALID; }
    *out = nullptr;
    dsm_options_t opt{};
    if (o) opt = *o;
    int rc = check_device(opt.device);
    if (rc) return rc;
    return guarded(nullptr, [&] {
        DSM_CUDA(cudaSetDevice(opt.device));
        auto* c = new dsm_ctx;
        try {
            c->eng.reset(dsm::make_psv_engine(setups, nsrc, &opt));
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

extern "C" int dsm_run_freqs(dsm_ctx_t* ctx, const int* ilist, int n, dsm_out_t* out) {
    if (!ctx || !ilist || !out) return DSM_ERR_INVALID;
    if (ctx->eng->nsrc != 1) {
        ctx->err = "a context with several sources takes dsm_run_freqs_multi";
        return DSM_ERR_INVALID;
    }
    return guarded(ctx, [&] {
        DSM_CUDA(cudaSetDevice(ctx->eng->opt.device));
        ctx->eng->run(ilist, n, out, nullptr, nullptr, nullptr, nullptr);
    });
}

extern "C" int dsm_run_freqs_multi(dsm_ctx_t* ctx, const int* ilist, int n, dsm_out_t* outs, int nout) {
    if (!ctx || !ilist || !outs) return DSM_ERR_INVALID;
    if (nout != ctx->eng->nsrc) {
        ctx->err = "dsm_run_freqs_multi needs one output set per source of the context";
        return DSM_ERR_INVALID;
    }
    return guarded(ctx, [&] {
        DSM_CUDA(cudaSetDevice(ctx->eng->opt.device));
        ctx->eng->run(ilist, n, outs, nullptr, nullptr, nullptr, nullptr);
    });
}

extern "C" int dsm_run_request(dsm_ctx_t* const* ctxs, int nctx, const int* const* ilists, const int* ns,
                               dsm_out_t* const* outs, int* rcs) {
    if (!ctxs || nctx <= 0 || !ilists || !ns) return DSM_ERR_INVALID;
    if (rcs)
        for (int k = 0; k < nctx; ++k) rcs[k] = DSM_OK;
    auto reject = [&](int k, const char* why) {
        if (why) ctxs[k]->err = why;
        if (rcs) rcs[k] = DSM_ERR_INVALID;
        return DSM_ERR_INVALID;
    };
    for (int k = 0; k < nctx; ++k) {
        if (!ctxs[k]) return DSM_ERR_INVALID;
        if (!ilists[k] || ns[k] <= 0) return reject(k, "a request context without frequencies");
        for (int j = 0; j < k; ++j)
            if (ctxs[j] == ctxs[k]) return reject(k, "a context appears twice in one request");
        if (ctxs[k]->eng->opt.device != ctxs[0]->eng->opt.device)
            return reject(k, "the contexts of a request share one device");
    }
    std::vector<int> rc(nctx, DSM_OK);
    std::vector<std::thread> th;
    th.reserve(nctx);
    for (int k = 0; k < nctx; ++k)
        th.emplace_back([&, k] {
            dsm_ctx_t* c = ctxs[k];
            rc[k] = guarded(c, [&] {
                DSM_CUDA(cudaSetDevice(c->eng->opt.device));
                c->eng->run(ilists[k], ns[k], outs ? outs[k] : nullptr, nullptr, nullptr, nullptr, nullptr);
            });
        });
    for (auto& t : th) t.join();
    int first = DSM_OK;
    for (int k = 0; k < nctx; ++k) {
        if (rcs) rcs[k] = rc[k];
        if (first == DSM_OK) first = rc[k];
    }
    return first;
}

extern "C" int dsm_run_freqs_device(dsm_ctx_t* ctx, const int* ilist, int n, const void** d_tsgt,
                                    const void** d_rsgt, const void** d_synn, int* llog) {
    if (!ctx || !ilist) return DSM_ERR_INVALID;
    return guarded(ctx, [&] {
        DSM_CUDA(cudaSetDevice(ctx->eng->opt.device));
        ctx->eng->run(ilist, n, nullptr, d_tsgt, d_rsgt, d_synn, llog);
    });
}

extern "C" int dsm_lmax_features(const dsm_ctx_t* ctx, const int* ilist, int n, float* feats) {
    if (!ctx || !ilist || !feats || n <= 0) return DSM_ERR_INVALID;
    ctx->eng->lmax_features(ilist, n, feats);
    return DSM_OK;
}

extern "C" int dsm_cutoffs(dsm_ctx_t* ctx, const int* ilist, int n, int* llog) {
    if (!ctx || !ilist || !llog) return DSM_ERR_INVALID;
    return guarded(ctx, [&] {
        DSM_CUDA(cudaSetDevice(ctx->eng->opt.device));
        ctx->eng->cutoffs_only = true;
        try {
            ctx->eng->run(ilist, n, nullptr, nullptr, nullptr, nullptr, llog);
        } catch (...) {
            ctx->eng->cutoffs_only = false;
            throw;
        }
        ctx->eng->cutoffs_only = false;
    });
}

extern "C" int dsm_lmax_init(const float* feats, const float* target, int n, unsigned seed, float* params) {
    if (!feats || !target || !params || n <= 0) return DSM_ERR_INVALID;
    return guarded(nullptr, [&] { dsm::lmax::init_params(feats, target, n, seed, params); });
}

extern "C" int dsm_lmax_train(const float* feats, const float* target, int n, int epochs, int batch, float lr,
                              float weight_decay, unsigned seed, float* params, float* losses, int device) {
    if (!feats || !target || !params || n <= 0) return DSM_ERR_INVALID;
    int rc = check_device(device);
    if (rc) return rc;
    return guarded(nullptr, [&] {
        dsm::lmax::train(feats, target, n, epochs, batch, lr, weight_decay, seed, params, losses, device);
    });
}

extern "C" int dsm_lmax_grad(const float* params, const float* feats, const float* target, int n, float* grad,
                             float* loss, int device) {
    if (!feats || !target || !params || !grad || !loss || n <= 0) return DSM_ERR_INVALID;
    int rc = check_device(device);
    if (rc) return rc;
    return guarded(nullptr, [&] { dsm::lmax::grad(params, feats, target, n, grad, loss, device); });
}

extern "C" int dsm_set_lmax_model(dsm_ctx_t* ctx, const float* params) {
    if (!ctx || !params) return DSM_ERR_INVALID;
    return guarded(ctx, [&] {
        DSM_CUDA(cudaSetDevice(ctx->eng->opt.device));
        ctx->eng->pred.load(params, ctx->eng->st);
    });
}

extern "C" int dsm_lmax_predict(dsm_ctx_t* ctx, const int* ilist, int n, float* out) {
    if (!ctx || !ilist || !out || n <= 0) return DSM_ERR_INVALID;
    return guarded(ctx, [&] {
        DSM_CUDA(cudaSetDevice(ctx->eng->opt.device));
        std::vector<float> f((size_t)n * DSM_LMAX_NFEAT);
        ctx->eng->lmax_features(ilist, n, f.data());
        ctx->eng->pred.predict(f.data(), n, out, ctx->eng->st);
        for (int k = 0; k < n; ++k) out[k] += f[(size_t)k * DSM_LMAX_NFEAT];  // log(lmax)
    });
}

extern "C" int dsm_ctx_destroy(dsm_ctx_t* ctx) {
    if (!ctx) return DSM_OK;
    delete ctx;
    return DSM_OK;
}

// Diagnostics: copies an internal device buffer of the last run to host
// memory ("amps": per-order cutoff probes, [F][Lcap][k]).  Returns the
// number of bytes copied, or a negative error code.
extern "C" long long dsm_debug_copy(dsm_ctx_t* ctx, const char* name, void* dst, long long bytes) {
    if (!ctx || !name || !dst) return -DSM_ERR_INVALID;
    dsm::Engine& e = *ctx->eng;
    const void* src = nullptr;
    size_t have = 0;
    if (std::strcmp(name, "amps") == 0) { src = e.amps.p; have = e.amps.n * sizeof(double); }
    for (int m = 0; m < 3; ++m) {
        char nm[8] = {'a', 'f', 'l', 'd', (char)('0' + m), 0};
        if (std::strcmp(name, nm) == 0) { src = e.Afld[m].p; have = e.Afld[m].n * sizeof(double); }
    }
    if (std::strcmp(name, "lcap") == 0) {
        long long v = e.Lcap;
        std::memcpy(dst, &v, sizeof(v));
        return sizeof(v);
    }
    if (!src) return -DSM_ERR_INVALID;
    size_t nb = std::min((size_t)bytes, have);
    if (cudaMemcpy(dst, src, nb, cudaMemcpyDeviceToHost) != cudaSuccess) return -DSM_ERR_CUDA;
    return (long long)nb;
}

// Test hooks of the error paths (no effect on results when unused).
// "tc_stall" = 1: the next run's tensor-core l-sum withholds one stage's
// copies in one CTA with a 20 ms wait limit, so it must report
// DSM_ERR_TIMEOUT and leave the context usable.
extern "C" int dsm_debug_set(dsm_ctx_t* ctx, const char* name, int value) {
    if (!ctx || !name) return DSM_ERR_INVALID;
    if (std::strcmp(name, "tc_stall") == 0) {
        if (!ctx->eng->mixed()) {
            ctx->err = "tc_stall needs a mixed-precision context";
            return DSM_ERR_INVALID;
        }
        ctx->eng->test_tc_stall = value != 0;
        return DSM_OK;
    }
    ctx->err = std::string("unknown debug setting ") + name;
    return DSM_ERR_INVALID;
}

extern "C" int dsm_set_fp64_check(dsm_ctx_t* ctx, dsm_ctx_t* ref, int stride) {
    if (!ctx) return DSM_ERR_INVALID;
    return guarded(ctx, [&] {
        dsm::Engine& e = *ctx->eng;
        if (!ref || stride <= 0) {
            e.check_ref = nullptr;
            e.check_stride = 0;
            return;
        }
        const dsm::Engine& r = *ref->eng;
        if (e.nsrc != 1 || r.nsrc != 1)
            throw Error(DSM_ERR_INVALID, "the FP64 check covers single-source contexts");
        if (ref == ctx || r.opt.precision != DSM_PREC_FP64)
            throw Error(DSM_ERR_INVALID, "the check context must be another context in DSM_PREC_FP64");
        if (r.mode != e.mode || r.R != e.R || r.Th != e.Th || r.opt.device != e.opt.device ||
            r.rsgt_sw != e.rsgt_sw || r.synn_sw != e.synn_sw)
            throw Error(DSM_ERR_INVALID, "the check context has another mode, grid, switches or device");
        e.check_ref = ref->eng.get();
        e.check_stride = stride;
    });
}

extern "C" int dsm_get_accuracy(const dsm_ctx_t* ctx, dsm_accuracy_t* a) {
    if (!ctx || !a) return DSM_ERR_INVALID;
    *a = ctx->eng->acc;
    return DSM_OK;
}

extern "C" int dsm_set_depth_cutoff(dsm_ctx_t* ctx, double bound) {
    if (!ctx) return DSM_ERR_INVALID;
    if (ctx->eng->mode != 1) {
        ctx->err = "the depth cut-off applies to P-SV contexts";
        return DSM_ERR_INVALID;
    }
    if (!(bound >= 0.0 && bound < 1.0)) {
        ctx->err = "depth cut-off bound must lie in [0, 1)";
        return DSM_ERR_INVALID;
    }
    ctx->eng->depth_bound = bound;
    return DSM_OK;
}

extern "C" int dsm_get_tuning(const dsm_ctx_t* ctx, dsm_tuning_t* t) {
    if (!ctx || !t) return DSM_ERR_INVALID;
    *t = ctx->eng->tune;
    return DSM_OK;
}

extern "C" int dsm_set_tuning(dsm_ctx_t* ctx, const dsm_tuning_t* t) {
    if (!ctx || !t) return DSM_ERR_INVALID;
    if ((t->fac_rows != 8 && t->fac_rows != 16) || (t->fld_orders != 16 && t->fld_orders != 32) ||
        (t->tc_orders != 32 && t->tc_orders != 64) || (t->fwd_merge != 0 && t->fwd_merge != 1)) {
        ctx->err = "tuning: fac_rows 8 or 16, fld_orders 16 or 32, tc_orders 32 or 64, fwd_merge 0 or 1";
        return DSM_ERR_INVALID;
    }
    ctx->eng->tune = *t;
    ctx->eng->tc_bk = t->tc_orders;
    return DSM_OK;
}

extern "C" int dsm_autotune(dsm_ctx_t* ctx, const int* ilist, int n, int reps, dsm_tuning_t* best,
                            double* ms_best) {
    if (!ctx || !ilist || n <= 0 || reps <= 0) return DSM_ERR_INVALID;
    return guarded(ctx, [&] {
        dsm::Engine& e = *ctx->eng;
        DSM_CUDA(cudaSetDevice(e.opt.device));
        const dsm_tuning_t keep = e.tune;
        std::vector<dsm_tuning_t> cand;
        const bool psv = e.mode == 1;
        for (int fr : {16, 8}) {
            if (!psv && fr != keep.fac_rows) continue;
            for (int fo : {32, 16}) {
                if (!psv && fo != keep.fld_orders) continue;
                for (int tb : {64, 32}) {
                    if (!e.mixed() && tb != keep.tc_orders) continue;
                    for (int fm : {1, 0}) {
                        if (!psv && fm != keep.fwd_merge) continue;
                        cand.push_back({psv ? fr : keep.fac_rows, psv ? fo : keep.fld_orders,
                                        e.mixed() ? tb : keep.tc_orders, psv ? fm : keep.fwd_merge});
                    }
                }
            }
        }
        double best_ms = 1e300;
        dsm_tuning_t win = keep;
        try {
            for (const auto& c : cand) {
                e.tune = c;
                e.tc_bk = c.tc_orders;
                e.run(ilist, n, nullptr, nullptr, nullptr, nullptr, nullptr);  // untimed
                double ms = 0.0;
                for (int r = 0; r < reps; ++r) {
                    e.run(ilist, n, nullptr, nullptr, nullptr, nullptr, nullptr);
                    ms += e.stats.ms_total;
                }
                ms /= reps;
                if (ms < best_ms) {
                    best_ms = ms;
                    win = c;
                }
            }
        } catch (...) {
            e.tune = keep;
            e.tc_bk = keep.tc_orders;
            throw;
        }
        e.tune = win;
        e.tc_bk = win.tc_orders;
        if (best) *best = win;
        if (ms_best) *ms_best = best_ms;
    });
}

extern "C" int dsm_set_profiling(dsm_ctx_t* ctx, int on) {
    if (!ctx) return DSM_ERR_INVALID;
    ctx->eng->prof = on != 0;
    return DSM_OK;
}

extern "C" int dsm_get_stats(const dsm_ctx_t* ctx, dsm_stats_t* s) {
    if (!ctx || !s) return DSM_ERR_INVALID;
    *s = ctx->eng->stats;
    return DSM_OK;
}
