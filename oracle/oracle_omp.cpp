// Oracle (test infrastructure only): frequency-parallel drivers of the
// CPU restatement, used for the timed CPU baseline.  The reference spreads
// frequencies over MPI ranks (src/SGTpsv/SGTpsv-MPI.f90:550); here the same
// independence is used with host threads pulling frequencies from a queue.
#include "dsmsgt.h"

#include <atomic>
#include <thread>
#include <vector>

extern "C" int oracle_sh_run(const dsm_sh_setup_t*, const int*, int, double*, double*, double*, int*);
extern "C" int oracle_psv_run(const dsm_psv_setup_t*, const int*, int, double*, double*, double*, int*);

namespace {
template <class F>
void run_pool(int n, int nthreads, F f) {
    if (nthreads < 1) nthreads = 1;
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&] {
            for (int k = next++; k < n; k = next++) f(k);
        });
    for (auto& x : th) x.join();
}
}  // namespace

extern "C" int oracle_sh_run_parallel(const dsm_sh_setup_t* s, const int* ilist, int n,
                                      double* tsgt, double* rsgt, double* synn, int* llog,
                                      int nthreads) {
    long nt = 2L * DSM_SH_NUM_TSGT * s->r_n * s->theta_n;
    long nr = 2L * DSM_SH_NUM_RSGT * s->r_n * s->theta_n;
    long ns = 2L * DSM_SH_NUM_SYNN * s->theta_n;
    run_pool(n, nthreads, [&](int k) {
        oracle_sh_run(s, ilist + k, 1, tsgt ? tsgt + nt * k : nullptr, rsgt ? rsgt + nr * k : nullptr,
                      synn ? synn + ns * k : nullptr, llog ? llog + k : nullptr);
    });
    return 0;
}

extern "C" int oracle_psv_run_parallel(const dsm_psv_setup_t* s, const int* ilist, int n,
                                       double* tsgt, double* rsgt, double* synn, int* llog,
                                       int nthreads) {
    long nt = 2L * DSM_PSV_NUM_TSGT * s->r_n * s->theta_n;
    long nr = 2L * DSM_PSV_NUM_RSGT * s->r_n * s->theta_n;
    long ns = 2L * DSM_PSV_NUM_SYNN * s->theta_n;
    run_pool(n, nthreads, [&](int k) {
        oracle_psv_run(s, ilist + k, 1, tsgt ? tsgt + nt * k : nullptr, rsgt ? rsgt + nr * k : nullptr,
                       synn ? synn + ns * k : nullptr, llog ? llog + k : nullptr);
    });
    return 0;
}
