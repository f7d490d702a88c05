// Engine context: device state of one SGT computation (SH or PSV).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "lmax.cuh"
#include "lsum_tc.cuh"

namespace dsm {

// Per-frequency cutoff state of the plain DSM l-cutoff (calamp + the
// ismall > 20 exit, src/SGTpsv/SGTpsv-MPI.f90:606-609, 902-905).
struct CutState {
    int ismall;
    int done;     // 1 once the exit condition fired (or maxlmax reached)
    int llog;     // the reference's llog
    int norders;  // orders summed: llog if the exit fired, else maxlmax+1
    double maxamp;
};

// Ragged work list of a solve launch: system sys belongs to batch frequency
// w with off[w] <= sys < off[w+1] and solves order l = lb[w] + sys - off[w].
struct WorkList {
    const int* off;  // [nw + 1]
    const int* lb;   // [nw]
    int nw;
};
__device__ __forceinline__ void wl_map(const WorkList& wl, int sys, int& w, int& l) {
    int k = 0;
    while (k + 1 < wl.nw && wl.off[k + 1] <= sys) ++k;
    w = k;
    l = wl.lb[k] + sys - wl.off[k];
}

// angular tables shared by both modes
struct ThetaTables {
    int th_n = 0;
    std::vector<double> h_x, h_s;   // cos, sin of theta (host libm)
    std::vector<int> h_pole;        // 0, 1 (theta = 0), 2 (theta = pi)
    DBuf<double> x, s;              // device copies
    DBuf<int> pole;
};

class Engine {
  public:
    int mode = 0;                    // 0 SH, 1 PSV
    dsm_options_t opt{};
    std::string err;
    cudaStream_t st = nullptr;
    cudaStream_t st2 = nullptr;      // side stream (independent per-batch work)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // copy stream for host records: a group's records go out while the
    // next group's l-sum runs
    cudaStream_t stc = nullptr;
    static constexpr int MAX_OUT_GROUPS = 8;
    cudaEvent_t ev_grp[MAX_OUT_GROUPS] = {};
    // mixed l-sum of a batch in frequency groups, in order on stt (high
    // priority): the first group's split, contraction and epilogue, then
    // the other groups' splits and each group's contraction and epilogue;
    // the records of a group go to the host (stc) while later groups run
    cudaStream_t stt = nullptr;
    cudaEvent_t ev_lp = nullptr, ev_lj = nullptr;
    int lsum_groups = 1;             // frequency groups of a batch without host records (DSM_LSUM_GROUPS)
    bool side_pending = false;
    cublasHandle_t cub = nullptr;
    cudaEvent_t ev[8] = {};
    long long launches = 0;
    dsm_stats_t stats{};

    // common geometry
    int R = 0, Th = 0;              // receivers, epicentral distances
    int num_t = 0, num_r = 0, num_s = 0;
    double tlen = 0, omegai = 0, ratl = 0;
    int maxlmax = 0, imin = 0, imax = 0;
    int rsgt_sw = 0, synn_sw = 0;
    ThetaTables th;

    // vector-harmonic basis tables B[m][col][l], col = basis*Th + itheta,
    // basis 0 = c_lm P_l^m, 1 = c_lm (m x/sin P_l^m + P_l^{m+1})
    int lcapB = 0;
    int m_lo = 0;                    // 0 (PSV) or 1 (SH)
    DBuf<double> basis[3];

    // receivers: interpolation weights (value, d/dr) from the three nodes
    DBuf<double> wv, wd;             // [R][3]

    // batch work buffers
    int F = 0, Lc = 0, Lcap = 0;     // frequencies per batch, l chunk, A capacity
    // Several source depths can share one banded factorisation per (omega,
    // l) (P-SV): the per-frequency buffers below (field matrices, cutoff
    // probes and states, outputs) hold nsrc slots of F frequencies, and src
    // selects the slot the mode hooks and the l-sum work on.
    int nsrc = 1, src = 0;
    // run-time tile shapes (dsm_set_tuning, dsm_autotune)
    dsm_tuning_t tune{16, 32, 64, 1};
    // depth cut-off amplitude bound (P-SV; 0: the whole band, as the reference)
    double depth_bound = 0.0;
    int amp_k = 1;                   // cutoff probes stored per order
    DBuf<double> Afld[3];            // field matrices per |m| [F][rows][Lcap]
    int afld_bytes = 8;              // their element: FP64, or FP32 where the mode's mixed path stores them so
    DBuf<double> Cgemm;              // GEMM output of one (omega, |m|)
    DBuf<CutState> cut;              // [F]
    DBuf<double> amps;               // [F][Lcap][5]
    DBuf<double> out_t, out_r, out_s;  // complex128 outputs of a batch
    DBuf<float> out32;                 // complex64 catalogue packing
    DBuf<int> d_freqs;
    std::vector<int> h_norders;

    // source src's slot of the per-frequency buffers
    size_t fld_off(int m) const { return (size_t)src * F * rows_m[m] * Lcap; }  // elements of Afld[m]
    CutState* cut_src() const { return cut.p + (size_t)src * F; }
    double* amps_src() const { return amps.p + (size_t)src * F * Lcap * amp_k; }
    double* out_t_src() const;
    double* out_r_src() const;
    double* out_s_src() const;

    // rows of the field matrix per |m| (set by the mode)
    int rows_m[3] = {0, 0, 0};
    // leading rows of each field matrix contracted with all 2 Th basis
    // columns; the remaining rows need only the first Th (set by the mode,
    // all rows unless it groups its fields)
    int rows_full[3] = {-1, -1, -1};
    int full_rows(int m) const { return rows_full[m] < 0 ? rows_m[m] : rows_full[m]; }
    // Layout of the contraction outputs: column-major (ld = rows of the |m|
    // block), or row-major with row stride c_ld >= 2 Th (a multiple of 4)
    // where the mode's epilogue reads a row's distances together
    bool c_rowmajor = false;
    int c_ld = 0;
    // offset of the |m| block inside Cgemm (one frequency)
    size_t c_off(int mi) const {
        size_t off = 0;
        for (int m = m_lo; m < mi; ++m) off += (size_t)rows_m[m] * (c_rowmajor ? (size_t)c_ld : 2 * (size_t)Th);
        return off;
    }
    size_t c_total() const { return c_off(3); }
    void init_common(int dev);
    virtual ~Engine();

    void build_basis(int lneed);
    void build_weights(const double* r, const double* rrsta);
    void gemm_fp64(int w, int mi, int K);

    // mixed precision: the l-sum as split 16-bit products on the tensor
    // cores (fields and bases split once per batch / per table build)
    bool mixed() const { return opt.precision == DSM_PREC_MIXED || opt.precision == DSM_PREC_MIXED_BF16; }
    int tc_fmt = tc::PIECE_F16, tc_bk = 64, nsm = 148;
    uint32_t tc_flags = tc::TC_REVERSE;
    int tc_chunk = 1;                // stages (of tc_bk orders) per hi*hi chunk: 64 orders
    int kcA = 0, kcB = 0;            // order capacities of the pieces (x64)
    DBuf<uint16_t> Apc[3];           // [2][F][rows][kcA]
    DBuf<float> sA[3];               // [F][rows]
    DBuf<uint16_t> Bpc[3];           // [2][2Th][kcB]
    DBuf<float> sB[3];               // [2Th]
    DBuf<float> Cmix;                // [F][c_total] column-major blocks
    DBuf<int> lnzA[3];               // [F][rows]: one past each field row's last nonzero order
    // Where the mode knows that a receiver's fields are zero from some order
    // on (P-SV with the depth cut), zfirst[src][F][R+1] holds that order per
    // receiver row (INT_MAX-like: none) and rowrec[m][row] the receiver row of
    // each field row; the split reads a row only up to it
    DBuf<int> zfirst, rowrec[3];
    bool use_zfirst = false;
    DBuf<int> tcKb;                  // order blocks of each row tile of the batch's problems
    DBuf<tc::Problem> tcp;
    DBuf<int> d_nord;
    DBuf<int> dflags;                // status words (DEV_WORD_TC, DEV_WORD_STATUS)
    int* tc_err() const { return dflags.p + DEV_WORD_TC; }
    int* dstatus() const { return dflags.p + DEV_WORD_STATUS; }
    // test hook: the next run's tensor-core launches withhold one stage's
    // copies in one CTA and wait at most 20 ms, so the bounded wait gives up
    int test_tc_stall = 0;
    // mixed l-sum of a batch: buffers, tensor maps and order counts once,
    // then the split and the tensor-core launches of frequencies [w0, w1)
    void lsum_prepare(int nf, const std::vector<int>& norders);
    // problem lists of all groups (each a list of batch slots), one upload
    void lsum_plan(const std::vector<std::vector<int>>& groups, const std::vector<int>& norders);
    // group g: split, contraction launches (both on stt)
    void lsum_split(int g);
    void lsum_contract(int g);
    struct TcLaunch { size_t first; int np, tiles; };
    struct TcGroup { std::vector<int> slots; std::vector<TcLaunch> launches; double split_bytes, flops, bytes; };
    std::vector<TcGroup> tc_groups;
    std::vector<tc::Problem> tc_plan;  // the problems of the last plan (host copy)
    size_t tc_kbn = 0;                 // row-tile entries of the last plan
    void count_exec_flops();           // adds the executed contraction flops (profiling)
    tc::Maps tcmaps;
    size_t tcp_next = 0;  // next free slot of tcp in this batch
    void check_device_flags();
    // contraction output of (frequency w, |m|) for the epilogue
    const double* c64(int mi) const { return Cgemm.p + c_off(mi); }
    const float* c32(int w, int mi) const { return Cmix.p + (size_t)w * c_total() + c_off(mi); }
    // optional per-kernel event timing
    bool prof = false;
    std::vector<cudaEvent_t> evpool;
    struct Rec { int id; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    int kid(const char* name);
    void kbegin(int id, cudaStream_t s = nullptr);
    void kend(int id, double bytes, double flops, cudaStream_t s = nullptr);
    void fork_side();   // side stream waits for the main stream
    void join_side();   // main stream waits for the side stream
    void kcollect();
    std::vector<int> pend_id;
    void grow_orders(int need);

    // mode hooks
    virtual void omega_pieces(const int* freqs_dev, int nf) = 0;
    virtual void solve_chunk(const int* freqs_dev, int nf, const WorkList& wl, int nsys) = 0;
    virtual void scan_chunk(int nf, const WorkList& wl) = 0;
    int nsys_max = 0;                // systems per solve launch (scratch size)
    double vtop_ = 1.0, rtop_ = 1.0;  // top-zone Vsv sum and radius (callsuf)
    int first_span(int ifreq) const;
    double span_hint = 1.0;          // first-range scale learned from earlier batches (run)
    DBuf<int> wl_off, wl_lb;
    std::vector<int> wl_host_off;    // host copy of the current round's work-list offsets
    virtual void epilogue(const int* freqs_dev, int w, int nf, cudaStream_t s) = 0;
    virtual size_t out_sizes(size_t* nt, size_t* nr, size_t* ns) const = 0;

    // learned cutoff: per-context model summaries, the device network, and
    // the cutoff-only mode used to harvest training data
    float summ[10] = {};             // r_src/rmax, r_rcv/rmax, 8 model summaries
    lmax::Predictor pred;
    bool cutoffs_only = false;
    void set_summaries(int is_psv, int nzone, const double* vrmin, const double* vrmax, const double* vsv,
                       const double* qmu, double r0, double rrcv);
    void lmax_features(const int* ilist, int n, float* out) const;
    long long rounds = 0;            // solve rounds of the last run

    // FP64 accuracy report: an FP64 engine of the same set-up recomputes
    // every check_stride-th frequency of a run on the device; per-component
    // sums of |x - x64|^2 and |x64|^2 accumulate in acc_sums
    Engine* check_ref = nullptr;
    int check_stride = 0;
    DBuf<double> acc_sums;           // [num_t + num_r + num_s][2]
    dsm_accuracy_t acc{};
    double ms_check = 0.0;
    void check_batch(const int* ilist, int b0, int nf, const std::vector<CutState>& hc);
    void finish_accuracy();

    // drivers; host_out holds nsrc output sets (or is null)
    void run(const int* ilist, int n, dsm_out_t* host_out, const void** dt, const void** dr,
             const void** ds, int* llog);
};

Engine* make_sh_engine(const dsm_sh_setup_t* s, const dsm_options_t* o);
Engine* make_psv_engine(const dsm_psv_setup_t* const* s, int nsrc, const dsm_options_t* o);

// shared kernels (tables.cu)
void launch_basis_tables(Engine& e, int lcap);
void launch_interp_weights(Engine& e, const double* d_r, const double* d_rrsta);
// complex64 records of frequencies [w0, w1) of a batch of nf into out32
void launch_pack32(Engine& e, int nf, int w0, int w1, size_t per_t, size_t per_r, size_t per_s, cudaStream_t s);

}  // namespace dsm

struct dsm_ctx {
    std::unique_ptr<dsm::Engine> eng;
    std::string err;
};
