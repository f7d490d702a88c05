/*
 * dsmsgt.h -- C-ABI of the B200 strain Green's tensor (SGT) engine.
 *
 * The engine replaces the body of the frequency loop of the DSM Kernel
 * Suite programs SGTsh and SGTpsv:
 *   SH : src/SGTsh/SGTsh-MPI.f90:404-555   (per-omega operator, l loop,
 *        m loop, sources, banded solve, receiver l-sum)
 *   PSV: src/SGTpsv/SGTpsv-MPI.f90:551-1095
 * Everything before that loop (parameter parsing, grid, element integrals)
 * and after it (catalogue files, logs) stays with the caller, which in the
 * reference is the Fortran driver.  The caller fills one of the setup
 * structs below with the arrays that driver holds after its set-up phase
 * (1-based indices are kept exactly as the Fortran computes them), creates
 * a context, and asks for any list of frequency indices.
 *
 * All pointers are plain host pointers; sizes are element counts.  Complex
 * numbers are interleaved (re, im) pairs of double (complex128) or float
 * (complex64).  No type in this header depends on CUDA or on PyTorch.
 *
 * Error behaviour: every entry point returns DSM_OK (0) or one of the
 * DSM_ERR_* codes.  The library never prints, stops or pauses (the
 * reference pauses on bad input, src/SGTpsv/others.f90:536); the text of
 * the last error of a context is available from dsm_last_error().
 */
#ifndef DSMSGT_H
#define DSMSGT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSM_ABI_VERSION 3

/* return codes */
#define DSM_OK               0
#define DSM_ERR_INVALID      1  /* bad argument or inconsistent set-up        */
#define DSM_ERR_CUDA         2  /* CUDA runtime / driver / library error      */
#define DSM_ERR_NONFINITE    3  /* a pivot, cutoff probe or output became
                                   Inf/NaN (the reference prints and carries
                                   on, src/SGTsh/dclib.f90:36-40; the outputs
                                   of such a call are not meaningful)        */
#define DSM_ERR_LMAX         4  /* a cutoff needs more orders than allowed    */
#define DSM_ERR_TIMEOUT      5  /* a bounded device wait gave up              */
#define DSM_ERR_NOMEM        6  /* device or host allocation failed           */
#define DSM_ERR_NODEVICE     7  /* no CUDA device / kernels not loadable      */

/* precision modes of a context */
#define DSM_PREC_FP64        0  /* plain path: every stage in FP64            */
#define DSM_PREC_MIXED       1  /* l-sum as split fp16 products (hi/lo of
                                   both operands, three products) on the
                                   tensor cores with FP32 accumulation      */
#define DSM_PREC_MIXED_BF16  2  /* same with bf16 pieces                   */

/* number of output components per point (src/SGTsh/modules.f90:371-373,
   src/SGTpsv/modules.f90:112-114) */
#define DSM_SH_NUM_TSGT   10
#define DSM_SH_NUM_RSGT    5
#define DSM_SH_NUM_SYNN    5
#define DSM_PSV_NUM_TSGT  20
#define DSM_PSV_NUM_RSGT  10
#define DSM_PSV_NUM_SYNN  10

/* ------------------------------------------------------------------------
 * SH set-up: the state of SGTsh after src/SGTsh/SGTsh-MPI.f90:33-347.
 * ---------------------------------------------------------------------- */
typedef struct dsm_sh_setup {
    int nzone;                 /* solid zones kept (outer core cut, :96-102)   */
    const double *vrmin;       /* [nzone] km                                   */
    const double *vrmax;       /* [nzone] km                                   */
    const double *vsv;         /* [4*nzone] column-major (4,nzone), for callsuf */
    const double *qmu;         /* [nzone]                                      */
    const int    *nlayer;      /* [nzone]                                      */
    const int    *isp;         /* [nzone] 1-based first node of each zone      */
    const int    *jsp;         /* [nzone] 1-based first element entry          */
    int           nnlayer;     /* total layers; the system has nnlayer+1 rows  */
    const double *t, *h1, *h2, *h3, *h4;   /* [4*nnlayer] element integrals   */
    /* source (single depth, src/SGTsh/others.f90:37-41) */
    int           spn;         /* zone of the source                           */
    double        spo;         /* position inside the zone (calspo)            */
    double        r0;          /* source radius after calspo adjustment        */
    double        mu0;         /* rigidity at the source (calgstg)             */
    int           ins;         /* 1-based element entry of the source layer    */
    const double *gt, *gh1, *gh2, *gh3, *gh4;  /* [8] split source element     */
    /* receivers */
    int           r_n;
    const double *r;           /* [r_n] km                                     */
    const double *rrsta;       /* [3*r_n] (3,r_n) interpolation node radii     */
    const int    *iista;       /* [3*r_n] (3,r_n) 1-based node indices         */
    int           theta_n;
    const double *theta;       /* [theta_n] degrees                            */
    /* DSM parameters */
    double        tlen;        /* s                                            */
    double        omegai;      /* imaginary frequency, already -ln(conf)/tlen  */
    double        ratl;        /* l-cutoff amplitude ratio                     */
    int           maxlmax;
    int           imin, imax;  /* frequency range of the run (zig-zag owner)   */
    int           rsgt_switch, tsgt_switch, synn_switch;
} dsm_sh_setup_t;

/* ------------------------------------------------------------------------
 * PSV set-up: the state of SGTpsv after src/SGTpsv/SGTpsv-MPI.f90:39-477.
 * Element arrays are passed whole, with the Fortran 1-based offsets the
 * driver uses to address them (itmp = isdr+issp(isl) etc.).
 * ---------------------------------------------------------------------- */
typedef struct dsm_psv_setup {
    int nzone;
    const int    *iphase;      /* [nzone] 1 solid, 2 fluid (calnl)             */
    const int    *nlayer;      /* [nzone]                                      */
    const int    *isp;         /* [nzone] 1-based first node (calsp)           */
    const int    *kkdr;        /* [nzone] 1-based first unknown (calspdr)      */
    const int    *elem;        /* [nzone] 1-based element offset: solid
                                  isdr+issp(isl), fluid ildr+ilsp(ill)         */
    const int    *hmoff;       /* [nzone] solid: 1-based column jsdr+jssp(isl)
                                  of the modified-derivative arrays; fluid 0   */
    const double *vrmin, *vrmax, *qmu, *qkappa;   /* [nzone]                   */
    const double *vsv;         /* [4*nzone] (4,nzone), for callsuf             */
    int           nn;          /* unknowns: kkdr(nzone)+2*nlayer(nzone)+1      */
    double        rmin, rmax;
    /* solid element arrays, each n_sel entries, order fixed by
       DSM_PSV_SOLID_* below; fluid arrays p1,p2,p3 each n_fel entries;
       modified first-derivative operators, each (4, n_hm) column-major with
       the first index running over the Fortran bounds (-2:1) or (-1:2).    */
    int           n_sel, n_fel, n_hm;
    const double *solid_el;    /* [DSM_PSV_NSOLID * n_sel]                     */
    const double *fluid_el;    /* [3 * n_fel]                                  */
    const double *hm_el;       /* [DSM_PSV_NHM * 4 * n_hm]                     */
    /* source */
    int           spn;
    double        spo;
    double        r0;          /* after calspo adjustment                      */
    double        ecC0, ecF0, ecL0;  /* elastic constants at r0 (calstg)      */
    double        ra_src[2];   /* ra(mtmp), ra(mtmp+1) around the source       */
    double        src_poly[24];/* rho,vpv,vph,vsv,vsh,eta (4 each), zone spn  */
    int           jsrc;        /* 1-based first excitation row (jtmp, :636)    */
    /* receivers */
    int           r_n;
    const double *r;           /* [r_n]                                        */
    const double *rrsta;       /* [3*r_n]                                      */
    const int    *iista;       /* [3*r_n] zone-local node indices (calra2_psv) */
    const int    *istazone;    /* [r_n]                                        */
    const double *lambda;      /* [r_n] A at the receiver (fluid receivers)    */
    const double *qkp;         /* [r_n] Qkappa at the receiver                 */
    int           theta_n;
    const double *theta;       /* [theta_n] degrees                            */
    double        tlen, omegai, ratl;
    int           maxlmax;
    int           imin, imax;
    int           rsgt_switch, tsgt_switch, synn_switch;
} dsm_psv_setup_t;

/* packing order of dsm_psv_setup_t.solid_el */
enum {
    DSM_PSV_T = 0, DSM_PSV_H1X, DSM_PSV_H2L, DSM_PSV_H2N, DSM_PSV_H3AY,
    DSM_PSV_H4AL, DSM_PSV_H4AN, DSM_PSV_H5AY, DSM_PSV_H6AL, DSM_PSV_H6AN,
    DSM_PSV_H7Y, DSM_PSV_H7Z, DSM_PSV_H8L, DSM_PSV_H8N, DSM_PSV_H3Y,
    DSM_PSV_H4L, DSM_PSV_H4N, DSM_PSV_H5Y, DSM_PSV_H6L, DSM_PSV_H6N,
    DSM_PSV_NSOLID
};
/* packing order of dsm_psv_setup_t.hm_el */
enum {
    DSM_PSV_H3MY = 0,   /* (-2:1) */
    DSM_PSV_H5MY,       /* (-1:2) */
    DSM_PSV_H4M1L,      /* (-1:2) */
    DSM_PSV_H4M2N,      /* (-2:1) */
    DSM_PSV_H6M1N,      /* (-1:2) */
    DSM_PSV_H6M2L,      /* (-2:1) */
    DSM_PSV_NHM
};

/* ------------------------------------------------------------------------
 * Context options and outputs
 * ---------------------------------------------------------------------- */
typedef struct dsm_options {
    int precision;        /* DSM_PREC_FP64, DSM_PREC_MIXED(_BF16)           */
    int device;           /* CUDA device ordinal                             */
    int use_lmax_predictor;/* 1: size l batches with the learned cutoff      */
    int l_chunk;          /* orders solved speculatively per batch (0: auto) */
    int freq_batch;       /* frequencies processed together (0: auto)        */
} dsm_options_t;

/* Host output buffers for dsm_run_freqs.  Any pointer may be NULL.  For
 * frequency k of the request (0 <= k < n):
 *   tsgt   complex128, column-major (num_tsgt, r_n, theta_n), block k
 *   rsgt   complex128, column-major (num_rsgt, r_n, theta_n), block k
 *   synn   complex128, column-major (num_synn, theta_n),      block k
 *   tsgt32/rsgt32/synn32: complex64 in catalogue record order, i.e. for each
 *          receiver the (num, theta_n) record the reference writes to one
 *          file (SGTpsv-MPI.f90:1113-1116): layout [k][ir][itheta][comp]
 *   llog   the reference's cutoff variable per frequency (the log line
 *          prints llog-1, SGTpsv-MPI.f90:1098)
 */
typedef struct dsm_out {
    double *tsgt, *rsgt, *synn;
    float  *tsgt32, *rsgt32, *synn32;
    int    *llog;
} dsm_out_t;

typedef struct dsm_ctx dsm_ctx_t;

/* Context creation uploads the set-up to the device, builds the
 * omega-independent tables (vector-harmonic bases, interpolation weights)
 * and reserves device memory.  Replaces the reference's per-run state in
 * src/SGTsh/modules.f90 / src/SGTpsv/modules.f90. */
int dsm_sh_create(const dsm_sh_setup_t *setup, const dsm_options_t *opt,
                  dsm_ctx_t **ctx);
int dsm_psv_create(const dsm_psv_setup_t *setup, const dsm_options_t *opt,
                   dsm_ctx_t **ctx);

/* Computes the SGTs of n frequency indices (each in [imin, imax], i != 0;
 * replaces one pass of the omega loop per index, SGTsh-MPI.f90:389-613,
 * SGTpsv-MPI.f90:535-1152).  Output is copied to the host buffers. */
int dsm_run_freqs(dsm_ctx_t *ctx, const int *ilist, int n, dsm_out_t *out);

/* Same computation with outputs left on the device: *d_tsgt etc. receive
 * device pointers owned by the context, valid until the next call.  Used
 * by callers that consume the SGT on the GPU. */
int dsm_run_freqs_device(dsm_ctx_t *ctx, const int *ilist, int n,
                         const void **d_tsgt, const void **d_rsgt,
                         const void **d_synn, int *llog);

/* Several source depths in one P-SV context.  No counterpart in the
 * reference, which takes one source depth per run (r0max = r0min,
 * src/SGTpsv/others.f90:52-54) and factors the band of every (omega, l)
 * once per run (SGTpsv-MPI.f90:885-890).  setups[0..nsrc) describe the same
 * model, grid, receivers and distances (the arrays must be equal) and differ
 * only in the source fields (spn, spo, r0, ecC0/F0/L0, ra_src, src_poly,
 * jsrc); each (omega, l) band is assembled and factored once and solved for
 * every source.  Each source keeps its own cutoff test and outputs, the same
 * values as a context of that source alone. */
int dsm_psv_create_multi(const dsm_psv_setup_t *const *setups, int nsrc,
                         const dsm_options_t *opt, dsm_ctx_t **ctx);
/* dsm_run_freqs for a context of nout = nsrc sources: outs[s] receives
 * source s's outputs (RSGT, which does not depend on the source, in every
 * set that asks for it); complex64 records are packed when outs[0] asks for
 * them.  dsm_run_freqs refuses a context with more than one source, and the
 * FP64 accuracy check covers single-source contexts. */
int dsm_run_freqs_multi(dsm_ctx_t *ctx, const int *ilist, int n, dsm_out_t *outs, int nout);

/* A request of several contexts -- other models, P-SV and SH, each with one
 * or several source depths -- run together: each context on its own host
 * thread and CUDA streams, so the GPU overlaps one context's latency-bound
 * band solves with another's l-sum.  No counterpart in the reference (one
 * MPI job per model and depth).  ctxs must be distinct and on one device;
 * for context k: ilists[k][0..ns[k]) and outs[k] (nsrc output sets, as
 * dsm_run_freqs_multi takes them; outs or outs[k] NULL: nothing is copied
 * to the host, the run only computes -- for timing, as dsm_autotune runs
 * its candidates).  rcs[k] (if rcs is not NULL) receives
 * each context's code; the call returns the first code that is not DSM_OK
 * (the texts stay with the contexts). */
int dsm_run_request(dsm_ctx_t *const *ctxs, int nctx, const int *const *ilists, const int *ns,
                    dsm_out_t *const *outs, int *rcs);

int dsm_ctx_destroy(dsm_ctx_t *ctx);
const char *dsm_last_error(const dsm_ctx_t *ctx);
const char *dsm_strerror(int code);
int dsm_abi_version(void);

/* Per-kernel device time of the last run, recorded with CUDA events on the
 * context's stream when profiling is on (dsm_set_profiling). */
#define DSM_MAX_KSTATS 24
typedef struct dsm_kstat {
    char      name[32];
    double    ms;          /* summed device time                          */
    long long launches;
    double    alg_bytes;   /* algorithmic bytes moved by these launches   */
    double    alg_flops;   /* algorithmic flops of these launches         */
} dsm_kstat_t;

/* Stage timing of the last run (device time in ms, CUDA events): the
 * per-(omega,l) solve, the l-sum contraction, the epilogue/packing, and
 * the whole call.  Also the number of kernel launches of the call. */
typedef struct dsm_stats {
    double ms_total, ms_solve, ms_lsum, ms_pack, ms_h2d, ms_d2h;
    long long launches;
    long long systems;      /* (omega,l) systems solved                    */
    long long orders_used;  /* sum over frequencies of the realised cutoff */
    long long orders_padded;/* orders solved beyond the cutoff             */
    double lsum_flops;      /* algorithmic flops of the contraction        */
    double solve_bytes;     /* algorithmic bytes of the banded solves      */
    int nk;                 /* entries of kern[] in use                    */
    dsm_kstat_t kern[DSM_MAX_KSTATS];
    long long solve_rounds;  /* order ranges solved per batch, summed        */
    long long freqs_extended;/* frequencies whose cutoff lay beyond their
                                first order range (the learned cutoff's
                                misses when it sized that range)            */
    double lsum_flops_exec;  /* flops the mixed contraction executed: row
                                tiles stop at their rows' last nonzero order
                                (counted when profiling is on, else 0)      */
} dsm_stats_t;
int dsm_get_stats(const dsm_ctx_t *ctx, dsm_stats_t *stats);

/* Accuracy report of a mixed-precision context (the per-output relative
 * L2 error the precision plan asks for).  No counterpart in the reference.
 * dsm_set_fp64_check attaches a DSM_PREC_FP64 context of the same set-up
 * (same mode, receivers and distances, same device; the caller keeps
 * ownership and must not destroy it while attached; NULL detaches): every
 * later dsm_run_freqs / dsm_run_freqs_device call then recomputes every
 * stride-th frequency of its request (request positions 0, stride, ...) on
 * that context and compares on the device.  The comparison's time is not
 * counted in dsm_stats_t.ms_total.  dsm_get_accuracy returns the report of
 * the last call: per component, sqrt(sum |x - x64|^2 / sum |x64|^2) over
 * the compared frequencies, receivers and distances; a component whose FP64
 * values vanish identically (below 1e-10 of its array's norm, e.g. SH has no
 * radial displacement) is measured against the whole array's norm.
 * Entries past the mode's component count are 0. */
typedef struct dsm_accuracy {
    int    nfreq;           /* frequencies recomputed by the last call       */
    int    llog_equal;      /* 1: each recomputed cutoff equals the call's   */
    double tsgt[DSM_PSV_NUM_TSGT], rsgt[DSM_PSV_NUM_RSGT], synn[DSM_PSV_NUM_SYNN];
    double tsgt_max, rsgt_max, synn_max;
} dsm_accuracy_t;
int dsm_set_fp64_check(dsm_ctx_t *ctx, dsm_ctx_t *fp64_ctx, int stride);
int dsm_get_accuracy(const dsm_ctx_t *ctx, dsm_accuracy_t *acc);

/* Tile shapes of a context, chosen at run time.  No counterpart in the
 * reference (a CPU program with no tiles).  The defaults are the measured
 * best on the benchmark; dsm_autotune measures the alternatives on the
 * caller's own request and keeps the fastest. */
/* Depth cut-off of the P-SV band (no counterpart in the reference, which
 * factors every band from the centre, SGTpsv-MPI.f90:662; the DSM config's
 * ratc names the same idea).  Below the turning depth of the slowest wave an
 * (omega, l) solution decays; rows where a WKB bound on its amplitude
 * relative to the source falls under `bound` leave the system (a zero
 * displacement boundary there), which changes the outputs by about bound^2
 * relative.  0 turns it off.  Default: 1e-20 in the mixed precision modes,
 * 0 in DSM_PREC_FP64 (the reference's results).  P-SV contexts only. */
int dsm_set_depth_cutoff(dsm_ctx_t *ctx, double bound);

typedef struct dsm_tuning {
    int fac_rows;    /* band rows a factorisation block stages per chunk: 8 or 16 (P-SV) */
    int fld_orders;  /* consecutive orders per warp of the receiver-field kernel: 16 or 32 (P-SV) */
    int tc_orders;   /* orders per tensor-core stage (and FP64 chunk sum): 32 or 64 (mixed precision) */
    int fwd_merge;   /* 1: the first source's forward substitution inside the P-SV factorisation
                        (2 blocks per SM), 0: in its own kernel after it (3 blocks per SM) */
} dsm_tuning_t;
int dsm_get_tuning(const dsm_ctx_t *ctx, dsm_tuning_t *t);
int dsm_set_tuning(dsm_ctx_t *ctx, const dsm_tuning_t *t);
/* Runs the request ilist[0..n) reps times (after one untimed run) with each
 * combination of the tile shapes that applies to the context's mode and
 * precision, keeps the one with the least device time and returns it in
 * *best (and its mean time per request in *ms_best, ms).  Outputs of these
 * runs are discarded; every combination gives results within the context's
 * accuracy (FP64: identical values). */
int dsm_autotune(dsm_ctx_t *ctx, const int *ilist, int n, int reps, dsm_tuning_t *best, double *ms_best);

/* Turns per-kernel event timing on (1) or off (0) for later runs. */
int dsm_set_profiling(dsm_ctx_t *ctx, int on);

/* Test hook of the error paths; no counterpart in the reference (whose
 * solvers print and carry on).  name "tc_stall", value 1: the next run of a
 * mixed-precision context withholds one stage's copies in the tensor-core
 * l-sum and shortens its bounded waits to 20 ms, so that run returns
 * DSM_ERR_TIMEOUT and the context stays usable.  Unknown names return
 * DSM_ERR_INVALID. */
int dsm_debug_set(dsm_ctx_t *ctx, const char *name, int value);

/* SH angular-order cutoff without allocating device memory.  No
 * counterpart in the reference: it returns in llog[k] the cutoff the SH
 * engine reaches for frequency ilist[k] (the same value dsm_run_freqs
 * reports), for callers that size their work before the SGT run but cannot
 * call cudaMalloc -- a process whose GPU memory is already reserved by
 * another framework's caching allocator, or one that must not cause the
 * implicit device-wide synchronisation of cudaMalloc/cudaFree while other
 * streams run.  All device buffers live in one fixed 64 MiB array per GPU,
 * held until the process exits; set-ups needing more are rejected with
 * DSM_ERR_INVALID (text in dsm_last_error(NULL)).  Runs on the current
 * device.  The first call on a device looks up the array's address, so
 * make it before any stream capture.  Calls that overlap on the GPU share
 * the array and race. */
int dsm_sh_cutoff_noalloc(const dsm_sh_setup_t *setup, const int *ilist, int n, int *llog);

/* ------------------------------------------------------------------------
 * Learned angular-order cutoff.  No counterpart in the reference.  A
 * 4-layer MLP (width 128, GELU, bf16 weights, FP32 accumulation) maps
 * DSM_LMAX_NFEAT features of a frequency to log(lmax) - log(1 + omega
 * r_top / v_top) (the cutoff relative to the reference's lsuf scale); a
 * context with
 * opt.use_lmax_predictor = 1 and a loaded parameter block sizes the first
 * order range of each frequency with it.  The plain amplitude test still
 * runs on the device and extends any short range, so the cutoff (llog) and
 * the outputs are those of the plain method; only padded work changes.
 * ---------------------------------------------------------------------- */
#define DSM_LMAX_NFEAT   11
#define DSM_LMAX_WIDTH   128
#define DSM_LMAX_NPARAM  34713   /* floats in a parameter block          */

/* Features of frequencies ilist[0..n) for the context's set-up, n x NFEAT:
 * log(1 + omega rtop / vtop) (the reference's lsuf scale, callsuf),
 * source radius / rmax, probe receiver radius / rmax, and 8 model
 * summaries: surface Vs, Vs at the source, min and max zone Vs (/10),
 * source depth (/1000 km), top-zone thickness (/100 km), mode (0 SH,
 * 1 P-SV), log10(Qmu at the source) / 3. */
int dsm_lmax_features(const dsm_ctx_t *ctx, const int *ilist, int n, float *feats);

/* Realised cutoffs only (banded solves and the amplitude test, no l-sum):
 * llog[k] as dsm_run_freqs reports it.  Used to harvest training data. */
int dsm_cutoffs(dsm_ctx_t *ctx, const int *ilist, int n, int *llog);

/* Parameter block: standardisation from (feats, target), He-initialised
 * weights from seed.  The network's target is the cutoff relative to the
 * lsuf scale: target = log(llog) - feats[0] per row. */
int dsm_lmax_init(const float *feats, const float *target, int n, unsigned seed, float *params);
/* AdamW on the GPU (device ordinal, decoupled weight decay):
 * params in/out, losses[epochs] out. */
int dsm_lmax_train(const float *feats, const float *target, int n, int epochs, int batch,
                   float lr, float weight_decay, unsigned seed, float *params,
                   float *losses, int device);
/* Loss (mean squared error of the standardised output) and its gradient
 * with respect to every parameter, on the n rows given. */
int dsm_lmax_grad(const float *params, const float *feats, const float *target, int n,
                  float *grad, float *loss, int device);
/* Attaches a parameter block to a context.  dsm_lmax_predict writes the
 * predicted log(lmax) (network output + feats[0]) of frequencies
 * ilist[0..n) to out. */
int dsm_set_lmax_model(dsm_ctx_t *ctx, const float *params);
int dsm_lmax_predict(dsm_ctx_t *ctx, const int *ilist, int n, float *out);

/* ------------------------------------------------------------------------
 * Catalogue consumer: the SGT records of one receiver radius (frequency
 * indices fmin..fmax at every catalogue distance, as SGTpsv / SGTsh write
 * them) turned into windowed time series at arbitrary epicentral distances
 * on the device.  Replaces KernelMaker's
 *   rdsgtomega        src/KernelMaker/fourier.f90:1-123
 *   clsgt             src/KernelMaker/fourier.f90:128-162
 *   findIdeltaRegion  src/KernelMaker/fourier.f90:165-190
 *   vectorFFT_double  src/KernelMaker/fourier.f90:418-450 (with cdft/bitrv2)
 * and the transform set-up of src/KernelMaker/KernelMaker-1.0.0.f90:311-330.
 * The per-point real combination of components that KernelMaker applies
 * before its transform (synn2h3freq, rsgt2h3freq, tsgt2h4freq and the
 * moment-tensor sums) can be passed as a matrix per point.
 * ---------------------------------------------------------------------- */
typedef struct dsm_cat_params {
    int    num;            /* components of the frequency-domain SGT (<= 32) */
    int    theta_n;        /* catalogue distances theta_min + k theta_delta  */
    double theta_min, theta_delta;      /* degrees                           */
    int    fmin, fmax;     /* frequency indices of the records               */
    int    np1;            /* half transform length: power of two >= fmax    */
    double tlen;           /* time length (s)                                */
    double omegai;         /* imaginary frequency (1/s), -ln(x)/tlen as
                              KernelMaker-1.0.0.f90:86 computes it           */
    double ipdistance;     /* sinc interpolation window (deg)                */
    double c_red_reci;     /* reducing slowness (s/deg), 0: none             */
    int    iwin_start, iwin_end;        /* output samples, 0 <= s <= e < 2 np1 */
    int    device;         /* CUDA device ordinal                            */
} dsm_cat_params_t;

typedef struct dsm_cat dsm_cat_t;

/* np1, the redefined sampling rate and the window samples of a time window
 * [start, end] (s), from lsmoothfinder (src/KernelMaker/others.f90:288-308)
 * and KernelMaker-1.0.0.f90:311-330.  Any output pointer but np1 may be
 * NULL. */
int dsm_cat_np1(double tlen, int fmax, double sampling_hz, double start, double end,
                int *np1, double *sampling_hz_out, int *iwin_start, int *iwin_end);

int dsm_cat_create(const dsm_cat_params_t *p, dsm_cat_t **cat);

/* Adds one record set to the frequency-domain SGT (rdsgtomega, one call per
 * catalogue kind).  rec holds [fmax-fmin+1][theta_n][ncomp] complex numbers
 * (elem_bytes 8: complex64 as in the catalogue files; 16: complex128), record
 * k being frequency index fmin + k; the record of index 0 is never read.
 * Component k is multiplied by scale[k] (NULL: 1; the reference halves
 * SYNN_PSV components 2, 8-10 and SYNN_SH 3-5, fourier.f90:78-85), by 1e-21
 * and by the reduction phase, and added to component dst[k] (NULL: k; the
 * reference puts SH sets into P-SV slots, fourier.f90:103-116).  With
 * on_device = 1, rec is a device pointer that must stay valid until
 * dsm_cat_clear or dsm_cat_destroy; otherwise it is copied to the device.
 * At most 4 sets. */
int dsm_cat_add(dsm_cat_t *cat, const void *rec, int elem_bytes, int ncomp,
                const int *dst, const double *scale, int on_device);

/* Forgets every record set (tsgtomega = 0). */
int dsm_cat_clear(dsm_cat_t *cat);

/* Time series at npoint distances (deg): out[p][j][t], t over the window,
 * j < nout, from the component combination coef[p][j][c] (c < num; NULL:
 * the num components themselves, nout ignored).  With out_on_device = 1,
 * out is a device pointer. */
int dsm_cat_series(dsm_cat_t *cat, int npoint, const double *distance, int nout,
                   const double *coef, double *out, int out_on_device);

/* The same points' combined spectra before the transform: out holds
 * complex128 [point][j][fmax-fmin+1] for frequency indices fmin..fmax (index
 * 0 is zero).  These are clsgt's interpolated SGT (fourier.f90:128-162)
 * combined per point, e.g. the h3 / h4 sums that KernelMaker's kernel
 * formulas multiply frequency by frequency before their transform
 * (src/KernelMaker/calculateK.f90:237-323, isovpfreq). */
int dsm_cat_spectra(dsm_cat_t *cat, int npoint, const double *distance, int nout,
                    const double *coef, void *out, int out_on_device);

/* vectorFFT_double (src/KernelMaker/fourier.f90:418-450) of nseries arbitrary
 * spectra, complex128 [series][fmax-fmin+1] for indices fmin..fmax: the
 * Hermitian extension, the length-2 np1 inverse transform and the window
 * samples times exp(omegai t) / tlen * 1e3, out[series][t].  Needs no record
 * set. */
int dsm_cat_transform(dsm_cat_t *cat, int nseries, const void *spectra, int spectra_on_device,
                      double *out, int out_on_device);

/* The per-point combination matrices that turn interpolated catalogue
 * components into the h3 / h4 spectra of the kernel formulas, for
 * dsm_cat_spectra's coef argument.  Replaces
 *   rsgt2h3freq  src/KernelMaker/fourier.f90:278-320 (receiver side, 10
 *                RSGT components, compo 'Z', 'R' or 'T')
 *   tsgt2h4freq  src/KernelMaker/fourier.f90:322-415 (source side, 20 TSGT
 *                components double-dotted with the moment tensor mt(1..6))
 * ang holds per point the 12 factors of the angles module, in the order
 * crq, srq, crq2, srq2, csq, ssq, csq2, ssq2, cqs, sqs, cqs2, sqs2
 * (calculateSineCosine, src/KernelMaker/others.f90:768-826).  coef3
 * receives [point][6][10], coef4 [point][6][20] (rows rr, tt, pp, rt, rp,
 * tp); either may be NULL.  Host arithmetic only; needs no device.  For
 * compo 'T' the pp row is minus the tt row (the reference negates the
 * previous call's h3(3), fourier.f90:314). */
int dsm_cat_h3h4_coef(int npoint, const double *ang, char compo, const double *mt, double *coef3,
                      double *coef4);

/* Per-point isotropic sensitivity kernels from the h3 / h4 spectra, the
 * body of KernelMaker's calculateKernel after its rsgt2h3freq /
 * tsgt2h4freq (src/KernelMaker/calculateK.f90:131-235):
 *   isovpfreq  calculateK.f90:237-323  types 1, 3, 4 (P-wave speed)
 *   isovsfreq  calculateK.f90:327-518  types 5, 7, 8 (S-wave speed, Q_mu
 *              through jacobianFuji)
 *   bwfilt / rekurs / bpcoeff  src/KernelMaker/bwfilt.f90 (forward
 *              recursive Butterworth band-pass, irek = 0)
 * Per point: the frequency products (x 1e3), vectorFFT_double of each
 * product, the Butterworth filter of every filter ift = 0..nfilter, and the
 * trapezoid sum over samples nt1(ift)..nt2(ift) against coeff.
 * dsm_cat_set_kernel_params uploads what every point shares; the arrays
 * are the reference's own, in Fortran order. */
#define DSM_KER_VP 1   /* types 1, 3, 4 (isovpfreq) */
#define DSM_KER_VS 2   /* types 5, 7, 8 (isovsfreq) */
typedef struct dsm_cat_kernel_params {
    int    types;          /* DSM_KER_VP | DSM_KER_VS                          */
    int    nfilter;        /* filters 0..nfilter (nfilter < 16)               */
    const double *fclp, *fchp;   /* corner frequencies (Hz), nfilter+1 each */
    int    npoles;         /* npButterworth, 1..10                            */
    double sampling_hz;    /* samplingHz; the filter's step is 1/sampling_hz  */
    const int *nt1, *nt2;  /* integration samples per filter (same indices as
                              iwin_start/iwin_end, iwin_start <= nt1 <= nt2 <=
                              iwin_end), nfilter+1 each                      */
    int    nr;             /* radii of coeff and jacobian                      */
    int    nktype;         /* tmpker(0:nktype, ...) and coeff(.., 1:nktype, ..);
                              >= 8 (the reference's nktype is 8)              */
    const double *coeff;   /* coeff(0:nfilter, 1:nktype, 1:nr,
                              iwin_start:iwin_end), host                      */
    const void *jacobian;  /* jacobianFuji(1:nr, fmin:fmax) complex128, host;
                              needed for DSM_KER_VS                          */
} dsm_cat_kernel_params_t;

int dsm_cat_set_kernel_params(dsm_cat_t *cat, const dsm_cat_kernel_params_t *kp);

/* Kernels of npoint points.  ir[p] (0-based) selects point p's radius in
 * coeff and jacobian; h3 and h4 are complex128 [point][6][fmax-fmin+1]
 * (rr, tt, pp, rt, rp, tp, as rsgt2h3freq / tsgt2h4freq order them; e.g.
 * the output of dsm_cat_spectra with the per-point combinations), on the
 * device when spectra_on_device = 1.  ker receives tmpker(0:nktype,
 * 0:nfilter) of every point, [point][nfilter+1][nktype+1] (types not
 * computed are 0).  filtered (NULL: not written) receives the filtered
 * series duf of P, duf of S and duqf, each present type's series in that
 * order, [point][series][nfilter+1][nwin].  With out_on_device = 1, ker
 * and filtered are device pointers. */
int dsm_cat_kernels(dsm_cat_t *cat, int npoint, const int *ir, const void *h3, const void *h4,
                    int spectra_on_device, double *ker, double *filtered, int out_on_device);

/* The Butterworth filters of dsm_cat_set_kernel_params (every filter
 * ift = 0..nfilter, forward recursion of bwfilt, src/KernelMaker/bwfilt.f90)
 * applied to arbitrary window series: in [nseries][nwin], out
 * [nseries][nfilter+1][nwin] (device pointers when on_device = 1).  With
 * dsm_cat_series on the h3 / h4 matrices of dsm_cat_h3h4_coef this is
 * calculateRSGT / calculateTSGT (src/KernelMaker/calculateK.f90:1-130),
 * whose video outputs sample the filtered series every jtstep samples. */
int dsm_cat_filter(dsm_cat_t *cat, int nseries, const double *in, double *out, int on_device);

/* Per-stage device time of the last dsm_cat_series when profiling is on:
 * kern[] holds cat_interp, cat_fft, cat_window (ms, launches, algorithmic
 * bytes); ms_total covers the whole call.  After dsm_cat_kernels: ker_spec
 * (products into transform rows), ker_fft, ker_filter (segment end states,
 * their chain, the filter reruns with the trapezoid parts and their sum);
 * ms_total covers the device work between the uploads and the copies back. */
int dsm_cat_set_profiling(dsm_cat_t *cat, int on);
int dsm_cat_get_stats(const dsm_cat_t *cat, dsm_stats_t *stats);

/* Upper bound of the transform buffer (bytes, >= 1 MiB; default 2 GiB):
 * points are processed in batches that fit it. */
int dsm_cat_set_batch_bytes(dsm_cat_t *cat, size_t bytes);

int dsm_cat_destroy(dsm_cat_t *cat);
const char *dsm_cat_last_error(const dsm_cat_t *cat);

/* FP64 fused multiply-add throughput of a device (TFLOP/s, independent
 * chains, all SMs).  No counterpart in the reference; measurement support
 * for the interpolation's roofline. */
int dsm_fp64_peak(int device, double *tflops);
/* The same for FP64 tensor-core products (mma.m16n8k4.f64, independent
 * accumulators, all SMs). */
int dsm_fp64_mma_peak(int device, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* DSMSGT_H */
