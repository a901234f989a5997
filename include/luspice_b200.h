/*
 * luspice_b200.h - batched refactor-and-solve C-ABI for one B200.
 *
 * This interface is added beside the reference's headers (it replaces none
 * of them): it exposes the pattern cache, the batched persistent launch and
 * the serving loop that the reference only sketches (src/lu_static.h:73-75
 * is a stub; batching exists only as benchmarks, src/mp/batch_spmv.cu).
 *
 * Model:
 *   lusp_pattern : one sparsity pattern after host analysis (COLAMD column
 *                  order, pivoting fp64 LU that fixes P and the L/U pattern,
 *                  level schedules) and its device-resident static layout.
 *   lusp_batch   : N systems (pattern + values + right-hand side) processed
 *                  by one persistent kernel: one CTA per system, systems
 *                  taken from a device work queue, columns and rows taken in
 *                  level order inside the CTA.
 *   lusp_server  : continuous-batching request loop on top of batches.
 *
 * Index conventions: CSC inputs are 0-based (Ap[n+1], Ai[nnz] = row, Ax[nnz]
 * in the same entry order); rows may be unsorted; duplicate entries are
 * summed.  All pointers are host pointers unless the name says d_.  Every
 * function returns an int status (LUSP_OK = 0) and never throws.  A stream
 * argument is a cudaStream_t passed as void* (NULL = legacy default stream).
 */
#ifndef LUSPICE_B200_H
#define LUSPICE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    LUSP_OK = 0,
    LUSP_ESINGULAR = 1,   /* no nonzero pivot in some column */
    LUSP_EALLOC = 2,      /* host or device allocation failed */
    LUSP_EARG = 3,        /* invalid argument */
    LUSP_ECUDA = 4,       /* a CUDA call failed (see lusp_last_error) */
    LUSP_ENODEV = 5,      /* no usable sm_100 device */
    LUSP_EBUSY = 6        /* request not finished (lusp_serve_poll) */
};

/* Per-system status bits (lusp_sys_stats.status). */
enum {
    LUSP_ST_SINGULAR = 1,
    LUSP_ST_PIVOT_WEAK = 2,
    LUSP_ST_STAGNATED = 4,
    LUSP_ST_NOT_CONVERGED = 8,
    LUSP_ST_NONFINITE = 16,
    LUSP_ST_WAIT_TIMEOUT = 32,
    LUSP_ST_CAPACITY = 64,
    LUSP_ST_ESCALATED = 128,  /* result comes from the fp64 path (server
                                 re-queue, or a ladder rung) */
    LUSP_ST_SHIFTED = 256,    /* ... from the ladder's P-hard rung */
    LUSP_ST_LADDER_FULL = 512,/* the ladder had no slot left: P-fast result */
    LUSP_ST_FP16_OFF = 1024   /* inner_prec 2 asked for, the scaled range does
                                 not fit fp16: fp32 inner products used */
};

enum { LUSP_MIXED = 0, LUSP_FP64 = 1 };
/* what: bit 1 refactor, bit 2 solve; LUSP_RUN_DIRECT makes the solve a
 * plain x = Q U^-1 L^-1 P b with the stored factors (no iteration). */
enum { LUSP_RUN_REFACTOR = 1, LUSP_RUN_SOLVE = 2, LUSP_RUN_BOTH = 3, LUSP_RUN_DIRECT = 4 };

typedef struct lusp_pattern lusp_pattern;
typedef struct lusp_batch lusp_batch;
typedef struct lusp_server lusp_server;

typedef struct {
    int n, nnz_a;
    long lnnz, unnz, cap;          /* splu-convention counts; cap = merged slots */
    int ncol_levels, nfwd_levels, nbwd_levels;
    int max_col, nslices, sell_total;
    long flops;                    /* multiply-adds of one refactorization */
    long gathered;                 /* L entries gathered by one refactorization */
    unsigned long long hash;
    size_t device_bytes;
    int singular_col;              /* -1 unless creation failed as singular */
    int dense_tail;                /* columns of the dense trailing block (0: none) */
    int tail_start;                /* its first position (n when there is none) */
} lusp_pattern_info;

typedef struct {
    double min_abs_pivot, min_pivot_ratio, max_abs_u;
    double res[16];                /* ||b - A x|| / ||b|| history */
    int nres, inner_iters, outer_iters, status, singular_col;
    int rung;                      /* what produced the result: 0 the batch's own
                                      precision, 1 ladder P-safe, 2 ladder P-hard */
    /* SM cycles summed over warps: refactor waits for dependency columns,
     * gathers of their L parts, updates (0 unless the library is built with
     * -DLUSP_REFACTOR_PHASE_CYCLES=1: the clock reads cost ~3 % of the
     * refactor); refactor wall cycles of the CTA (always) */
    long long cyc_wait, cyc_gather, cyc_update, cyc_refactor;
    /* SM cycles of the solve phase (CTA wall time): L sweeps, dense-tail
     * solves, U sweeps, SpMVs, the whole solve */
    long long cyc_lsolve, cyc_tail, cyc_usolve, cyc_spmv, cyc_solve;
    /* SM cycles of the refactor's dense trailing block: panels, U-row
     * solves, trailing updates */
    long long cyc_tpanel, cyc_ttrsm, cyc_tupdate;
    /* SM cycles of the dense-tail solves: diagonal-block chains, products
     * with the block columns */
    long long cyc_tdiag, cyc_tgemv;
} lusp_sys_stats;

typedef struct {
    int prec;                      /* LUSP_MIXED (fp32 factors + GMRES-IR) or LUSP_FP64 (direct) */
    int krylov;                    /* GMRES restart length (default 30, max 64) */
    int max_outer;                 /* outer corrections (default 3) */
    double rtol;                   /* ||b-Ax||/||b|| target (default 1e-10) */
    double inner_rel;              /* inner stop vs current residual (default 1e-4: the
                                      outer loop corrects the rest; a tighter inner
                                      stop only adds preconditioner applications) */
    double stag_ratio;             /* required residual reduction per outer (default 0.5) */
    double pivot_tol;              /* frozen-pivot acceptance (default 1e-3) */
    int block_threads;             /* CTA size of the solve kernel: 0 auto (512 when the
                                      batch has at most one system per SM, else 256) */
    int ctas_per_sm;               /* solve kernel shared-memory plan target: 0 auto
                                      (1 or 2 with the same rule) */
    int solve_sweep;               /* triangular solves: 0 auto, 1 dataflow (per-row
                                      ready bits), 2 level-synchronous (barrier per
                                      level; descriptors in shared memory when they
                                      fit, else read from global memory) */
    int refactor_mode;             /* gathers of dependency columns: 0 staged in
                                      shared memory by asynchronous copies with
                                      precomputed relative slots, 1 loaded per
                                      dependency with a search of the column's rows */
    int inner_prec;                /* A in the inner GMRES products (mixed path):
                                      0 fp32 values (default), 1 fp64 values (first
                                      escalation step for ill-conditioned systems),
                                      2 Ruiz-scaled fp16 values where every scaled
                                      nonzero lies in the fp16 normal range, checked
                                      per system on the device at each solve (else
                                      fp32, with LUSP_ST_FP16_OFF) */
    double xtol;                   /* forward-error target: the refinement stops when
                                      the residual is <= rtol and the error estimated
                                      from the last two corrections is <= xtol
                                      (default 1e-8) */
    int refactor_threads;          /* CTA size of the refactorization kernel: 0 auto
                                      (768 when the batch has at most one system per
                                      SM, else 512), or 64..1024, a multiple of 32 */
    int refactor_cluster;          /* CTAs (one thread-block cluster) that share one
                                      system's refactorization: 0 auto (2 when every
                                      system of the batch gets its own pair of SMs,
                                      else 1), or 1..8 */
    int ladder;                    /* device-side escalation in the same launch, for a
                                      LUSP_MIXED system whose solve fails (a status
                                      failure bit, or a final residual above rtol):
                                      0 off (default); 1 P-safe: refactor in fp64 and
                                      solve by GMRES-IR with the fp64 factor; 2 P-hard:
                                      the fp64 factor of A + hard_shift diag|A(i,i)|
                                      (the residual still uses A); 3 P-safe, then
                                      P-hard for the systems P-safe fails */
    int ladder_slots;              /* systems the ladder takes per launch: 0 auto (all
                                      systems up to 256, else max(256, nsys / 8)); a
                                      failed system beyond them keeps its P-fast result
                                      with LUSP_ST_LADDER_FULL */
    double factor_shift;           /* factor A + factor_shift diag|A(i,i)| instead of A
                                      (the residual still uses A; default 0) */
    double hard_shift;             /* the P-hard rung's shift (default 1e-7) */
    int refactor_spread;           /* CTAs that share one system's refactorization
                                      anywhere on the GPU, synchronizing through
                                      global memory, for batches of a few large
                                      systems: 0 auto (every SM for a batch of at
                                      most SMs / 8 systems with at least 16 M
                                      gathered updates each), -1 never, > 0 that
                                      many CTAs per system (at most SMs / nsys) */
} lusp_batch_opts;

/* ---- library ---- */
const char *lusp_last_error(void);
const char *lusp_version(void);
int lusp_device_count(void);

/* ---- patterns ---- */
/* q: column order (NULL -> COLAMD computed here).  Ax: the values used to
 * choose pivots (the first Newton step).  On LUSP_ESINGULAR *out is NULL
 * and lusp_last_error names the column. */
int lusp_pattern_create(int n, const int *Ap, const int *Ai, const double *Ax,
                        const int *q, lusp_pattern **out);
/* As lusp_pattern_create, with the size of the dense trailing block: the
 * last dense_tail columns (and rows) are refactored and solved as one dense
 * block (at most 768; -1: chosen by a cost model, which lusp_pattern_create
 * uses; 0: none).  The factor values are the same either way. */
int lusp_pattern_create_ex(int n, const int *Ap, const int *Ai, const double *Ax,
                           const int *q, int dense_tail, lusp_pattern **out);
void lusp_pattern_destroy(lusp_pattern *p);
int lusp_pattern_get_info(const lusp_pattern *p, lusp_pattern_info *info);
/* pinv[orig_row] = position; q[position] = original column. */
int lusp_pattern_get_perm(const lusp_pattern *p, int *pinv, int *q);
/* merged columns in position space: cp[n+1], ri[cap], dg[n]. */
int lusp_pattern_get_structure(const lusp_pattern *p, int *cp, int *ri, int *dg);
/* column levels (level.c semantics) */
int lusp_pattern_get_levels(const lusp_pattern *p, int *col_level);

/* ---- host analysis entry points (no device needed) ---- */
int lusp_colamd(int n_row, int n_col, const int *Ap, const int *Ai,
                double knob_dense_row, double knob_dense_col, int *q);
/* Pivoting fp64 LU in splu layout (test and tooling use). Arrays sized by
 * the caller: pinv[n], Lp[n+1], Up[n+1]; Li/Lx/Ui/Ux with capacities
 * lcap/ucap (returns LUSP_EALLOC with *lnnz/*unnz set when too small).
 * Returns LUSP_OK or LUSP_ESINGULAR (*singular_col set). */
int lusp_pivot_factor(int n, const int *Ap, const int *Ai, const double *Ax,
                      const int *q, double tol, int *pinv,
                      int *Lp, int *Li, double *Lx, long lcap,
                      int *Up, int *Ui, double *Ux, long ucap,
                      long *lnnz, long *unnz, int *singular_col);

/* ---- batches ---- */
void lusp_batch_opts_default(lusp_batch_opts *o);
int lusp_batch_create(int nsys, lusp_pattern *const *pats, const lusp_batch_opts *opts,
                      lusp_batch **out);
void lusp_batch_destroy(lusp_batch *b);
/* Device buffers of system sys (valid for the batch lifetime). */
int lusp_batch_device_ptrs(lusp_batch *b, int sys, double **d_vals, double **d_rhs, double **d_x);
/* Host <-> device copies for all systems, concatenated in system order
 * (values: nnz_a of each system; rhs / x: n of each system). */
int lusp_batch_upload(lusp_batch *b, const double *vals, const double *rhs, void *stream);
int lusp_batch_download(lusp_batch *b, double *x, void *stream);
/* One persistent launch: refactor and/or solve every system. */
int lusp_batch_run(lusp_batch *b, int what, void *stream);
/* Same as lusp_batch_run, replayed from a CUDA graph captured on first use
 * (one graph per (what, stream)). */
int lusp_batch_run_graph(lusp_batch *b, int what, void *stream);
/* Copy per-system statistics to the host (synchronizes the stream). */
int lusp_batch_stats(lusp_batch *b, lusp_sys_stats *out, void *stream);
/* Merged factor values of one system (cap entries; float for LUSP_MIXED,
 * double for LUSP_FP64), synchronizing copy.  The engine's refactor keeps
 * only the strict-L part current in this layout (the solves read U, the
 * diagonal and the dense trailing block from their own arrays); this call
 * completes the array on `stream` before copying it. */
int lusp_batch_factor_values(lusp_batch *b, int sys, void *out, void *stream);
/* Device-to-device copy of all input values from src to dst (both batches
 * must hold the same patterns in the same order). */
int lusp_batch_copy_values(lusp_batch *dst, const lusp_batch *src, void *stream);
/* Device pointer to the merged factor values of one system, completed
 * (as lusp_batch_factor_values does) by a kernel on the default stream;
 * later runs leave only the strict-L part current until the next call. */
int lusp_batch_factor_device_ptr(lusp_batch *b, int sys, void **d_values);
/* Update max_outer, rtol, inner_rel, stag_ratio, pivot_tol, xtol,
 * factor_shift and hard_shift, for the ladder's rungs too (prec, krylov,
 * ladder, ladder_slots and the launch shape are fixed at creation). */
int lusp_batch_set_params(lusp_batch *b, const lusp_batch_opts *opts);
/* Kernel launches issued by the last lusp_batch_run (for accounting). */
int lusp_batch_launch_count(const lusp_batch *b);
/* on != 0: later lusp_batch_run calls (not graph replays) record CUDA events
 * on their stream around the refactor, dense-block and solve kernels;
 * lusp_batch_kernel_ms then waits for the last such run and returns the
 * three kernels' device times in ms (0 for a kernel that run did not
 * launch; LUSP_EARG while timing is off). */
int lusp_batch_time_kernels(lusp_batch *b, int on);
int lusp_batch_kernel_ms(lusp_batch *b, float *ms3);
/* Launch shape the batch chose (for reports): shape[0..9] = refactor grid,
 * refactor CTA threads, CTAs per system in one thread-block cluster, CTAs
 * per system in spread mode (0: none; the refactor_spread_kernel instance
 * runs), dense-block grid (0: no dense block) and CTA threads, solve grid
 * and CTA threads, triangular sweeps (1 dataflow, 2 level-synchronous),
 * dense-block CTAs per system (a thread-block cluster when 2). */
int lusp_batch_launch_shape(const lusp_batch *b, int *shape10);

/* ---- serving loop ----
 * Continuous batching of refactor+solve requests from concurrent callers
 * (Newton steps of Monte-Carlo and corner sweeps).  A scheduler thread keeps
 * up to `streams` persistent launches in flight; every launch packs the
 * requests that are ready when a stream frees up (any mix of patterns), so
 * requests that arrive while others run are admitted as slots free up and
 * their work overlaps on the device.  Patterns are analysed once on a
 * separate host thread and kept on the device in an LRU cache keyed by a
 * hash of (n, Ap, Ai), within hbm_budget_gb together with the launch arenas.
 * A system whose mixed-precision solve fails (IR stagnation, no
 * convergence, non-finite, weak or zero pivot) is escalated to fp64 as
 * `escalate` says: on the device in the same launch, or re-queued once
 * with an fp64 factor and GMRES-IR (LUSP_ST_ESCALATED in its result either
 * way).  Results do not
 * depend on what else is in the launch (one CTA runs each system the same
 * way). */
typedef struct {
    lusp_batch_opts solver;        /* prec = LUSP_MIXED (escalating) or LUSP_FP64 */
    int max_batch;                 /* systems per launch (default 128) */
    int streams;                   /* launches in flight (default 3) */
    double hbm_budget_gb;          /* pattern cache + arenas (default 150) */
    double arena_gb;               /* device arena per stream (default 2) */
    double staging_mb;             /* pinned host staging per stream (default 256) */
    int escalate;                  /* failed mixed systems: 0 kept as they are; 1 (default)
                                      the device ladder's P-safe rung in the same launch
                                      (lusp_batch_opts.ladder), and a system the ladder
                                      had no slot for re-queued once with an fp64 factor
                                      and GMRES-IR; 2 as 1 with P-safe then P-hard; 3
                                      only the re-queue */
    int analysis_threads;          /* host threads analysing new patterns (default 4) */
} lusp_server_opts;

typedef struct {
    int rc;                        /* LUSP_OK, LUSP_ESINGULAR (analysis), LUSP_EARG,
                                      LUSP_EALLOC (refused: larger than a stream arena or
                                      than the pattern cache's HBM budget) */
    int status;                    /* LUSP_ST_* of the final attempt */
    double latency_ms;             /* submit -> result available */
    double queue_ms;               /* submit -> launch */
    double device_ms;              /* launch that produced the result (device time) */
    double residual;               /* final ||b - A x|| / ||b|| */
    int inner_iters, outer_iters, batch_size, cache_hit, escalated, pad_;
    unsigned long long pattern_hash;
} lusp_serve_result;

typedef struct {
    long long submitted, completed, escalated, cache_hits, cache_misses, evictions, launches;
    long long patterns_resident, max_batch_seen;
    double pattern_gb;
    long long refused;             /* patterns refused by admission: larger than the
                                      pattern cache's share of hbm_budget_gb (their
                                      requests complete with LUSP_EALLOC and
                                      LUSP_ST_CAPACITY) */
    long long promoted;            /* times a pattern started its requests on the fp64
                                      factor + GMRES-IR path after two escalations in a
                                      row (one mixed trial every 16 requests) */
    long long fp64_starts;         /* requests started on that path */
} lusp_server_stats;

void lusp_server_opts_default(lusp_server_opts *o);
int lusp_server_create(const lusp_server_opts *o, lusp_server **out);
/* Waits for requests in flight, then frees everything. */
void lusp_server_destroy(lusp_server *s);
/* Copies the inputs; returns a request id >= 0, or -LUSP_E* on error. */
long long lusp_serve_submit(lusp_server *s, int n, const int *Ap, const int *Ai, const double *Ax,
                            const double *b);
/* wait_ms: 0 poll, > 0 wait at most that long, < 0 wait until done.  Returns
 * LUSP_OK with x (n doubles, may be NULL) and res filled and the request
 * released, or LUSP_EBUSY while it runs, or LUSP_EARG for an unknown id. */
int lusp_serve_poll(lusp_server *s, long long id, double *x, lusp_serve_result *res, int wait_ms);
int lusp_server_get_stats(lusp_server *s, lusp_server_stats *st);

/* ---- netlist matrix ingest (host; no device needed) ----
 * COO triplets with 1-based indices, as s0 files and dsh_symbolic carry
 * them.  cap: allocated entries. */
typedef struct {
    int n;
    long long nnz, cap;
    int *row, *col;
    double *val;
} lusp_coo;
/* s0 file (header "n <n>", "A <i> <j> <val>" lines; spmv.h's format). */
int lusp_read_s0_coo(const char *path, lusp_coo *A);
/* Matrix Market coordinate file (real, integer or pattern; general,
 * symmetric or skew-symmetric, the mirrored entries appended after each
 * stored one), square. */
int lusp_read_mtx_coo(const char *path, lusp_coo *A);
/* Floating-node list: "F <row>" lines (1-based, other lines ignored) ->
 * rows[0..*count) 0-based; LUSP_EALLOC with *count set when cap is short. */
int lusp_read_flt(const char *path, int n, int *rows, int cap, int *count);
/* pin > 0 onto the diagonal of each listed row (0-based): the first stored
 * (i, i) entry gains pin, a row without one gets a new (i, i) = pin entry
 * at the end (the replay programs' rule, bench/test_lu.c:71-93). */
int lusp_coo_pin_rows(lusp_coo *A, const int *rows, int count, double pin);
/* COO -> 0-based CSC (Ap[n+1], Ai/Ax[nnz]), entries of a column in
 * storage order, duplicates kept. */
int lusp_coo_to_csc(const lusp_coo *A, int *Ap, int *Ai, double *Ax);
void lusp_coo_free(lusp_coo *A);

/* ---- CSR SpMV with fp32 values (fp64 x, y and accumulation); the fp64
 * version is spmv_launch in spmv.h.  Device pointers. ---- */
int lusp_csr_spmv32(int n, const int *d_rowptr, const int *d_colidx, const float *d_values,
                    const double *d_x, double *d_y, void *stream);

/* ---- SELL-C-sigma SpMV (standalone, whole GPU) ---- */
typedef struct lusp_sell lusp_sell;
/* Build from a 0-based CSR: C in {8,16,32}, sigma >= C (row sort window),
 * value storage 0 = fp64, 1 = fp32, 2 = fp16 with Ruiz scaling (values are
 * stored as D_r A D_c in fp16, y = D_r^-1 (S (D_c^-1 x)); creation fails
 * with LUSP_EARG when a scaled value is outside the fp16 normal range).
 * Rows longer than max(256, 8 x the mean row length) are kept out of the
 * slices (one would set its whole slice's width) and computed in the same
 * launch by a warp each; `stored` counts slice slots plus their entries. */
int lusp_sell_create(int n, const int *rowptr, const int *colidx, const double *vals,
                     int C, int sigma, int value_kind, lusp_sell **out);
void lusp_sell_destroy(lusp_sell *s);
/* y = A x, fp64 accumulation; d_x, d_y device pointers of n doubles. */
int lusp_sell_spmv(const lusp_sell *s, const double *d_x, double *d_y, void *stream);
int lusp_sell_info(const lusp_sell *s, long *stored, long *nnz, double *fp16_scaled_min,
                   double *fp16_scaled_max);

/* ---- autotuning (measured on this GPU) ---- */
/* Times refactor + solve of nsys copies of (Ax, b) for candidate
 * configurations — dense trailing block (none, the cost model's choice,
 * half of it, larger), refactor shape (the engine's own rules, returned as
 * refactor_threads = refactor_cluster = 0, which also choose spread mode for
 * a batch of medium systems; or an explicit CTA size, the automatic one and
 * its neighbour, on cluster sizes 1 and 2), solve-kernel CTA (256, 512
 * threads) and sweep kind (level-synchronous, dataflow) — and
 * returns the fastest: *opts is updated (its other fields are kept),
 * *dense_tail is the block size to pass to lusp_pattern_create_ex, and
 * *best_ms the time of one launch.  Takes about a second per candidate
 * block size for matrices of a few thousand rows. */
int lusp_tune(int n, const int *Ap, const int *Ai, const double *Ax, const double *b, int nsys,
              lusp_batch_opts *opts, int *dense_tail, double *best_ms);
/* Fastest SELL slice height C in {8,16,32} and sort window sigma in
 * {32,256,1024} for this CSR matrix and value storage (as lusp_sell_create). */
int lusp_sell_tune(int n, const int *rowptr, const int *colidx, const double *vals, int value_kind,
                   int *C, int *sigma, double *best_us);

#ifdef __cplusplus
}
#endif

#endif /* LUSPICE_B200_H */
