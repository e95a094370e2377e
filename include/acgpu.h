/*
 * acgpu — C ABI of the B200 solve phase for Laplacians.jl's approxchol_lap.
 *
 * The reference (Laplacians.jl v1.4.1) builds, in Julia,
 *     f = approxchol_lap(a; tol, maxits, maxtime, verbose, pcgIts, params)
 * (src/approxChol.jl:1522-1545) whose closure (src/approxChol.jl:1624) runs
 *     pcg(lap(a), b .- mean(b), b -> LDLsolver(ldli, b); stag_test = 5)
 * (src/pcg.jl:256-445, src/approxChol.jl:1347-1408).  This library replaces
 * that closure body: the host hands over the adjacency matrix and the LDLinv
 * factor once (acg_create), and every solve runs on the GPU (acg_solve).
 *
 * Conventions
 *   - Plain C types only.  Index arrays are int64 as Julia stores them; the
 *     `index_base` argument says whether they are 1-based (Julia) or 0-based.
 *   - Every function returns an int status: 0 = ACG_OK, > 0 = a convergence
 *     outcome of a finished solve (mirrors the reference's PCG stop reasons),
 *     < 0 = an error; acg_last_error() then holds a message (thread-local).
 *   - No exception crosses the ABI.  The caller keeps ownership of every
 *     array it passes; the library copies what it needs.
 *   - A solver handle is used by one host thread at a time.
 */
#ifndef ACGPU_H
#define ACGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define ACG_OK 0
/* convergence outcomes (>0): the solve finished and x holds the best iterate */
#define ACG_STOP_MAXITS 1      /* itcnt reached maxits            (src/pcg.jl:288)     */
#define ACG_STOP_STAG_X 2      /* al*|p|_1 < eps*|x|_1            (src/pcg.jl:308-317) */
#define ACG_STOP_STAG_R 3      /* al*|q|_1 < eps*|r|_1            (src/pcg.jl:330-338) */
#define ACG_STOP_STAG_RHO 4    /* rho stagnation test             (src/pcg.jl:370-383) */
#define ACG_STOP_INF 5         /* rho or beta infinite            (src/pcg.jl:385-400) */
#define ACG_STOP_STAG_P 6      /* beta*|p|_1 < eps*|z|_1          (src/pcg.jl:406-414) */
#define ACG_STOP_MAXTIME 7     /* wall time above maxtime         (src/pcg.jl:425-430) */
/* errors (<0) */
#define ACG_ERR_INVALID -1     /* bad argument or malformed input  */
#define ACG_ERR_NOMEM -2       /* host or device allocation failed */
#define ACG_ERR_CUDA -3        /* a CUDA runtime call failed       */
#define ACG_ERR_TIMEOUT -4     /* a bounded device wait gave up    */
#define ACG_ERR_NODEVICE -5    /* no usable sm_100 device          */
#define ACG_ERR_BUSY -6        /* admission refused (memory budget)*/

/* Last error message of the calling thread ("" if none). */
const char* acg_last_error(void);

/* ---- host: Julia-compatible random stream ------------------------------ */
/* Random.seed!(seed) of Julia 1.8 (stdlib Random, Xoshiro256++ seeded through
 * SHA-256 of the seed's 32-bit limbs).  Writes the 4-word state. */
int acg_rng_seed(uint64_t seed, uint64_t state[4]);
/* `count` draws of Julia's rand()::Float64 from `state` (advanced in place). */
int acg_rng_rand(uint64_t state[4], double* out, int64_t count);
/* SHA-256 digest, exposed for the known-answer test of the seeding path. */
int acg_sha256(const uint8_t* data, int64_t len, uint8_t out[32]);

/* ---- host: approximate Cholesky elimination ---------------------------- */
typedef struct acg_factor acg_factor;
/* approxChol(LLmatp(a)) with the default :deg order (src/approxChol.jl:864-977,
 * 102-136, 2085-2239).  `a` is the adjacency matrix in CSC form: n columns,
 * colptr[n+1] (0- or 1-based, detected from colptr[0]), sorted rowval, weights
 * nzval >= 0, structurally symmetric, zero diagonal, every vertex with an
 * edge.  Draws from `rng_state` exactly where the reference calls rand(), and
 * advances it.  On success *out owns the factor (free with acg_factor_free). */
int acg_approxchol(int64_t n, const int64_t* colptr, const int64_t* rowval,
                   const double* nzval, uint64_t rng_state[4], acg_factor** out);
/* approxChol in a fixed elimination order (src/approxChol.jl:758-862 on
 * LLMatOrd, src/approxChol.jl:203-229 and 265-294): perm (1-based, length n,
 * perm[k] = the vertex eliminated k-th) or NULL for the given order 1..n; the
 * factor comes back in the original vertex ids, as approxchol_lapGiven /
 * approxchol_lapWdeg / approxchol_lapRandom build it (src/approxChol.jl:1628-1789). */
int acg_approxchol_ordered(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                           const int64_t* perm, uint64_t rng_state[4], acg_factor** out);
/* The split/merge elimination of approxchol_lap2 (split = merge = 2 there):
 * approxChol(LLmatp(a, split), split, merge) (src/approxChol.jl:979-1157,
 * 138-183) with compressAvgCol! (src/approxChol.jl:541-600); merge < 1 is
 * approxChol(LLmatp(a, split), split) (src/approxChol.jl:1162-1322, avgCol!). */
int acg_approxchol_split(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval, int64_t split,
                         int64_t merge, uint64_t rng_state[4], acg_factor** out);
/* Opt-in, not the reference's elimination: a parallel approximate Cholesky
 * elimination in rounds.  Each round takes an independent set of live
 * vertices whose degree is a local minimum and at most max(2, the median live
 * degree) (ties by pseudo-random priorities), and eliminates the set at once
 * on `threads` host threads with
 * the reference's per-vertex step (src/approxChol.jl:888-966: merge parallel
 * edges, order by weight, sample and join neighbours).  Its random numbers are
 * keyed by (seed, vertex, entry) rather than drawn from Julia's rand() stream,
 * so the factor is a different sample than approxChol's (not bit-identical to
 * the reference); it does not depend on `threads`.  The last vertices (at
 * most 4,096, more when rounds find few vertices) are eliminated one at a
 * time in order of degree; before them the factor's dependency DAG is at most
 * `*rounds` levels deep.  Same LDLinv layout and the same requirements on `a`
 * as acg_approxchol (a connected graph). */
int acg_approxchol_parallel(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval,
                            uint64_t seed, int threads, int64_t* rounds, acg_factor** out);
/* n and F = length(ldli.fval). */
int acg_factor_dims(const acg_factor* f, int64_t* n, int64_t* nnz);
/* Copy out the LDLinv arrays in the reference layout (src/approxCholTypes.jl:73-79),
 * 1-based: col[n-1], colptr[n], rowval[F], fval[F], d[n]. */
int acg_factor_export(const acg_factor* f, int64_t* col, int64_t* colptr, int64_t* rowval,
                      double* fval, double* d);
void acg_factor_free(acg_factor* f);
/* Binary LDLinv file (little-endian): "ACGLDLI1", int64 n, int64 F, int64 1
 * (index base), then col[n-1], colptr[n], rowval[F] (int64) and fval[F], d[n]
 * (float64), the fields of LDLinv (src/approxCholTypes.jl:73-79) as Julia
 * stores them.  The reference has no such file: it lets a host that runs the
 * reference's own elimination hand the factor over, and factors be cached.
 * acg_ldlinv_load checks the header, the size and the structure (colptr from
 * 1 to F+1 without decreasing, ids in [1, n]); read the arrays back with
 * acg_factor_dims / acg_factor_export. */
int acg_ldlinv_save(const char* path, int64_t n, const int64_t* col, const int64_t* colptr, const int64_t* rowval,
                    const double* fval, const double* d, int64_t nnz);
int acg_ldlinv_load(const char* path, acg_factor** out);

/* ---- device solver ------------------------------------------------------ */
typedef struct acg_solver acg_solver;

/* Optional tuning knobs of acg_create (0 = automatic). */
typedef struct {
  int sweep_lanes;     /* sweep engine: 0 = sync-free dataflow sweep (one cooperative
                          launch per sweep), 1 = one launch per level          */
  int spmv_lanes;      /* lanes per row in the Laplacian mat-vec: 2, 4, 8 or 16     */
  int wide_level_min;  /* levels at least this wide get a grid launch each; runs of
                          narrower levels whose values fit in shared memory run in
                          one CTA with block barriers (default 2048)              */
  int sweep_blocks_per_sm;   /* resident blocks per SM of the single-vector sweeps (0 = by the
                                DAG: 1, 2 or 4 as the tasks per level grow)              */
  int poll_mode;             /* waits on a pending value: 0 = automatic, 1 tight+sleep,
                                2 tight only, 3 backoff                               */
  int tail;                  /* 2 = sweep the final narrow levels in one CTA from shared
                                memory (experimental); 0 = off                         */
  int batch_bwd_heavy;       /* batched sweeps: vertices with more entries than this get a
                                whole warp (0 = 8); backward and forward tables       */
  int batch_fwd_heavy;
  int batch_blocks_per_sm;   /* resident blocks per SM of the batched sweeps (0 = the
                                occupancy limit)                                       */
  int sweep_heavy;           /* single-vector sweeps: vertices with more entries than this
                                get a whole warp (0 = 16)                              */
  int dense_tail;            /* largest number of final-level vertices whose substitution
                                is replaced by a dense triangular product (0 = 4096,
                                -1 = none; at most 8192 and n/4)                       */
  int sweep_stride;          /* 1 = one value per vertex in the one-vector sweep vectors;
                                0 = one 32-byte sector per vertex (faster: values that
                                different SMs write at once never share a sector)     */
  int level_order;           /* vertex order inside a DAG level: 0 = by decreasing in-degree,
                                1 = by the caller's vertex id (keeps the caller's locality
                                for the mat-vec and the sweeps' gathers)               */
  int spin_limit;            /* polls of a pending value before a sweep wait gives up and
                                the solve returns ACG_ERR_TIMEOUT (0 = 4,194,304, a few
                                seconds)                                                */
  int test_unproduced_task;  /* testing only (0 = off): k > 0 blanks the k-th record of
                                the forward sweep tables, so its vertices' values are never
                                produced and the waits on them run out; a test of the
                                bounded waits that neither faults nor hangs the GPU     */
  double min_inner_tol;      /* mixed precision: the smallest relative residual an inner
                                FP32 solve is asked for (0 = 2e-5)                      */
} acg_options;

/* Shape of an uploaded solver. */
typedef struct {
  int64_t n;           /* vertices                                   */
  int64_t nnz_lap;     /* stored entries of lap(a) = nnz(a) + n       */
  int64_t nnz_factor;  /* F = length(ldli.fval)                       */
  int64_t levels;      /* depth of the LDLinv dependency DAG          */
  int64_t wide_levels; /* levels swept with one grid launch each (FP32 plan) */
  int64_t thin_runs;   /* runs of thin levels swept by one CTA (FP32 plan) */
  int sweep_lanes, spmv_lanes;
  int64_t device_bytes;   /* device memory held by this solver now           */
  int64_t batch_capacity; /* right-hand sides its batch buffers hold (0 = none) */
  int64_t tail_levels;    /* final levels swept by one CTA from shared memory    */
  int64_t tail_vertices;  /* vertices of those levels                           */
  int64_t dense_levels;   /* final levels replaced by the dense triangular block */
  int64_t dense_vertices; /* K: vertices of that block (0 = none)                */
} acg_stats;

/* Outcome of one solve (one right-hand side). */
typedef struct {
  int64_t iterations;  /* PCG iterations = pcgIts[1] (mixed: inner iterations summed) */
  int64_t refinements; /* FP64 refinement steps (mixed precision), 0 for FP64        */
  double relres;       /* |r|/|b| of the recursive residual when PCG stopped         */
  double best_relres;  /* smallest recursive |r|/|b| (that of the returned bestx)    */
  double true_relres;  /* |(b - mean b) - L x| / |b - mean b| of the returned x, FP64 */
  double solve_ms;     /* device time of the solve graph (CUDA events)               */
  int status;          /* 0 converged, else the ACG_STOP_* code                      */
  int levels;          /* depth of the LDLinv dependency DAG                         */
} acg_solve_info;

/* Device time of the solve's kernels (milliseconds per call). */
typedef struct {
  double spmv_ms;           /* q = L p (one launch)                          */
  double forward_ms;        /* forward LDLinv sweep (all its launches)       */
  double backward_ms;       /* backward LDLinv sweep                         */
  double iteration_ms;      /* the kernels of one PCG iteration              */
  int launches_per_iteration;
  int forward_launches;
  /* algorithmic bytes per call: every structure entry, task record and vector
     element the kernel must touch once (re-reads not counted) */
  double spmv_bytes, forward_bytes, backward_bytes;
  /* the sweep kernel alone, without the dense tail products (equal to
     forward_ms / backward_ms when the solver has no dense tail) */
  double forward_sweep_ms, backward_sweep_ms;
  double dense_ms;          /* both dense tail products (forward + backward) */
  double forward_sweep_bytes, backward_sweep_bytes, dense_bytes;
  /* the batched loop body's vector kernels, one call each (acg_time_kernels_batch
     only; 0 otherwise): p.q and |p|_1, |q|_1; the x and r update; the sums of
     y, y.r and r; the p update; and their algorithmic bytes */
  double pq_ms, update_ms, yzr_ms, pupdate_ms;
  double pq_bytes, update_bytes, yzr_bytes, pupdate_bytes;
  /* a batched solve's set-up and wrap-up (acg_time_kernels_batch only): the
     gather of the right-hand-side block into vertex-major rows, the scatter
     of x back, and one FP64 true residual b - L x of the block */
  double gather_ms, scatter_ms, true_residual_ms;
} acg_kernel_times;

/* 0 if the current CUDA device is usable (sm_100), else an error code. */
int acg_device_check(void);

/* Upload lap(a) and an LDLinv factor to the current device.
 * Replaces the captures `la = lap(a)` and `F(b) = LDLsolver(ldli, b)` of the
 * closure built at src/approxChol.jl:1597-1624.
 *   a_*: adjacency CSC (n columns, colptr[n+1], sorted rowval, nzval >= 0).
 *   ldli_*: the LDLinv arrays (src/approxCholTypes.jl:73-79) with F = ldli_nnz
 *           entries; index_base 1 for Julia arrays, 0 for 0-based ones.
 * Builds the level schedule of the factor's dependency DAG, renumbers vertices
 * by level, folds the running products of forward!/backward! into per-entry
 * coefficients, and keeps FP64 and FP32 copies on the device. */
int acg_create(int64_t n, const int64_t* a_colptr, const int64_t* a_rowval, const double* a_nzval,
               const int64_t* ldli_col, const int64_t* ldli_colptr, const int64_t* ldli_rowval,
               const double* ldli_fval, const double* ldli_d, int64_t ldli_nnz, int index_base,
               const acg_options* opts, acg_solver** out);
void acg_destroy(acg_solver* h);
int acg_solver_stats(const acg_solver* h, acg_stats* out);

/* x = f(b): the closure body of src/approxChol.jl:1624, i.e.
 * pcg(la, b .- mean(b), LDLsolver; tol, maxits, maxtime, stag_test) with the
 * stop rules of src/pcg.jl:256-445, returning bestx.  Host arrays; nrhs
 * right-hand sides stored column-major with leading dimension ldb (>= n when
 * nrhs > 1), info[nrhs] optional; more than one right-hand side is solved in
 * batched launches of up to 64 columns (each column its own PCG system).
 *   precision 0: FP64 PCG (the reference algorithm).
 *   precision 1: FP32 PCG (SpMV, LDLinv sweeps, vectors) inside FP64 iterative
 *                refinement on the true residual; tol is then on
 *                |b - L x| / |b| and maxits bounds the inner iterations.
 * Returns 0 (all converged), the largest ACG_STOP_* code, or an error (<0). */
int acg_solve(acg_solver* h, const double* b, double* x, int64_t nrhs, int64_t ldb, double tol, int64_t maxits,
              double maxtime, int stag_test, int precision, acg_solve_info* info);
/* ---- asynchronous solves (serving) ---------------------------------------
 * acg_solve_async enqueues one batched solve of 1 <= nrhs <= 64 columns of b
 * (column-major, ldb >= n; x has the same layout) and returns at once with a
 * request.  A solver runs its requests in submission order; while one solves,
 * the next one's copy in and the previous one's copy out proceed on their own
 * streams (two requests in flight per solver: a third submit first waits for
 * the oldest to finish).  b and x must stay valid until acg_wait; copies run
 * asynchronously for page-locked b and x, and x in pageable memory is filled
 * by acg_wait.  acg_poll returns 1 when the request has finished (acg_wait
 * will not block), 0 while it runs, < 0 on error.  acg_wait blocks until the
 * request has finished, fills info[nrhs] (optional), frees the request and
 * returns what acg_solve would have.  Requests still open when their solver
 * is destroyed are finished first and may still be waited.  The reference
 * has no asynchronous entry: its closure solves one vector per call
 * (src/approxChol.jl:1624, src/pcg.jl:256). */
typedef struct acg_request acg_request;
int acg_solve_async(acg_solver* h, const double* b, double* x, int64_t nrhs, int64_t ldb, double tol,
                    int64_t maxits, double maxtime, int stag_test, int precision, acg_request** out);
int acg_poll(acg_request* r);
int acg_wait(acg_request* r, acg_solve_info* info);
/* As acg_solve for one right-hand side already in device memory (on the
 * solver's device).  The solve is ordered after the work already queued on the
 * legacy default stream; a caller that wrote b_dev on a stream of its own
 * synchronizes that stream first.  Other streams are not waited for, so
 * serving loops and copies elsewhere on the GPU keep running.  Returns when x_dev
 * holds the result. */
int acg_solve_device(acg_solver* h, const double* b_dev, double* x_dev, double tol, int64_t maxits, double maxtime,
                     int stag_test, int precision, acg_solve_info* info);
/* Block of nrhs right-hand sides already in device memory (column-major,
 * leading dimension ld >= n; ordered as acg_solve_device): solved 64 at a time in one batched launch, each
 * column its own PCG system with the same stop rules as acg_solve; info[nrhs]
 * optional.  The reference solves one vector per call (src/pcg.jl:256). */
int acg_solve_batch_device(acg_solver* h, const double* b_dev, double* x_dev, int64_t nrhs, int64_t ld, double tol,
                           int64_t maxits, double maxtime, int stag_test, int precision, acg_solve_info* info);
/* ---- many graphs in one launch ------------------------------------------- */
/* The block-diagonal union of ngraphs graphs: graph g owns vertices
 * [offsets[g], offsets[g+1]) (contiguous blocks of the union adjacency a_*),
 * and the factor is the union of the graphs' LDLinv factors with vertex ids
 * shifted to the union (ncol = n - ngraphs eliminated columns: one root per
 * graph).  Every graph keeps its own PCG (FP64, its own scalars and stop
 * rules, src/pcg.jl:256-445), as blockSolver solves components
 * (src/solverInterface.jl:152-188), but all graphs share every launch. */
int acg_create_group(int64_t ngraphs, const int64_t* offsets, int64_t n, const int64_t* a_colptr,
                     const int64_t* a_rowval, const double* a_nzval, const int64_t* ldli_col, int64_t ncol,
                     const int64_t* ldli_colptr, const int64_t* ldli_rowval, const double* ldli_fval,
                     const double* ldli_d, int64_t ldli_nnz, int index_base, const acg_options* opts,
                     acg_solver** out);
/* One right-hand side per graph (b: n values of the union, host); info[ngraphs].
 * precision 0: FP64 PCG per graph; 1: each graph's FP32 PCG inside its own FP64
 * refinement on the true residual (as acg_solve's precision 1), all graphs in
 * the same launches.  A group of one graph (or any one-graph solver) is solved
 * as acg_solve does. */
int acg_solve_group(acg_solver* h, const double* b, double* x, double tol, int64_t maxits, double maxtime,
                    int stag_test, int precision, acg_solve_info* info);

/* y = LDLsolver(ldli, r) (src/approxChol.jl:1347-1366) on the device; host arrays. */
int acg_ldlsolve(acg_solver* h, const double* r, double* y, int precision);
/* y = lap(a) * x on the device (FP64 or FP32 values); host arrays. */
int acg_lap_mul(acg_solver* h, const double* x, double* y, int precision);
/* Time the solve's kernels: each captured `reps` times into a CUDA graph and
 * timed with CUDA events on the solver's stream (no reference counterpart). */
int acg_time_kernels(acg_solver* h, int precision, int reps, acg_kernel_times* out);
/* The same for the batched kernels with nrhs (<= 64) right-hand sides
 * (iteration_ms is not measured there). */
int acg_time_kernels_batch(acg_solver* h, int precision, int nrhs, int reps, acg_kernel_times* out);

/* The batched sweeps cut at given levels of the factor's dependency DAG.  For
 * each levels[i] = L: fwd_ms[i] is the forward sweep over the tasks of levels
 * 0..L and bwd_ms[i] the backward sweep over the tasks of levels >= L (the
 * swept head; the dense tail's levels are never swept), each per launch with
 * nrhs right-hand sides; fwd_tasks[i] / bwd_tasks[i] are those tasks.  Levels
 * are clamped to [0, levels - 1]; times are differences of two timings, and a
 * prefix shorter than the timing noise reads 0.  The differences between points show what
 * each range of levels costs.  Diagnostic only: it uses the batch buffers, so a
 * solver that serves answers ACG_ERR_BUSY; a group solver ACG_ERR_INVALID. */
int acg_time_sweep_levels(acg_solver* h, int precision, int nrhs, int reps, int npts, const int* levels,
                          double* fwd_ms, double* bwd_ms, int* fwd_tasks, int* bwd_tasks);

/* ---- serving loop: continuous batching on the device -------------------- */
/* The reference has no server: its closure solves one vector per call
 * (src/approxChol.jl:1624).  A serving loop turns a one-graph solver's batched
 * kernels into slots: one device-resident loop (a CUDA graph with a WHILE
 * node) runs PCG iterations for every busy slot and, between iterations,
 * admits waiting requests into free slots and hands finished solves back.
 * Requests that arrive while others are on the GPU join the running loop as
 * soon as a slot frees up; every right-hand side is its own PCG system with
 * the reference's stop rules, so a result matches the same request solved
 * alone up to the rounding of its first rho (summed in the loop body's form).
 *   acg_serve_open: `slots` columns (rounded up to 8, 16, 32 or 64) in
 *     `precision` 0 (FP64 PCG) or 1 (FP32 PCG inside FP64 refinement, each
 *     column refining on its own schedule); `queue` more requests may wait
 *     (0 = as many as slots).  Staging buffers for them are allocated here.
 *     While the loop is open the solver's batched entry points return
 *     ACG_ERR_BUSY; its one-vector entry points still work.
 *   acg_serve_submit: nrhs right-hand sides (column-major, ldb >= n when
 *     nrhs > 1), each its own solve; b is copied before the call returns; x
 *     (same layout) is written by the time acg_serve_wait returns.  Blocks
 *     while the queue is full.
 *   acg_serve_poll: 1 when every column of the ticket has finished, else 0.
 *   acg_serve_wait: blocks until then, fills info[nrhs], frees the ticket and
 *     returns what acg_solve would have.
 *   acg_serve_stats: launches of the loop so far (an idle loop ends and the
 *     next request relaunches it) and right-hand sides finished.
 *   acg_serve_close: waits for the loop to go idle and frees it; every
 *     ticket must have been waited (else ACG_ERR_BUSY).  acg_destroy closes a
 *     solver's open loop. */
typedef struct acg_server acg_server;
typedef struct acg_ticket acg_ticket;
int acg_serve_open(acg_solver* h, int precision, int slots, int queue, acg_server** out);
int acg_serve_submit(acg_server* s, const double* b, double* x, int64_t nrhs, int64_t ldb, double tol,
                     int64_t maxits, double maxtime, int stag_test, acg_ticket** out);
int acg_serve_poll(acg_ticket* t);
int acg_serve_wait(acg_ticket* t, acg_solve_info* info);
int acg_serve_stats(acg_server* s, int64_t* launches, int64_t* completed);
int acg_serve_close(acg_server* s);

/* ---- allocation-free preconditioner application ------------------------ */
/* No counterpart in the reference (its Julia LDLsolver allocates freely).
 * y_dev = LDLsolver(ldli, r_dev), as acg_ldlsolve computes it, for vectors
 * already in device memory, without allocating: every piece of scratch comes
 * from one fixed device array inside the library (ACG_NOALLOC_MAX_N vertices
 * at most, about 6.4 MB, reserved on each GPU that loads the library until
 * the process exits).  Meant for callers that must not allocate while they
 * solve: a serving loop whose device memory is a fixed pool sized at start-up,
 * a host runtime whose own allocator owns the GPU's memory, or a caller that
 * cannot let cudaMalloc/cudaFree synchronize the device under its other
 * streams.  The scratch address is looked up once per device inside
 * acg_create (set-up).  Work is enqueued on `stream` (a cudaStream_t; NULL =
 * the legacy default stream); the call then waits for it and reports a sweep
 * that gave up as ACG_ERR_TIMEOUT.  The array keeps the last call's contents;
 * each call clears the state that must start at zero (the stop flags and
 * reduction tickets) itself.  Every call shares the one array: calls whose work
 * overlaps on the GPU (different streams, or different solvers, at the same
 * time) race and corrupt each other's results.  Graphs with more than
 * ACG_NOALLOC_MAX_N vertices are rejected with ACG_ERR_INVALID, and so are a
 * group solver (acg_create_group), a current device other than the solver's
 * and a stream that belongs to another device: the call checks these on the
 * host before it enqueues anything. */
#define ACG_NOALLOC_MAX_N 131072
int acg_ldlsolve_noalloc(acg_solver* h, const double* r_dev, double* y_dev, int precision, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ACGPU_H */
