/*
 * rumb: B200-native (sm_100a) subset-lattice kernels for certified random-utility (RUM) distances.
 *
 * C ABI of librumb.so. Every entry point returns an int status (RUMB_OK or an RUMB_E_* code) and
 * never aborts, traps or prints; rumb_last_error() gives the calling thread's last message.
 * Buffers are plain pointers owned by the caller: host memory unless a field says otherwise.
 * A context (rumb_ctx) owns all device memory, streams, graphs and cached lattice tables of one
 * GPU; calls on one context are serialized by the caller, except rumb_cancel, which any thread
 * may call at any time.
 *
 * Slab layout: one value per (alternative x, menu S containing x) at x * 2^(n-1) + compress(S, x),
 * compress = drop bit x and shift the higher bits down (the reference's layout,
 * solver/bm_admm/kernels.py:24-35). A slab has n * 2^(n-1) entries.
 *
 * Reference interfaces replaced (file:line in mingxiz/rum-testing-gpu):
 *   rumb_bm_solve            solve_kadmm_v2 + the certified runner's hooks
 *                            (solver/bm_admm/solver.py:148-377, solver/rum_solver.py:869-911)
 *   rumb_bm_iterate          one_iter, replayed `iters` times (solver/bm_admm/solver.py:240-254)
 *   rumb_butterfly           Bfly2.apply / butterfly_fast (solver/bm_admm/butterfly2.py:275-282,
 *                            solver/common/butterfly.py:381-422)
 *   rumb_prox                prox_all (solver/bm_admm/solver.py:66-139)
 *   rumb_push_ub64           push_to_ub64 (solver/common/transforms.py:94-98)
 *   rumb_fw_lb64             fw_lb_rows_gpu (solver/common/transforms.py:101-114)
 *   rumb_mem_info            machine.gpu_free_bytes (solver/machine.py:156-159)
 *   rumb_cg_pricer_create    StreamPricer.__init__ / the mask sweep's scaffolding
 *                            (solver/flow_cg/pricing_stream.py:270-299, solver/flow_cg/solver.py:69-77)
 *   rumb_cg_price            StreamPricer.price (solver/flow_cg/pricing_stream.py:407-412) and the mask
 *                            sweep + backtrace (solver/flow_cg/solver.py:169-200)
 */
#ifndef RUMB_H
#define RUMB_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RUMB_API __attribute__((visibility("default")))
#else
#define RUMB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define RUMB_VERSION 100

/* status codes */
#define RUMB_OK 0
#define RUMB_E_INVAL 1    /* bad argument: sizes, dtype, n out of range */
#define RUMB_E_OOM 2      /* device memory exhausted */
#define RUMB_E_CUDA 3     /* any other CUDA error (message says which) */
#define RUMB_E_TIMEOUT 4  /* a bounded device wait gave up */
#define RUMB_E_CANCEL 5   /* rumb_cancel was called */
#define RUMB_E_NODEV 6    /* no usable CUDA device */
#define RUMB_E_INTERNAL 7 /* anything else */

/* state dtypes of the ADMM iterate (the certificate is float64 in every mode) */
#define RUMB_F64 0   /* float64 state */
#define RUMB_F32 1   /* float32 state */
#define RUMB_MIXED 2 /* float32 state until progress stalls, then float64 to the end */

/* stop reasons of rumb_bm_solve */
#define RUMB_STOP_GAP_ABS 1
#define RUMB_STOP_GAP_REL 2
#define RUMB_STOP_TIME 3
#define RUMB_STOP_MAX_ITER 4
#define RUMB_STOP_UB_TARGET 5
#define RUMB_STOP_LB_TARGET 6
#define RUMB_STOP_CANCEL 7
#define RUMB_STOP_STALL 8    /* float32 state (RUMB_F32, stall_checks > 0): the bracket stopped closing */

typedef struct rumb_ctx rumb_ctx;
typedef struct rumb_bm_state rumb_bm_state;
typedef struct rumb_cg_pricer rumb_cg_pricer;

RUMB_API int rumb_version(void);
/* copies the calling thread's last error message (NUL-terminated, truncated to len) */
RUMB_API int rumb_last_error(char *buf, size_t len);

RUMB_API int rumb_ctx_create(int device, rumb_ctx **out);
RUMB_API int rumb_ctx_destroy(rumb_ctx *ctx);
/* run subsequent work on `stream` (a cudaStream_t of the context's device; NULL = the context's
 * own stream) */
RUMB_API int rumb_ctx_set_stream(rumb_ctx *ctx, void *stream);
RUMB_API int rumb_ctx_sync(rumb_ctx *ctx);
RUMB_API int rumb_mem_info(rumb_ctx *ctx, size_t *free_bytes, size_t *total_bytes);
/* ask a running solve on ctx to stop at its next check (thread-safe) */
RUMB_API int rumb_cancel(rumb_ctx *ctx);

/* ---------------------------------------------------------------- primitives (host slabs) */
/* out = the (a,b,c,d) 2x2 butterfly over the n-1 rest bits of every alternative block:
 * pair (l, l | 2^j), lo' = a*lo + b*hi, hi' = c*lo + d*hi; dtype RUMB_F64 or RUMB_F32. */
RUMB_API int rumb_butterfly(rumb_ctx *ctx, int n, int dtype, const void *in, void *out, double a, double b,
                   double c, double d);
/* rumb_butterfly with no device allocation (no counterpart in the reference). It stages the slab
 * in a 4 MiB static device array, one per device, instead of the context's scratch, so it holds
 * n <= 16 in either dtype; a larger slab returns RUMB_E_INVAL. The first call on each device looks
 * the array up (cudaGetSymbolAddress). Which kernels a call launches depends on n and dtype (n <= 5
 * takes one small butterfly kernel, larger n one transform kernel per window of the plan), and with
 * lazy module loading (CUDA's default) the first launch of a kernel can still allocate in the
 * driver: before a region where nothing may allocate, make one call for every (n, dtype) the region
 * will use. Nothing in the array has to start at zero. Every context on a device shares the array:
 * calls on one device must not overlap (they race; nothing serializes them). */
RUMB_API int rumb_butterfly_noalloc(rumb_ctx *ctx, int n, int dtype, const void *in, void *out, double a,
                                    double b, double c, double d);
/* out = the per-menu simplex prox of v (all 2^n - 1 menus); xhat holds p_hat at observed entries,
 * wmask is 1 at observed entries and 0 elsewhere. */
RUMB_API int rumb_prox(rumb_ctx *ctx, int n, int dtype, const void *v, const void *xhat, const void *wmask,
              double beta2, void *out);
/* float64 upper bound at slab iterate x (dtype of x): the point pushed to an exact unit flow;
 * ub = its distance to p on the mp observed rows, p_fit[mp] its values there (may be NULL). */
RUMB_API int rumb_push_ub64(rumb_ctx *ctx, int n, int dtype, const void *x, long long mp, const uint32_t *menu,
                   const int32_t *alt, const double *p, double *ub, double *p_fit);
/* float64 Frank-Wolfe lower bound at the point with values y[mp] on the observed rows. */
RUMB_API int rumb_fw_lb64(rumb_ctx *ctx, int n, long long mp, const uint32_t *menu, const int32_t *alt,
                 const double *y, const double *p, double *lb);

/* ---------------------------------------------------------------- BM-ADMM */
typedef struct {
    int n;               /* alternatives, 2 <= n <= 30 */
    long long mp;        /* observed (menu, alternative) rows, menus with >= 2 members */
    const uint32_t *menu;
    const int32_t *alt;
    const double *p;     /* p_hat (any finite values) */
    int on_device;       /* 1: menu, alt, p are device pointers of the context's device */
} rumb_bm_problem;

typedef struct {
    double beta;         /* penalty (beta1 = beta2) */
    double alpha;        /* over-relaxation */
    double precond_p;    /* per-bit preconditioner p of the inequality block */
    int check;           /* iterations between upper bounds */
    int lb_every;        /* upper-bound checks between lower bounds */
    long long max_iter;
    double abs_tol;      /* stop at ub - lb <= abs_tol (< 0: off) */
    double rel_tol;      /* stop at (ub - lb) / lb <= rel_tol (< 0: off) */
    double time_limit;   /* seconds from the start of the call (<= 0: none) */
    double ub_target;    /* stop once ub <= ub_target (NaN: none) */
    double lb_target;    /* stop once lb >= lb_target (NaN: none) */
    int dtype;           /* RUMB_F64, RUMB_F32 or RUMB_MIXED */
    int use_graph;       /* 1: replay each check interval as one CUDA graph */
    int stall_checks;    /* float32 state: window of checks over which the gap must keep shrinking
                            (RUMB_F32 with 0: no stall test) */
    double stall_rtol;   /* float32 state: once the gap shrank by less than this fraction over the
                            last stall_checks checks, RUMB_MIXED hands over to float64 and
                            RUMB_F32 stops with RUMB_STOP_STALL */
    int overlap_check;   /* 1 (with use_graph): each check runs on a second stream on a snapshot
                            of the state while the next interval's iterations run; a stop takes
                            effect one interval later (iters counts the work done), the bracket is
                            the check's. 0: checks in line (the reference's sequence) */
} rumb_bm_params;

typedef struct {
    double lb, ub;       /* best certified bracket on the observed rows */
    double phi;          /* distance of the last iterate (not a bound) */
    long long iters;     /* ADMM iterations run */
    long long iters_f32; /* of which in float32 (RUMB_F32 / RUMB_MIXED) */
    int stop;            /* RUMB_STOP_* */
    int n_push, n_lb;
    double setup_s, solve_s, push_s, per_iter_ms;
    double device_ms;    /* CUDA-event time of the solve on the context's stream */
    long long launches;  /* kernels the call launched (graph replays count their kernels) */
} rumb_bm_result;

/* called once per check with (iterations, seconds since the call, phi, best ub, best lb) */
typedef void (*rumb_trace_fn)(void *user, long long iter, double wall_s, double phi, double ub, double lb);

/* Device bytes one rumb_bm_solve of (n, mp, dtype) allocates: the state and scratch slabs (both
 * dtypes for RUMB_MIXED), the snapshot slab of overlapped checks, the float64 certificate slabs and
 * node arrays, the observation masks and the uploaded rows -- what the caller compares with
 * rumb_mem_info's free bytes before choosing the method. Computed without touching the device;
 * ctx may be NULL. 2 <= n <= 30, mp >= 1, else RUMB_E_INVAL. Replaces the reference's planner
 * sizing (_PLAN["bm_admm"] with _bm_admm_bytes, solver/rum_solver.py:735-770). */
RUMB_API int rumb_bm_plan(rumb_ctx *ctx, int n, long long mp, int dtype, size_t *bytes);

/* Certified solve. warm: start from a kept state (NULL: the cold start prox(xhat)); keep: if not
 * NULL, receives a new handle holding the final state (free with rumb_bm_state_destroy);
 * p_fit[mp] (may be NULL): the observed values of the best upper-bound point. */
RUMB_API int rumb_bm_solve(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par,
                  const rumb_bm_state *warm, rumb_bm_state **keep, rumb_bm_result *res, double *p_fit,
                  rumb_trace_fn trace, void *user);
RUMB_API int rumb_bm_state_destroy(rumb_bm_state *st);
/* Runs `iters` ADMM iterations from the host state (x2, s, y, z: slabs in par->dtype, float32
 * for RUMB_MIXED) and writes the state back; cold_start = 1 first sets x2 = prox(xhat), s = y = z
 * = 0. For iterate-level parity checks. */
RUMB_API int rumb_bm_iterate(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par, void *x2,
                    void *s, void *y, void *z, int iters, int cold_start);

/* ---------------------------------------------------------------- batched draws */
typedef struct {
    int slots;            /* draws resident at once; 0 = as many as fit mem_fraction of free memory */
    double mem_fraction;  /* share of free device memory the slots may take (0 = 0.8) */
    double draw_time;     /* seconds per draw (<= 0: none), of the GPU's time: the K resident draws
                             share it, so a draw stops after draw_time x K seconds of wall time */
    const double *y0;     /* NULL, or B x mp predicted fits: each draw's bracket starts from the
                             Frank-Wolfe lower bound at its y0 (certified for any y0) */
    int y0_state;         /* with y0: also write y0 into the start state's observed entries */
    double *p_fit;        /* NULL, or B x mp out: each draw's best upper-bound point on the rows */
} rumb_batch_params;

typedef struct {
    int slots;            /* draws resident at once */
    double bytes_per_slot;
    long long total_iters;/* slot-iterations run */
    double setup_s, solve_s, device_ms;
    int lo_bits;          /* transform split used */
    long long launches;   /* kernels the call launched (graph replays count their kernels) */
} rumb_batch_info;

/* B draws of one menu structure (prob->menu, prob->alt; prob->p is the structure's reference
 * point and is not solved), each to the certified bracket of par (abs_tol / rel_tol / max_iter,
 * dtype RUMB_F32 or RUMB_F64; a float32 draw whose gap stops shrinking ends with RUMB_STOP_STALL),
 * with per-draw thresholds below[b] (stop once ub <= below) and above[b] (stop once lb >= above),
 * NaN or NULL for none. P is B x mp row-major (host). Every draw starts from warm (e.g. the kept
 * state of p_hat's solve) or from the cold start. res[B] receives each draw's bracket.
 * The bootstrap's per-draw solves (solver/inference/bootstrap.py:308-335) run here together. */
RUMB_API int rumb_bm_solve_batch(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par,
                                 const rumb_batch_params *bp, int B, const double *P, const double *below,
                                 const double *above, const rumb_bm_state *warm, rumb_bm_result *res,
                                 rumb_batch_info *info);

/* ---------------------------------------------------------------- Flow-CG pricing */
/* pricing storage of the lattice values */
#define RUMB_PRICE_MASK 0 /* float32 per subset (2^n values and 2^n predecessor bytes, n <= 34) */
#define RUMB_PRICE_F32 1  /* float32 values: stored by mask when 5 * 2^n bytes fit half the free device
                           * memory (the same bits as two live rank-indexed layers, and the mask's
                           * speed), else rank-indexed with two live layers */
#define RUMB_PRICE_U16 2  /* rank-indexed, 16-bit mantissa per rank + float32 (offset, step) per 1024 ranks */
#define RUMB_PRICE_U24 3  /* rank-indexed, 24-bit mantissa per rank + float32 (offset, step) per 1024 ranks */
/* OR-ed into mode: evaluate w(x, D) by scanning x's rows in every sweep. Without it the pricer
 * builds, once, for every pair (D, x in D) the list of x's rows whose menu is a subset of D, in
 * row order (when n <= 26, the lists have < 2^32 entries and fit a quarter of the free device
 * memory), and a sweep adds exactly those rows' scores: the same float32 sums, far fewer tests. */
#define RUMB_PRICE_SCAN 16
/* OR-ed into RUMB_PRICE_F32: keep the rank-indexed two-layer storage whatever the free memory. */
#define RUMB_PRICE_STREAM 32

/* A pricer over the rows (menu bitmask, alternative) in x-major order: offsets[x]..offsets[x+1]
 * are alternative x's rows (offsets has n+1 entries, offsets[n] = mp). k_pred: predecessors are
 * kept for layers >= k_pred and the rest is solved on the sub-lattice (<= 0: n - 10).
 * fma_decode: decode block-scaled values as fma(q, step, offset) (1) or multiply-then-add (0). */
RUMB_API int rumb_cg_pricer_create(rumb_ctx *ctx, int n, long long mp, const uint64_t *menus,
                                   const int64_t *offsets, int mode, int k_pred, int fma_decode,
                                   rumb_cg_pricer **out);
/* One pricing call on float32 row scores (host memory, or device memory of the pricer's GPU when
 * on_device = 1): vmax = the longest path value (float64 decode of the stored top value),
 * rank_pos[n] = the priced ranking (rank_pos[a] = position of a, 0 = best), margin = the
 * quantization margin (0 for float32 storage), layer_step[n+1] (may be NULL) = each layer's
 * largest quantization step. */
RUMB_API int rumb_cg_price(rumb_cg_pricer *pricer, const float *scores, int on_device, double *vmax,
                           int32_t *rank_pos, double *margin, float *layer_step);
RUMB_API int rumb_cg_pricer_destroy(rumb_cg_pricer *pricer);
/* list_entries = the number of cover-list entries (-1 when the pricer scans rows), list_bytes =
 * their device bytes with the offsets. Either pointer may be NULL. (No counterpart in the
 * reference, which always scans.) */
RUMB_API int rumb_cg_pricer_info(const rumb_cg_pricer *pricer, long long *list_entries, long long *list_bytes);
/* sweep_max64 (solver/flow_cg/pricing_stream.py:236-249) on the pricer's rows: V[full] of the
 * longest path with float64 scores (host memory, the pricer's row order), two float64 layers of
 * C(n, n/2) ranks live (allocated on the first call, kept with the pricer). The Frank-Wolfe bound's
 * sweep where its float64 slab does not fit (solver/common/transforms.py:117-129). */
RUMB_API int rumb_cg_pricer_max64(rumb_cg_pricer *pricer, const double *scores, double *vmax);

/* The CG master's column bookkeeping on the pricer's GPU (replaces the host maintainers
 * solver/flow_cg/qp_bitset_incremental.py:36-141 and the column builder
 * solver/flow_cg/cg_core.py:63-80; the QP stays with the caller). alts[mp] = each row's
 * alternative and p_obs[mp] = its observed share, in the pricer's x-major row order; up to
 * max_cols columns. Columns are packed bits (W = ceil(mp / 64) words, bit s = row s). */
typedef struct rumb_cg_master rumb_cg_master;
RUMB_API int rumb_cg_master_create(rumb_cg_pricer *pricer, const int32_t *alts, const double *p_obs, int max_cols,
                                   rumb_cg_master **out);
/* Append a column: the column of the ranking rank_pos[n] (row s is 1 when its alternative is
 * the best-ranked member of its menu), or the packed column bits_in (exactly one of the two).
 * bits_out (W words, may be NULL) receives the column; gram_row (k + 1 values, may be NULL) the
 * new column's Gram entries Q[k][0..k] (popcounts; k = the new column's index). *index = k. */
RUMB_API int rumb_cg_master_add_column(rumb_cg_master *master, const int32_t *rank_pos, const uint64_t *bits_in,
                                       uint64_t *bits_out, double *gram_row, int *index);
/* p_out += sum_t delta[t] V[:, cols[t]] with cols increasing, each row adding in that order (the
 * host maintainer's float64 sums, bit for bit), then the residual p_obs - p_out as float32 for the
 * next pricing. */
RUMB_API int rumb_cg_master_apply(rumb_cg_master *master, const int32_t *cols, const double *delta, int count);
/* Price the current residual with the master's pricer (rumb_cg_price's outputs). */
RUMB_API int rumb_cg_master_price(rumb_cg_master *master, double *vmax, int32_t *rank_pos, double *margin);
/* p_out[mp] to host memory. */
RUMB_API int rumb_cg_master_p_out(rumb_cg_master *master, double *out);
RUMB_API int rumb_cg_master_destroy(rumb_cg_master *master);

/* ---------------------------------------------------------------- bootstrap draws
 * Resampled shares of a respondent panel on the GPU (replaces the host block builder
 * solver/inference/draws.py:273-285 and the screen solver/inference/bootstrap.py:290-306).
 * B draws, each a row of R respondent weights W (row-major B x R; integer counts). Respondent r
 * was offered menu u offered_count times and chose row j chose_count times, given as lists:
 * offered_ptr[u]..offered_ptr[u+1] index (offered_resp, offered_count) for menu u (n_menus + 1
 * offsets), chose_ptr[j]..chose_ptr[j+1] index (chose_resp, chose_count) for row j (M + 1
 * offsets); row_menu[j] = row j's menu. Draw b's row j is chose / seen with
 * seen = sum_r W[b, r] offered[r, row_menu[j]] and chose = sum_r W[b, r] chose[r, j], and p_hat[j]
 * where seen <= 0 (bit for bit the host's values: the sums are exact). At most 20,480
 * respondents. All arrays are host memory; create copies them to the context's GPU. */
typedef struct rumb_draws rumb_draws;
RUMB_API int rumb_draws_create(rumb_ctx *ctx, long long B, int R, long long M, int n_menus, const double *W,
                               const int64_t *offered_ptr, const int32_t *offered_resp,
                               const double *offered_count, const int64_t *chose_ptr, const int32_t *chose_resp,
                               const double *chose_count, const int32_t *row_menu, const double *p_hat,
                               rumb_draws **out);
/* The draws idx[0..count) as rows of out (count x M, host): perturbed = 1 gives
 * p_hat + scale (p_b - p_hat) (the Hong-Li perturbation, scale = eps_n r_n), 0 the shares p_b. */
RUMB_API int rumb_draws_rows(rumb_draws *draws, const int64_t *idx, long long count, int perturbed, double scale,
                             double *out);
/* The screen over all B draws: dev[b] = ||p_b - p_hat|| and, with fit (M values, a RUM point),
 * ub[b] = ||p_hat + scale (p_b - p_hat) - fit||, an upper bound of draw b's distance. dev or ub
 * may be NULL; ub needs fit. The norms are float64 sums in a fixed order (equal to a host sum
 * to rounding). */
RUMB_API int rumb_draws_screen(rumb_draws *draws, const double *fit, double scale, double *dev, double *ub);
RUMB_API int rumb_draws_destroy(rumb_draws *draws);

/* ---------------------------------------------------------------- profiling */
typedef struct {
    char name[64];            /* kernel and launch shape */
    long long launches;
    double total_ms;          /* CUDA-event time summed over the launches */
    double bytes_per_launch;  /* algorithmic bytes one launch must move */
    int graph;                /* 1: timed inside the replayed CUDA graph; 0: eager launches */
} rumb_kernel_stat;

/* Runs `warmup` untimed ADMM iterations from the cold start, then captures `iters` iterations
 * (plus one float64 check when par->lb_every > 0) as a CUDA graph with an event pair around every
 * kernel launch, replays it twice and reports per kernel of the second replay: launches, total
 * time and algorithmic bytes per launch -- the kernels timed as a solve's graph replays run them
 * (where the driver cannot time a graph's events, eager launches instead; `graph` says which).
 * Fills at most cap entries. This is the library's counterpart of the reference's per-phase
 * timers (solver/flow_cg/solver.py:174-188). */
RUMB_API int rumb_bm_profile(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par, int warmup,
                             int iters, rumb_kernel_stat *stats, int cap, int *count);

/* ---------------------------------------------------------------- learned warm start
 * No counterpart in the reference. A small multilayer perceptron (BF16 weights and activations,
 * FP32 accumulation and master weights, GELU after every layer but the last, mean-squared-error
 * loss, Adam) whose matrix products run on the tensor cores (tcgen05); the bootstrap trains it on
 * solved draws to predict a new draw's fitted cells. */
typedef struct rumb_mlp rumb_mlp;

/* C[M x N] = A[M x K] . B[N x K]^T on the tensor cores: A and B bf16 (16-bit patterns), row-major;
 * C float32; M and N multiples of 128, K a multiple of 64. Host buffers. */
RUMB_API int rumb_gemm_bf16(rumb_ctx *ctx, int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C);
/* n_layers layers of widths dims[0] -> dims[1] -> ... -> dims[n_layers]; weights drawn
 * uniform(+-1/sqrt(fan_in)) from seed. */
RUMB_API int rumb_mlp_create(rumb_ctx *ctx, int n_layers, const int *dims, unsigned long long seed,
                             rumb_mlp **out);
RUMB_API int rumb_mlp_destroy(rumb_mlp *mlp);
/* parameters in the layout of get/set_params: per layer W (dims[l+1] x dims[l], row-major), then b */
RUMB_API int rumb_mlp_num_params(rumb_mlp *mlp, long long *count);
RUMB_API int rumb_mlp_get_params(rumb_mlp *mlp, float *params);
RUMB_API int rumb_mlp_set_params(rumb_mlp *mlp, const float *params);
/* Y[rows x dims[L]] = the network at X[rows x dims[0]] (float32 host rows) */
RUMB_API int rumb_mlp_forward(rumb_mlp *mlp, const float *X, long long rows, float *Y);
/* loss = mean over rows x dims[L] of (net(X) - T)^2 and, if grad is not NULL, its gradient in the
 * parameter layout (rows <= 16384) */
RUMB_API int rumb_mlp_loss_grad(rumb_mlp *mlp, const float *X, const float *T, long long rows, double *loss,
                                float *grad);
/* epochs of Adam (lr) over shuffled mini-batches of `batch` rows; loss = the last epoch's mean */
RUMB_API int rumb_mlp_train(rumb_mlp *mlp, const float *X, const float *T, long long rows, int epochs, int batch,
                            double lr, unsigned long long seed, double *loss);

#ifdef __cplusplus
}
#endif
#endif
