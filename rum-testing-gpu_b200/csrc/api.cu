// The C ABI of librumb.so (include/rumb.h): argument checks, the context, error capture.
// Every entry point catches everything, records a message for rumb_last_error and returns a
// status code; nothing here aborts, traps or prints.
#include <cstdio>
#include <cstring>
#include <new>

#include "bm.cuh"
#include "cgmaster.cuh"
#include "ctx.cuh"
#include "draws.cuh"
#include "mlp.cuh"
#include "pricer.cuh"

namespace rumb {
static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace rumb

using rumb::Error;

#define RUMB_API_BEGIN try {
#define RUMB_API_END                                                   \
    }                                                                  \
    catch (const Error &e) {                                           \
        rumb::set_last_error(e.what());                                \
        return e.code;                                                 \
    }                                                                  \
    catch (const std::bad_alloc &) {                                   \
        rumb::set_last_error("host memory exhausted");                 \
        return RUMB_E_OOM;                                             \
    }                                                                  \
    catch (const std::exception &e) {                                  \
        rumb::set_last_error(e.what());                                \
        return RUMB_E_INTERNAL;                                        \
    }                                                                  \
    catch (...) {                                                      \
        rumb::set_last_error("unknown error");                         \
        return RUMB_E_INTERNAL;                                        \
    }

#define NEED_CTX(ctx)                                                  \
    if (!(ctx)) rumb::fail(RUMB_E_INVAL, "context is NULL");           \
    rumb::DeviceGuard _dg((ctx)->c.device)

extern "C" {

int rumb_version(void) { return RUMB_VERSION; }

int rumb_last_error(char *buf, size_t len) {
    if (!buf || len == 0) return RUMB_E_INVAL;
    std::snprintf(buf, len, "%s", rumb::g_last_error.c_str());
    return RUMB_OK;
}

int rumb_ctx_create(int device, rumb_ctx **out) {
    RUMB_API_BEGIN
    if (!out) rumb::fail(RUMB_E_INVAL, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        rumb::fail(RUMB_E_NODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (device < 0 || device >= count) rumb::fail(RUMB_E_INVAL, "device index out of range");
    rumb::DeviceGuard dg(device);
    rumb_ctx *c = new rumb_ctx();
    c->c.device = device;
    try {
        RUMB_CUDA(cudaStreamCreateWithFlags(&c->c.own, cudaStreamNonBlocking));
        RUMB_CUDA(cudaEventCreateWithFlags(&c->c.ev_a, cudaEventDisableTiming));
        RUMB_CUDA(cudaEventCreateWithFlags(&c->c.ev_b, cudaEventDisableTiming));
    } catch (...) {
        delete c;
        throw;
    }
    *out = c;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_ctx_destroy(rumb_ctx *ctx) {
    RUMB_API_BEGIN
    if (!ctx) return RUMB_OK;
    {
        rumb::DeviceGuard dg(ctx->c.device);
        cudaStreamSynchronize(ctx->c.own);
        ctx->c.bm64.reset();
        ctx->c.bm32.reset();
        ctx->c.batch64.reset();
        ctx->c.batch32.reset();
        ctx->c.cert.reset();
        ctx->c.scratch.reset();
        ctx->c.layers.clear();
        if (ctx->c.aux) {
            cudaStreamSynchronize(ctx->c.aux);
            cudaStreamDestroy(ctx->c.aux);
        }
        if (ctx->c.ev_snap) cudaEventDestroy(ctx->c.ev_snap);
        if (ctx->c.ev_done) cudaEventDestroy(ctx->c.ev_done);
        if (ctx->c.res_host) cudaFreeHost(ctx->c.res_host);
        if (ctx->c.ev_a) cudaEventDestroy(ctx->c.ev_a);
        if (ctx->c.ev_b) cudaEventDestroy(ctx->c.ev_b);
        if (ctx->c.own) cudaStreamDestroy(ctx->c.own);
    }
    delete ctx;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_ctx_set_stream(rumb_ctx *ctx, void *stream) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    ctx->c.user = reinterpret_cast<cudaStream_t>(stream);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_ctx_sync(rumb_ctx *ctx) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    RUMB_CUDA(cudaStreamSynchronize(ctx->c.own));
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mem_info(rumb_ctx *ctx, size_t *free_bytes, size_t *total_bytes) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    size_t f = 0, t = 0;
    RUMB_CUDA(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cancel(rumb_ctx *ctx) {
    if (!ctx) return RUMB_E_INVAL;
    ctx->c.cancel.store(1);
    return RUMB_OK;
}

int rumb_butterfly(rumb_ctx *ctx, int n, int dtype, const void *in, void *out, double a, double b, double c,
                   double d) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    return rumb::butterfly_host(ctx->c, n, dtype, in, out, a, b, c, d);
    RUMB_API_END
}

int rumb_butterfly_noalloc(rumb_ctx *ctx, int n, int dtype, const void *in, void *out, double a, double b,
                           double c, double d) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    return rumb::butterfly_noalloc_host(ctx->c, n, dtype, in, out, a, b, c, d);
    RUMB_API_END
}

int rumb_prox(rumb_ctx *ctx, int n, int dtype, const void *v, const void *xhat, const void *wmask, double beta2,
              void *out) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    return rumb::prox_host(ctx->c, n, dtype, v, xhat, wmask, beta2, out);
    RUMB_API_END
}

int rumb_push_ub64(rumb_ctx *ctx, int n, int dtype, const void *x, long long mp, const uint32_t *menu,
                   const int32_t *alt, const double *p, double *ub, double *p_fit) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    return rumb::push_ub64_host(ctx->c, n, dtype, x, mp, menu, alt, p, ub, p_fit);
    RUMB_API_END
}

int rumb_fw_lb64(rumb_ctx *ctx, int n, long long mp, const uint32_t *menu, const int32_t *alt, const double *y,
                 const double *p, double *lb) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    return rumb::fw_lb64_host(ctx->c, n, mp, menu, alt, y, p, lb);
    RUMB_API_END
}

int rumb_bm_plan(rumb_ctx *ctx, int n, long long mp, int dtype, size_t *bytes) {
    (void)ctx;
    RUMB_API_BEGIN
    if (!bytes) rumb::fail(RUMB_E_INVAL, "bm_plan: bytes is NULL");
    *bytes = rumb::bm_plan_bytes(n, mp, dtype);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_bm_solve(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par, const rumb_bm_state *warm,
                  rumb_bm_state **keep, rumb_bm_result *res, double *p_fit, rumb_trace_fn trace, void *user) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    if (keep) *keep = nullptr;
    return rumb::bm_solve(ctx->c, prob, par, warm, keep, res, p_fit, trace, user);
    RUMB_API_END
}

int rumb_bm_state_destroy(rumb_bm_state *st) {
    RUMB_API_BEGIN
    if (!st) return RUMB_OK;
    rumb::DeviceGuard dg(st->device);
    delete st;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_bm_iterate(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par, void *x2, void *s,
                    void *y, void *z, int iters, int cold_start) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    if (!x2 || !s || !y || !z) rumb::fail(RUMB_E_INVAL, "state buffers must not be NULL");
    if (iters < 0) rumb::fail(RUMB_E_INVAL, "iters must be >= 0");
    return rumb::bm_iterate(ctx->c, prob, par, x2, s, y, z, iters, cold_start);
    RUMB_API_END
}

int rumb_bm_solve_batch(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par,
                        const rumb_batch_params *bp, int B, const double *P, const double *below, const double *above,
                        const rumb_bm_state *warm, rumb_bm_result *res, rumb_batch_info *info) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    return rumb::bm_solve_batch(ctx->c, prob, par, bp, B, P, below, above, warm, res, info);
    RUMB_API_END
}

int rumb_bm_profile(rumb_ctx *ctx, const rumb_bm_problem *prob, const rumb_bm_params *par, int warmup, int iters,
                    rumb_kernel_stat *stats, int cap, int *count) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    if (iters < 1) rumb::fail(RUMB_E_INVAL, "iters must be >= 1");
    return rumb::bm_profile(ctx->c, prob, par, warmup, iters, stats, cap, count);
    RUMB_API_END
}

int rumb_cg_pricer_create(rumb_ctx *ctx, int n, long long mp, const uint64_t *menus, const int64_t *offsets,
                          int mode, int k_pred, int fma_decode, rumb_cg_pricer **out) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    if (!out) rumb::fail(RUMB_E_INVAL, "out is NULL");
    *out = nullptr;
    ctx->c.join_in();
    rumb_cg_pricer *h = new rumb_cg_pricer();
    try {
        h->p = rumb::pricer_create(ctx->c, n, mp, menus, offsets, mode, k_pred, fma_decode);
    } catch (...) {
        delete h;
        throw;
    }
    h->device = ctx->c.device;
    ctx->c.join_out();
    *out = h;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_price(rumb_cg_pricer *pr, const float *scores, int on_device, double *vmax, int32_t *rank_pos,
                  double *margin, float *layer_step) {
    RUMB_API_BEGIN
    if (!pr || !pr->p) rumb::fail(RUMB_E_INVAL, "pricer is NULL");
    if (!scores || !vmax || !rank_pos || !margin) rumb::fail(RUMB_E_INVAL, "NULL output");
    rumb::DeviceGuard dg(pr->device);
    rumb::pricer_price(pr->p, scores, on_device, vmax, rank_pos, margin, layer_step);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_pricer_max64(rumb_cg_pricer *pr, const double *scores, double *vmax) {
    RUMB_API_BEGIN
    if (!pr || !pr->p) rumb::fail(RUMB_E_INVAL, "pricer is NULL");
    if (!scores || !vmax) rumb::fail(RUMB_E_INVAL, "scores / vmax must not be NULL");
    rumb::DeviceGuard dg(pr->device);
    rumb::pricer_max64(pr->p, scores, vmax);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_pricer_info(const rumb_cg_pricer *pr, long long *list_entries, long long *list_bytes) {
    RUMB_API_BEGIN
    if (!pr || !pr->p) rumb::fail(RUMB_E_INVAL, "pricer is NULL");
    rumb::pricer_info(pr->p, list_entries, list_bytes);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_pricer_destroy(rumb_cg_pricer *pr) {
    RUMB_API_BEGIN
    if (!pr) return RUMB_OK;
    {
        rumb::DeviceGuard dg(pr->device);
        rumb::pricer_destroy(pr->p);
    }
    delete pr;
    return RUMB_OK;
    RUMB_API_END
}

// ---------------------------------------------------------------- CG master
#define NEED_MASTER(h)                                                 \
    if (!(h) || !(h)->m) rumb::fail(RUMB_E_INVAL, "master is NULL");  \
    rumb::DeviceGuard _dg((h)->device)

int rumb_cg_master_create(rumb_cg_pricer *pr, const int32_t *alts, const double *p_obs, int max_cols,
                          rumb_cg_master **out) {
    RUMB_API_BEGIN
    if (!pr || !pr->p) rumb::fail(RUMB_E_INVAL, "pricer is NULL");
    if (!out) rumb::fail(RUMB_E_INVAL, "out is NULL");
    *out = nullptr;
    rumb::DeviceGuard dg(pr->device);
    rumb_cg_master *h = new rumb_cg_master();
    try {
        h->m = rumb::cgmaster_create(pr->p, alts, p_obs, max_cols);
    } catch (...) {
        delete h;
        throw;
    }
    h->device = pr->device;
    *out = h;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_master_add_column(rumb_cg_master *h, const int32_t *rank_pos, const uint64_t *bits_in, uint64_t *bits_out,
                              double *gram_row, int *index) {
    RUMB_API_BEGIN
    NEED_MASTER(h);
    int k = rumb::cgmaster_add_column(h->m, rank_pos, bits_in, bits_out, gram_row);
    if (index) *index = k;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_master_apply(rumb_cg_master *h, const int32_t *cols, const double *delta, int count) {
    RUMB_API_BEGIN
    NEED_MASTER(h);
    rumb::cgmaster_apply(h->m, cols, delta, count);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_master_price(rumb_cg_master *h, double *vmax, int32_t *rank_pos, double *margin) {
    RUMB_API_BEGIN
    NEED_MASTER(h);
    if (!vmax || !rank_pos || !margin) rumb::fail(RUMB_E_INVAL, "NULL output");
    rumb::cgmaster_price(h->m, vmax, rank_pos, margin);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_master_p_out(rumb_cg_master *h, double *out) {
    RUMB_API_BEGIN
    NEED_MASTER(h);
    if (!out) rumb::fail(RUMB_E_INVAL, "out is NULL");
    rumb::cgmaster_p_out(h->m, out);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_cg_master_destroy(rumb_cg_master *h) {
    RUMB_API_BEGIN
    if (!h) return RUMB_OK;
    {
        rumb::DeviceGuard dg(h->device);
        rumb::cgmaster_destroy(h->m);
    }
    delete h;
    return RUMB_OK;
    RUMB_API_END
}

// ---------------------------------------------------------------- bootstrap draws
int rumb_draws_create(rumb_ctx *ctx, long long B, int R, long long M, int n_menus, const double *W,
                      const int64_t *offered_ptr, const int32_t *offered_resp, const double *offered_count,
                      const int64_t *chose_ptr, const int32_t *chose_resp, const double *chose_count,
                      const int32_t *row_menu, const double *p_hat, rumb_draws **out) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    if (!out) rumb::fail(RUMB_E_INVAL, "out is NULL");
    *out = nullptr;
    ctx->c.join_in();
    rumb_draws *h = new rumb_draws();
    try {
        h->d = rumb::draws_create(ctx->c, B, R, M, n_menus, W, offered_ptr, offered_resp, offered_count, chose_ptr,
                                  chose_resp, chose_count, row_menu, p_hat);
    } catch (...) {
        delete h;
        throw;
    }
    h->device = ctx->c.device;
    ctx->c.join_out();
    *out = h;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_draws_rows(rumb_draws *d, const int64_t *idx, long long count, int perturbed, double scale, double *out) {
    RUMB_API_BEGIN
    if (!d || !d->d) rumb::fail(RUMB_E_INVAL, "draws is NULL");
    rumb::DeviceGuard dg(d->device);
    rumb::draws_rows(d->d, idx, count, perturbed, scale, out);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_draws_screen(rumb_draws *d, const double *fit, double scale, double *dev, double *ub) {
    RUMB_API_BEGIN
    if (!d || !d->d) rumb::fail(RUMB_E_INVAL, "draws is NULL");
    rumb::DeviceGuard dg(d->device);
    rumb::draws_screen(d->d, fit, scale, dev, ub);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_draws_destroy(rumb_draws *d) {
    RUMB_API_BEGIN
    if (!d) return RUMB_OK;
    {
        rumb::DeviceGuard dg(d->device);
        rumb::draws_destroy(d->d);
    }
    delete d;
    return RUMB_OK;
    RUMB_API_END
}

// ---------------------------------------------------------------- tensor-core GEMM and MLP
struct rumb_mlp {
    rumb_ctx *ctx = nullptr;
    rumb::Mlp *m = nullptr;
};

#define NEED_MLP(h)                                                    \
    if (!(h) || !(h)->m) rumb::fail(RUMB_E_INVAL, "mlp is NULL");      \
    rumb::DeviceGuard _dg((h)->ctx->c.device)

int rumb_gemm_bf16(rumb_ctx *ctx, int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    return rumb::gemm_bf16_host(ctx->c, M, N, K, A, B, C);
    RUMB_API_END
}

int rumb_mlp_create(rumb_ctx *ctx, int n_layers, const int *dims, unsigned long long seed, rumb_mlp **out) {
    RUMB_API_BEGIN
    NEED_CTX(ctx);
    if (!out) rumb::fail(RUMB_E_INVAL, "out is NULL");
    *out = nullptr;
    rumb_mlp *h = new rumb_mlp();
    h->ctx = ctx;
    try {
        h->m = rumb::mlp_create(ctx->c, n_layers, dims, seed);
    } catch (...) {
        delete h;
        throw;
    }
    *out = h;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mlp_destroy(rumb_mlp *h) {
    RUMB_API_BEGIN
    if (!h) return RUMB_OK;
    if (h->m) {
        rumb::DeviceGuard dg(h->ctx->c.device);
        rumb::mlp_destroy(h->m);
    }
    delete h;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mlp_num_params(rumb_mlp *h, long long *count) {
    RUMB_API_BEGIN
    NEED_MLP(h);
    if (!count) rumb::fail(RUMB_E_INVAL, "count is NULL");
    *count = rumb::mlp_num_params(*h->m);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mlp_get_params(rumb_mlp *h, float *params) {
    RUMB_API_BEGIN
    NEED_MLP(h);
    if (!params) rumb::fail(RUMB_E_INVAL, "params is NULL");
    rumb::mlp_get_params(*h->m, params, false);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mlp_set_params(rumb_mlp *h, const float *params) {
    RUMB_API_BEGIN
    NEED_MLP(h);
    if (!params) rumb::fail(RUMB_E_INVAL, "params is NULL");
    rumb::mlp_set_params(*h->m, params);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mlp_forward(rumb_mlp *h, const float *X, long long rows, float *Y) {
    RUMB_API_BEGIN
    NEED_MLP(h);
    rumb::mlp_forward(*h->m, X, rows, Y);
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mlp_loss_grad(rumb_mlp *h, const float *X, const float *T, long long rows, double *loss, float *grad) {
    RUMB_API_BEGIN
    NEED_MLP(h);
    double l = rumb::mlp_loss_grad(*h->m, X, T, rows, grad);
    if (loss) *loss = l;
    return RUMB_OK;
    RUMB_API_END
}

int rumb_mlp_train(rumb_mlp *h, const float *X, const float *T, long long rows, int epochs, int batch, double lr,
                   unsigned long long seed, double *loss) {
    RUMB_API_BEGIN
    NEED_MLP(h);
    double l = rumb::mlp_train(*h->m, X, T, rows, epochs, batch, lr, seed);
    if (loss) *loss = l;
    return RUMB_OK;
    RUMB_API_END
}

}  // extern "C"
