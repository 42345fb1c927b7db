// Internal entry points of the BM-ADMM translation unit (called by the C ABI in api.cu).
#pragma once
#include "ctx.cuh"

namespace rumb {
size_t bm_plan_bytes(int n, ll mp, int dtype);
int bm_solve(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, const rumb_bm_state *warm,
             rumb_bm_state **keep, rumb_bm_result *out, double *p_fit, rumb_trace_fn trace, void *user);
int bm_iterate(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, void *x2, void *s, void *y, void *z,
               int iters, int cold);
int butterfly_host(Ctx &c, int n, int dtype, const void *in, void *out, double a, double b, double cc, double d);
int butterfly_noalloc_host(Ctx &c, int n, int dtype, const void *in, void *out, double a, double b, double cc,
                           double d);
int prox_host(Ctx &c, int n, int dtype, const void *v, const void *xhat, const void *wmask, double beta2, void *out);
int push_ub64_host(Ctx &c, int n, int dtype, const void *x, ll mp, const uint32_t *menu, const int32_t *alt,
                   const double *p, double *ub, double *p_fit);
int fw_lb64_host(Ctx &c, int n, ll mp, const uint32_t *menu, const int32_t *alt, const double *y, const double *p,
                 double *lb);
int bm_profile(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, int warmup, int iters, rumb_kernel_stat *stats,
               int cap, int *count);
int bm_solve_batch(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, const rumb_batch_params *bp, int B,
                   const double *P, const double *below, const double *above, const rumb_bm_state *warm,
                   rumb_bm_result *out, rumb_batch_info *info);
}  // namespace rumb
