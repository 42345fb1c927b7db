// Internal interface of the Flow-CG pricer translation unit.
#pragma once
#include "ctx.cuh"

namespace rumb {
struct Pricer;
Pricer *pricer_create(Ctx &c, int n, ll mp, const uint64_t *menus, const int64_t *offsets, int mode, int k_pred,
                      int fma_decode);
void pricer_destroy(Pricer *P);
void pricer_price(Pricer *P, const float *scores, int on_device, double *vmax, int32_t *rank_pos, double *margin,
                  float *layer_step_out);
int pricer_device(const Pricer *P);
void pricer_info(const Pricer *P, long long *list_entries, long long *list_bytes);
void pricer_max64(Pricer *P, const double *scores_host, double *vmax);
// the pricer's context, n, row count and device rows (x-major menus), for the CG master
Ctx &pricer_ctx(const Pricer *P);
int pricer_n(const Pricer *P);
ll pricer_rows(const Pricer *P);
const ull *pricer_menus(const Pricer *P);
}  // namespace rumb

struct rumb_cg_pricer {
    rumb::Pricer *p = nullptr;
    int device = 0;
};
