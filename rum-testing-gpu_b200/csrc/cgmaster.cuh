// Internal interface of the Flow-CG master translation unit.
#pragma once
#include "ctx.cuh"
#include "pricer.cuh"

namespace rumb {
struct CgMaster;
CgMaster *cgmaster_create(Pricer *pr, const int32_t *alts, const double *p_obs, int max_cols);
void cgmaster_destroy(CgMaster *m);
int cgmaster_device(const CgMaster *m);
int cgmaster_add_column(CgMaster *m, const int32_t *rank_pos, const uint64_t *bits_in, uint64_t *bits_out,
                        double *gram_row);
void cgmaster_apply(CgMaster *m, const int32_t *cols, const double *delta, int count);
void cgmaster_price(CgMaster *m, double *vmax, int32_t *rank_pos, double *margin);
void cgmaster_p_out(CgMaster *m, double *out);
}  // namespace rumb

struct rumb_cg_master {
    rumb::CgMaster *m = nullptr;
    int device = 0;
};
