// Internal interface of the bootstrap-draws translation unit.
#pragma once
#include "ctx.cuh"

namespace rumb {
struct Draws;
Draws *draws_create(Ctx &c, ll B, int R, ll M, int n_menus, const double *W, const int64_t *optr,
                    const int32_t *oresp, const double *ocnt, const int64_t *cptr, const int32_t *cresp,
                    const double *ccnt, const int32_t *row_menu, const double *p_hat);
void draws_destroy(Draws *D);
int draws_device(const Draws *D);
void draws_rows(Draws *D, const int64_t *idx, ll count, int perturbed, double scale, double *out);
void draws_screen(Draws *D, const double *fit, double scale, double *dev, double *ub);
}  // namespace rumb

struct rumb_draws {
    rumb::Draws *d = nullptr;
    int device = 0;
};
