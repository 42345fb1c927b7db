// Bootstrap draws on the GPU: each draw's resampled shares and the screen's distances.
//
// Reference behaviour (mingxiz/rum-testing-gpu):
//   draw rows   solver/inference/draws.py:273-285 (_build: seen = W offered[:, row_menu],
//               chose = W chose, p_b = chose / seen, p_hat where a menu went unseen)
//   perturb     solver/inference/hong_li.py (p_hat + eps_n r_n (p_b - p_hat))
//   screen      solver/inference/bootstrap.py:290-306 (dev_b = ||p_b - p_hat||,
//               U_b = min(U_b, ||perturb(p_b) - p_fit||): p_fit is a RUM point)
//
// A draw is a row of respondent weights W[b, :] (multinomial counts). Respondent r was offered
// menu u offered[r, u] times and chose row j chose[r, j] times; the draw's row j is
//     seen = sum_r W[b, r] offered[r, menu(j)],  chose = sum_r W[b, r] chose[r, j],
//     p_b[j] = chose / seen (p_hat[j] when seen <= 0).
// The weights and counts are integers, so both sums are exact in any order and the rows equal the
// host's bit for bit (the division and the perturbation are single IEEE operations, written
// without contraction). The two norms of the screen are float64 sums in a fixed tree order here,
// in numpy's order on the host: they agree to rounding.
//
// Layout: W row-major (B x R, float64); offered by menu and chose by row as CSR lists of
// (respondent, count). One CTA per draw: the draw's R weights staged in shared memory, the
// threads striding over the M rows with the lists' gathers served from there.
#include <algorithm>
#include <cmath>
#include <memory>
#include <string>

#include "ctx.cuh"
#include "draws.cuh"

namespace rumb {

constexpr int DR_THREADS = 512;

struct DrawArgs {
    int R;
    ll M;
    const double *W;
    const ll *optr;
    const int *oresp;
    const double *ocnt;
    const ll *cptr;
    const int *cresp;
    const double *ccnt;
    const int *row_menu;
    const double *p_hat;
};

// rows: count x M output (perturbed with scale when perturbed = 1, else the raw shares), or null;
// dev / ub: per draw ||p_b - p_hat|| and ||perturb(p_b) - fit|| (ub needs fit), or null.
__global__ void __launch_bounds__(DR_THREADS) draw_rows_kernel(DrawArgs A, const ll *idx, int perturbed, double scale,
                                                               const double *fit, double *rows, double *dev,
                                                               double *ub) {
    extern __shared__ double sw[];
    __shared__ double red_d[DR_THREADS / 32], red_u[DR_THREADS / 32];
    const ll b = idx ? idx[blockIdx.x] : (ll)blockIdx.x;
    const double *wrow = A.W + b * (ll)A.R;
    for (int r = threadIdx.x; r < A.R; r += blockDim.x) sw[r] = wrow[r];
    __syncthreads();
    double sd = 0.0, su = 0.0;
    double *out = rows ? rows + (ll)blockIdx.x * A.M : nullptr;
    for (ll j = threadIdx.x; j < A.M; j += blockDim.x) {
        const int u = A.row_menu[j];
        double seen = 0.0, chose = 0.0;
        for (ll k = A.optr[u]; k < A.optr[u + 1]; ++k) seen = __dadd_rn(seen, __dmul_rn(sw[A.oresp[k]], A.ocnt[k]));
        for (ll k = A.cptr[j]; k < A.cptr[j + 1]; ++k) chose = __dadd_rn(chose, __dmul_rn(sw[A.cresp[k]], A.ccnt[k]));
        const double ph = A.p_hat[j];
        const double pb = seen <= 0.0 ? ph : __ddiv_rn(chose, seen);
        const double P = __dadd_rn(ph, __dmul_rn(scale, __dsub_rn(pb, ph)));
        if (out) out[j] = perturbed ? P : pb;
        const double d = __dsub_rn(pb, ph);
        sd = __dadd_rn(sd, __dmul_rn(d, d));
        if (fit) {
            const double e = __dsub_rn(P, fit[j]);
            su = __dadd_rn(su, __dmul_rn(e, e));
        }
    }
    if (!dev && !ub) return;
    for (int o = 16; o > 0; o >>= 1) {
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
        su += __shfl_xor_sync(0xffffffffu, su, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red_d[w] = sd;
        red_u[w] = su;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double td = 0.0, tu = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            td += red_d[i];
            tu += red_u[i];
        }
        if (dev) dev[blockIdx.x] = sqrt(td);
        if (ub) ub[blockIdx.x] = sqrt(tu);
    }
}

struct Draws {
    Ctx *c = nullptr;
    ll B = 0, M = 0;
    int R = 0, n_menus = 0;
    DevBuf W, optr, oresp, ocnt, cptr, cresp, ccnt, row_menu, p_hat;
    DevBuf fit, idx, rows, dev, ub;
};

static void check_csr(const int64_t *ptr, const int32_t *resp, ll n, int R, const char *what) {
    if (!ptr) fail(RUMB_E_INVAL, std::string(what) + ": NULL pointer");
    if (ptr[0] != 0) fail(RUMB_E_INVAL, std::string(what) + ": lists must start at 0");
    for (ll i = 0; i < n; ++i)
        if (ptr[i + 1] < ptr[i]) fail(RUMB_E_INVAL, std::string(what) + ": list offsets must be nondecreasing");
    if (ptr[n] > 0 && !resp) fail(RUMB_E_INVAL, std::string(what) + ": NULL respondents");
    for (ll k = 0; k < ptr[n]; ++k)
        if (resp[k] < 0 || resp[k] >= R) fail(RUMB_E_INVAL, std::string(what) + ": respondent out of range");
}

template <class T>
static void upload(DevBuf &d, const T *h, size_t count, cudaStream_t st) {
    d.ensure(std::max<size_t>(count, 1) * sizeof(T));
    if (count) RUMB_CUDA(cudaMemcpyAsync(d.ptr, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
}

Draws *draws_create(Ctx &c, ll B, int R, ll M, int n_menus, const double *W, const int64_t *optr,
                    const int32_t *oresp, const double *ocnt, const int64_t *cptr, const int32_t *cresp,
                    const double *ccnt, const int32_t *row_menu, const double *p_hat) {
    if (B < 1 || R < 1 || M < 1 || n_menus < 1) fail(RUMB_E_INVAL, "draws: B, R, M and n_menus must be >= 1");
    if ((size_t)R * sizeof(double) > 160 * 1024) fail(RUMB_E_INVAL, "draws: at most 20480 respondents");
    if (!W || !row_menu || !p_hat) fail(RUMB_E_INVAL, "draws: NULL weights, row menus or p_hat");
    check_csr(optr, oresp, n_menus, R, "offered");
    check_csr(cptr, cresp, M, R, "chose");
    if ((optr[n_menus] > 0 && !ocnt) || (cptr[M] > 0 && !ccnt)) fail(RUMB_E_INVAL, "draws: NULL counts");
    for (ll j = 0; j < M; ++j)
        if (row_menu[j] < 0 || row_menu[j] >= n_menus) fail(RUMB_E_INVAL, "draws: row menu out of range");
    std::unique_ptr<Draws> D(new Draws());
    D->c = &c;
    D->B = B;
    D->R = R;
    D->M = M;
    D->n_menus = n_menus;
    cudaStream_t st = c.own;
    upload(D->W, W, (size_t)B * R, st);
    upload(D->optr, optr, (size_t)n_menus + 1, st);
    upload(D->oresp, oresp, (size_t)optr[n_menus], st);
    upload(D->ocnt, ocnt, (size_t)optr[n_menus], st);
    upload(D->cptr, cptr, (size_t)M + 1, st);
    upload(D->cresp, cresp, (size_t)cptr[M], st);
    upload(D->ccnt, ccnt, (size_t)cptr[M], st);
    upload(D->row_menu, row_menu, (size_t)M, st);
    upload(D->p_hat, p_hat, (size_t)M, st);
    RUMB_CUDA(cudaStreamSynchronize(st));
    return D.release();
}

void draws_destroy(Draws *D) { delete D; }

int draws_device(const Draws *D) { return D->c->device; }

static DrawArgs args_of(const Draws &D) {
    DrawArgs A;
    A.R = D.R;
    A.M = D.M;
    A.W = D.W.as<double>();
    A.optr = D.optr.as<ll>();
    A.oresp = D.oresp.as<int>();
    A.ocnt = D.ocnt.as<double>();
    A.cptr = D.cptr.as<ll>();
    A.cresp = D.cresp.as<int>();
    A.ccnt = D.ccnt.as<double>();
    A.row_menu = D.row_menu.as<int>();
    A.p_hat = D.p_hat.as<double>();
    return A;
}

static void launch(const Draws &D, ll count, const ll *idx, int perturbed, double scale, const double *fit,
                   double *rows, double *dev, double *ub) {
    cudaStream_t st = D.c->own;
    const size_t smem = (size_t)D.R * sizeof(double);
    // the opt-in above 48 KB is a per-device attribute: set it on the draws' device when it is needed
    if (smem > 48 * 1024)
        RUMB_CUDA(cudaFuncSetAttribute(draw_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (ll lo = 0; lo < count; lo += 65535) {
        const ll nb = std::min<ll>(65535, count - lo);
        draw_rows_kernel<<<(unsigned)nb, DR_THREADS, smem, st>>>(args_of(D), idx ? idx + lo : nullptr, perturbed, scale,
                                                                  fit, rows ? rows + lo * D.M : nullptr,
                                                                  dev ? dev + lo : nullptr, ub ? ub + lo : nullptr);
        RUMB_LAUNCH("draw_rows_kernel");
    }
}

void draws_rows(Draws *D, const int64_t *idx, ll count, int perturbed, double scale, double *out) {
    if (count < 0 || (count > 0 && (!idx || !out))) fail(RUMB_E_INVAL, "draws: NULL indices or output");
    if (count == 0) return;
    for (ll i = 0; i < count; ++i)
        if (idx[i] < 0 || idx[i] >= D->B) fail(RUMB_E_INVAL, "draws: draw index out of range");
    cudaStream_t st = D->c->own;
    upload(D->idx, idx, (size_t)count, st);
    D->rows.ensure((size_t)count * D->M * sizeof(double));
    launch(*D, count, D->idx.as<ll>(), perturbed, scale, nullptr, D->rows.as<double>(), nullptr, nullptr);
    RUMB_CUDA(cudaMemcpyAsync(out, D->rows.ptr, (size_t)count * D->M * sizeof(double), cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
}

void draws_screen(Draws *D, const double *fit, double scale, double *dev, double *ub) {
    if (!dev && !ub) return;
    if (ub && !fit) fail(RUMB_E_INVAL, "draws: the screen's bound needs a fit");
    cudaStream_t st = D->c->own;
    if (fit) upload(D->fit, fit, (size_t)D->M, st);
    D->dev.ensure((size_t)D->B * sizeof(double));
    D->ub.ensure((size_t)D->B * sizeof(double));
    launch(*D, D->B, nullptr, 1, scale, fit ? D->fit.as<double>() : nullptr, nullptr, D->dev.as<double>(),
           ub ? D->ub.as<double>() : nullptr);
    if (dev) RUMB_CUDA(cudaMemcpyAsync(dev, D->dev.ptr, (size_t)D->B * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (ub) RUMB_CUDA(cudaMemcpyAsync(ub, D->ub.ptr, (size_t)D->B * sizeof(double), cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace rumb
