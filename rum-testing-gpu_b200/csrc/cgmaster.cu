// The Flow-CG master's per-column bookkeeping on the GPU, next to the pricer: the column of a
// ranking, its row of the Gram matrix Q = V'V, the fitted shares p_out = V lam kept up to date,
// and the float32 residual the pricer reads, so that a CG iteration sends the pricer nothing but
// the change in lam.
//
// Reference behaviour (mingxiz/rum-testing-gpu):
//   ranking -> column   solver/flow_cg/cg_core.py:63-80 (row s is 1 when its alternative is the
//                       best-ranked member of its menu)
//   Gram row            solver/flow_cg/qp_bitset_incremental.py:51-77 (popcount of the packed
//                       columns' AND: Q[k, j], and Q[k, k])
//   p_out update        solver/flow_cg/qp_bitset_incremental.py:127-141 (for every column a with
//                       |delta_a| > 1e-12, in increasing a: p_out[rows of a] += delta_a)
//   residual            solver/flow_cg/solver.py:166-168 ((p_obs - p_out) as float32)
//
// All of it is exact against the host arithmetic: the column and the popcounts are integers, and
// each p_out entry receives the same float64 additions in the same order (one thread per row walks
// the active columns in increasing order), so the residual and therefore the priced column are the
// host's bit for bit. The QP and h = V'p_obs stay on the host (LAPACK's factorizations and numpy's
// summation order are part of the column sequence).
//
// Layout: columns as packed bits, column a at bits[a W .. a W + W) (W = ceil(M / 64) words, bit s
// of the column = row s in the pricer's x-major order).
#include <algorithm>
#include <memory>
#include <vector>

#include "cgmaster.cuh"
#include "ctx.cuh"

namespace rumb {

// column of a ranking: thread per 64-row word
__global__ void ranking_column_kernel(const ull *menus, const int *alts, const int *rank_pos, int n, ll M, int W,
                                      ull *col) {
    __shared__ int rp[64];
    if (threadIdx.x < n) rp[threadIdx.x] = rank_pos[threadIdx.x];
    __syncthreads();
    const ll w = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (w >= W) return;
    ull word = 0;
    const ll s0 = w * 64;
    const int cnt = (int)std::min<ll>(64, M - s0);
    for (int t = 0; t < cnt; ++t) {
        const ull m = menus[s0 + t];
        int best = -1, br = 0x7fffffff;
        for (ull mm = m; mm; mm &= mm - 1ULL) {
            const int x = __ffsll((long long)mm) - 1;
            if (rp[x] < br) { br = rp[x]; best = x; }
        }
        if (best == alts[s0 + t]) word |= 1ULL << t;
    }
    col[w] = word;
}

// Gram row of column k against columns 0..k: a warp per column j, popcount of the AND
__global__ void gram_row_kernel(const ull *bits, int W, int k, double *row) {
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j > k) return;
    const ull *a = bits + (ll)j * W, *b = bits + (ll)k * W;
    long long c = 0;
    for (int w = lane; w < W; w += 32) c += __popcll(a[w] & b[w]);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) row[j] = (double)c;
}

// p_out[i] += delta_t for the listed columns in list order (increasing), then the residual
__global__ void pout_apply_kernel(const ull *bits, int W, const int *cols, const double *delta, int count, ll M,
                                  double *p_out, const double *p_obs, float *scores) {
    const ll i = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (i >= M) return;
    const ll wi = i >> 6;
    const int bi = (int)(i & 63);
    double v = p_out[i];
    for (int t = 0; t < count; ++t) {
        if ((bits[(ll)cols[t] * W + wi] >> bi) & 1ULL) v = __dadd_rn(v, delta[t]);
    }
    p_out[i] = v;
    scores[i] = __double2float_rn(__dsub_rn(p_obs[i], v));
}

struct CgMaster {
    Pricer *pr = nullptr;
    Ctx *c = nullptr;
    int n = 0, W = 0, max_cols = 0, K = 0;
    ll M = 0;
    DevBuf alts, p_obs, p_out, scores, bits, rank, gram, cols, delta;
};

CgMaster *cgmaster_create(Pricer *pr, const int32_t *alts, const double *p_obs, int max_cols) {
    if (!pr) fail(RUMB_E_INVAL, "pricer is NULL");
    if (!alts || !p_obs) fail(RUMB_E_INVAL, "alternatives / p_obs must not be NULL");
    if (max_cols < 1) fail(RUMB_E_INVAL, "max_cols must be >= 1");
    const ll M = pricer_rows(pr);
    const int n = pricer_n(pr);
    if (M < 1) fail(RUMB_E_INVAL, "the pricer has no rows");
    if (n > 64) fail(RUMB_E_INVAL, "n must be <= 64");
    for (ll s = 0; s < M; ++s)
        if (alts[s] < 0 || alts[s] >= n) fail(RUMB_E_INVAL, "alternative out of range");
    std::unique_ptr<CgMaster> m(new CgMaster());
    m->pr = pr;
    m->c = &pricer_ctx(pr);
    m->n = n;
    m->M = M;
    m->W = (int)((M + 63) / 64);
    m->max_cols = max_cols;
    cudaStream_t st = m->c->own;
    m->alts.ensure((size_t)M * 4);
    m->p_obs.ensure((size_t)M * 8);
    m->p_out.ensure((size_t)M * 8);
    m->scores.ensure((size_t)M * 4);
    m->bits.ensure((size_t)max_cols * m->W * 8);
    m->rank.ensure(64 * 4);
    m->gram.ensure((size_t)max_cols * 8);
    m->cols.ensure((size_t)max_cols * 4);
    m->delta.ensure((size_t)max_cols * 8);
    RUMB_CUDA(cudaMemcpyAsync(m->alts.ptr, alts, (size_t)M * 4, cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(m->p_obs.ptr, p_obs, (size_t)M * 8, cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemsetAsync(m->p_out.ptr, 0, (size_t)M * 8, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    return m.release();
}

void cgmaster_destroy(CgMaster *m) { delete m; }

int cgmaster_device(const CgMaster *m) { return m->c->device; }

int cgmaster_add_column(CgMaster *m, const int32_t *rank_pos, const uint64_t *bits_in, uint64_t *bits_out,
                        double *gram_row) {
    if (m->K >= m->max_cols) fail(RUMB_E_INVAL, "the master holds max_cols columns already");
    if ((rank_pos == nullptr) == (bits_in == nullptr)) fail(RUMB_E_INVAL, "give a ranking or a column, not both");
    cudaStream_t st = m->c->own;
    ull *col = m->bits.as<ull>() + (ll)m->K * m->W;
    if (rank_pos) {
        std::vector<int> seen(m->n, 0);
        for (int x = 0; x < m->n; ++x) {
            if (rank_pos[x] < 0 || rank_pos[x] >= m->n || seen[rank_pos[x]]) fail(RUMB_E_INVAL, "rank_pos is not a permutation");
            seen[rank_pos[x]] = 1;
        }
        RUMB_CUDA(cudaMemcpyAsync(m->rank.ptr, rank_pos, (size_t)m->n * 4, cudaMemcpyHostToDevice, st));
        ranking_column_kernel<<<grid_for(m->W, 128), 128, 0, st>>>(pricer_menus(m->pr), m->alts.as<int>(),
                                                                   m->rank.as<int>(), m->n, m->M, m->W, col);
        RUMB_LAUNCH("ranking_column_kernel");
    } else {
        if (m->M % 64 && (bits_in[m->W - 1] >> (m->M % 64)) != 0) fail(RUMB_E_INVAL, "column bits beyond the rows");
        RUMB_CUDA(cudaMemcpyAsync(col, bits_in, (size_t)m->W * 8, cudaMemcpyHostToDevice, st));
    }
    const int k = m->K;
    gram_row_kernel<<<(unsigned)((k + 1 + 7) / 8), 256, 0, st>>>(m->bits.as<ull>(), m->W, k, m->gram.as<double>());
    RUMB_LAUNCH("gram_row_kernel");
    if (bits_out) RUMB_CUDA(cudaMemcpyAsync(bits_out, col, (size_t)m->W * 8, cudaMemcpyDeviceToHost, st));
    if (gram_row) RUMB_CUDA(cudaMemcpyAsync(gram_row, m->gram.ptr, (size_t)(k + 1) * 8, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    m->K = k + 1;
    return k;
}

void cgmaster_apply(CgMaster *m, const int32_t *cols, const double *delta, int count) {
    if (count < 0 || count > m->K) fail(RUMB_E_INVAL, "count must be in 0 .. columns held");
    if (count > 0 && (!cols || !delta)) fail(RUMB_E_INVAL, "cols / delta must not be NULL");
    for (int t = 0; t < count; ++t) {
        if (cols[t] < 0 || cols[t] >= m->K) fail(RUMB_E_INVAL, "column index out of range");
        if (t > 0 && cols[t] <= cols[t - 1]) fail(RUMB_E_INVAL, "columns must be increasing");
    }
    cudaStream_t st = m->c->own;
    if (count) {
        RUMB_CUDA(cudaMemcpyAsync(m->cols.ptr, cols, (size_t)count * 4, cudaMemcpyHostToDevice, st));
        RUMB_CUDA(cudaMemcpyAsync(m->delta.ptr, delta, (size_t)count * 8, cudaMemcpyHostToDevice, st));
    }
    pout_apply_kernel<<<grid_for(m->M, 256), 256, 0, st>>>(m->bits.as<ull>(), m->W, m->cols.as<int>(),
                                                          m->delta.as<double>(), count, m->M, m->p_out.as<double>(),
                                                          m->p_obs.as<double>(), m->scores.as<float>());
    RUMB_LAUNCH("pout_apply_kernel");
}

void cgmaster_price(CgMaster *m, double *vmax, int32_t *rank_pos, double *margin) {
    pricer_price(m->pr, m->scores.as<float>(), 1, vmax, rank_pos, margin, nullptr);
}

void cgmaster_p_out(CgMaster *m, double *out) {
    cudaStream_t st = m->c->own;
    RUMB_CUDA(cudaMemcpyAsync(out, m->p_out.ptr, (size_t)m->M * 8, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace rumb
