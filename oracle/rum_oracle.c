/*
 * CPU restatement of the reference's two subset-lattice hot paths -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the parity checker (the "oracle") for the CUDA library in rum-testing-gpu_b200/.
 * Only the test suite, the smoke check and the CPU-baseline leg of bench.py load it; the
 * library never does. Compile with -ffp-contract=off so every a*b+c stays two roundings except
 * where fmaf() is written out on purpose (the pricer's block-scaled decode, see price_* below).
 *
 * Reference (mingxiz/rum-testing-gpu), the behaviour restated here:
 *   slab layout / compress       solver/bm_admm/kernels.py:24-35, solver/common/transforms.py:59-65
 *   2x2 butterfly, bits ascending solver/common/butterfly.py:23-48, solver/bm_admm/butterfly2.py:62-65
 *   prox_all                     solver/bm_admm/solver.py:66-139
 *   one ADMM iteration           solver/bm_admm/solver.py:33-54 (_EW_SRC), :240-254 (one_iter)
 *   float64 push (upper bound)   solver/common/arcflow_kernels.py:357-386, :415-434
 *   float64 longest path (LB)    solver/common/arcflow_kernels.py:388-397, :437-448
 *   mask Bellman-Ford pricing    solver/flow_cg/bf_pricing.py:8-47
 *   rank-indexed stream pricing  solver/flow_cg/pricing_stream.py:61-182 (f32/u16/u24), :302-412
 *   ranking -> 0/1 column        solver/flow_cg/cg_core.py:63-80
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef long long ll;
typedef unsigned long long ull;

/* thread count of the parallel loops (every loop writes disjoint outputs, so results do not
 * depend on it) */
void ora_set_threads(int t) {
#ifdef _OPENMP
    omp_set_num_threads(t > 0 ? t : omp_get_num_procs());
#else
    (void)t;
#endif
}

int ora_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ slab layout */

/* rest index of menu-without-x inside alternative x's block: drop bit x, shift the higher bits
 * down (solver/bm_admm/kernels.py:30-33). */
static inline ull compress_bit(ull mask, int x) {
    ull low = mask & ((1ULL << x) - 1ULL);
    ull high = mask >> (x + 1);
    return low | (high << x);
}

/* inverse: put a 0 bit back at position x */
static inline ull expand_bit(ull rest, int x) {
    return (rest & ((1ULL << x) - 1ULL)) | ((rest >> x) << (x + 1));
}

void ora_slab_index(int n, ll mp, const ull *menu, const ll *alt, ll *idx) {
    ll Nloc = 1LL << (n - 1);
    for (ll j = 0; j < mp; ++j) {
        int x = (int)alt[j];
        ull m = menu[j] & ~(1ULL << x);
        idx[j] = (ll)x * Nloc + (ll)compress_bit(m, x);
    }
}

/* ------------------------------------------------------------------ butterflies */

/* (a,b,c,d) butterfly over the n-1 rest bits of every alternative's block, bits ascending:
 * pair (l, l|2^j): lo' = a*X + b*Y, hi' = c*X + d*Y (X = lo, Y = hi). In place. */
#define BFLY_BODY(T)                                                                        \
    ll Nloc = 1LL << (n - 1);                                                               \
    for (int x = 0; x < n; ++x) {                                                           \
        T *blk = v + (ll)x * Nloc;                                                          \
        for (int j = 0; j < n - 1; ++j) {                                                   \
            ll h = 1LL << j;                                                                \
            _Pragma("omp parallel for schedule(static) if (Nloc >= 4096)")                  \
            for (ll base = 0; base < Nloc; base += 2 * h)                                   \
                for (ll i = base; i < base + h; ++i) {                                      \
                    T X = blk[i], Y = blk[i + h];                                           \
                    blk[i] = a * X + b * Y;                                                 \
                    blk[i + h] = c * X + d * Y;                                             \
                }                                                                           \
        }                                                                                   \
    }

void ora_bfly_f64(int n, double *v, double a, double b, double c, double d) { BFLY_BODY(double) }
void ora_bfly_f32(int n, float *v, float a, float b, float c, float d) { BFLY_BODY(float) }

/* ------------------------------------------------------------------ prox (per menu) */

/* Simplex prox of every menu S (all 2^n - 1 masks), one reference thread's work per menu
 * (solver/bm_admm/solver.py:66-139); T is the state dtype, sorting and thresholds in double. */
#define PROX_BODY(T)                                                                        \
    ll Nloc = 1LL << (n - 1);                                                               \
    ull full = (1ULL << n);                                                                 \
    _Pragma("omp parallel for schedule(dynamic, 1024) if (full >= 4096)")                  \
    for (ull S = 1; S < full; ++S) {                                                        \
        T vals[64]; ll pos_arr[64]; double srt[64];                                         \
        int k = __builtin_popcountll(S);                                                    \
        ull SS = S; int kk = 0; T w0 = (T)0; int mixed = 0; int single = 0;                 \
        while (SS) {                                                                        \
            ull bit = SS & (0ULL - SS);                                                     \
            int i = __builtin_ctzll(bit);                                                   \
            ll pos = (ll)i * Nloc + (ll)compress_bit(S & ~(1ULL << i), i);                  \
            if (k == 1) { out[pos] = (T)1; single = 1; break; }                             \
            T v = in[pos], w = wmask[pos], xh = xhat[pos];                                  \
            if (kk == 0) w0 = w; else if (w != w0) mixed = 1;                               \
            vals[kk] = (beta2 * v + (T)2 * w * xh) / (beta2 + (T)2 * w);                    \
            pos_arr[kk] = pos;                                                              \
            SS ^= bit; kk++;                                                                \
        }                                                                                   \
        if (single) continue;                                                               \
        if (mixed) {                                                                        \
            for (int a2 = 0; a2 < k; ++a2) {                                                \
                ll q = pos_arr[a2];                                                         \
                srt[a2] = (double)beta2 * (double)in[q] + 2.0 * (double)wmask[q] * (double)xhat[q]; \
            }                                                                               \
            for (int a2 = 1; a2 < k; ++a2) {                                                \
                double key = srt[a2]; ll kp = pos_arr[a2]; int b = a2 - 1;                  \
                while (b >= 0 && srt[b] < key) { srt[b + 1] = srt[b]; pos_arr[b + 1] = pos_arr[b]; --b; } \
                srt[b + 1] = key; pos_arr[b + 1] = kp;                                      \
            }                                                                               \
            double stc = 0.0, sic = 0.0, mu = 0.0;                                          \
            for (int a2 = 0; a2 < k; ++a2) {                                                \
                double cc = (double)beta2 + 2.0 * (double)wmask[pos_arr[a2]];               \
                stc += srt[a2] / cc; sic += 1.0 / cc;                                       \
                double th = (stc - 1.0) / sic;                                              \
                if (srt[a2] - th > 0.0) mu = th;                                            \
            }                                                                               \
            for (int a2 = 0; a2 < k; ++a2) {                                                \
                double cc = (double)beta2 + 2.0 * (double)wmask[pos_arr[a2]];               \
                double yv = (srt[a2] - mu) / cc;                                            \
                out[pos_arr[a2]] = yv > 0.0 ? (T)yv : (T)0.0;                               \
            }                                                                               \
            continue;                                                                       \
        }                                                                                   \
        for (int a2 = 0; a2 < k; ++a2) srt[a2] = (double)vals[a2];                          \
        for (int a2 = 1; a2 < k; ++a2) {                                                    \
            double key = srt[a2]; int b = a2 - 1;                                           \
            while (b >= 0 && srt[b] < key) { srt[b + 1] = srt[b]; --b; }                    \
            srt[b + 1] = key;                                                               \
        }                                                                                   \
        double css = 0.0, tau = 0.0;                                                        \
        for (int a2 = 0; a2 < k; ++a2) {                                                    \
            css += srt[a2];                                                                 \
            double th = (css - 1.0) / (double)(a2 + 1);                                     \
            if (srt[a2] - th > 0.0) tau = th;                                               \
        }                                                                                   \
        for (int a2 = 0; a2 < k; ++a2) {                                                    \
            double yv = (double)vals[a2] - tau;                                             \
            out[pos_arr[a2]] = yv > 0.0 ? (T)yv : (T)0.0;                                   \
        }                                                                                   \
    }

void ora_prox_f64(int n, const double *in, double *out, const double *xhat, const double *wmask,
                  double beta2) { PROX_BODY(double) }
void ora_prox_f32(int n, const float *in, float *out, const float *xhat, const float *wmask,
                  float beta2) { PROX_BODY(float) }

/* ------------------------------------------------------------------ one ADMM iteration */

/* The iteration of solve_kadmm_v2 (solver/bm_admm/solver.py:240-254) on host slabs, `iters`
 * times. co[0..3] = Qt (row-major 2x2), co[4..7] = Q, inv_gl[Nloc] = 1/(gamma + lambda(rest)).
 * scratch: 6 slabs (w, AT, rhs, x, Ax, x2n; xk reuses w). */
#define ITER_BODY(T, BF, PX)                                                                \
    ll Nloc = 1LL << (n - 1), m2 = (ll)n * Nloc;                                            \
    T *w = scratch, *AT = scratch + m2, *rhs = scratch + 2 * m2, *x = scratch + 3 * m2;     \
    T *Ax = scratch + 4 * m2, *x2n = scratch + 5 * m2, *xk = w;                             \
    T one = (T)1;                                                                           \
    for (int it = 0; it < iters; ++it) {                                                    \
        _Pragma("omp parallel for schedule(static)")                                        \
        for (ll i = 0; i < m2; ++i) w[i] = y[i] - b1 * s[i];                                \
        memcpy(AT, w, (size_t)m2 * sizeof(T));                                              \
        BF(n, AT, (T)1, (T)0, (T)-1, p);                                                    \
        _Pragma("omp parallel for schedule(static)")                                        \
        for (ll i = 0; i < m2; ++i) rhs[i] = (z[i] + b2 * x2[i] - AT[i]) * ib1;             \
        memcpy(x, rhs, (size_t)m2 * sizeof(T));                                             \
        BF(n, x, (T)co[0], (T)co[1], (T)co[2], (T)co[3]);                                   \
        _Pragma("omp parallel for schedule(static)")                                        \
        for (ll i = 0; i < m2; ++i) x[i] *= inv_gl[i % Nloc];                               \
        BF(n, x, (T)co[4], (T)co[5], (T)co[6], (T)co[7]);                                   \
        memcpy(Ax, x, (size_t)m2 * sizeof(T));                                              \
        BF(n, Ax, (T)1, (T)-1, (T)0, p);                                                    \
        _Pragma("omp parallel for schedule(static)")                                        \
        for (ll i = 0; i < m2; ++i) xk[i] = alpha * x[i] + (one - alpha) * x2[i] - ib2 * z[i]; \
        PX(n, xk, x2n, xhat, wmask, b2);                                                    \
        _Pragma("omp parallel for schedule(static)")                                        \
        for (ll i = 0; i < m2; ++i) {                                                       \
            T xo = alpha * x[i] + (one - alpha) * x2[i];                                    \
            z[i] -= b2 * (xo - x2n[i]);                                                     \
        }                                                                                   \
        _Pragma("omp parallel for schedule(static)")                                        \
        for (ll i = 0; i < m2; ++i) {                                                       \
            T axor = -alpha * Ax[i] - (one - alpha) * s[i];                                 \
            T sn = ib1 * y[i] - axor; sn = sn > (T)0 ? sn : (T)0;                           \
            y[i] -= b1 * (axor + sn); s[i] = sn;                                            \
        }                                                                                   \
        memcpy(x2, x2n, (size_t)m2 * sizeof(T));                                            \
    }

void ora_admm_iter_f64(int n, double *x2, double *s, double *y, double *z, const double *xhat,
                       const double *wmask, const double *inv_gl, const double *co, double b1,
                       double b2, double ib1, double ib2, double alpha, double p, double *scratch,
                       int iters) { ITER_BODY(double, ora_bfly_f64, ora_prox_f64) }
void ora_admm_iter_f32(int n, float *x2, float *s, float *y, float *z, const float *xhat,
                       const float *wmask, const float *inv_gl, const double *co, float b1,
                       float b2, float ib1, float ib2, float alpha, float p, float *scratch,
                       int iters) { ITER_BODY(float, ora_bfly_f32, ora_prox_f32) }

/* ------------------------------------------------------------------ lattice layers */

/* node ids grouped by popcount, ascending inside a group; bounds[c]..bounds[c+1] is layer c
 * (solver/common/arcflow_kernels.py:317-326). bounds has n+2 entries. */
void ora_layers(int n, ll *order, ll *bounds) {
    ll N = 1LL << n;
    ll *cnt = (ll *)calloc((size_t)n + 2, sizeof(ll));
    for (ll v = 0; v < N; ++v) cnt[__builtin_popcountll((ull)v) + 1]++;
    bounds[0] = 0;
    for (int c = 0; c <= n; ++c) bounds[c + 1] = bounds[c] + cnt[c + 1];
    ll *fill = (ll *)malloc(((size_t)n + 1) * sizeof(ll));
    for (int c = 0; c <= n; ++c) fill[c] = bounds[c];
    for (ll v = 0; v < N; ++v) order[fill[__builtin_popcountll((ull)v)]++] = v;
    free(cnt); free(fill);
}

/* ------------------------------------------------------------------ float64 push */

/* x (slab, float64) -> the arc flow pushed to an exact unit flow, rf (slab). The Mobius
 * butterfly is applied by the caller. Follows wmax64 / outwt64 / massg64 / extract64. */
void ora_make_feasible64(int n, const double *q, double *rf, double eps) {
    ll Nloc = 1LL << (n - 1), m2 = (ll)n * Nloc, N = 1LL << n;
    double *w = (double *)malloc((size_t)m2 * sizeof(double));
    double *outw = (double *)malloc((size_t)N * sizeof(double));
    double *mass = (double *)calloc((size_t)N, sizeof(double));
    ll *order = (ll *)malloc((size_t)N * sizeof(ll));
    ll *bounds = (ll *)malloc(((size_t)n + 2) * sizeof(ll));
    #pragma omp parallel for schedule(static)
    for (ll i = 0; i < m2; ++i) w[i] = (q[i] > 0.0 ? q[i] : 0.0) + eps;
    #pragma omp parallel for schedule(static)
    for (ll D = 0; D < N; ++D) {
        double sum = 0.0;
        for (int x = 0; x < n; ++x) {
            ll bit = 1LL << x;
            if (!(D & bit)) sum += w[(ll)x * Nloc + (ll)compress_bit((ull)D, x)];
        }
        outw[D] = sum;
    }
    ora_layers(n, order, bounds);
    mass[0] = 1.0;
    for (int c = 1; c <= n; ++c) {
        #pragma omp parallel for schedule(static)
        for (ll i = bounds[c]; i < bounds[c + 1]; ++i) {
            ll C = order[i];
            double sum = 0.0;
            for (int x = 0; x < n; ++x) {
                ll bit = 1LL << x;
                if (C & bit) {
                    ll P = C ^ bit;
                    double ow = outw[P];
                    if (ow > 0.0) sum += mass[P] * w[(ll)x * Nloc + (ll)compress_bit((ull)P, x)] / ow;
                }
            }
            mass[C] = sum;
        }
    }
    #pragma omp parallel for schedule(static)
    for (ll a = 0; a < m2; ++a) {
        ll x = a / Nloc, rest = a - x * Nloc;
        ll T = (ll)expand_bit((ull)rest, (int)x);
        double ow = outw[T];
        rf[a] = (ow > 0.0) ? mass[T] * w[a] / ow : 0.0;
    }
    free(w); free(outw); free(mass); free(order); free(bounds);
}

/* value of the best path from the empty set to the full set where the arc S -> S+{x} is worth
 * R[x*Nloc + compress(S, x)] (lpath64 + longest_path_gpu64). */
double ora_longest_path64(int n, const double *R) {
    ll Nloc = 1LL << (n - 1), N = 1LL << n;
    double *dp = (double *)malloc((size_t)N * sizeof(double));
    ll *order = (ll *)malloc((size_t)N * sizeof(ll));
    ll *bounds = (ll *)malloc(((size_t)n + 2) * sizeof(ll));
    ora_layers(n, order, bounds);
    dp[0] = 0.0;
    for (int c = 1; c <= n; ++c) {
        #pragma omp parallel for schedule(static)
        for (ll i = bounds[c]; i < bounds[c + 1]; ++i) {
            ll C = order[i];
            double best = -1e300;
            for (int x = 0; x < n; ++x) {
                ll bit = 1LL << x;
                if (C & bit) {
                    ll P = C ^ bit;
                    double v = dp[P] + R[(ll)x * Nloc + (ll)compress_bit((ull)P, x)];
                    if (v > best) best = v;
                }
            }
            dp[C] = best;
        }
    }
    double out = dp[N - 1];
    free(dp); free(order); free(bounds);
    return out;
}

/* ------------------------------------------------------------------ Flow-CG pricing */

/* C(b, t) table, entry b*(n+1)+t (solver/flow_cg/cg_core.py:53-60) */
static ull *binom_table(int n) {
    ull *tab = (ull *)calloc((size_t)(n + 1) * (n + 1), sizeof(ull));
    for (int b = 0; b <= n; ++b) {
        tab[b * (n + 1) + 0] = 1;
        for (int t = 1; t <= b; ++t)
            tab[b * (n + 1) + t] = tab[(b - 1) * (n + 1) + t - 1] + (t <= b - 1 ? tab[(b - 1) * (n + 1) + t] : 0);
    }
    return tab;
}

ull ora_colex_rank(ull mask) {
    ull r = 0, t = 0, b = 0;
    while (mask) {
        if (mask & 1ULL) {
            ++t;
            /* C(b, t) */
            ull c = 1;
            for (ull i = 0; i < t; ++i) c = c * (b - i) / (i + 1);
            if (t > b) c = 0;
            r += c;
        }
        mask >>= 1; ++b;
    }
    return r;
}

/* w(x, D): sequential float32 sum of x's row scores whose menu is a subset of D */
static inline float wsum(const ull *menus, const float *scores, ll lo, ll hi, ull D) {
    float w = 0.0f;
    for (ll i = lo; i < hi; ++i) {
        ull Dp = menus[i];
        if ((Dp & D) == Dp) w += scores[i];
    }
    return w;
}

/* Mask-indexed sweep restricted to the subsets of `within` (all of them when within = full):
 * V and pred are indexed by the mask over the original n alternatives (2^n entries; only the
 * subsets of `within` are touched). Layers ascending by popcount, x ascending, strict '>'
 * (bf_update). */
static void mask_sweep(int n, const ull *menus, const float *scores, const ll *offsets, ull within,
                       float *V, unsigned char *pred) {
    int K = __builtin_popcountll(within);
    int elems[64], j = 0;
    for (int b = 0; b < n; ++b) if ((within >> b) & 1ULL) elems[j++] = b;
    ull Nsub = 1ULL << K;
    /* sub-masks by popcount, ascending (Gosper order) */
    for (int c = 1; c <= K; ++c)
        for (ull ds = 0; ds < Nsub; ++ds) {
            if (__builtin_popcountll(ds) != c) continue;
            ull D = 0;
            for (int t = 0; t < K; ++t) if ((ds >> t) & 1ULL) D |= 1ULL << elems[t];
            float best = 0.0f; int seen = 0;
            for (int t = 0; t < K; ++t) {
                if (!((ds >> t) & 1ULL)) continue;
                int x = elems[t];
                ull prev = D ^ (1ULL << x);
                float w = wsum(menus, scores, offsets[x], offsets[x + 1], D);
                float cand = V[prev] + w;
                if (!seen || cand > best) { best = cand; seen = 1; pred[D] = (unsigned char)x; }
            }
            V[D] = best;
        }
}

/* Full mask pricing (n <= 30): returns V[full] and rank_pos (0 = most preferred). */
float ora_price_mask(int n, const ull *menus, const float *scores, const ll *offsets, int *rank_pos) {
    ull N = 1ULL << n;
    float *V = (float *)calloc((size_t)N, sizeof(float));
    unsigned char *pred = (unsigned char *)calloc((size_t)N, 1);
    mask_sweep(n, menus, scores, offsets, N - 1, V, pred);
    float vmax = V[N - 1];
    ull D = N - 1;
    for (int i = 0; i < n; ++i) { int x = pred[D]; rank_pos[x] = i; D ^= 1ULL << x; }
    free(V); free(pred);
    return vmax;
}

#define SBLOCK 1024
/* One layer k of the rank-indexed sweep in mode 0 = f32, 1 = u16, 2 = u24, reproducing
 * bf_stream_{f32,u16,u24} block by block (1024 ranks per quantization block). The previous
 * layer is decoded with fmaf (m + q*e) when fma_decode, else with a separate multiply and add. */
static void stream_layer(int mode, int fma_decode, int n, int k, ull count, const ull *binom,
                         const void *vprev, const unsigned char *lprev, const float *mprev,
                         const float *eprev, void *vcur, unsigned char *lcur, float *mcur,
                         float *ecur, unsigned char *pred, const ull *menus, const float *scores,
                         const ll *offsets) {
    ull nblk = (count + SBLOCK - 1) / SBLOCK;
    float *vals = (float *)malloc(SBLOCK * sizeof(float));
    for (ull blk = 0; blk < nblk; ++blk) {
        float tmin = 3.0e38f, tmax = -3.0e38f;
        for (int j = 0; j < SBLOCK; ++j) {
            ull r = blk * SBLOCK + (ull)j;
            vals[j] = 0.0f;
            if (r >= count) continue;
            ull rr = r; int b = n - 1; int elems[64]; ull D = 0ULL;
            for (int t = k; t >= 1; --t) {
                while (binom[b * (n + 1) + t] > rr) --b;
                elems[t - 1] = b; D |= (1ULL << b); rr -= binom[b * (n + 1) + t]; --b;
            }
            float best = 0.0f; int seen = 0, bestx = 0;
            ull suf = 0ULL, remain = r;
            for (int t = k - 1; t >= 0; --t) {
                int x = elems[t];
                remain -= binom[x * (n + 1) + (t + 1)];
                ull rp = remain + suf;
                suf += binom[x * (n + 1) + t];
                float vp;
                if (mode == 0) vp = ((const float *)vprev)[rp];
                else {
                    unsigned int q = ((const unsigned short *)vprev)[rp];
                    if (mode == 2) q = (q << 8) | (unsigned int)lprev[rp];
                    float qf = (float)q, m = mprev[rp / SBLOCK], e = eprev[rp / SBLOCK];
                    if (fma_decode) vp = fmaf(qf, e, m);
                    else { float t2 = qf * e; vp = m + t2; }
                }
                float w = wsum(menus, scores, offsets[x], offsets[x + 1], D);
                float cand = vp + w;
                if (!seen || cand >= best) { best = cand; seen = 1; bestx = x; }
            }
            vals[j] = best;
            if (pred) pred[r] = (unsigned char)bestx;
            if (best < tmin) tmin = best;
            if (best > tmax) tmax = best;
        }
        if (mode == 0) {
            for (int j = 0; j < SBLOCK; ++j) {
                ull r = blk * SBLOCK + (ull)j;
                if (r < count) ((float *)vcur)[r] = vals[j];
            }
            continue;
        }
        float levels = (mode == 1) ? 65535.0f : 16777215.0f;
        float step = (tmax - tmin) / levels;
        mcur[blk] = tmin; ecur[blk] = step;
        for (int j = 0; j < SBLOCK; ++j) {
            ull r = blk * SBLOCK + (ull)j;
            if (r >= count) continue;
            float q = (step > 0.0f) ? rintf((vals[j] - tmin) / step) : 0.0f;
            q = fminf(fmaxf(q, 0.0f), levels);
            unsigned int qi = (unsigned int)q;
            if (mode == 1) ((unsigned short *)vcur)[r] = (unsigned short)qi;
            else { ((unsigned short *)vcur)[r] = (unsigned short)(qi >> 8); lcur[r] = (unsigned char)(qi & 255u); }
        }
    }
    free(vals);
}

/* sweep_max64 (solver/flow_cg/pricing_stream.py:190-249): V[full] = the longest path over the
 * subset lattice with float64 scores, two rank-indexed layers live: for every k-subset D (colex
 * rank r), V[D] = max over x in D of V[D \ {x}] + w(x, D), w a sequential float64 sum of x's row
 * scores whose menu is a subset of D, in row order. Only the maximum is kept (no predecessors). */
double ora_sweep_max64(int n, const ull *menus, const double *scores, const ll *offsets) {
    ull *binom = binom_table(n);
    ull cap = 1;
    for (int k = 0; k <= n; ++k) if (binom[n * (n + 1) + k] > cap) cap = binom[n * (n + 1) + k];
    double *prev = (double *)calloc((size_t)cap, sizeof(double));
    double *cur = (double *)calloc((size_t)cap, sizeof(double));
    for (int k = 1; k <= n; ++k) {
        ull count = binom[n * (n + 1) + k];
        for (ull r = 0; r < count; ++r) {
            /* elements of the subset of rank r, ascending */
            int el[64];
            ull rr = r, D = 0ULL;
            int b = n - 1;
            for (int t = k; t >= 1; --t) {
                while (binom[b * (n + 1) + t] > rr) --b;
                el[t - 1] = b;
                D |= 1ULL << b;
                rr -= binom[b * (n + 1) + t];
                --b;
            }
            double best = 0.0;
            int seen = 0;
            for (int j = 0; j < k; ++j) {
                /* rank of D without el[j]: the elements below keep their positions, those above move down one */
                ull rp = 0;
                for (int i = 0; i < k; ++i) {
                    if (i == j) continue;
                    int pos = i < j ? i : i - 1;
                    rp += binom[el[i] * (n + 1) + pos + 1];
                }
                double w = 0.0;
                int x = el[j];
                for (ll i = offsets[x]; i < offsets[x + 1]; ++i)
                    if ((menus[i] & D) == menus[i]) w += scores[i];
                double cand = prev[rp] + w;
                if (!seen || cand > best) { best = cand; seen = 1; }
            }
            cur[r] = best;
        }
        double *t = prev; prev = cur; cur = t;
    }
    double v = prev[0];
    free(prev); free(cur); free(binom);
    return v;
}

/* StreamPricer.price: the sweep, then the backtrace through the stored predecessor layers and
 * the mask DP on the sub-lattice of the node reached at layer k_pred
 * (solver/flow_cg/pricing_stream.py:302-412). Returns 0; vmax (float64 decode as the host does),
 * margin (0.5 * sum of per-layer max steps for u16, the sum for u24, 0 for f32) and
 * layer_step[n+1] (per-layer largest step, float32). */
int ora_price_stream(int mode, int fma_decode, int n, int k_pred, const ull *menus, const float *scores,
                     const ll *offsets, double *vmax, int *rank_pos, double *margin, float *layer_step) {
    ull *binom = binom_table(n);
    ull cap = 0, counts[65];
    for (int k = 0; k <= n; ++k) { counts[k] = binom[n * (n + 1) + k]; if (counts[k] > cap) cap = counts[k]; }
    ull nblk = (cap + SBLOCK - 1) / SBLOCK;
    size_t isz = mode == 0 ? 4 : 2;
    void *vb[2] = {calloc(cap, isz), calloc(cap, isz)};
    unsigned char *lb[2] = {(unsigned char *)calloc(cap, 1), (unsigned char *)calloc(cap, 1)};
    float *mb[2] = {(float *)calloc(nblk, 4), (float *)calloc(nblk, 4)};
    float *eb[2] = {(float *)calloc(nblk, 4), (float *)calloc(nblk, 4)};
    unsigned char **preds = (unsigned char **)calloc((size_t)n + 1, sizeof(unsigned char *));
    for (int k = k_pred; k <= n; ++k) preds[k] = (unsigned char *)calloc(counts[k], 1);
    int cur = 0, prev = 1;
    for (int k = 0; k <= n; ++k) layer_step[k] = 0.0f;
    for (int k = 1; k <= n; ++k) {
        stream_layer(mode, fma_decode, n, k, counts[k], binom, vb[prev], lb[prev], mb[prev], eb[prev],
                     vb[cur], lb[cur], mb[cur], eb[cur], k >= k_pred ? preds[k] : NULL, menus, scores,
                     offsets);
        if (mode != 0) {
            ull g = (counts[k] + SBLOCK - 1) / SBLOCK;
            float mx = eb[cur][0];
            for (ull i = 1; i < g; ++i) if (eb[cur][i] > mx) mx = eb[cur][i];
            layer_step[k] = mx;
        }
        int t = cur; cur = prev; prev = t;
    }
    double ms = 0.0;
    for (int k = 1; k <= n; ++k) ms += (double)layer_step[k];
    if (mode == 0) { *vmax = (double)((float *)vb[prev])[0]; *margin = 0.0; }
    else {
        unsigned int q = ((unsigned short *)vb[prev])[0];
        if (mode == 2) q = (q << 8) | lb[prev][0];
        *vmax = (double)mb[prev][0] + (double)q * (double)eb[prev][0];
        *margin = mode == 1 ? 0.5 * ms : ms;
    }
    /* backtrace */
    ull D = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
    int pos = 0;
    for (int k = n; k > k_pred; --k) {
        ull r = ora_colex_rank(D);
        int x = preds[k][r];
        rank_pos[x] = pos++;
        D ^= 1ULL << x;
    }
    /* sub-lattice of D: mask DP over the subsets of D with the original menus and order */
    {
        float *V = (float *)calloc((size_t)1 << n, sizeof(float));
        unsigned char *pr = (unsigned char *)calloc((size_t)1 << n, 1);
        mask_sweep(n, menus, scores, offsets, D, V, pr);
        ull Dm = D;
        int K = __builtin_popcountll(D);
        for (int i = 0; i < K; ++i) { int x = pr[Dm]; rank_pos[x] = pos + i; Dm ^= 1ULL << x; }
        free(V); free(pr);
    }
    for (int k = k_pred; k <= n; ++k) free(preds[k]);
    free(preds); free(binom);
    for (int i = 0; i < 2; ++i) { free(vb[i]); free(lb[i]); free(mb[i]); free(eb[i]); }
    return 0;
}

/* 0/1 column of a ranking (rank_pos[a] = position of a, 0 = best): row s is 1 when its
 * alternative is the best-ranked member of its menu (map_ranking_to_choice). */
void ora_ranking_column(int n, ll M, const ull *menus, const int *alts, const int *rank_pos,
                        unsigned char *out) {
    for (ll s = 0; s < M; ++s) {
        ull mask = menus[s];
        int best_alt = -1, best_rank = n + 1;
        for (int a = 0; a < n; ++a)
            if ((mask >> a) & 1ULL) {
                int r = rank_pos[a];
                if (r < best_rank) { best_rank = r; best_alt = a; }
            }
        out[s] = best_alt == alts[s] ? 1 : 0;
    }
}
