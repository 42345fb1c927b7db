// BM-ADMM on the Block-Marschak slab (sm_100a): the fused per-menu prox, the float64
// certificate (feasibility push -> upper bound, Frank-Wolfe longest path -> lower bound) and the
// certified solve loop.
//
// Reference behaviour (mingxiz/rum-testing-gpu):
//   iteration        solver/bm_admm/solver.py:33-54 (_EW_SRC), :240-254 (one_iter)
//   prox             solver/bm_admm/solver.py:66-139 (prox_all)
//   setup            solver/bm_admm/solver.py:184-238 (scatter, eigen data, cold start)
//   check loop       solver/bm_admm/solver.py:308-367 with the runner's hooks
//                    solver/rum_solver.py:869-911 (running-min push, lower bound every lb_every)
//   push (UB)        solver/common/transforms.py:94-98, solver/common/arcflow_kernels.py:357-434
//   Frank-Wolfe LB   solver/common/transforms.py:101-114, solver/common/arcflow_kernels.py:388-448
//
// Per iteration this runs 4 butterflies (A', Q^T with the eigen-space diagonal fused into its
// last store, Q, A) with the w / rhs elementwise steps fused into the A' loads and stores, and
// ONE prox kernel that also does the over-relaxed point, the z update, the s/y update with its
// nonnegativity clamp and the x2 copy (the reference's fuse_xk, prox_all, fuse_z, fuse_sy and
// copyto). The prox walks menus in mask order, so a warp's members of one alternative are 32
// consecutive entries of that alternative's block (coalesced), and projects with Michelot's
// active-set iteration in registers instead of an insertion sort.
#include <atomic>
#include <chrono>
#include <cstring>
#include <string>

#include "bfly.cuh"
#include "xform.cuh"
#include "prox.cuh"
#include "bm.cuh"
#include "ctx.cuh"

namespace rumb {

// ================================================================= prox
template <class T>
struct ProxArgs {
    int n;
    ll Nloc, nmenus;
    const T *v;         // PROX mode input
    T *out;             // PROX mode output
    const T *x;         // ITER mode input
    T *x2, *z;          // ITER mode state (updated in place)
    const T *xhat;
    const uint32_t *obsbits;
    T alpha, b1, b2, ib1, ib2;
};

enum { PROX_ONLY = 0, PROX_ITER = 1 };

template <class T, int N, int MODE>
__global__ void __launch_bounds__(128) prox_kernel(ProxArgs<T> P) {
    ll gid = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (gid >= P.nmenus) return;
    const uint32_t S = (uint32_t)(gid + 1);
    const int n = P.n;
    const int k = __popc(S);
    // observed members
    uint32_t wb = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (i < n && ((S >> i) & 1u)) {
            ll pos = (ll)i * P.Nloc + (ll)compress_bit(S ^ (1u << i), i);
            if ((P.obsbits[pos >> 5] >> (pos & 31)) & 1u) wb |= 1u << i;
        }
    }
    const bool mixed = wb != 0 && wb != S;
    double t[N];
    T q[N];
    const T two = (T)2, one = (T)1;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        t[i] = 0.0;
        q[i] = (T)0;
        if (i < n && ((S >> i) & 1u)) {
            ll pos = (ll)i * P.Nloc + (ll)compress_bit(S ^ (1u << i), i);
            T v;
            if (MODE == PROX_ITER) {
                T xi = P.x[pos], x2i = P.x2[pos], zi = P.z[pos];
                T xo = P.alpha * xi + (one - P.alpha) * x2i;
                v = xo - P.ib2 * zi;
                q[i] = zi - P.b2 * xo;                 // z' = z - b2 (xo - u) = q + b2 u
            } else {
                v = P.v[pos];
            }
            bool w = (wb >> i) & 1u;
            T xh = w ? P.xhat[pos] : (T)0;
            T wt = w ? one : (T)0;
            if (mixed) t[i] = (double)P.b2 * (double)v + 2.0 * (double)wt * (double)xh;
            else t[i] = (double)((P.b2 * v + two * wt * xh) / (P.b2 + two * wt));
        }
    }
    // threshold (Michelot's active-set iteration: the active set only shrinks, <= k rounds)
    double tau = 0.0;
    if (k > 1) {
        if (!mixed) {
            uint32_t A = S;
            double sum = 0.0;
#pragma unroll
            for (int i = 0; i < N; ++i)
                if ((A >> i) & 1u) sum += t[i];
            tau = (sum - 1.0) / (double)k;
            for (int round = 0; round < N; ++round) {
                uint32_t A2 = 0;
                double s2 = 0.0;
                int c2 = 0;
#pragma unroll
                for (int i = 0; i < N; ++i)
                    if (((A >> i) & 1u) && t[i] > tau) { A2 |= 1u << i; s2 += t[i]; ++c2; }
                if (A2 == A) break;
                A = A2;
                tau = (s2 - 1.0) / (double)c2;
            }
        } else {
            const double cw = (double)P.b2 + 2.0, cu = (double)P.b2;   // curvature observed / not
            uint32_t A = S;
            double stc = 0.0, sic = 0.0;
#pragma unroll
            for (int i = 0; i < N; ++i)
                if ((A >> i) & 1u) {
                    double c = ((wb >> i) & 1u) ? cw : cu;
                    stc += t[i] / c;
                    sic += 1.0 / c;
                }
            tau = (stc - 1.0) / sic;
            for (int round = 0; round < N; ++round) {
                uint32_t A2 = 0;
                double s2 = 0.0, i2 = 0.0;
#pragma unroll
                for (int i = 0; i < N; ++i)
                    if (((A >> i) & 1u) && t[i] > tau) {
                        double c = ((wb >> i) & 1u) ? cw : cu;
                        A2 |= 1u << i; s2 += t[i] / c; i2 += 1.0 / c;
                    }
                if (A2 == A) break;
                A = A2;
                tau = (s2 - 1.0) / i2;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (i < n && ((S >> i) & 1u)) {
            ll pos = (ll)i * P.Nloc + (ll)compress_bit(S ^ (1u << i), i);
            T u;
            if (k == 1) {
                u = one;
            } else if (mixed) {
                double c = ((wb >> i) & 1u) ? (double)P.b2 + 2.0 : (double)P.b2;
                double yv = (t[i] - tau) / c;
                u = yv > 0.0 ? (T)yv : (T)0;
            } else {
                double yv = t[i] - tau;
                u = yv > 0.0 ? (T)yv : (T)0;
            }
            if (MODE == PROX_ITER) {
                P.z[pos] = q[i] + P.b2 * u;
                P.x2[pos] = u;
            } else {
                P.out[pos] = u;
            }
        }
    }
}

template <class T, int MODE>
static void launch_prox_n(const ProxArgs<T> &P, cudaStream_t st) {
    const int TB = 128;
    unsigned grid = grid_for(P.nmenus, TB);
    int n = P.n;
    if (g_prof) {
        double S = (double)P.Nloc * n, e = sizeof(T);
        double bytes = (MODE == PROX_ITER ? 5.0 : 2.0) * S * e + S / 8.0;
        prof_begin(MODE == PROX_ITER ? (e == 8 ? "prox_fused<f64>" : "prox_fused<f32>")
                                     : (e == 8 ? "prox_only<f64>" : "prox_only<f32>"), bytes, st);
    }
#define RUMB_PROX_CASE(NN)                                          \
    if (n <= NN) {                                                  \
        prox_kernel<T, NN, MODE><<<grid, TB, 0, st>>>(P);           \
        RUMB_LAUNCH("prox_kernel");                                 \
        prof_end(st);                                               \
        return;                                                     \
    }
    RUMB_PROX_CASE(8)
    RUMB_PROX_CASE(12)
    RUMB_PROX_CASE(16)
    RUMB_PROX_CASE(20)
    RUMB_PROX_CASE(24)
    RUMB_PROX_CASE(28)
    RUMB_PROX_CASE(30)
#undef RUMB_PROX_CASE
    fail(RUMB_E_INVAL, "prox: n > 30");
}

// ================================================================= observation setup
template <class T>
__global__ void obs_setup_kernel(const uint32_t *menu, const int32_t *alt, const double *p, ll mp, int n,
                                 ll Nloc, ll *obs, T *xhat, uint32_t *obsbits, int *bad) {
    ll j = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (j >= mp) return;
    int x = alt[j];
    uint32_t m = menu[j];
    if (x < 0 || x >= n || !((m >> x) & 1u) || (n < 32 && (m >> n) != 0) || __popc(m) < 2) {
        atomicExch(bad, 1);
        obs[j] = 0;
        return;
    }
    ll pos = (ll)x * Nloc + (ll)compress_bit(m & ~(1u << x), x);
    obs[j] = pos;
    xhat[pos] = (T)p[j];
    atomicOr(&obsbits[pos >> 5], 1u << (pos & 31));
}

// ================================================================= float64 certificate
// The push works on q = Mobius(x) and recomputes the clipped weights w = max(q, 0) + eps where
// they are read, instead of storing a w slab.
__device__ __forceinline__ double wclip(double q, double eps) { return (q > 0.0 ? q : 0.0) + eps; }

__global__ void outw_kernel(const double *q, double *outw, int n, ll Nloc, double eps) {
    ll D = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    ll N = 1LL << n;
    if (D >= N) return;
    double s = 0.0;
    for (int x = 0; x < n; ++x) {
        ll bit = 1LL << x;
        if (!(D & bit)) s += wclip(q[(ll)x * Nloc + (ll)compress_bit((ull)D, x)], eps);
    }
    outw[D] = s;
}

__global__ void mass_layer_kernel(const double *q, const double *outw, double *mass, const int *nodes, ll ns,
                                  int n, ll Nloc, double eps) {
    ll i = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (i >= ns) return;
    ll C = nodes[i];
    double s = 0.0;
    for (int x = 0; x < n; ++x) {
        ll bit = 1LL << x;
        if (C & bit) {
            ll P = C ^ bit;
            double ow = outw[P];
            if (ow > 0.0) s += mass[P] * wclip(q[(ll)x * Nloc + (ll)compress_bit((ull)P, x)], eps) / ow;
        }
    }
    mass[C] = s;
}

__global__ void extract_kernel(const double *q, const double *outw, const double *mass, double *rf, int n,
                               ll Nloc, double eps) {
    ll a = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    ll m2 = (ll)n * Nloc;
    if (a >= m2) return;
    ll x = a / Nloc, rest = a - x * Nloc;
    ll T = (ll)expand_bit((ull)rest, (int)x);
    double ow = outw[T];
    rf[a] = (ow > 0.0) ? mass[T] * wclip(q[a], eps) / ow : 0.0;
}

__global__ void lpath_layer_kernel(const double *R, double *dp, const int *nodes, ll ns, int n, ll Nloc) {
    ll i = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (i >= ns) return;
    ll C = nodes[i];
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

constexpr int RED_THREADS = 1024;

// Deterministic single-block sum of the per-thread partials (fixed order for a fixed size).
__device__ __forceinline__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

// Result slots of one check (device doubles)
enum { R_PHI2 = 0, R_RY = 1, R_UB_NOW = 2, R_UB_BEST = 3, R_LB_NOW = 4, R_LB_SEED = 5, R_SLOTS = 8 };

// phi^2 = sum (p - x2[obs])^2 and sum (p - y) y at the iterate; LB scatter g[obs] = r if g
template <class T>
__global__ void obs_stats_kernel(const T *x2, const ll *obs, const double *p, ll mp, double *g, double *res,
                                 const double *yv = nullptr) {
    __shared__ double sh[32];
    double f = 0.0, ry = 0.0;
    for (ll j = threadIdx.x; j < mp; j += blockDim.x) {
        double y = yv ? yv[j] : (double)x2[obs[j]];     // yv: the observed values given directly
        double r = p[j] - y;
        f += r * r;
        ry += r * y;
        if (g) g[obs[j]] = r;
    }
    double F = block_sum(f, sh);
    double RY = block_sum(ry, sh);
    if (threadIdx.x == 0) { res[R_PHI2] = F; res[R_RY] = RY; }
}

__global__ void ub_eval_kernel(const double *xub, const ll *obs, const double *p, ll mp, double *pfit_cur,
                               double *res) {
    __shared__ double sh[32];
    double f = 0.0;
    for (ll j = threadIdx.x; j < mp; j += blockDim.x) {
        double v = xub[obs[j]];
        pfit_cur[j] = v;
        double d = v - p[j];
        f += d * d;
    }
    double F = block_sum(f, sh);
    if (threadIdx.x == 0) res[R_UB_NOW] = sqrt(F);
}

__global__ void ub_commit_kernel(const double *pfit_cur, double *pfit_best, ll mp, const double *res) {
    ll j = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (j >= mp) return;
    if (res[R_UB_NOW] < res[R_UB_BEST]) pfit_best[j] = pfit_cur[j];
}

__global__ void ub_best_kernel(double *res) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && res[R_UB_NOW] < res[R_UB_BEST]) res[R_UB_BEST] = res[R_UB_NOW];
}

__global__ void lb_final_kernel(const double *dp, ll N, double *res) {
    double rc = dp[N - 1] - res[R_RY];
    double v = res[R_PHI2] - 2.0 * rc;
    res[R_LB_NOW] = sqrt(v > 0.0 ? v : 0.0);
}

__global__ void set_doubles_kernel(double *p, int count, double v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i] = v;
}

template <class TI, class TO>
__global__ void convert_kernel(const TI *in, TO *out, ll m) {
    ll i = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (i < m) out[i] = (TO)in[i];
}

// s/y update of the reference's fuse_sy (solver/bm_admm/solver.py:47-51), small-n path
template <class T>
__global__ void sy_update_kernel(const T *Ax, T *s, T *y, ll m, T alpha, T b1, T ib1) {
    ll i = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (i >= m) return;
    T one = (T)1;
    T axor = -alpha * Ax[i] - (one - alpha) * s[i];
    T sn = ib1 * y[i] - axor;
    sn = sn > (T)0 ? sn : (T)0;
    y[i] -= b1 * (axor + sn);
    s[i] = sn;
}

// ----------------------------------------------------------------- layers (host build, cached)
const int *Ctx::layer_table(int n, std::vector<ll> &bounds) {
    auto it = layers.find(n);
    if (it != layers.end()) {
        bounds = layer_bounds[n];
        return it->second->as<int>();
    }
    ll N = 1LL << n;
    std::vector<ll> cnt(n + 2, 0);
    for (ll v = 0; v < N; ++v) cnt[__builtin_popcountll((ull)v) + 1]++;
    std::vector<ll> b(n + 2, 0);
    for (int c = 0; c <= n; ++c) b[c + 1] = b[c] + cnt[c + 1];
    std::vector<ll> fill(b.begin(), b.end() - 1);
    std::vector<int> order(N);
    for (ll v = 0; v < N; ++v) order[fill[__builtin_popcountll((ull)v)]++] = (int)v;
    auto buf = std::make_shared<DevBuf>();
    buf->ensure((size_t)N * sizeof(int));
    RUMB_CUDA(cudaMemcpy(buf->ptr, order.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice));
    layers[n] = buf;
    layer_bounds[n] = b;
    bounds = b;
    return buf->as<int>();
}

// Generic full transform in -> out (K_PLAIN passes; the certificate's Mobius, zeta and
// subset-sum butterflies). in may be float32 while out is float64 (the first pass converts).
template <class T, class TI>
static void xf_transform(int n, const TI *in, T *out, Co<T> k, cudaStream_t st) {
    if (n - 1 < 5) {
        bf_transform<T, TI>(n, in, out, k.a, k.b, k.c, k.d, st);
        return;
    }
    std::vector<XfShape> plan = xf_plan(n - 1);
    ll Nloc = 1LL << (n - 1);
    for (size_t i = 0; i < plan.size(); ++i) {
        if (i == 0) {
            XfArgs<T, TI> A{};
            A.in = in; A.out = out; A.k1 = k; A.Nloc = Nloc; A.s0 = plan[i].s0; A.B = plan[i].B;
            xf_launch<T, TI, K_PLAIN>(A, plan[i], n, st);
        } else {
            XfArgs<T, T> A{};
            A.in = out; A.out = out; A.k1 = k; A.Nloc = Nloc; A.s0 = plan[i].s0; A.B = plan[i].B;
            xf_launch<T, T, K_PLAIN>(A, plan[i], n, st);
        }
    }
}

// ----------------------------------------------------------------- certificate workspace
struct CertWork : public BmWorkBase {
    DevBuf qa, qb;            // float64 slabs
    DevBuf outw, mass, dp;    // float64 node arrays
    DevBuf obs, p;            // observed positions and p (mp)
    DevBuf pfit_cur, pfit_best;
    DevBuf res;               // R_SLOTS doubles
    ll mp = 0;
    int n = 0;
    void ensure(int n_, ll mp_) {
        n = n_;
        mp = mp_;
        ll m2 = (ll)n << (n - 1), N = 1LL << n;
        qa.ensure((size_t)m2 * 8);
        qb.ensure((size_t)m2 * 8);
        outw.ensure((size_t)N * 8);
        mass.ensure((size_t)N * 8);
        dp.ensure((size_t)N * 8);
        obs.ensure((size_t)mp * 8);
        p.ensure((size_t)mp * 8);
        pfit_cur.ensure((size_t)mp * 8);
        pfit_best.ensure((size_t)mp * 8);
        res.ensure(R_SLOTS * 8);
    }
};

static CertWork &cert_work(Ctx &c) {
    if (!c.cert) c.cert.reset(new CertWork());
    return *static_cast<CertWork *>(c.cert.get());
}

// UB part of a check: x2 (dtype T) -> q = Mobius -> push -> zeta -> ub_now, pfit; running best.
template <class T>
static void enqueue_push(Ctx &c, CertWork &W, int n, const T *x2, cudaStream_t st, const double *p_ovr = nullptr,
                         double *res_ovr = nullptr, double *pfit_ovr = nullptr) {
    const double *pp = p_ovr ? p_ovr : W.p.as<double>();
    double *rr = res_ovr ? res_ovr : W.res.as<double>();
    // the best point's observed values: the workspace's own, a batched draw's own row, or none
    double *pfit_best = res_ovr == nullptr ? W.pfit_best.as<double>() : pfit_ovr;
    ll Nloc = 1LL << (n - 1), m2 = (ll)n * Nloc, N = 1LL << n;
    const double eps = 1e-12;
    double *qa = W.qa.as<double>(), *qb = W.qb.as<double>();
    xf_transform<double, T>(n, x2, qa, Co<double>{1.0, -1.0, 0.0, 1.0}, st);     // Mobius
    outw_kernel<<<grid_for(N, 256), 256, 0, st>>>(qa, W.outw.as<double>(), n, Nloc, eps);
    RUMB_LAUNCH("outw_kernel");
    std::vector<ll> bounds;
    const int *nodes = c.layer_table(n, bounds);
    set_doubles_kernel<<<1, 32, 0, st>>>(W.mass.as<double>(), 1, 1.0);    // mass[empty set] = 1
    RUMB_LAUNCH("set_doubles");
    for (int cc = 1; cc <= n; ++cc) {
        ll lo = bounds[cc], ns = bounds[cc + 1] - lo;
        if (ns <= 0) continue;
        mass_layer_kernel<<<grid_for(ns, 256), 256, 0, st>>>(qa, W.outw.as<double>(), W.mass.as<double>(),
                                                             nodes + lo, ns, n, Nloc, eps);
        RUMB_LAUNCH("mass_layer_kernel");
    }
    extract_kernel<<<grid_for(m2, 256), 256, 0, st>>>(qa, W.outw.as<double>(), W.mass.as<double>(), qb, n, Nloc,
                                                      eps);
    RUMB_LAUNCH("extract_kernel");
    xf_transform<double, double>(n, qb, qa, Co<double>{1.0, 1.0, 0.0, 1.0}, st);  // zeta -> x_ub in qa
    ub_eval_kernel<<<1, RED_THREADS, 0, st>>>(qa, W.obs.as<ll>(), pp, W.mp, W.pfit_cur.as<double>(), rr);
    RUMB_LAUNCH("ub_eval_kernel");
    if (pfit_best) {
        ub_commit_kernel<<<grid_for(W.mp, 256), 256, 0, st>>>(W.pfit_cur.as<double>(), pfit_best, W.mp, rr);
        RUMB_LAUNCH("ub_commit_kernel");
    }
    ub_best_kernel<<<1, 32, 0, st>>>(rr);
    RUMB_LAUNCH("ub_best_kernel");
}

// phi (and the LB's residual sums); with_lb also scatters g and runs the longest path.
template <class T>
static void enqueue_stats_lb(Ctx &c, CertWork &W, int n, const T *x2, bool with_lb, cudaStream_t st,
                             const double *p_ovr = nullptr, double *res_ovr = nullptr, const double *y_ovr = nullptr) {
    const double *pp = p_ovr ? p_ovr : W.p.as<double>();
    double *rr = res_ovr ? res_ovr : W.res.as<double>();
    ll Nloc = 1LL << (n - 1), m2 = (ll)n * Nloc, N = 1LL << n;
    double *g = W.qb.as<double>();
    if (with_lb) RUMB_CUDA(cudaMemsetAsync(g, 0, (size_t)m2 * 8, st));
    obs_stats_kernel<T><<<1, RED_THREADS, 0, st>>>(x2, W.obs.as<ll>(), pp, W.mp, with_lb ? g : nullptr, rr, y_ovr);
    RUMB_LAUNCH("obs_stats_kernel");
    if (!with_lb) return;
    xf_transform<double, double>(n, g, g, Co<double>{1.0, 0.0, 1.0, 1.0}, st);    // subset sums
    std::vector<ll> bounds;
    const int *nodes = c.layer_table(n, bounds);
    double *dp = W.dp.as<double>();
    set_doubles_kernel<<<1, 32, 0, st>>>(dp, 1, 0.0);
    RUMB_LAUNCH("set_doubles");
    for (int cc = 1; cc <= n; ++cc) {
        ll lo = bounds[cc], ns = bounds[cc + 1] - lo;
        if (ns <= 0) continue;
        lpath_layer_kernel<<<grid_for(ns, 256), 256, 0, st>>>(g, dp, nodes + lo, ns, n, Nloc);
        RUMB_LAUNCH("lpath_layer_kernel");
    }
    lb_final_kernel<<<1, 1, 0, st>>>(dp, N, rr);
    RUMB_LAUNCH("lb_final_kernel");
}

// ================================================================= ADMM workspace
template <class T>
struct BmWork : public BmWorkBase {
    DevBuf x2, s, y, z, x, Ax, t1, t2, xhat, obsbits, diag, err, menu_obs;
    DevBuf snap;                 // overlapped checks: the snapshot of x2 a check reads
    int n = 0;
    void ensure(int n_) {
        n = n_;
        ll m2 = (ll)n << (n - 1);
        size_t sb = (size_t)m2 * sizeof(T);
        for (DevBuf *b : {&x2, &s, &y, &z, &x, &Ax, &t1, &t2, &xhat}) b->ensure(sb);
        obsbits.ensure((size_t)((m2 + 31) / 32) * 4);
        menu_obs.ensure((size_t)4 << n);
        diag.ensure(64 * sizeof(T));
        err.ensure(16);
    }
};

template <class T>
static BmWork<T> &bm_work(Ctx &c) {
    std::unique_ptr<BmWorkBase> &slot = sizeof(T) == 8 ? c.bm64 : c.bm32;
    if (!slot) slot.reset(new BmWork<T>());
    return *static_cast<BmWork<T> *>(slot.get());
}

// Per-bit eigen data of G = [[1, -1], [-1, 1 + p^2]] (ascending eigenvalues, orthonormal
// eigenvectors as columns of Q) and the eigen-space diagonal 1/(gamma + lambda(rest)) by the
// popcount of the rest index, lambda = ev1^pc * ev0^(nb - pc) multiplied bit by bit.
struct Eigen {
    double Q[2][2];
    double ev[2];
};

static Eigen eigen2(double p) {
    double a = 1.0, b = -1.0, d = 1.0 + p * p;
    double mid = 0.5 * (a + d), rad = std::sqrt(0.25 * (a - d) * (a - d) + b * b);
    Eigen E;
    E.ev[0] = mid - rad;
    E.ev[1] = mid + rad;
    for (int k = 0; k < 2; ++k) {
        double vx = b, vy = E.ev[k] - a;                     // (G - ev I) v = 0
        double nr = std::sqrt(vx * vx + vy * vy);
        E.Q[0][k] = vx / nr;
        E.Q[1][k] = vy / nr;
    }
    return E;
}

struct BmCoef {
    double b1, b2, ib1, ib2, alpha, p;
    double Qt[4], Q[4], AQ[4];
    // the register-tiled passes (n >= 8): Q and Q^T as q00 (1, t, t, -1) applied in unit form and
    // A Q divided by q00; the scales q00^(n-1) of Q and of Q^T move into the diagonal
    double Qu[4], AQu[4];
    std::vector<double> diag;   // by popcount: entries 0..nb as is, 32..32+nb times q00^(2 nb)
    int lo_bits = 12;           // transform window split (tuned)
    int prox_form = PROX_TILE;  // prox kernel form (tuned)
    int fuse = 1;               // two windows: P4 carries the next A' (three passes an iteration; tuned)
};

static BmCoef make_coef(int n, double beta, double alpha, double p) {
    BmCoef C;
    C.b1 = C.b2 = beta;
    C.ib1 = C.ib2 = 1.0 / beta;
    C.alpha = alpha;
    C.p = p;
    Eigen E = eigen2(p);
    C.Qt[0] = E.Q[0][0]; C.Qt[1] = E.Q[1][0]; C.Qt[2] = E.Q[0][1]; C.Qt[3] = E.Q[1][1];
    C.Q[0] = E.Q[0][0]; C.Q[1] = E.Q[0][1]; C.Q[2] = E.Q[1][0]; C.Q[3] = E.Q[1][1];
    // A Q with A = [[1, -1], [0, p]] (the raw A butterfly, solver/bm_admm/solver.py:247)
    C.AQ[0] = C.Q[0] - C.Q[2]; C.AQ[1] = C.Q[1] - C.Q[3]; C.AQ[2] = p * C.Q[2]; C.AQ[3] = p * C.Q[3];
    // Q is a reflection (det < 0): [[q00, q01], [q01, -q00]], symmetric, so Q^T = Q
    for (int i = 0; i < 4; ++i) {
        C.Qu[i] = C.Q[i] / C.Q[0];
        C.AQu[i] = C.AQ[i] / C.Q[0];
    }
    C.Qu[3] = -1.0;
    int nb = n - 1;
    double gamma = 1.0;                                  // beta2 / beta1
    C.diag.assign(64, 0.0);
    const double scale = std::pow(C.Q[0], 2.0 * nb);
    for (int pc = 0; pc <= nb; ++pc) {
        double lam = 1.0;
        for (int bit = 0; bit < nb; ++bit) lam *= (bit < pc) ? E.ev[1] : E.ev[0];
        C.diag[pc] = 1.0 / (gamma + lam);
        C.diag[32 + pc] = C.diag[pc] * scale;
    }
    return C;
}


// The reference's one_iter (solver/bm_admm/solver.py:240-254) for n <= 5: separate butterflies.
template <class T>
static void enqueue_iteration_small(BmWork<T> &W, const BmCoef &C, int n, cudaStream_t st) {
    T *x2 = W.x2.template as<T>(), *s = W.s.template as<T>(), *y = W.y.template as<T>(), *z = W.z.template as<T>();
    T *x = W.x.template as<T>(), *Ax = W.Ax.template as<T>(), *t1 = W.t1.template as<T>(), *t2 = W.t2.template as<T>();
    T p = (T)C.p;
    bf_transform<T, T>(n, t1, t1, (T)1, (T)0, (T)-1, p, st, PRO_W, y, s, (T)C.b1, EPI_RHS, z, x2, (T)C.b2,
                       (T)C.ib1);
    bf_transform<T, T>(n, t1, t2, (T)C.Qt[0], (T)C.Qt[1], (T)C.Qt[2], (T)C.Qt[3], st, PRO_PLAIN, nullptr, nullptr,
                       (T)0, EPI_DIAG, nullptr, nullptr, (T)0, (T)0, W.diag.template as<T>());
    bf_transform<T, T>(n, t2, x, (T)C.Q[0], (T)C.Q[1], (T)C.Q[2], (T)C.Q[3], st);
    bf_transform<T, T>(n, x, Ax, (T)1, (T)-1, (T)0, p, st);
    sy_update_kernel<T><<<grid_for((ll)n << (n - 1), 256), 256, 0, st>>>(Ax, s, y, (ll)n << (n - 1), (T)C.alpha,
                                                                       (T)C.b1, (T)C.ib1);
    RUMB_LAUNCH("sy_update_kernel");
}

// Device pointers of one or more draws' ADMM state (slots of bstride elements, grid.y = slot).
template <class T>
struct IterPtrs {
    T *x2, *s, *y, *z, *x, *Ax, *t1, *t2;
    const T *xhat, *diag;
    const uint32_t *menu_obs;
    unsigned int *err;
    int slots = 1;
    ll bstride = 0;
    const int *active = nullptr;
};

template <class T>
static IterPtrs<T> iter_ptrs(BmWork<T> &W) {
    IterPtrs<T> P;
    P.x2 = W.x2.template as<T>(); P.s = W.s.template as<T>(); P.y = W.y.template as<T>(); P.z = W.z.template as<T>();
    P.x = W.x.template as<T>(); P.Ax = W.Ax.template as<T>(); P.t1 = W.t1.template as<T>(); P.t2 = W.t2.template as<T>();
    P.xhat = W.xhat.template as<T>(); P.diag = W.diag.template as<T>();
    P.menu_obs = W.menu_obs.template as<uint32_t>();
    P.err = W.err.template as<unsigned int>();
    return P;
}

// One ADMM iteration: register-tiled transform passes (1 for n <= 13; with two windows 3, or 4
// unfused; more for n >= 21) and the fused prox, for every slot of I (n >= 8). seq_i / seq_n place
// the iteration in a sequence: with C.fuse and two windows, the first iteration of a sequence
// starts with P1 on the low window, iteration i applies P2 and P4A on window Y (high for even i,
// low for odd i) and P3 on the other, and the last one ends with a plain P4.
template <class T>
static void enqueue_iteration_ptrs(const IterPtrs<T> &I, const BmCoef &C, int n, cudaStream_t st, int seq_i = 0,
                                   int seq_n = 1) {
    T *x2 = I.x2, *s = I.s, *y = I.y, *z = I.z, *x = I.x, *Ax = I.Ax, *t1 = I.t1, *t2 = I.t2;
    const int K = I.slots;
    {
        T p = (T)C.p;
        Co<T> kA{(T)1, (T)0, (T)-1, p};                                    // A' (sign folded)
        Co<T> kQt{(T)C.Qu[0], (T)C.Qu[1], (T)C.Qu[2], (T)C.Qu[3]};      // Q^T = Q, unit form
        Co<T> kQ = kQt;
        Co<T> kAQ{(T)C.AQu[0], (T)C.AQu[1], (T)C.AQu[2], (T)C.AQu[3]};  // A Q / q00, A = [[1,-1],[0,p]]
        Co<T> kAr{(T)1, (T)-1, (T)0, p};                                   // A itself
        std::vector<XfShape> plan = xf_plan(n - 1, C.lo_bits);
        XfArgs<T, T> base{};
        base.Nloc = 1LL << (n - 1);
        base.b1 = (T)C.b1; base.b2 = (T)C.b2; base.ib1 = (T)C.ib1; base.alpha = (T)C.alpha;
        base.diag = I.diag + 32;                                           // with the folded scales
        base.bstride = I.bstride;
        base.active = I.active;
        auto at = [&](const XfShape &sh) { XfArgs<T, T> A = base; A.s0 = sh.s0; A.B = sh.B; return A; };
        const size_t m = plan.size() - 1;                                  // high windows
        if (m == 0) {
            XfArgs<T, T> A = at(plan[0]);
            A.y = y; A.s = s; A.z = z; A.x2 = x2; A.out = x; A.s_io = s; A.y_io = y;
            A.k1 = kA; A.k2 = kQt; A.k3 = kQ; A.k4 = kAQ;
            xf_launch<T, T, K_FULL>(A, plan[0], n, st, K);
        } else if (m == 1 && C.fuse) {
            if (seq_i == 0) {
                XfArgs<T, T> A = at(plan[0]); A.y = y; A.s = s; A.out = t1; A.k1 = kA;
                xf_launch<T, T, K_P1>(A, plan[0], n, st, K);
            }
            const XfShape &Y = (seq_i % 2 == 0) ? plan[1] : plan[0], &Xw = (seq_i % 2 == 0) ? plan[0] : plan[1];
            { XfArgs<T, T> A = at(Y); A.in = t1; A.out = t2; A.z = z; A.x2 = x2; A.k1 = kA; A.k2 = kQt;
              xf_launch<T, T, K_P2>(A, Y, n, st, K); }
            { XfArgs<T, T> A = at(Xw); A.in = t2; A.out = x; A.out2 = Ax; A.k1 = kQt; A.k2 = kQ; A.k3 = kAQ;
              A.k4 = kAr;
              xf_launch<T, T, K_P3>(A, Xw, n, st, K); }
            { XfArgs<T, T> A = at(Y); A.in = x; A.in2 = Ax; A.out = x; A.s_io = s; A.y_io = y; A.k1 = kQ;
              A.k3 = kAQ;
              if (seq_i + 1 < seq_n) {
                  A.out2 = t1; A.k4 = kA;
                  xf_launch<T, T, K_P4A>(A, Y, n, st, K);
              } else {
                  xf_launch<T, T, K_P4>(A, Y, n, st, K);
              }
            }
        } else {
            { XfArgs<T, T> A = at(plan[0]); A.y = y; A.s = s; A.out = t1; A.k1 = kA;
              xf_launch<T, T, K_P1>(A, plan[0], n, st, K); }
            for (size_t i = 1; i < m; ++i) {
                XfArgs<T, T> A = at(plan[i]); A.in = t1; A.out = t1; A.k1 = kA;
                xf_launch<T, T, K_PLAIN>(A, plan[i], n, st, K);
            }
            { XfArgs<T, T> A = at(plan[m]); A.in = t1; A.out = t2; A.z = z; A.x2 = x2; A.k1 = kA; A.k2 = kQt;
              xf_launch<T, T, K_P2>(A, plan[m], n, st, K); }
            for (size_t i = 1; i < m; ++i) {
                XfArgs<T, T> A = at(plan[i]); A.in = t2; A.out = t2; A.k1 = kQt;
                xf_launch<T, T, K_PLAIN>(A, plan[i], n, st, K);
            }
            { XfArgs<T, T> A = at(plan[0]); A.in = t2; A.out = x; A.out2 = Ax; A.k1 = kQt; A.k2 = kQ; A.k3 = kAQ;
              A.k4 = kAr;
              xf_launch<T, T, K_P3>(A, plan[0], n, st, K); }
            for (size_t i = 1; i < m; ++i) {
                XfArgs<T, T> A = at(plan[i]); A.in = x; A.in2 = Ax; A.out = x; A.out2 = Ax; A.k1 = kQ; A.k3 = kAQ;
                xf_launch<T, T, K_DUAL>(A, plan[i], n, st, K);
            }
            { XfArgs<T, T> A = at(plan[m]); A.in = x; A.in2 = Ax; A.out = x; A.s_io = s; A.y_io = y; A.k1 = kQ;
              A.k3 = kAQ;
              xf_launch<T, T, K_P4>(A, plan[m], n, st, K); }
        }
    }
    // fused prox + z + x2
    ProxTileArgs<T> P{};
    P.n = n;
    P.Nloc = 1LL << (n - 1);
    P.x = x; P.x2 = x2; P.z = z;
    P.xhat = I.xhat;
    P.menu_obs = I.menu_obs;
    P.alpha = (T)C.alpha; P.b2 = (T)C.b2; P.ib2 = (T)C.ib2;
    P.inv_c0 = (T)(1.0 / C.b2); P.inv_c1 = (T)(1.0 / (C.b2 + 2.0));
    P.err = I.err;
    P.bstride = I.bstride;
    P.active = I.active;
    if (g_prof) {
        double S = (double)P.Nloc * n * K, e = sizeof(T);
        static const char *form_name[PROX_FORMS] = {"prox_tile", "prox_lanes2", "prox_lanes4", "prox_lanes8", "prox_tau",
                                                    "prox_tau2", "prox_pair"};
        const int f = (n > PROX_LANES_MAX_N && C.prox_form != PROX_TAU && C.prox_form != PROX_TAU2 &&
                       C.prox_form != PROX_PAIR) ? PROX_TILE : C.prox_form;
        prof_begin(std::string(form_name[f]) + (e == 8 ? "<f64>" : "<f32>"), 5.0 * S * e + 4.0 * (1LL << n), st);
    }
    launch_prox_tile<T>(P, st, K, C.prox_form);
    prof_end(st);
}

// `count` iterations as one sequence (see enqueue_iteration_ptrs) for every slot of I.
template <class T>
static void enqueue_iterations_ptrs(const IterPtrs<T> &I, const BmCoef &C, int n, cudaStream_t st, int count) {
    for (int i = 0; i < count; ++i) enqueue_iteration_ptrs<T>(I, C, n, st, i, count);
}

template <class T>
static void enqueue_iteration(BmWork<T> &W, const BmCoef &C, int n, cudaStream_t st, int seq_i = 0, int seq_n = 1) {
    if (n >= PT_M + 1) {
        enqueue_iteration_ptrs<T>(iter_ptrs<T>(W), C, n, st, seq_i, seq_n);
        return;
    }
    // small lattices: separate butterflies and the thread-per-menu prox
    enqueue_iteration_small<T>(W, C, n, st);
    T *x2 = W.x2.template as<T>(), *z = W.z.template as<T>(), *x = W.x.template as<T>();
    ProxArgs<T> P{};
    P.n = n;
    P.Nloc = 1LL << (n - 1);
    P.nmenus = (1LL << n) - 1;
    P.x = x; P.x2 = x2; P.z = z;
    P.xhat = W.xhat.template as<T>();
    P.obsbits = W.obsbits.template as<uint32_t>();
    P.alpha = (T)C.alpha; P.b1 = (T)C.b1; P.b2 = (T)C.b2; P.ib1 = (T)C.ib1; P.ib2 = (T)C.ib2;
    launch_prox_n<T, PROX_ITER>(P, st);
}

template <class T>
static void enqueue_iterations(BmWork<T> &W, const BmCoef &C, int n, cudaStream_t st, int count) {
    for (int i = 0; i < count; ++i) enqueue_iteration<T>(W, C, n, st, i, count);
}

template <class T>
static void enqueue_cold_start(BmWork<T> &W, const BmCoef &C, int n, cudaStream_t st) {
    ll m2 = (ll)n << (n - 1);
    ProxArgs<T> P{};
    P.n = n;
    P.Nloc = 1LL << (n - 1);
    P.nmenus = (1LL << n) - 1;
    P.v = W.xhat.template as<T>();
    P.out = W.x2.template as<T>();
    P.xhat = W.xhat.template as<T>();
    P.obsbits = W.obsbits.template as<uint32_t>();
    P.b2 = (T)C.b2;
    launch_prox_n<T, PROX_ONLY>(P, st);
    for (DevBuf *b : {&W.s, &W.y, &W.z}) RUMB_CUDA(cudaMemsetAsync(b->ptr, 0, (size_t)m2 * sizeof(T), st));
}

// The iteration's autotuner: times a few iterations of each candidate on the workspace and keeps
// the fastest, one knob at a time -- the transform passes' low-window size (10, 11 or 12 bits;
// it sets the high-window split), then the prox kernel's form (the shared-memory tile, or 2, 4 or
// 8 lanes per menu), then with two windows the fused three-pass sequence against four passes.
// Cached per context, n and dtype; the state is reset by the caller. The environment variables
// RUMB_PROX_FORM (0 tile, 1..3 lanes 2/4/8) and RUMB_FUSE (0 / 1) pin those knobs.
static int forced_knob(const char *name, int count) {
    const char *e = getenv(name);
    if (!e || !*e) return -1;
    int v = atoi(e);
    return (v >= 0 && v < count) ? v : -1;
}
static void apply_forced(BmCoef &C) {
    int f = forced_knob("RUMB_PROX_FORM", PROX_FORMS);
    if (f >= 0) C.prox_form = f;
    f = forced_knob("RUMB_FUSE", 2);
    if (f >= 0) C.fuse = f;
}

template <class T>
static void tune_iteration(Ctx &c, BmWork<T> &W, BmCoef &C, int n, cudaStream_t st) {
    auto key = std::make_pair(n, (int)sizeof(T));
    auto it = c.tuned.find(key);
    if (it == c.tuned.end()) {
        BmCoef K = C;
        cudaEvent_t a, b;
        RUMB_CUDA(cudaEventCreate(&a));
        RUMB_CUDA(cudaEventCreate(&b));
        auto time_it = [&]() -> float {
            enqueue_iterations<T>(W, K, n, st, 2);
            RUMB_CUDA(cudaEventRecord(a, st));
            enqueue_iterations<T>(W, K, n, st, 6);
            RUMB_CUDA(cudaEventRecord(b, st));
            RUMB_CUDA(cudaEventSynchronize(b));
            float ms = 0.f;
            RUMB_CUDA(cudaEventElapsedTime(&ms, a, b));
            return ms;
        };
        int best_lo = 12, best_form = n <= PROX_LANES_MAX_N ? PROX_LANES4 : PROX_TILE, best_fuse = 1;
        if (n >= PT_M + 1) {
            K.prox_form = best_form;
            K.fuse = best_fuse;
            if (n - 1 > 10) {
                float best_ms = 1e30f;
                for (int lb : {10, 11, 12}) {
                    if (lb > n - 1) continue;
                    K.lo_bits = lb;
                    float ms = time_it();
                    if (ms < best_ms) { best_ms = ms; best_lo = lb; }
                }
            }
            K.lo_bits = best_lo;
            if (n <= PROX_LANES_MAX_N) {
                float best_ms = 1e30f;
                for (int f = 0; f < PROX_FORMS; ++f) {
                    K.prox_form = f;
                    float ms = time_it();
                    if (ms < best_ms) { best_ms = ms; best_form = f; }
                }
            }
            K.prox_form = best_form;
            if (xf_plan(n - 1, best_lo).size() == 2) {
                float best_ms = 1e30f;
                for (int f = 0; f < 2; ++f) {
                    K.fuse = f;
                    float ms = time_it();
                    if (ms < best_ms) { best_ms = ms; best_fuse = f; }
                }
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        it = c.tuned.emplace(key, std::array<int, 3>{best_lo, best_form, best_fuse}).first;
    }
    C.lo_bits = it->second[0];
    C.prox_form = it->second[1];
    C.fuse = it->second[2];
    apply_forced(C);
}

// The tuned schedule of (n, dtype) when it is known, else the defaults.
template <class T>
static void tuned_or_default(Ctx &c, BmCoef &C, int n) {
    auto it = c.tuned.find(std::make_pair(n, (int)sizeof(T)));
    if (it != c.tuned.end()) {
        C.lo_bits = it->second[0];
        C.prox_form = it->second[1];
        C.fuse = it->second[2];
    }
    apply_forced(C);
}

// ----------------------------------------------------------------- problem upload
struct DevProblem {
    DevBuf menu, alt, p;
    const uint32_t *d_menu = nullptr;
    const int32_t *d_alt = nullptr;
    const double *d_p = nullptr;
};

static void upload_problem(const rumb_bm_problem &pr, DevProblem &D, cudaStream_t st) {
    if (pr.on_device) {
        D.d_menu = pr.menu; D.d_alt = pr.alt; D.d_p = pr.p;
        return;
    }
    D.menu.ensure((size_t)pr.mp * 4);
    D.alt.ensure((size_t)pr.mp * 4);
    D.p.ensure((size_t)pr.mp * 8);
    RUMB_CUDA(cudaMemcpyAsync(D.menu.ptr, pr.menu, (size_t)pr.mp * 4, cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(D.alt.ptr, pr.alt, (size_t)pr.mp * 4, cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(D.p.ptr, pr.p, (size_t)pr.mp * 8, cudaMemcpyHostToDevice, st));
    D.d_menu = D.menu.as<uint32_t>(); D.d_alt = D.alt.as<int32_t>(); D.d_p = D.p.as<double>();
}

// observations -> obs positions + p (cert workspace), xhat + obsbits (ADMM workspace of dtype T)
template <class T>
static void setup_obs(Ctx &c, CertWork &CW, BmWork<T> *W, const rumb_bm_problem &pr, const DevProblem &D,
                      cudaStream_t st) {
    int n = pr.n;
    ll Nloc = 1LL << (n - 1), m2 = (ll)n * Nloc;
    DevBuf bad;
    bad.ensure(4);
    RUMB_CUDA(cudaMemsetAsync(bad.ptr, 0, 4, st));
    DevBuf tmpx, tmpb;
    T *xhat;
    uint32_t *bits;
    if (W) {
        xhat = W->xhat.template as<T>();
        bits = W->obsbits.template as<uint32_t>();
    } else {
        tmpx.ensure((size_t)m2 * sizeof(T));
        tmpb.ensure((size_t)((m2 + 31) / 32) * 4);
        xhat = tmpx.as<T>();
        bits = tmpb.as<uint32_t>();
    }
    RUMB_CUDA(cudaMemsetAsync(xhat, 0, (size_t)m2 * sizeof(T), st));
    RUMB_CUDA(cudaMemsetAsync(bits, 0, (size_t)((m2 + 31) / 32) * 4, st));
    obs_setup_kernel<T><<<grid_for(pr.mp, 256), 256, 0, st>>>(D.d_menu, D.d_alt, D.d_p, pr.mp, n, Nloc,
                                                              CW.obs.as<ll>(), xhat, bits, bad.as<int>());
    RUMB_LAUNCH("obs_setup_kernel");
    RUMB_CUDA(cudaMemcpyAsync(CW.p.ptr, D.d_p, (size_t)pr.mp * 8, cudaMemcpyDeviceToDevice, st));
    if (W) {
        launch_menu_obs(bits, n, Nloc, W->menu_obs.template as<uint32_t>(), st);
    }
    int hbad = 0;
    RUMB_CUDA(cudaMemcpyAsync(&hbad, bad.ptr, 4, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    if (hbad) fail(RUMB_E_INVAL, "an observed row's alternative is not in its menu, is out of range, or its menu has "
                                 "fewer than 2 members");
}

static void check_problem(const rumb_bm_problem *pr) {
    if (!pr) fail(RUMB_E_INVAL, "problem is NULL");
    if (pr->n < 2 || pr->n > 30) fail(RUMB_E_INVAL, "bm_admm handles 2 <= n <= 30");
    if (pr->mp < 1) fail(RUMB_E_INVAL, "no observed rows");
    if (!pr->menu || !pr->alt || !pr->p) fail(RUMB_E_INVAL, "menu, alt and p must not be NULL");
}

static void check_params(const rumb_bm_params *par) {
    if (!par) fail(RUMB_E_INVAL, "params is NULL");
    if (par->check < 1 || par->lb_every < 1 || par->max_iter < 1)
        fail(RUMB_E_INVAL, "check, lb_every and max_iter must be >= 1");
    if (!(par->beta > 0.0) || !std::isfinite(par->beta)) fail(RUMB_E_INVAL, "beta must be > 0");
    if (!std::isfinite(par->alpha) || !std::isfinite(par->precond_p)) fail(RUMB_E_INVAL, "alpha and precond_p must be finite");
    if (par->dtype < RUMB_F64 || par->dtype > RUMB_MIXED) fail(RUMB_E_INVAL, "dtype must be RUMB_F64, RUMB_F32 or RUMB_MIXED");
}


template <class T>
static void copy_state_in(BmWork<T> &W, const rumb_bm_state &st, ll m2, cudaStream_t s) {
    DevBuf *dst[4] = {&W.x2, &W.s, &W.y, &W.z};
    const DevBuf *src[4] = {&st.x2, &st.s, &st.y, &st.z};
    for (int i = 0; i < 4; ++i) {
        if ((st.dtype == RUMB_F64) == (sizeof(T) == 8)) {
            RUMB_CUDA(cudaMemcpyAsync(dst[i]->ptr, src[i]->ptr, (size_t)m2 * sizeof(T), cudaMemcpyDeviceToDevice, s));
        } else if (st.dtype == RUMB_F64) {
            convert_kernel<double, T><<<grid_for(m2, 256), 256, 0, s>>>(src[i]->as<double>(), dst[i]->as<T>(), m2);
            RUMB_LAUNCH("convert_kernel");
        } else {
            convert_kernel<float, T><<<grid_for(m2, 256), 256, 0, s>>>(src[i]->as<float>(), dst[i]->as<T>(), m2);
            RUMB_LAUNCH("convert_kernel");
        }
    }
}

template <class T>
static rumb_bm_state *copy_state_out(BmWork<T> &W, int n, int device, cudaStream_t s) {
    ll m2 = (ll)n << (n - 1);
    rumb_bm_state *st = new rumb_bm_state();
    st->n = n;
    st->dtype = sizeof(T) == 8 ? RUMB_F64 : RUMB_F32;
    st->device = device;
    try {
        DevBuf *dst[4] = {&st->x2, &st->s, &st->y, &st->z};
        const DevBuf *src[4] = {&W.x2, &W.s, &W.y, &W.z};
        for (int i = 0; i < 4; ++i) {
            dst[i]->ensure((size_t)m2 * sizeof(T));
            RUMB_CUDA(cudaMemcpyAsync(dst[i]->ptr, src[i]->ptr, (size_t)m2 * sizeof(T), cudaMemcpyDeviceToDevice, s));
        }
    } catch (...) {
        delete st;
        throw;
    }
    return st;
}

// Converts a float32 state into the float64 workspace (the mixed mode's hand-over).
static void promote_state(BmWork<float> &F, BmWork<double> &D, ll m2, cudaStream_t s) {
    const DevBuf *src[4] = {&F.x2, &F.s, &F.y, &F.z};
    DevBuf *dst[4] = {&D.x2, &D.s, &D.y, &D.z};
    for (int i = 0; i < 4; ++i) {
        convert_kernel<float, double><<<grid_for(m2, 256), 256, 0, s>>>(src[i]->as<float>(), dst[i]->as<double>(), m2);
        RUMB_LAUNCH("convert_kernel");
    }
}

// ----------------------------------------------------------------- graphs
struct Graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    long long kernels = 0;     // kernel launches captured (each replay launches them all)
    ~Graph() { reset(); }
    void reset() {
        if (e) cudaGraphExecDestroy(e);
        if (g) cudaGraphDestroy(g);
        e = nullptr;
        g = nullptr;
    }
    template <class F>
    void capture(cudaStream_t st, F &&fn) {
        reset();
        RUMB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const long long before = g_launches;
        try {
            fn();
        } catch (...) {
            g_launches = before;
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(st, &tmp);
            if (tmp) cudaGraphDestroy(tmp);
            throw;
        }
        kernels = g_launches - before;     // captured, not yet run
        g_launches = before;
        RUMB_CUDA(cudaStreamEndCapture(st, &g));
        RUMB_CUDA(cudaGraphInstantiate(&e, g, 0));
    }
    void launch(cudaStream_t st) {
        RUMB_CUDA(cudaGraphLaunch(e, st));
        g_launches += kernels;
    }
};

static int graph_chunk(int check) {
    int k = 1;
    for (int d = 1; d <= 32 && d <= check; ++d)
        if (check % d == 0) k = d;
    return k;
}

using Clock = std::chrono::steady_clock;
static double secs(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

// One leg of the solve in dtype T: iterate + check until a stop. Returns true when the solve
// is over (any stop), false when a mixed-mode float32 leg stalled and float64 should take over.
struct LoopState {
    ll it = 0, it32 = 0;
    int checks = 0, n_lb = 0;
    double ub = INFINITY, lb = 0.0, phi = NAN;
    int stop = RUMB_STOP_MAX_ITER;
    double push_s = 0.0;
    std::vector<double> gaps;   // mixed mode: the bracket's gap at every check
};

// The check loop with every check overlapped with the next interval's iterations: the iterations
// run on the context's stream, a snapshot of x2 is copied there, and the check (phi, push, lower
// bound) runs on the second stream on the snapshot while the following interval iterates. The host
// reads check k after enqueueing interval k + 1, so a stop lands one interval after its check.
template <class T>
static bool run_leg_overlap(Ctx &c, CertWork &CW, BmWork<T> &W, const rumb_bm_problem &pr,
                            const rumb_bm_params &par, LoopState &L, Clock::time_point t0, bool stall_exit,
                            Graph &g_iter, int chunk, rumb_trace_fn trace, void *user) {
    const int n = pr.n;
    const ll m2 = (ll)n << (n - 1);
    cudaStream_t st = c.own;
    c.ensure_aux();
    cudaStream_t cs = c.aux;
    W.snap.ensure((size_t)m2 * sizeof(T));
    T *x2s = W.snap.template as<T>();
    Graph h_ub, h_ublb;
    h_ub.capture(cs, [&] {
        enqueue_stats_lb<T>(c, CW, n, x2s, false, cs);
        enqueue_push<T>(c, CW, n, x2s, cs);
    });
    h_ublb.capture(cs, [&] {
        enqueue_stats_lb<T>(c, CW, n, x2s, true, cs);
        enqueue_push<T>(c, CW, n, x2s, cs);
    });
    struct AuxSync {   // no check may outlive the loop (its graphs and the snapshot)
        cudaStream_t s;
        ~AuxSync() { cudaStreamSynchronize(s); }
    } aux_sync{cs};
    RUMB_CUDA(cudaEventRecord(c.ev_snap, st));        // the set-up on st comes before any check
    RUMB_CUDA(cudaStreamWaitEvent(cs, c.ev_snap, 0));
    RUMB_CUDA(cudaEventRecord(c.ev_done, cs));
    double *res = c.res_host;
    bool pending = false, pend_lb = false;
    ll pend_it = 0;
    // 0 go on, 1 stop, 2 float32 stall (hand over)
    auto process = [&]() -> int {
        RUMB_CUDA(cudaEventSynchronize(c.ev_done));
        pending = false;
        L.checks++;
        L.phi = std::sqrt(res[R_PHI2]);
        L.ub = res[R_UB_BEST];
        if (pend_lb) {
            L.n_lb++;
            if (res[R_LB_NOW] > L.lb) L.lb = res[R_LB_NOW];
        }
        if (trace) trace(user, pend_it, secs(t0, Clock::now()), L.phi, L.ub, L.lb);
        if (std::isfinite(par.ub_target) && L.ub <= par.ub_target) { L.stop = RUMB_STOP_UB_TARGET; return 1; }
        if (std::isfinite(par.lb_target) && L.lb >= par.lb_target) { L.stop = RUMB_STOP_LB_TARGET; return 1; }
        double gap = L.ub - L.lb;
        if (par.abs_tol >= 0 && gap <= par.abs_tol) { L.stop = RUMB_STOP_GAP_ABS; return 1; }
        if (par.rel_tol >= 0 && L.lb > 0 && gap / L.lb <= par.rel_tol) { L.stop = RUMB_STOP_GAP_REL; return 1; }
        if (stall_exit) {
            L.gaps.push_back(gap);
            size_t Wn = (size_t)(par.stall_checks > 0 ? par.stall_checks : 1);
            if (L.gaps.size() > Wn && gap > (1.0 - par.stall_rtol) * L.gaps[L.gaps.size() - 1 - Wn]) return 2;
        }
        return 0;
    };
    auto finish = [&](int r) -> bool {
        RUMB_CUDA(cudaStreamSynchronize(st));
        RUMB_CUDA(cudaStreamSynchronize(cs));
        return r != 2;
    };
    while (L.it < par.max_iter) {
        for (int i = 0; i < par.check / chunk; ++i) g_iter.launch(st);
        L.it += par.check;
        if (sizeof(T) == 4) L.it32 += par.check;
        RUMB_CUDA(cudaStreamWaitEvent(st, c.ev_done, 0));   // the last check no longer reads the snapshot
        RUMB_CUDA(cudaMemcpyAsync(x2s, W.x2.ptr, (size_t)m2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
        RUMB_CUDA(cudaEventRecord(c.ev_snap, st));
        if (pending) {
            auto tp = Clock::now();
            int r = process();
            L.push_s += secs(tp, Clock::now());
            if (r) return finish(r);
        }
        double el = secs(t0, Clock::now());
        if ((par.time_limit > 0 && el > par.time_limit) || c.cancel.load()) {
            L.stop = c.cancel.load() ? RUMB_STOP_CANCEL : RUMB_STOP_TIME;
            return finish(1);
        }
        const bool want_lb = (L.checks % par.lb_every) == 0;
        RUMB_CUDA(cudaStreamWaitEvent(cs, c.ev_snap, 0));
        (want_lb ? h_ublb : h_ub).launch(cs);
        RUMB_CUDA(cudaMemcpyAsync(res, CW.res.ptr, R_SLOTS * sizeof(double), cudaMemcpyDeviceToHost, cs));
        RUMB_CUDA(cudaEventRecord(c.ev_done, cs));
        pending = true;
        pend_lb = want_lb;
        pend_it = L.it;
    }
    if (pending) {
        int r = process();
        if (r) return finish(r);
    }
    L.stop = RUMB_STOP_MAX_ITER;
    return finish(1);
}

template <class T>
static bool run_leg(Ctx &c, CertWork &CW, BmWork<T> &W, const BmCoef &C, const rumb_bm_problem &pr,
                    const rumb_bm_params &par, LoopState &L, Clock::time_point t0, bool stall_exit,
                    rumb_trace_fn trace, void *user) {
    int n = pr.n;
    cudaStream_t st = c.own;
    int chunk = graph_chunk(par.check);
    Graph g_iter, g_ub, g_ublb;
    bool graphs = par.use_graph != 0;
    if (graphs) {
        g_iter.capture(st, [&] { enqueue_iterations<T>(W, C, n, st, chunk); });
        g_ub.capture(st, [&] {
            enqueue_stats_lb<T>(c, CW, n, W.x2.template as<T>(), false, st);
            enqueue_push<T>(c, CW, n, W.x2.template as<T>(), st);
        });
        g_ublb.capture(st, [&] {
            enqueue_stats_lb<T>(c, CW, n, W.x2.template as<T>(), true, st);
            enqueue_push<T>(c, CW, n, W.x2.template as<T>(), st);
        });
    }
    if (graphs && par.overlap_check) return run_leg_overlap<T>(c, CW, W, pr, par, L, t0, stall_exit, g_iter, chunk,
                                                              trace, user);
    double res[R_SLOTS];
    while (L.it < par.max_iter) {
        if (graphs) {
            for (int i = 0; i < par.check / chunk; ++i) g_iter.launch(st);
        } else {
            enqueue_iterations<T>(W, C, n, st, par.check);
        }
        L.it += par.check;
        if (sizeof(T) == 4) L.it32 += par.check;
        double el = secs(t0, Clock::now());
        if (par.time_limit > 0 && el > par.time_limit) {
            RUMB_CUDA(cudaStreamSynchronize(st));
            L.stop = RUMB_STOP_TIME;
            return true;
        }
        if (c.cancel.load()) {
            RUMB_CUDA(cudaStreamSynchronize(st));
            L.stop = RUMB_STOP_CANCEL;
            return true;
        }
        bool want_lb = (L.checks % par.lb_every) == 0;
        auto tp = Clock::now();
        if (graphs) {
            (want_lb ? g_ublb : g_ub).launch(st);
        } else {
            enqueue_stats_lb<T>(c, CW, n, W.x2.template as<T>(), want_lb, st);
            enqueue_push<T>(c, CW, n, W.x2.template as<T>(), st);
        }
        RUMB_CUDA(cudaMemcpyAsync(res, CW.res.ptr, sizeof(res), cudaMemcpyDeviceToHost, st));
        unsigned int dev_err = 0;
        RUMB_CUDA(cudaMemcpyAsync(&dev_err, W.err.ptr, 4, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaStreamSynchronize(st));
        if (dev_err) fail(RUMB_E_TIMEOUT, "a kernel's bounded wait for its TMA copies gave up");
        L.push_s += secs(tp, Clock::now());
        L.checks++;
        L.phi = std::sqrt(res[R_PHI2]);
        L.ub = res[R_UB_BEST];
        if (want_lb) {
            L.n_lb++;
            if (res[R_LB_NOW] > L.lb) L.lb = res[R_LB_NOW];
        }
        if (trace) trace(user, L.it, secs(t0, Clock::now()), L.phi, L.ub, L.lb);
        if (std::isfinite(par.ub_target) && L.ub <= par.ub_target) { L.stop = RUMB_STOP_UB_TARGET; return true; }
        if (std::isfinite(par.lb_target) && L.lb >= par.lb_target) { L.stop = RUMB_STOP_LB_TARGET; return true; }
        double gap = L.ub - L.lb;
        if (par.abs_tol >= 0 && gap <= par.abs_tol) { L.stop = RUMB_STOP_GAP_ABS; return true; }
        if (par.rel_tol >= 0 && L.lb > 0 && gap / L.lb <= par.rel_tol) { L.stop = RUMB_STOP_GAP_REL; return true; }
        if (stall_exit) {
            // A float32 state's bracket stops closing at its rounding floor: hand over to float64
            // once the gap has shrunk by less than stall_rtol over the last stall_checks checks.
            L.gaps.push_back(gap);
            size_t W = (size_t)(par.stall_checks > 0 ? par.stall_checks : 1);
            if (L.gaps.size() > W && gap > (1.0 - par.stall_rtol) * L.gaps[L.gaps.size() - 1 - W]) return false;
        }
    }
    L.stop = RUMB_STOP_MAX_ITER;
    return true;
}

// Device bytes of one solve, counted from the buffers it ensures: BmWork (9 slabs, the snapshot
// slab, observation bits, per-menu observed masks, diagonal, error word) per state dtype, the
// float64 certificate (2 slabs, 3 node arrays, 4 row arrays, result words), the popcount-ordered
// node ids and the uploaded rows.
size_t bm_plan_bytes(int n, ll mp, int dtype) {
    if (n < 2 || n > 30) fail(RUMB_E_INVAL, "bm_plan: 2 <= n <= 30");
    if (mp < 1) fail(RUMB_E_INVAL, "bm_plan: mp >= 1");
    if (dtype != RUMB_F64 && dtype != RUMB_F32 && dtype != RUMB_MIXED) fail(RUMB_E_INVAL, "bm_plan: dtype");
    const size_t m2 = (size_t)n << (n - 1), N = (size_t)1 << n;
    auto work = [&](size_t e) { return 10 * m2 * e + (m2 + 31) / 32 * 4 + 4 * N + 64 * e + 16; };
    size_t b = 0;
    if (dtype != RUMB_F64) b += work(4);
    if (dtype != RUMB_F32) b += work(8);
    b += 2 * m2 * 8 + 3 * N * 8 + 4 * (size_t)mp * 8 + R_SLOTS * 8;   // certificate
    b += 4 * N;                                                        // node ids by popcount
    b += 16 * (size_t)mp;                                              // rows: menu, alt, p
    return b;
}

int bm_solve(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, const rumb_bm_state *warm,
             rumb_bm_state **keep, rumb_bm_result *out, double *p_fit, rumb_trace_fn trace, void *user) {
    check_problem(pr);
    check_params(par);
    if (!out) fail(RUMB_E_INVAL, "result is NULL");
    auto t0 = Clock::now();
    const long long launches0 = g_launches;
    int n = pr->n;
    ll m2 = (ll)n << (n - 1);
    if (warm && (warm->n != n)) fail(RUMB_E_INVAL, "warm state was kept for another n");
    cudaStream_t st = c.own;
    c.cancel.store(0);
    c.join_in();
    cudaEvent_t e0, e1;
    RUMB_CUDA(cudaEventCreate(&e0));
    RUMB_CUDA(cudaEventCreate(&e1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } eg{e0, e1};
    RUMB_CUDA(cudaEventRecord(e0, st));

    CertWork &CW = cert_work(c);
    CW.ensure(n, pr->mp);
    DevProblem D;
    upload_problem(*pr, D, st);
    BmCoef C = make_coef(n, par->beta, par->alpha, par->precond_p);
    bool use32 = par->dtype != RUMB_F64;
    BmWork<double> *W64 = nullptr;
    BmWork<float> *W32 = nullptr;
    if (use32) { W32 = &bm_work<float>(c); W32->ensure(n); }
    if (!use32 || par->dtype == RUMB_MIXED) { W64 = &bm_work<double>(c); W64->ensure(n); }
    if (W32) setup_obs<float>(c, CW, W32, *pr, D, st);
    if (W64) setup_obs<double>(c, CW, W64, *pr, D, st);
    if (W32) RUMB_CUDA(cudaMemsetAsync(W32->err.ptr, 0, 16, st));
    if (W64) RUMB_CUDA(cudaMemsetAsync(W64->err.ptr, 0, 16, st));
    std::vector<float> d32(C.diag.begin(), C.diag.end());
    if (W32) RUMB_CUDA(cudaMemcpyAsync(W32->diag.ptr, d32.data(), d32.size() * 4, cudaMemcpyHostToDevice, st));
    if (W64) RUMB_CUDA(cudaMemcpyAsync(W64->diag.ptr, C.diag.data(), C.diag.size() * 8, cudaMemcpyHostToDevice, st));
    // transform split (tuned once per context, n and dtype), then the initial state
    BmCoef C64 = C;
    if (W32) {
        enqueue_cold_start<float>(*W32, C, n, st);
        tune_iteration<float>(c, *W32, C, n, st);
    }
    if (W64) {
        enqueue_cold_start<double>(*W64, C64, n, st);
        tune_iteration<double>(c, *W64, C64, n, st);
    }
    if (!W32) C = C64;
    if (use32) {
        if (warm) copy_state_in<float>(*W32, *warm, m2, st);
        else enqueue_cold_start<float>(*W32, C, n, st);
    } else {
        if (warm) copy_state_in<double>(*W64, *warm, m2, st);
        else enqueue_cold_start<double>(*W64, C, n, st);
    }
    set_doubles_kernel<<<1, 32, 0, st>>>(CW.res.as<double>(), R_SLOTS, 0.0);
    RUMB_LAUNCH("set_doubles");
    set_doubles_kernel<<<1, 32, 0, st>>>(CW.res.as<double>() + R_UB_BEST, 1, INFINITY);
    RUMB_LAUNCH("set_doubles");
    std::vector<ll> bounds;
    c.layer_table(n, bounds);
    RUMB_CUDA(cudaStreamSynchronize(st));
    auto t_setup = Clock::now();

    LoopState L;
    bool final_dtype64 = !use32;
    if (use32) {
        // a float32 state stops at its rounding floor: mixed hands over to float64, float32 ends
        bool stall_exit = par->dtype == RUMB_MIXED || par->stall_checks > 0;
        bool done = run_leg<float>(c, CW, *W32, C, *pr, *par, L, t0, stall_exit, trace, user);
        if (!done && par->dtype == RUMB_MIXED) {
            promote_state(*W32, *W64, m2, st);
            final_dtype64 = true;
            run_leg<double>(c, CW, *W64, C64, *pr, *par, L, t0, false, trace, user);
        } else if (!done) {
            L.stop = RUMB_STOP_STALL;
        }
    } else {
        run_leg<double>(c, CW, *W64, C, *pr, *par, L, t0, false, trace, user);
    }
    RUMB_CUDA(cudaEventRecord(e1, st));
    if (p_fit && std::isfinite(L.ub))
        RUMB_CUDA(cudaMemcpyAsync(p_fit, CW.pfit_best.ptr, (size_t)pr->mp * 8, cudaMemcpyDeviceToHost, st));
    if (keep) {
        *keep = final_dtype64 ? copy_state_out<double>(*W64, n, c.device, st)
                              : copy_state_out<float>(*W32, n, c.device, st);
    }
    RUMB_CUDA(cudaStreamSynchronize(st));
    float dms = 0.f;
    RUMB_CUDA(cudaEventElapsedTime(&dms, e0, e1));
    auto t_end = Clock::now();
    out->lb = L.lb;
    out->ub = L.ub;
    out->phi = L.phi;
    out->iters = L.it;
    out->iters_f32 = L.it32;
    out->stop = L.stop;
    out->n_push = L.checks;
    out->n_lb = L.n_lb;
    out->setup_s = secs(t0, t_setup);
    out->solve_s = secs(t_setup, t_end);
    out->push_s = L.push_s;
    out->per_iter_ms = L.it > 0 ? 1e3 * out->solve_s / (double)L.it : 0.0;
    out->device_ms = dms;
    out->launches = g_launches - launches0;
    c.join_out();
    return RUMB_OK;
}

int bm_iterate(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, void *x2, void *s, void *y, void *z,
               int iters, int cold) {
    check_problem(pr);
    check_params(par);
    int n = pr->n;
    ll m2 = (ll)n << (n - 1);
    cudaStream_t st = c.own;
    c.join_in();
    CertWork &CW = cert_work(c);
    CW.ensure(n, pr->mp);
    DevProblem D;
    upload_problem(*pr, D, st);
    BmCoef C = make_coef(n, par->beta, par->alpha, par->precond_p);
    auto run = [&](auto tag) {
        using T = decltype(tag);
        BmWork<T> &W = bm_work<T>(c);
        W.ensure(n);
        setup_obs<T>(c, CW, &W, *pr, D, st);
        RUMB_CUDA(cudaMemsetAsync(W.err.ptr, 0, 16, st));
        std::vector<T> dg(C.diag.begin(), C.diag.end());
        RUMB_CUDA(cudaMemcpyAsync(W.diag.ptr, dg.data(), dg.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        size_t sb = (size_t)m2 * sizeof(T);
        tuned_or_default<T>(c, C, n);
        if (cold) {
            enqueue_cold_start<T>(W, C, n, st);
        } else {
            RUMB_CUDA(cudaMemcpyAsync(W.x2.ptr, x2, sb, cudaMemcpyHostToDevice, st));
            RUMB_CUDA(cudaMemcpyAsync(W.s.ptr, s, sb, cudaMemcpyHostToDevice, st));
            RUMB_CUDA(cudaMemcpyAsync(W.y.ptr, y, sb, cudaMemcpyHostToDevice, st));
            RUMB_CUDA(cudaMemcpyAsync(W.z.ptr, z, sb, cudaMemcpyHostToDevice, st));
        }
        enqueue_iterations<T>(W, C, n, st, iters);
        RUMB_CUDA(cudaMemcpyAsync(x2, W.x2.ptr, sb, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaMemcpyAsync(s, W.s.ptr, sb, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaMemcpyAsync(y, W.y.ptr, sb, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaMemcpyAsync(z, W.z.ptr, sb, cudaMemcpyDeviceToHost, st));
        unsigned int dev_err = 0;
        RUMB_CUDA(cudaMemcpyAsync(&dev_err, W.err.ptr, 4, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaStreamSynchronize(st));
        if (dev_err) fail(RUMB_E_TIMEOUT, "a kernel's bounded wait for its TMA copies gave up");
    };
    if (par->dtype == RUMB_F64) run(double());
    else run(float());
    c.join_out();
    return RUMB_OK;
}

thread_local Prof *g_prof = nullptr;

// Runs `iters` iterations eagerly from the cold start with an event pair around every launch;
// returns per-kernel-name launches, total milliseconds and algorithmic bytes per launch.
int bm_profile(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, int warmup, int iters, rumb_kernel_stat *stats,
               int cap, int *count) {
    check_problem(pr);
    check_params(par);
    if (!stats || !count || cap < 1) fail(RUMB_E_INVAL, "profile: stats buffer");
    int n = pr->n;
    cudaStream_t st = c.own;
    c.join_in();
    CertWork &CW = cert_work(c);
    CW.ensure(n, pr->mp);
    DevProblem D;
    upload_problem(*pr, D, st);
    BmCoef C = make_coef(n, par->beta, par->alpha, par->precond_p);
    Prof prof;
    prof.st = st;
    bool prof_graph = true;
    auto run = [&](auto tag) {
        using T = decltype(tag);
        BmWork<T> &W = bm_work<T>(c);
        W.ensure(n);
        setup_obs<T>(c, CW, &W, *pr, D, st);
        RUMB_CUDA(cudaMemsetAsync(W.err.ptr, 0, 16, st));
        std::vector<T> dg(C.diag.begin(), C.diag.end());
        RUMB_CUDA(cudaMemcpyAsync(W.diag.ptr, dg.data(), dg.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        enqueue_cold_start<T>(W, C, n, st);
        tune_iteration<T>(c, W, C, n, st);
        enqueue_cold_start<T>(W, C, n, st);
        enqueue_iterations<T>(W, C, n, st, std::max(warmup, 3));      // warm-up
        RUMB_CUDA(cudaStreamSynchronize(st));
        // one check first, so that its cached tables exist before the capture (no allocation inside)
        if (par->lb_every > 0) {
            enqueue_stats_lb<T>(c, CW, n, W.x2.template as<T>(), true, st);
            enqueue_push<T>(c, CW, n, W.x2.template as<T>(), st);
            RUMB_CUDA(cudaStreamSynchronize(st));
        }
        auto body = [&] {
            enqueue_iterations<T>(W, C, n, st, iters);
            if (par->lb_every > 0) {
                enqueue_stats_lb<T>(c, CW, n, W.x2.template as<T>(), true, st);
                enqueue_push<T>(c, CW, n, W.x2.template as<T>(), st);
            }
        };
        // the profiled iterations and one check captured as a CUDA graph, as a solve replays them,
        // with an event recorded before and after every kernel; the graph runs twice and the
        // second run's events are read. Where the driver cannot time events recorded by a graph,
        // the same launches run eagerly instead.
        for (int i = 0; i < 64 * (iters + 4); ++i) {
            cudaEvent_t e;
            RUMB_CUDA(cudaEventCreate(&e));
            prof.pool.push_back(e);
        }
        Graph gp;
        g_prof = &prof;
        try {
            gp.capture(st, body);
        } catch (...) {
            g_prof = nullptr;
            throw;
        }
        g_prof = nullptr;
        gp.launch(st);
        RUMB_CUDA(cudaStreamSynchronize(st));
        gp.launch(st);
        RUMB_CUDA(cudaStreamSynchronize(st));
        float probe = 0.f;
        if (!prof.recs.empty() && cudaEventElapsedTime(&probe, prof.recs[0].a, prof.recs[0].b) != cudaSuccess) {
            cudaGetLastError();
            for (auto &r : prof.recs) {
                cudaEventDestroy(r.a);
                cudaEventDestroy(r.b);
            }
            prof.recs.clear();
            prof_graph = false;
            g_prof = &prof;
            try {
                body();
            } catch (...) {
                g_prof = nullptr;
                throw;
            }
            g_prof = nullptr;
            RUMB_CUDA(cudaStreamSynchronize(st));
        }
    };
    if (par->dtype == RUMB_F64) run(double());
    else run(float());
    std::vector<std::string> names;
    std::map<std::string, rumb_kernel_stat> agg;
    for (auto &r : prof.recs) {
        float ms = 0.f;
        if (r.b) RUMB_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        cudaEventDestroy(r.a);
        if (r.b) cudaEventDestroy(r.b);
        auto it = agg.find(r.name);
        if (it == agg.end()) {
            rumb_kernel_stat k{};
            snprintf(k.name, sizeof k.name, "%s", r.name.c_str());
            k.bytes_per_launch = r.bytes;
            it = agg.emplace(r.name, k).first;
            names.push_back(r.name);
        }
        it->second.launches += 1;
        it->second.total_ms += ms;
        it->second.graph = prof_graph ? 1 : 0;
    }
    int k = 0;
    for (auto &nm : names) {
        if (k >= cap) break;
        stats[k++] = agg[nm];
    }
    *count = k;
    c.join_out();
    return RUMB_OK;
}

// ================================================================= batched draws
// Many draws of one menu structure (the bootstrap's perturbed points) solved together: K slots of
// ADMM state live side by side (slot k at k * S), one CUDA graph advances every active slot by a
// check interval (grid.y = slot, retired slots skip their CTAs), each active slot then gets its
// float64 check, and the host retires finished draws and refills their slots from the queue.
// Slots are admitted by device memory: K = min(B, mem_fraction * free / bytes per slot).

// x[obs[j]] = y[j]: a draw's predicted fit written into its state's observed entries
template <class T>
__global__ void scatter_vals_kernel(const ll *obs, const double *y, ll mp, T *x) {
    ll j = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (j < mp) x[obs[j]] = (T)y[j];
}

__global__ void copy_double_kernel(double *dst, const double *src) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *src;
}

__global__ void scatter_rows_kernel(const ll *obs, const double *p, ll mp, double *p_dst, float *xf, double *xd) {
    ll j = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (j >= mp) return;
    double v = p[j];
    p_dst[j] = v;
    if (xf) xf[obs[j]] = (float)v;
    if (xd) xd[obs[j]] = v;
}

template <class T>
struct BatchWork : public BmWorkBase {
    DevBuf x2, s, y, z, x, Ax, t1, t2, xhat;   // K slabs each
    DevBuf obsbits, menu_obs, diag, err, active, p, res, pfit;
    int K = 0, n = 0;
    ll mp = 0;
    void ensure(int n_, ll mp_, int K_) {
        n = n_; mp = mp_; K = K_;
        ll m2 = (ll)n << (n - 1);
        size_t sb = (size_t)m2 * sizeof(T) * (size_t)K;
        for (DevBuf *b : {&x2, &s, &y, &z, &x, &Ax, &t1, &t2, &xhat}) b->ensure(sb);
        obsbits.ensure((size_t)((m2 + 31) / 32) * 4);
        menu_obs.ensure((size_t)4 << n);
        diag.ensure(64 * sizeof(T));
        err.ensure(16);
        active.ensure((size_t)K * 4);
        p.ensure((size_t)K * (size_t)mp * 8);
        pfit.ensure((size_t)K * (size_t)mp * 8);
        res.ensure((size_t)K * R_SLOTS * 8);
    }
};

template <class T>
static size_t batch_slot_bytes(int n, ll mp) {
    ll m2 = (ll)n << (n - 1);
    return (size_t)9 * (size_t)m2 * sizeof(T) + (size_t)mp * 16 + R_SLOTS * 8;
}

template <class T>
static int bm_solve_batch_t(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, const rumb_batch_params *bp,
                            int B, const double *P, const double *below, const double *above, const rumb_bm_state *warm,
                            rumb_bm_result *out, rumb_batch_info *info) {
    const int n = pr->n;
    const ll mp = pr->mp, m2 = (ll)n << (n - 1);
    cudaStream_t st = c.own;
    auto t0 = Clock::now();
    // slots by memory
    size_t fr = 0, tot = 0;
    RUMB_CUDA(cudaMemGetInfo(&fr, &tot));
    double frac = (bp && bp->mem_fraction > 0) ? bp->mem_fraction : 0.8;
    size_t per = batch_slot_bytes<T>(n, mp);
    CertWork &CW = cert_work(c);
    CW.ensure(n, mp);
    RUMB_CUDA(cudaMemGetInfo(&fr, &tot));
    ll fit = (ll)((double)fr * frac / (double)per);
    int K = (bp && bp->slots > 0) ? bp->slots : (int)std::min<ll>(fit, 256);
    K = std::max(1, std::min(K, B));
    if ((ll)K > fit && fit >= 1) K = (int)fit;
    if (fit < 1) fail(RUMB_E_OOM, "one draw's state does not fit the free device memory");
    std::unique_ptr<BmWorkBase> &slot = sizeof(T) == 8 ? c.batch64 : c.batch32;
    if (!slot) slot.reset(new BatchWork<T>());
    BatchWork<T> &W = *static_cast<BatchWork<T> *>(slot.get());
    W.ensure(n, mp, K);
    // shared structure: observed positions, bits, per-menu masks, diagonal
    DevProblem D;
    upload_problem(*pr, D, st);
    BmCoef C = make_coef(n, par->beta, par->alpha, par->precond_p);
    {
        DevBuf bad;
        bad.ensure(4);
        RUMB_CUDA(cudaMemsetAsync(bad.ptr, 0, 4, st));
        RUMB_CUDA(cudaMemsetAsync(W.xhat.ptr, 0, (size_t)m2 * sizeof(T) * K, st));
        RUMB_CUDA(cudaMemsetAsync(W.obsbits.ptr, 0, (size_t)((m2 + 31) / 32) * 4, st));
        obs_setup_kernel<T><<<grid_for(mp, 256), 256, 0, st>>>(D.d_menu, D.d_alt, D.d_p, mp, n, 1LL << (n - 1),
                                                               CW.obs.as<ll>(), W.xhat.template as<T>(),
                                                               W.obsbits.template as<uint32_t>(), bad.as<int>());
        RUMB_LAUNCH("obs_setup_kernel");
        launch_menu_obs(W.obsbits.template as<uint32_t>(), n, 1LL << (n - 1), W.menu_obs.template as<uint32_t>(), st);
        int hbad = 0;
        RUMB_CUDA(cudaMemcpyAsync(&hbad, bad.ptr, 4, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaStreamSynchronize(st));
        if (hbad) fail(RUMB_E_INVAL, "an observed row's alternative is not in its menu, or its menu is a singleton");
        std::vector<T> dg(C.diag.begin(), C.diag.end());
        RUMB_CUDA(cudaMemcpyAsync(W.diag.ptr, dg.data(), dg.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        RUMB_CUDA(cudaMemsetAsync(W.err.ptr, 0, 16, st));
    }
    IterPtrs<T> I;
    I.x2 = W.x2.template as<T>(); I.s = W.s.template as<T>(); I.y = W.y.template as<T>(); I.z = W.z.template as<T>();
    I.x = W.x.template as<T>(); I.Ax = W.Ax.template as<T>(); I.t1 = W.t1.template as<T>(); I.t2 = W.t2.template as<T>();
    I.xhat = W.xhat.template as<T>(); I.diag = W.diag.template as<T>();
    I.menu_obs = W.menu_obs.template as<uint32_t>();
    I.err = W.err.template as<unsigned int>();
    I.slots = K;
    I.bstride = m2;
    I.active = W.active.template as<int>();
    // the schedule tuned on a single-draw workspace, when known
    tuned_or_default<T>(c, C, n);
    DevBuf pbuf;                                    // the draws' rows, uploaded once
    pbuf.ensure((size_t)B * (size_t)mp * 8);
    RUMB_CUDA(cudaMemcpyAsync(pbuf.ptr, P, (size_t)B * (size_t)mp * 8, cudaMemcpyHostToDevice, st));
    const double *y0 = bp ? bp->y0 : nullptr;       // predicted fits: a lower-bound seed per draw
    double *fit_out = bp ? bp->p_fit : nullptr;
    DevBuf ybuf;
    if (y0) {
        ybuf.ensure((size_t)B * (size_t)mp * 8);
        RUMB_CUDA(cudaMemcpyAsync(ybuf.ptr, y0, (size_t)B * (size_t)mp * 8, cudaMemcpyHostToDevice, st));
    }
    std::vector<int> act(K, 0), draw_of(K, -1);
    std::vector<ll> it_of(K, 0);
    std::vector<double> ub_of(K, INFINITY), lb_of(K, 0.0), phi_of(K, NAN);
    std::vector<int> nlb_of(K, 0), npush_of(K, 0);
    std::vector<Clock::time_point> t_of(K);
    std::vector<std::vector<double>> gaps_of(K);
    int next = 0, done = 0;
    ll total_iters = 0;
    auto admit = [&](int k) {
        if (next >= B) { act[k] = 0; draw_of[k] = -1; return; }
        int b = next++;
        draw_of[k] = b; act[k] = 1; it_of[k] = 0; ub_of[k] = INFINITY; lb_of[k] = 0.0; phi_of[k] = NAN;
        nlb_of[k] = 0; npush_of[k] = 0; gaps_of[k].clear();
        t_of[k] = Clock::now();
        double *pk = W.p.template as<double>() + (size_t)k * mp;
        T *xk = W.xhat.template as<T>() + (size_t)k * m2;
        scatter_rows_kernel<<<grid_for(mp, 256), 256, 0, st>>>(CW.obs.as<ll>(), pbuf.as<double>() + (size_t)b * mp, mp,
                                                               pk, sizeof(T) == 4 ? (float *)xk : nullptr,
                                                               sizeof(T) == 8 ? (double *)xk : nullptr);
        RUMB_LAUNCH("scatter_rows_kernel");
        double *rk = W.res.template as<double>() + (size_t)k * R_SLOTS;
        set_doubles_kernel<<<1, 32, 0, st>>>(rk, R_SLOTS, 0.0);
        set_doubles_kernel<<<1, 32, 0, st>>>(rk + R_UB_BEST, 1, INFINITY);
        RUMB_LAUNCH("set_doubles");
        T *dst[4] = {I.x2 + (size_t)k * m2, I.s + (size_t)k * m2, I.y + (size_t)k * m2, I.z + (size_t)k * m2};
        if (warm) {
            const DevBuf *src[4] = {&warm->x2, &warm->s, &warm->y, &warm->z};
            for (int i = 0; i < 4; ++i) {
                if ((warm->dtype == RUMB_F64) == (sizeof(T) == 8))
                    RUMB_CUDA(cudaMemcpyAsync(dst[i], src[i]->ptr, (size_t)m2 * sizeof(T), cudaMemcpyDeviceToDevice, st));
                else if (warm->dtype == RUMB_F64)
                    convert_kernel<double, T><<<grid_for(m2, 256), 256, 0, st>>>(src[i]->as<double>(), dst[i], m2);
                else
                    convert_kernel<float, T><<<grid_for(m2, 256), 256, 0, st>>>(src[i]->as<float>(), dst[i], m2);
            }
            RUMB_LAUNCH("warm copy");
        } else {
            ProxArgs<T> Pa{};
            Pa.n = n; Pa.Nloc = 1LL << (n - 1); Pa.nmenus = (1LL << n) - 1;
            Pa.v = xk; Pa.out = dst[0]; Pa.xhat = xk;
            Pa.obsbits = W.obsbits.template as<uint32_t>();
            Pa.b2 = (T)C.b2;
            launch_prox_n<T, PROX_ONLY>(Pa, st);
            for (int i = 1; i < 4; ++i) RUMB_CUDA(cudaMemsetAsync(dst[i], 0, (size_t)m2 * sizeof(T), st));
        }
        if (y0) {
            // the Frank-Wolfe bound at the prediction is a certified lower bound for any y0: the
            // draw's bracket starts from it (R_LB_SEED); y0_state also moves the state's observed
            // entries to the prediction
            const double *yb = ybuf.as<double>() + (size_t)b * mp;
            if (bp->y0_state) {
                scatter_vals_kernel<T><<<grid_for(mp, 256), 256, 0, st>>>(CW.obs.as<ll>(), yb, mp, dst[0]);
                RUMB_LAUNCH("scatter_vals_kernel");
            }
            enqueue_stats_lb<T>(c, CW, n, dst[0], true, st, pk, rk, yb);
            copy_double_kernel<<<1, 32, 0, st>>>(rk + R_LB_SEED, rk + R_LB_NOW);
            RUMB_LAUNCH("copy_double_kernel");
        }
    };
    for (int k = 0; k < K; ++k) admit(k);
    RUMB_CUDA(cudaMemcpyAsync(W.active.ptr, act.data(), (size_t)K * 4, cudaMemcpyHostToDevice, st));
    std::vector<ll> bounds;
    c.layer_table(n, bounds);
    RUMB_CUDA(cudaStreamSynchronize(st));
    auto t_setup = Clock::now();
    const int chunk = graph_chunk(par->check);
    Graph g_iter;
    g_iter.capture(st, [&] { enqueue_iterations_ptrs<T>(I, C, n, st, chunk); });
    std::vector<double> res((size_t)K * R_SLOTS);
    cudaEvent_t e0, e1;
    RUMB_CUDA(cudaEventCreate(&e0));
    RUMB_CUDA(cudaEventCreate(&e1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } eg{e0, e1};
    RUMB_CUDA(cudaEventRecord(e0, st));
    while (done < B) {
        if (c.cancel.load()) fail(RUMB_E_CANCEL, "cancelled");
        if (par->time_limit > 0 && secs(t0, Clock::now()) > par->time_limit) break;
        for (int i = 0; i < par->check / chunk; ++i) g_iter.launch(st);
        int nact = 0;
        for (int k = 0; k < K; ++k) {
            if (!act[k]) continue;
            ++nact;
            it_of[k] += par->check;
            const T *x2k = I.x2 + (size_t)k * m2;
            const double *pk = W.p.template as<double>() + (size_t)k * mp;
            double *rk = W.res.template as<double>() + (size_t)k * R_SLOTS;
            bool want_lb = (npush_of[k] % par->lb_every) == 0;
            enqueue_stats_lb<T>(c, CW, n, x2k, want_lb, st, pk, rk);
            enqueue_push<T>(c, CW, n, x2k, st, pk, rk, fit_out ? W.pfit.template as<double>() + (size_t)k * mp : nullptr);
        }
        total_iters += (ll)nact * par->check;
        RUMB_CUDA(cudaMemcpyAsync(res.data(), W.res.ptr, res.size() * 8, cudaMemcpyDeviceToHost, st));
        unsigned int dev_err = 0;
        RUMB_CUDA(cudaMemcpyAsync(&dev_err, W.err.ptr, 4, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaStreamSynchronize(st));
        if (dev_err) fail(RUMB_E_TIMEOUT, "a kernel's bounded wait for its TMA copies gave up");
        bool changed = false;
        for (int k = 0; k < K; ++k) {
            if (!act[k]) continue;
            const double *r = &res[(size_t)k * R_SLOTS];
            bool want_lb = (npush_of[k] % par->lb_every) == 0;
            npush_of[k]++;
            phi_of[k] = std::sqrt(r[R_PHI2]);
            ub_of[k] = r[R_UB_BEST];
            if (want_lb) { nlb_of[k]++; if (r[R_LB_NOW] > lb_of[k]) lb_of[k] = r[R_LB_NOW]; }
            if (r[R_LB_SEED] > lb_of[k]) lb_of[k] = r[R_LB_SEED];
            int b = draw_of[k];
            int stop = 0;
            double gap = ub_of[k] - lb_of[k];
            double bl = below ? below[b] : NAN, ab = above ? above[b] : NAN;
            if (std::isfinite(bl) && ub_of[k] <= bl) stop = RUMB_STOP_UB_TARGET;
            else if (std::isfinite(ab) && lb_of[k] >= ab) stop = RUMB_STOP_LB_TARGET;
            else if (par->abs_tol >= 0 && gap <= par->abs_tol) stop = RUMB_STOP_GAP_ABS;
            else if (par->rel_tol >= 0 && lb_of[k] > 0 && gap / lb_of[k] <= par->rel_tol) stop = RUMB_STOP_GAP_REL;
            else if (it_of[k] >= par->max_iter) stop = RUMB_STOP_MAX_ITER;
            // the K resident draws share the GPU: a draw's budget is draw_time of its share
            else if (bp && bp->draw_time > 0 && secs(t_of[k], Clock::now()) > bp->draw_time * K) stop = RUMB_STOP_TIME;
            else if (par->stall_checks > 0) {
                // a float32 state's bracket stops closing at its rounding floor
                gaps_of[k].push_back(gap);
                size_t Wn = (size_t)par->stall_checks;
                if (sizeof(T) == 4 && gaps_of[k].size() > Wn &&
                    gap > (1.0 - par->stall_rtol) * gaps_of[k][gaps_of[k].size() - 1 - Wn])
                    stop = RUMB_STOP_STALL;
            }
            if (!stop) continue;
            rumb_bm_result &o = out[b];
            o.lb = lb_of[k]; o.ub = ub_of[k]; o.phi = phi_of[k]; o.iters = it_of[k];
            o.iters_f32 = sizeof(T) == 4 ? it_of[k] : 0; o.stop = stop; o.n_push = npush_of[k]; o.n_lb = nlb_of[k];
            o.setup_s = 0.0; o.solve_s = secs(t_of[k], Clock::now()); o.push_s = 0.0;
            o.per_iter_ms = 0.0; o.device_ms = 0.0;
            if (fit_out)
                RUMB_CUDA(cudaMemcpyAsync(fit_out + (size_t)b * mp, W.pfit.template as<double>() + (size_t)k * mp,
                                          (size_t)mp * 8, cudaMemcpyDeviceToHost, st));
            ++done;
            admit(k);
            changed = true;
        }
        if (changed) RUMB_CUDA(cudaMemcpyAsync(W.active.ptr, act.data(), (size_t)K * 4, cudaMemcpyHostToDevice, st));
    }
    // draws left when the time ran out
    for (int k = 0; k < K; ++k) {
        if (!act[k] || draw_of[k] < 0) continue;
        rumb_bm_result &o = out[draw_of[k]];
        o.lb = lb_of[k]; o.ub = ub_of[k]; o.phi = phi_of[k]; o.iters = it_of[k];
        o.iters_f32 = sizeof(T) == 4 ? it_of[k] : 0; o.stop = RUMB_STOP_TIME; o.n_push = npush_of[k];
        o.n_lb = nlb_of[k]; o.solve_s = secs(t_of[k], Clock::now());
        if (fit_out)
            RUMB_CUDA(cudaMemcpyAsync(fit_out + (size_t)draw_of[k] * mp, W.pfit.template as<double>() + (size_t)k * mp,
                                      (size_t)mp * 8, cudaMemcpyDeviceToHost, st));
    }
    for (int b = next; b < B; ++b) {
        out[b] = rumb_bm_result{};
        out[b].ub = INFINITY;
        out[b].stop = RUMB_STOP_TIME;
    }
    RUMB_CUDA(cudaEventRecord(e1, st));
    RUMB_CUDA(cudaEventSynchronize(e1));
    float dms = 0.f;
    RUMB_CUDA(cudaEventElapsedTime(&dms, e0, e1));
    if (info) {
        info->slots = K;
        info->bytes_per_slot = (double)per;
        info->total_iters = total_iters;
        info->setup_s = secs(t0, t_setup);
        info->solve_s = secs(t_setup, Clock::now());
        info->device_ms = dms;
        info->lo_bits = C.lo_bits;
    }
    return RUMB_OK;
}

int bm_solve_batch(Ctx &c, const rumb_bm_problem *pr, const rumb_bm_params *par, const rumb_batch_params *bp, int B,
                   const double *P, const double *below, const double *above, const rumb_bm_state *warm,
                   rumb_bm_result *out, rumb_batch_info *info) {
    check_problem(pr);
    check_params(par);
    if (pr->n < PT_M + 1) fail(RUMB_E_INVAL, "batched draws need n >= 8");
    if (B < 1 || !P || !out) fail(RUMB_E_INVAL, "B >= 1 draws, P and the results are required");
    if (warm && warm->n != pr->n) fail(RUMB_E_INVAL, "warm state was kept for another n");
    c.cancel.store(0);
    c.join_in();
    const long long launches0 = g_launches;
    int r;
    if (par->dtype == RUMB_F64) r = bm_solve_batch_t<double>(c, pr, par, bp, B, P, below, above, warm, out, info);
    else r = bm_solve_batch_t<float>(c, pr, par, bp, B, P, below, above, warm, out, info);
    for (int b = 0; b < B; ++b) out[b].launches = 0;     // shared by the batch: counted in info
    if (info) info->launches = g_launches - launches0;
    c.join_out();
    return r;
}

// ----------------------------------------------------------------- primitives on host slabs
struct Scratch : public BmWorkBase {
    DevBuf a, b, c, d;
};
static Scratch &scratch(Ctx &c) {
    if (!c.scratch) c.scratch.reset(new Scratch());
    return *static_cast<Scratch *>(c.scratch.get());
}

int butterfly_host(Ctx &c, int n, int dtype, const void *in, void *out, double a, double b, double cc, double d) {
    if (n < 2 || n > 30) fail(RUMB_E_INVAL, "butterfly: 2 <= n <= 30");
    if (dtype != RUMB_F64 && dtype != RUMB_F32) fail(RUMB_E_INVAL, "butterfly: dtype RUMB_F64 or RUMB_F32");
    if (!in || !out) fail(RUMB_E_INVAL, "butterfly: NULL buffer");
    ll m2 = (ll)n << (n - 1);
    size_t es = dtype == RUMB_F64 ? 8 : 4;
    Scratch &S = scratch(c);
    S.a.ensure((size_t)m2 * es);
    cudaStream_t st = c.own;
    c.join_in();
    RUMB_CUDA(cudaMemcpyAsync(S.a.ptr, in, (size_t)m2 * es, cudaMemcpyHostToDevice, st));
    if (dtype == RUMB_F64)
        xf_transform<double, double>(n, S.a.as<double>(), S.a.as<double>(), Co<double>{a, b, cc, d}, st);
    else
        xf_transform<float, float>(n, S.a.as<float>(), S.a.as<float>(),
                                   Co<float>{(float)a, (float)b, (float)cc, (float)d}, st);
    RUMB_CUDA(cudaMemcpyAsync(out, S.a.ptr, (size_t)m2 * es, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    c.join_out();
    return RUMB_OK;
}

// ----------------------------------------------------------------- butterfly without allocation
// butterfly_host stages the slab in the context's scratch, which grows by cudaMalloc/cudaFree.
// This variant stages it in a static device array of this module instead, so a call reaches no
// allocator: 4 MiB, which holds the slab up to n = 16 (16 * 2^15 float64 values). The array is
// per device and shared by every context on it; the host copy overwrites every entry the
// transform reads, so nothing in it has to start at zero. Two calls on one device that overlap
// (two threads, two contexts) race on the array; nothing here serializes them.
static constexpr size_t NOALLOC_SLAB_BYTES = size_t(4) << 20;
static constexpr int NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) unsigned char g_noalloc_slab[NOALLOC_SLAB_BYTES];
static std::atomic<void *> g_noalloc_addr[NOALLOC_MAX_DEVICES];

// The slab's address on `device`, which must be the current device. Found once per device by
// cudaGetSymbolAddress (which loads this module on that device if nothing has yet).
static void *noalloc_slab(int device) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) fail(RUMB_E_INVAL, "butterfly_noalloc: device index above 63");
    void *p = g_noalloc_addr[device].load(std::memory_order_acquire);
    if (p) return p;
    RUMB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_slab));
    if (!p || (reinterpret_cast<uintptr_t>(p) & 255)) fail(RUMB_E_INTERNAL, "butterfly_noalloc: slab address");
    g_noalloc_addr[device].store(p, std::memory_order_release);
    return p;
}

int butterfly_noalloc_host(Ctx &c, int n, int dtype, const void *in, void *out, double a, double b, double cc,
                           double d) {
    if (n < 2 || n > 30) fail(RUMB_E_INVAL, "butterfly_noalloc: 2 <= n <= 30");
    if (dtype != RUMB_F64 && dtype != RUMB_F32) fail(RUMB_E_INVAL, "butterfly_noalloc: dtype RUMB_F64 or RUMB_F32");
    if (!in || !out) fail(RUMB_E_INVAL, "butterfly_noalloc: NULL buffer");
    ll m2 = (ll)n << (n - 1);
    size_t es = dtype == RUMB_F64 ? 8 : 4;
    size_t bytes = (size_t)m2 * es;
    if (bytes > NOALLOC_SLAB_BYTES)
        fail(RUMB_E_INVAL, "butterfly_noalloc: the slab of n = " + std::to_string(n) + " needs " +
                               std::to_string(bytes) + " bytes; the static staging array holds " +
                               std::to_string(NOALLOC_SLAB_BYTES) + " (n <= 16)");
    void *slab = noalloc_slab(c.device);
    cudaStream_t st = c.own;
    c.join_in();
    RUMB_CUDA(cudaMemcpyAsync(slab, in, bytes, cudaMemcpyHostToDevice, st));
    if (dtype == RUMB_F64)
        xf_transform<double, double>(n, (const double *)slab, (double *)slab, Co<double>{a, b, cc, d}, st);
    else
        xf_transform<float, float>(n, (const float *)slab, (float *)slab,
                                   Co<float>{(float)a, (float)b, (float)cc, (float)d}, st);
    RUMB_CUDA(cudaMemcpyAsync(out, slab, bytes, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    c.join_out();
    return RUMB_OK;
}

template <class T>
static void prox_host_t(Ctx &c, int n, const T *v, const T *xhat, const T *wmask, double beta2, T *out) {
    ll m2 = (ll)n << (n - 1);
    ll nw = (m2 + 31) / 32;
    std::vector<uint32_t> bits((size_t)nw, 0u);
    for (ll i = 0; i < m2; ++i) {
        if (wmask[i] == (T)1) bits[(size_t)(i >> 5)] |= 1u << (i & 31);
        else if (wmask[i] != (T)0) fail(RUMB_E_INVAL, "prox: wmask entries must be 0 or 1");
    }
    Scratch &S = scratch(c);
    S.a.ensure((size_t)m2 * sizeof(T));
    S.b.ensure((size_t)m2 * sizeof(T));
    S.c.ensure((size_t)m2 * sizeof(T));
    S.d.ensure((size_t)nw * 4);
    cudaStream_t st = c.own;
    RUMB_CUDA(cudaMemcpyAsync(S.a.ptr, v, (size_t)m2 * sizeof(T), cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(S.b.ptr, xhat, (size_t)m2 * sizeof(T), cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(S.d.ptr, bits.data(), (size_t)nw * 4, cudaMemcpyHostToDevice, st));
    ProxArgs<T> P{};
    P.n = n;
    P.Nloc = 1LL << (n - 1);
    P.nmenus = (1LL << n) - 1;
    P.v = S.a.as<T>();
    P.out = S.c.as<T>();
    P.xhat = S.b.as<T>();
    P.obsbits = S.d.as<uint32_t>();
    P.b2 = (T)beta2;
    launch_prox_n<T, PROX_ONLY>(P, st);
    RUMB_CUDA(cudaMemcpyAsync(out, S.c.ptr, (size_t)m2 * sizeof(T), cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
}

int prox_host(Ctx &c, int n, int dtype, const void *v, const void *xhat, const void *wmask, double beta2, void *out) {
    if (n < 2 || n > 30) fail(RUMB_E_INVAL, "prox: 2 <= n <= 30");
    if (!v || !xhat || !wmask || !out) fail(RUMB_E_INVAL, "prox: NULL buffer");
    c.join_in();
    if (dtype == RUMB_F64)
        prox_host_t<double>(c, n, (const double *)v, (const double *)xhat, (const double *)wmask, beta2, (double *)out);
    else if (dtype == RUMB_F32)
        prox_host_t<float>(c, n, (const float *)v, (const float *)xhat, (const float *)wmask, beta2, (float *)out);
    else
        fail(RUMB_E_INVAL, "prox: dtype RUMB_F64 or RUMB_F32");
    c.join_out();
    return RUMB_OK;
}

static void small_problem(rumb_bm_problem &pr, int n, ll mp, const uint32_t *menu, const int32_t *alt,
                          const double *p) {
    pr.n = n;
    pr.mp = mp;
    pr.menu = menu;
    pr.alt = alt;
    pr.p = p;
    pr.on_device = 0;
    check_problem(&pr);
}

int push_ub64_host(Ctx &c, int n, int dtype, const void *x, ll mp, const uint32_t *menu, const int32_t *alt,
                   const double *p, double *ub, double *p_fit) {
    rumb_bm_problem pr;
    small_problem(pr, n, mp, menu, alt, p);
    if (!x || !ub) fail(RUMB_E_INVAL, "push: NULL buffer");
    if (dtype != RUMB_F64 && dtype != RUMB_F32) fail(RUMB_E_INVAL, "push: dtype RUMB_F64 or RUMB_F32");
    ll m2 = (ll)n << (n - 1);
    cudaStream_t st = c.own;
    c.join_in();
    CertWork &CW = cert_work(c);
    CW.ensure(n, mp);
    DevProblem D;
    upload_problem(pr, D, st);
    setup_obs<double>(c, CW, nullptr, pr, D, st);
    Scratch &S = scratch(c);
    size_t es = dtype == RUMB_F64 ? 8 : 4;
    S.a.ensure((size_t)m2 * es);
    RUMB_CUDA(cudaMemcpyAsync(S.a.ptr, x, (size_t)m2 * es, cudaMemcpyHostToDevice, st));
    set_doubles_kernel<<<1, 32, 0, st>>>(CW.res.as<double>() + R_UB_BEST, 1, INFINITY);
    RUMB_LAUNCH("set_doubles");
    if (dtype == RUMB_F64) enqueue_push<double>(c, CW, n, S.a.as<double>(), st);
    else enqueue_push<float>(c, CW, n, S.a.as<float>(), st);
    double res[R_SLOTS];
    RUMB_CUDA(cudaMemcpyAsync(res, CW.res.ptr, sizeof(res), cudaMemcpyDeviceToHost, st));
    if (p_fit) RUMB_CUDA(cudaMemcpyAsync(p_fit, CW.pfit_cur.ptr, (size_t)mp * 8, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    *ub = res[R_UB_NOW];
    c.join_out();
    return RUMB_OK;
}

// LB at observed values y: runs the LB on a slab whose observed entries are y (others unread).
int fw_lb64_host(Ctx &c, int n, ll mp, const uint32_t *menu, const int32_t *alt, const double *y, const double *p,
                 double *lb) {
    rumb_bm_problem pr;
    small_problem(pr, n, mp, menu, alt, p);
    if (!y || !lb) fail(RUMB_E_INVAL, "fw_lb: NULL buffer");
    ll m2 = (ll)n << (n - 1);
    cudaStream_t st = c.own;
    c.join_in();
    CertWork &CW = cert_work(c);
    CW.ensure(n, mp);
    DevProblem D;
    upload_problem(pr, D, st);
    // the y slab: scatter y at the observed positions through the xhat path (xhat := y)
    rumb_bm_problem py = pr;
    py.p = y;
    DevProblem Dy;
    upload_problem(py, Dy, st);
    Scratch &S = scratch(c);
    S.a.ensure((size_t)m2 * 8);
    S.d.ensure((size_t)((m2 + 31) / 32) * 4);
    // positions with xhat = y
    {
        DevBuf bad;
        bad.ensure(4);
        RUMB_CUDA(cudaMemsetAsync(bad.ptr, 0, 4, st));
        RUMB_CUDA(cudaMemsetAsync(S.a.ptr, 0, (size_t)m2 * 8, st));
        RUMB_CUDA(cudaMemsetAsync(S.d.ptr, 0, (size_t)((m2 + 31) / 32) * 4, st));
        obs_setup_kernel<double><<<grid_for(mp, 256), 256, 0, st>>>(Dy.d_menu, Dy.d_alt, Dy.d_p, mp, n, 1LL << (n - 1),
                                                                    CW.obs.as<ll>(), S.a.as<double>(),
                                                                    S.d.as<uint32_t>(), bad.as<int>());
        RUMB_LAUNCH("obs_setup_kernel");
        int hbad = 0;
        RUMB_CUDA(cudaMemcpyAsync(&hbad, bad.ptr, 4, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaStreamSynchronize(st));
        if (hbad) fail(RUMB_E_INVAL, "an observed row's alternative is not in its menu or is out of range");
    }
    RUMB_CUDA(cudaMemcpyAsync(CW.p.ptr, D.d_p, (size_t)mp * 8, cudaMemcpyDeviceToDevice, st));
    enqueue_stats_lb<double>(c, CW, n, S.a.as<double>(), true, st);
    double res[R_SLOTS];
    RUMB_CUDA(cudaMemcpyAsync(res, CW.res.ptr, sizeof(res), cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    *lb = res[R_LB_NOW];
    c.join_out();
    return RUMB_OK;
}

}  // namespace rumb
