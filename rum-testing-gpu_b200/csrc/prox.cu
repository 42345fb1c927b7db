// The per-menu prox tile kernel (formulas and the tile layout in prox.cuh) and its launchers.
//
// One thread per menu S; the member loops walk the set bits of S in increasing alternative order
// (the order of every sum), with the alternatives' run offsets in a shared table. Measured at
// n = 18 and 20 against two other forms of the same loop (all n alternatives unrolled with a
// predicate; the five lowest bits and the warp-uniform higher bits walked separately) and against
// loading x, x2, z straight from the slab into registers: equal in float64, 15-35 % faster in
// float32.
#include "prox.cuh"

namespace rumb {

__device__ __forceinline__ uint32_t cb32(uint32_t mask, int x) {
    return (mask & ((1u << x) - 1u)) | ((mask >> (x + 1)) << x);
}

// The previous iterate's support {i : x2_i > 0} is almost always this iteration's: the threshold
// is computed on it first and accepted when it satisfies the projection's optimality conditions
// (active t_i > tau, inactive t_i <= tau), which make tau unique; otherwise Michelot's iteration
// runs from the full set.

// ---------------------------------------------------------------- tile form

template <class T, int N>
__global__ void __launch_bounds__(PT_THREADS, 5) prox_tile_kernel(ProxTileArgs<T> P) {
    extern __shared__ __align__(128) unsigned char pt_smem[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(pt_smem);
    if (P.active && !P.active[blockIdx.y]) return;         // a retired slot (uniform per CTA)
    {
        const ll boff = (ll)blockIdx.y * P.bstride;
        P.x += boff;
        P.x2 += boff;
        P.z += boff;
        P.xhat += boff;
    }
    const int tid = threadIdx.x, lane = tid & 31;
    const ll Nloc = P.Nloc;
    constexpr int E_max = (int)prox_tile_elems(N);
    T *sx = reinterpret_cast<T *>(pt_smem + 256);
    T *sx2 = sx + E_max;
    T *sz = sx2 + E_max;
    const uint32_t base = (uint32_t)blockIdx.x << PT_M;
    int *roff = reinterpret_cast<int *>(pt_smem + 16);
    if (tid == 0) {
        mbar_init(mbar, 1);
        fence_mbar_init();
    }
    if (tid < N) roff[tid] = pt_roff(base, tid);
    __syncthreads();
    if (tid < 32) {
        // lane i issues alternative i's three copies; lane 0 first announces the byte count
        if (lane == 0) {
            unsigned elems = (unsigned)(PT_M * (1 << (PT_M - 1)) + __popc(base >> PT_M) * (1 << PT_M));
            mbar_expect_tx(mbar, (unsigned)(3u * elems * sizeof(T)));
        }
        __syncwarp();
        if (lane < N) {
            int len = pt_rlen(base, lane);
            if (len) {
                int off = pt_roff(base, lane);
                ll g = pt_rstart(base, lane, Nloc);
                unsigned b = (unsigned)(len * sizeof(T));
                tma_load_1d(sx + off, P.x + g, b, mbar);
                tma_load_1d(sx2 + off, P.x2 + g, b, mbar);
                tma_load_1d(sz + off, P.z + g, b, mbar);
            }
        }
    }
    const uint32_t low = (uint32_t)tid;
    const uint32_t S = base | low;
    const uint32_t wb = P.menu_obs[S];                 // observed members of S (one coalesced load)
    if (!mbar_wait_bounded(mbar, 0)) {
        if (tid == 0) atomicOr(P.err, 1u);
        mbar_wait_bounded(mbar, 0);                    // a second bounded chance for in-flight copies
        return;
    }
    const int k = __popc(S);
    const T one = (T)1, two = (T)2;
    const bool mixed = wb != 0 && wb != S;
    const double cw = (double)P.b2 + 2.0, cu = (double)P.b2, icw = 1.0 / cw, icu = 1.0 / cu;
    auto xhat_of = [&](int i) -> T { return P.xhat[(ll)i * Nloc + (ll)cb32(S, i)]; };
    uint32_t A0 = 0;
    double s1 = 0.0, s2 = 0.0, f1 = 0.0, f2 = 0.0;
    // pass 1: xo, v, q = z - b2 xo (kept in sz); the value the threshold works on goes to sx: the
    // equal-curvature value (b2 v + 2 w xh) / (b2 + 2 w) in the state dtype, or v itself for a
    // menu with observed and unobserved members (then t is b2 v + 2 xh, rebuilt in double where
    // it is read); sums over the previous support (s) and over all members (f)
    for (uint32_t SS = S; SS; SS &= SS - 1) {
        const int i = __ffs(SS) - 1;
        const int e = roff[i] + (int)(i < PT_M ? cb32(low, i) : low);
        T x2o = sx2[e];
        T xo = P.alpha * sx[e] + (one - P.alpha) * x2o;
        T zz = sz[e];
        T v = xo - P.ib2 * zz;
        sz[e] = zz - P.b2 * xo;
        const bool w = (wb >> i) & 1u;
        T xh = (T)0;
        if (w) xh = xhat_of(i);
        double ti, ic = 1.0;
        if (mixed) {
            sx[e] = v;
            ti = (double)P.b2 * (double)v + (w ? 2.0 * (double)xh : 0.0);
            ic = w ? icw : icu;
        } else {
            T val = (P.b2 * v + two * (w ? one : (T)0) * xh) * (w ? P.inv_c1 : P.inv_c0);
            sx[e] = val;
            ti = (double)val;
        }
        f1 += mixed ? ti * ic : ti;
        f2 += ic;
        if (x2o > (T)0) {
            A0 |= 1u << i;
            s1 += mixed ? ti * ic : ti;
            s2 += ic;
        }
    }
    auto t_of = [&](int i, int e) -> double {
        double ti = (double)sx[e];
        if (mixed) ti = (double)P.b2 * ti + (((wb >> i) & 1u) ? 2.0 * (double)xhat_of(i) : 0.0);
        return ti;
    };
    double tau = 0.0;
    bool ok = false;
    if (k > 1 && A0 != 0) {
        tau = (s1 - 1.0) / s2;
        ok = true;
        for (uint32_t SS = S; SS; SS &= SS - 1) {
            const int i = __ffs(SS) - 1;
            const double ti = t_of(i, roff[i] + (int)(i < PT_M ? cb32(low, i) : low));
            const bool in = (A0 >> i) & 1u;
            ok = ok && (in ? (ti > tau) : !(ti > tau));
        }
    }
    if (k > 1 && !ok) {
        uint32_t A = S;
        s1 = f1;
        s2 = f2;
        tau = (s1 - 1.0) / s2;
        for (int round = 0; round < 32; ++round) {
            uint32_t A2 = 0;
            s1 = 0.0;
            s2 = 0.0;
            for (uint32_t AA = A; AA; AA &= AA - 1) {
                const int i = __ffs(AA) - 1;
                const double ti = t_of(i, roff[i] + (int)(i < PT_M ? cb32(low, i) : low));
                const double ic = mixed ? (((wb >> i) & 1u) ? icw : icu) : 1.0;
                if (ti > tau) {
                    A2 |= 1u << i;
                    s1 += mixed ? ti * ic : ti;
                    s2 += ic;
                }
            }
            if (A2 == A) break;
            A = A2;
            tau = (s1 - 1.0) / s2;
        }
    }
    // pass 2: u = the projection, x2' = u, z' = q + b2 u
    for (uint32_t SS = S; SS; SS &= SS - 1) {
        const int i = __ffs(SS) - 1;
        const int e = roff[i] + (int)(i < PT_M ? cb32(low, i) : low);
        T u;
        if (k == 1) {
            u = one;
        } else if (mixed) {
            const bool w = (wb >> i) & 1u;
            double yv = (t_of(i, e) - tau) / (w ? cw : cu);
            u = yv > 0.0 ? (T)yv : (T)0;
        } else {
            double yv = (double)sx[e] - tau;
            u = yv > 0.0 ? (T)yv : (T)0;
        }
        sx2[e] = u;
        sz[e] = sz[e] + P.b2 * u;
    }
    fence_async_smem();
    __syncthreads();
    if (tid < 32 && lane < N) {
        int len = pt_rlen(base, lane);
        if (len) {
            int off = pt_roff(base, lane);
            ll g = pt_rstart(base, lane, Nloc);
            unsigned b = (unsigned)(len * sizeof(T));
            tma_store_1d(P.x2 + g, sx2 + off, b);
            tma_store_1d(P.z + g, sz + off, b);
            tma_commit();
            tma_wait_read();
        }
    }
}

// ---------------------------------------------------------------- launchers
template <class T, int N>
static void launch_tile_n(const ProxTileArgs<T> &P, cudaStream_t st, int slots) {
    static bool attr = false;   // the opt-in above 48 KB, once per kernel
    const size_t smem = prox_tile_smem<T>(N);
    if (!attr) {
        RUMB_CUDA(cudaFuncSetAttribute(prox_tile_kernel<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
        attr = true;
    }
    dim3 grid((unsigned)(1LL << (N - PT_M)), (unsigned)slots);
    prox_tile_kernel<T, N><<<grid, PT_THREADS, smem, st>>>(P);
    RUMB_LAUNCH("prox_tile_kernel");
}

template <class T>
void launch_prox_tile(const ProxTileArgs<T> &P, cudaStream_t st, int slots) {
    switch (P.n) {
#define RUMB_PT_CASE(NN) \
    case NN: launch_tile_n<T, NN>(P, st, slots); return;
        RUMB_PT_CASE(8) RUMB_PT_CASE(9) RUMB_PT_CASE(10) RUMB_PT_CASE(11) RUMB_PT_CASE(12) RUMB_PT_CASE(13)
        RUMB_PT_CASE(14) RUMB_PT_CASE(15) RUMB_PT_CASE(16) RUMB_PT_CASE(17) RUMB_PT_CASE(18) RUMB_PT_CASE(19)
        RUMB_PT_CASE(20) RUMB_PT_CASE(21) RUMB_PT_CASE(22) RUMB_PT_CASE(23) RUMB_PT_CASE(24) RUMB_PT_CASE(25)
        RUMB_PT_CASE(26) RUMB_PT_CASE(27) RUMB_PT_CASE(28) RUMB_PT_CASE(29) RUMB_PT_CASE(30)
#undef RUMB_PT_CASE
    default: break;
    }
    fail(RUMB_E_INVAL, "prox: 8 <= n <= 30");
}

template void launch_prox_tile<float>(const ProxTileArgs<float> &, cudaStream_t, int);
template void launch_prox_tile<double>(const ProxTileArgs<double> &, cudaStream_t, int);

// per-menu mask of observed members, from the observation bits of the slab
__global__ void menu_obs_kernel(const uint32_t *obsbits, int n, ll Nloc, uint32_t *menu_obs) {
    ll S = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (S >= (1LL << n)) return;
    uint32_t wb = 0;
    for (int i = 0; i < n; ++i) {
        if (!((S >> i) & 1)) continue;
        ll pos = (ll)i * Nloc + (ll)compress_bit((ull)S ^ (1ULL << i), i);
        if ((obsbits[pos >> 5] >> (pos & 31)) & 1u) wb |= 1u << i;
    }
    menu_obs[S] = wb;
}

void launch_menu_obs(const uint32_t *obsbits, int n, ll Nloc, uint32_t *menu_obs, cudaStream_t st) {
    menu_obs_kernel<<<grid_for(1LL << n, 256), 256, 0, st>>>(obsbits, n, Nloc, menu_obs);
    RUMB_LAUNCH("menu_obs_kernel");
}

}  // namespace rumb
