// The per-menu prox tile kernel (formulas and the tile layout in prox.cuh) and its launchers.
//
// A CTA stages its tile's runs of x, x2 and z in shared memory with 16-byte cp.async copies
// spread over all its threads (the runs are 64 or 128 values long: many small copies, which this
// moves faster than one TMA bulk copy per run did: 47 against 50 us at n = 18 float64, 32 against
// 35 us float32, 104 against 114 us at n = 20 float32), then one thread per menu S walks the
// members by set bits in increasing alternative order (the order of every sum), and x2 and z
// leave as 16-byte stores. The member loop by set bits measured equal or faster than two other
// forms (all alternatives unrolled with a predicate; the five lowest bits and the warp-uniform
// higher bits walked apart), and staging beat loading x, x2, z straight into registers by a third.
// Staging two arrays instead of three (x and x2 read through registers into the relaxed point xo,
// plus one bit per element for x2 > 0; 7 CTAs per SM instead of 5 in float64) measured 45.6
// against 47.2 us in float64 and 34.7 against 32.4 us in float32: more resident CTAs barely help,
// the per-menu dependent work is what bounds the kernel. Running the elementwise parts (the
// relaxed point, v, q, the threshold value; u and z') element by element over the tile, with one
// thread per menu for the threshold alone and the stores fused into the second pass, measured
// 51.5 against 47.3 us in float64 and 36.7 against 32.2 us in float32. Computing a member's tile
// position from the base mask in registers instead of reading the run offset from shared memory:
// no change (47.4 us float64).
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
    pdl_grid_sync();                                       // launched by launch_pdl
    extern __shared__ __align__(128) unsigned char pt_smem[];
    if (P.active && !P.active[blockIdx.y]) return;         // a retired slot (uniform per CTA)
    {
        const ll boff = (ll)blockIdx.y * P.bstride;
        P.x += boff;
        P.x2 += boff;
        P.z += boff;
        P.xhat += boff;
    }
    const int tid = threadIdx.x;
    const ll Nloc = P.Nloc;
    constexpr int E_max = (int)prox_tile_elems(N);
    T *sx = reinterpret_cast<T *>(pt_smem + 256);
    T *sx2 = sx + E_max;
    T *sz = sx2 + E_max;
    const uint32_t base = (uint32_t)blockIdx.x << PT_M;
    int *roff = reinterpret_cast<int *>(pt_smem + 16);
    __shared__ long long rg[32];     // global start of each alternative's run
    __shared__ int hi_alt[32];       // the j-th present high run's alternative
    if (tid < N) {
        roff[tid] = pt_roff(base, tid);
        rg[tid] = pt_rstart(base, tid, Nloc);
        if (tid >= PT_M && ((base >> tid) & 1u)) hi_alt[__popc(base & ((1u << tid) - 1u) & ~((1u << PT_M) - 1u))] = tid;
    }
    __syncthreads();
    constexpr int VEC = 16 / (int)sizeof(T);
    const int Et = PT_M * (1 << (PT_M - 1)) + __popc(base >> PT_M) * (1 << PT_M);
    // the run holding tile element e: the first PT_M runs are 2^(PT_M-1) long, the rest 2^PT_M
    auto run_of = [&](int e) -> int {
        return e < PT_M * (1 << (PT_M - 1)) ? (e >> (PT_M - 1)) : hi_alt[(e - PT_M * (1 << (PT_M - 1))) >> PT_M];
    };
    for (int c = tid; c < Et / VEC; c += PT_THREADS) {
        const int e = c * VEC;
        const int i = run_of(e);
        const ll g = rg[i] + (e - roff[i]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sx + e)), "l"(P.x + g) : "memory");
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sx2 + e)), "l"(P.x2 + g) : "memory");
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sz + e)), "l"(P.z + g) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    const uint32_t low = (uint32_t)tid;
    const uint32_t S = base | low;
    const uint32_t wb = P.menu_obs[S];                 // observed members of S (one coalesced load)
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
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
    __syncthreads();
    for (int c = tid; c < Et / VEC; c += PT_THREADS) {
        const int e = c * VEC;
        const int i = run_of(e);
        const ll g = rg[i] + (e - roff[i]);
        *reinterpret_cast<uint4 *>(P.x2 + g) = *reinterpret_cast<const uint4 *>(sx2 + e);
        *reinterpret_cast<uint4 *>(P.z + g) = *reinterpret_cast<const uint4 *>(sz + e);
    }
}

// ---------------------------------------------------------------- tile form, thresholds per menu
// The tile form with the member loops cut to one: each menu's thread walks its members once,
// staging the value the threshold works on (over x) and q = z - b2 xo (over z) and collecting the
// sums over the previous support together with the smallest value on it and the largest value
// off it; those two decide the optimality test without a second walk. The threshold (Michelot's
// iteration on the rare failure) goes to shared memory with a per-menu flag, and the projection,
// x2' = u and z' = q + b2 u are then formed element by element by all threads on the way out
// (16-byte stores). The arithmetic, the sums' order and so the results are the tile form's.
constexpr int PT_PLAIN = 0, PT_SINGLE = 1, PT_MIXED = 2;

template <class T, int N>
__global__ void __launch_bounds__(PT_THREADS, 5) prox_tau_kernel(ProxTileArgs<T> P) {
    pdl_grid_sync();                                       // launched by launch_pdl
    extern __shared__ __align__(128) unsigned char pt_smem[];
    if (P.active && !P.active[blockIdx.y]) return;         // a retired slot (uniform per CTA)
    {
        const ll boff = (ll)blockIdx.y * P.bstride;
        P.x += boff;
        P.x2 += boff;
        P.z += boff;
        P.xhat += boff;
    }
    const int tid = threadIdx.x;
    const ll Nloc = P.Nloc;
    constexpr int E_max = (int)prox_tile_elems(N);
    T *sx = reinterpret_cast<T *>(pt_smem + 256);
    T *sx2 = sx + E_max;
    T *sz = sx2 + E_max;
    const uint32_t base = (uint32_t)blockIdx.x << PT_M;
    int *roff = reinterpret_cast<int *>(pt_smem + 16);
    __shared__ long long rg[32];     // global start of each alternative's run
    __shared__ int hi_alt[32];       // the j-th present high run's alternative
    __shared__ double stau[PT_THREADS];
    __shared__ uint32_t sobs[PT_THREADS];
    __shared__ unsigned char sflag[PT_THREADS];
    if (tid < N) {
        roff[tid] = pt_roff(base, tid);
        rg[tid] = pt_rstart(base, tid, Nloc);
        if (tid >= PT_M && ((base >> tid) & 1u)) hi_alt[__popc(base & ((1u << tid) - 1u) & ~((1u << PT_M) - 1u))] = tid;
    }
    __syncthreads();
    constexpr int VEC = 16 / (int)sizeof(T);
    const int Et = PT_M * (1 << (PT_M - 1)) + __popc(base >> PT_M) * (1 << PT_M);
    auto run_of = [&](int e) -> int {
        return e < PT_M * (1 << (PT_M - 1)) ? (e >> (PT_M - 1)) : hi_alt[(e - PT_M * (1 << (PT_M - 1))) >> PT_M];
    };
    for (int c = tid; c < Et / VEC; c += PT_THREADS) {
        const int e = c * VEC;
        const int i = run_of(e);
        const ll g = rg[i] + (e - roff[i]);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sx + e)), "l"(P.x + g) : "memory");
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sx2 + e)), "l"(P.x2 + g) : "memory");
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sz + e)), "l"(P.z + g) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    const uint32_t low = (uint32_t)tid;
    const uint32_t S = base | low;
    const uint32_t wb = P.menu_obs[S];
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const int k = __popc(S);
    const T one = (T)1, two = (T)2;
    const bool mixed = wb != 0 && wb != S;
    const double cw = (double)P.b2 + 2.0, cu = (double)P.b2, icw = 1.0 / cw, icu = 1.0 / cu;
    auto xhat_of = [&](int i) -> T { return P.xhat[(ll)i * Nloc + (ll)cb32(S, i)]; };
    uint32_t A0 = 0;
    double s1 = 0.0, s2 = 0.0, f1 = 0.0, f2 = 0.0;
    double min_on = INFINITY, max_off = -INFINITY;
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
            min_on = ti < min_on ? ti : min_on;
        } else {
            max_off = ti > max_off ? ti : max_off;
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
        ok = (min_on > tau) && !(max_off > tau);
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
    stau[low] = tau;
    sobs[low] = wb;
    sflag[low] = (unsigned char)(k == 1 ? PT_SINGLE : (mixed ? PT_MIXED : PT_PLAIN));
    __syncthreads();
    // the projection and the write-back, element by element: element e of run i belongs to the
    // menu base | low, low = e - roff[i] for a high run, the lows containing i in order for a low run
    for (int c = tid; c < Et / VEC; c += PT_THREADS) {
        const int e = c * VEC;
        const int i = run_of(e);
        const int pos = e - roff[i];
        const ll g = rg[i] + pos;
        T u2[VEC], z2[VEC];
#pragma unroll
        for (int t = 0; t < VEC; ++t) {
            const int ps = pos + t;
            const uint32_t lw = i >= PT_M ? (uint32_t)ps
                                          : ((((uint32_t)ps >> i) << (i + 1)) | ((uint32_t)ps & ((1u << i) - 1u)) | (1u << i));
            const double tau_m = stau[lw];
            const int fl = sflag[lw];
            T u;
            if (fl == PT_SINGLE) {
                u = one;
            } else if (fl == PT_MIXED) {
                const bool w = (sobs[lw] >> i) & 1u;
                const double ti = (double)P.b2 * (double)sx[e + t] + (w ? 2.0 * (double)P.xhat[g + t] : 0.0);
                const double yv = (ti - tau_m) / (w ? cw : cu);
                u = yv > 0.0 ? (T)yv : (T)0;
            } else {
                const double yv = (double)sx[e + t] - tau_m;
                u = yv > 0.0 ? (T)yv : (T)0;
            }
            u2[t] = u;
            z2[t] = sz[e + t] + P.b2 * u;
        }
        if constexpr (sizeof(T) == 8) {
            *reinterpret_cast<double2 *>(P.x2 + g) = make_double2(u2[0], u2[1]);
            *reinterpret_cast<double2 *>(P.z + g) = make_double2(z2[0], z2[1]);
        } else {
            *reinterpret_cast<float4 *>(P.x2 + g) = make_float4(u2[0], u2[1], u2[2], u2[3]);
            *reinterpret_cast<float4 *>(P.z + g) = make_float4(z2[0], z2[1], z2[2], z2[3]);
        }
    }
}

// The one-walk form with two staged arrays (more CTAs per SM): xo formed while staging, the
// previous support kept as one bit per element. TPM = 2: two threads per menu (a lane pair), each
// walking every other member, the walk's sums, extremes and support joined by one shuffle each
// (more resident warps for the same shared memory, half of each thread's dependent chain).
template <class T, int N, int TPM = 1>
__global__ void __launch_bounds__(PT_THREADS * TPM, TPM == 1 ? 6 : 5) prox_tau2_kernel(ProxTileArgs<T> P) {
    pdl_grid_sync();                                       // launched by launch_pdl
    constexpr int NT = PT_THREADS * TPM;
    extern __shared__ __align__(128) unsigned char pt_smem[];
    if (P.active && !P.active[blockIdx.y]) return;         // a retired slot (uniform per CTA)
    {
        const ll boff = (ll)blockIdx.y * P.bstride;
        P.x += boff;
        P.x2 += boff;
        P.z += boff;
        P.xhat += boff;
    }
    const int tid = threadIdx.x;
    const ll Nloc = P.Nloc;
    constexpr int E_max = (int)prox_tile_elems(N);
    T *sx = reinterpret_cast<T *>(pt_smem + 256);        // xo, then the threshold's value
    T *sz = sx + E_max;                                    // z, then q
    uint32_t *sbit = reinterpret_cast<uint32_t *>(sz + E_max);   // x2 > 0, a bit per element
    const uint32_t base = (uint32_t)blockIdx.x << PT_M;
    int *roff = reinterpret_cast<int *>(pt_smem + 16);
    __shared__ long long rg[32];     // global start of each alternative's run
    __shared__ int hi_alt[32];       // the j-th present high run's alternative
    __shared__ double stau[PT_THREADS];
    __shared__ uint32_t sobs[PT_THREADS];
    __shared__ unsigned char sflag[PT_THREADS];
    if (tid < N) {
        roff[tid] = pt_roff(base, tid);
        rg[tid] = pt_rstart(base, tid, Nloc);
        if (tid >= PT_M && ((base >> tid) & 1u)) hi_alt[__popc(base & ((1u << tid) - 1u) & ~((1u << PT_M) - 1u))] = tid;
    }
    __syncthreads();
    constexpr int VEC = 16 / (int)sizeof(T);
    const int Et = PT_M * (1 << (PT_M - 1)) + __popc(base >> PT_M) * (1 << PT_M);
    auto run_of = [&](int e) -> int {
        return e < PT_M * (1 << (PT_M - 1)) ? (e >> (PT_M - 1)) : hi_alt[(e - PT_M * (1 << (PT_M - 1))) >> PT_M];
    };
    const T one = (T)1, two = (T)2;
    // z staged as it is; the relaxed point xo = alpha x + (1 - alpha) x2 formed on the way in, with
    // one bit per element for x2 > 0 (the previous support): two staged arrays instead of three
    // SU chunks per thread in flight: every load of a round is issued before any is used
    constexpr int SU = 4;
    const int nch = Et / VEC;
    for (int c0 = tid; c0 < nch; c0 += NT * SU) {
        T xv[SU][VEC], x2v[SU][VEC];
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            const int c = c0 + u * NT;
            if (c < nch) {
                const int e = c * VEC;
                const int i = run_of(e);
                const ll g = rg[i] + (e - roff[i]);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sz + e)), "l"(P.z + g)
                             : "memory");
                *reinterpret_cast<uint4 *>(xv[u]) = *reinterpret_cast<const uint4 *>(P.x + g);
                *reinterpret_cast<uint4 *>(x2v[u]) = *reinterpret_cast<const uint4 *>(P.x2 + g);
            }
        }
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            const int c = c0 + u * NT;
            if (c < nch) {
                const int e = c * VEC;
                const unsigned am = __activemask();
#pragma unroll
                for (int t = 0; t < VEC; ++t) {
                    sx[e + t] = P.alpha * xv[u][t] + (one - P.alpha) * x2v[u][t];
                    const unsigned b = __ballot_sync(am, x2v[u][t] > (T)0);
                    if ((threadIdx.x & 31) == __ffs(am) - 1) sbit[(c >> 5) * VEC + t] = b;
                }
            }
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    const uint32_t low = (uint32_t)(tid / TPM);
    const int h = tid % TPM;                              // this thread's share of the members
    const unsigned pm = TPM == 2 ? 3u << ((threadIdx.x & 31) & ~1) : 0u;
    const uint32_t S = base | low;
    const uint32_t wb = P.menu_obs[S];
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const int k = __popc(S);
    const bool mixed = wb != 0 && wb != S;
    const double cw = (double)P.b2 + 2.0, cu = (double)P.b2, icw = 1.0 / cw, icu = 1.0 / cu;
    auto xhat_of = [&](int i) -> T { return P.xhat[(ll)i * Nloc + (ll)cb32(S, i)]; };
    uint32_t A0 = 0;
    double s1 = 0.0, s2 = 0.0, f1 = 0.0, f2 = 0.0;
    double min_on = INFINITY, max_off = -INFINITY;
    uint32_t SS = S;
    if (TPM == 2 && h) SS &= SS - 1;
    for (; SS; SS &= SS - 1) {
        const int i = __ffs(SS) - 1;
        const int e = roff[i] + (int)(i < PT_M ? cb32(low, i) : low);
        const int ce = e / VEC;
        const bool on = (sbit[(ce >> 5) * VEC + (e % VEC)] >> (ce & 31)) & 1u;
        T xo = sx[e];
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
        if (on) {
            A0 |= 1u << i;
            s1 += mixed ? ti * ic : ti;
            s2 += ic;
            min_on = ti < min_on ? ti : min_on;
        } else {
            max_off = ti > max_off ? ti : max_off;
        }
        if (TPM == 2) SS &= SS - 1;                        // the partner's member
    }
    if constexpr (TPM == 2) {
        A0 |= __shfl_xor_sync(pm, A0, 1);
        s1 += __shfl_xor_sync(pm, s1, 1);
        s2 += __shfl_xor_sync(pm, s2, 1);
        f1 += __shfl_xor_sync(pm, f1, 1);
        f2 += __shfl_xor_sync(pm, f2, 1);
        min_on = fmin(min_on, __shfl_xor_sync(pm, min_on, 1));
        max_off = fmax(max_off, __shfl_xor_sync(pm, max_off, 1));
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
        ok = (min_on > tau) && !(max_off > tau);
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
            uint32_t AA = A;
            if (TPM == 2 && h) AA &= AA - 1;
            for (; AA; AA &= AA - 1) {
                const int i = __ffs(AA) - 1;
                const double ti = t_of(i, roff[i] + (int)(i < PT_M ? cb32(low, i) : low));
                const double ic = mixed ? (((wb >> i) & 1u) ? icw : icu) : 1.0;
                if (ti > tau) {
                    A2 |= 1u << i;
                    s1 += mixed ? ti * ic : ti;
                    s2 += ic;
                }
                if (TPM == 2) AA &= AA - 1;
            }
            if constexpr (TPM == 2) {
                A2 |= __shfl_xor_sync(pm, A2, 1);
                s1 += __shfl_xor_sync(pm, s1, 1);
                s2 += __shfl_xor_sync(pm, s2, 1);
            }
            if (A2 == A) break;
            A = A2;
            tau = (s1 - 1.0) / s2;
        }
    }
    if (h == 0) {
        stau[low] = tau;
        sobs[low] = wb;
        sflag[low] = (unsigned char)(k == 1 ? PT_SINGLE : (mixed ? PT_MIXED : PT_PLAIN));
    }
    __syncthreads();
    // the projection and the write-back, element by element: element e of run i belongs to the
    // menu base | low, low = e - roff[i] for a high run, the lows containing i in order for a low run
    for (int c = tid; c < Et / VEC; c += NT) {
        const int e = c * VEC;
        const int i = run_of(e);
        const int pos = e - roff[i];
        const ll g = rg[i] + pos;
        T u2[VEC], z2[VEC];
#pragma unroll
        for (int t = 0; t < VEC; ++t) {
            const int ps = pos + t;
            const uint32_t lw = i >= PT_M ? (uint32_t)ps
                                          : ((((uint32_t)ps >> i) << (i + 1)) | ((uint32_t)ps & ((1u << i) - 1u)) | (1u << i));
            const double tau_m = stau[lw];
            const int fl = sflag[lw];
            T u;
            if (fl == PT_SINGLE) {
                u = one;
            } else if (fl == PT_MIXED) {
                const bool w = (sobs[lw] >> i) & 1u;
                const double ti = (double)P.b2 * (double)sx[e + t] + (w ? 2.0 * (double)P.xhat[g + t] : 0.0);
                const double yv = (ti - tau_m) / (w ? cw : cu);
                u = yv > 0.0 ? (T)yv : (T)0;
            } else {
                const double yv = (double)sx[e + t] - tau_m;
                u = yv > 0.0 ? (T)yv : (T)0;
            }
            u2[t] = u;
            z2[t] = sz[e + t] + P.b2 * u;
        }
        if constexpr (sizeof(T) == 8) {
            *reinterpret_cast<double2 *>(P.x2 + g) = make_double2(u2[0], u2[1]);
            *reinterpret_cast<double2 *>(P.z + g) = make_double2(z2[0], z2[1]);
        } else {
            *reinterpret_cast<float4 *>(P.x2 + g) = make_float4(u2[0], u2[1], u2[2], u2[3]);
            *reinterpret_cast<float4 *>(P.z + g) = make_float4(z2[0], z2[1], z2[2], z2[3]);
        }
    }
}

// ---------------------------------------------------------------- lane-group form
// G consecutive lanes share one menu S (a warp holds 32 / G consecutive menus); lane gl of the
// group owns the members i = gl, gl + G, gl + 2G, ... of S. Every member's x, x2 and z are read
// straight from the slab into registers and x2', z' written back: for i >= log2(32 / G) bit i of S
// is the same for all the warp's menus, so the active lanes read 32 / G consecutive rests of block
// i (one contiguous segment per member slot and lane parity), and for lower i half of them do.
// Nothing is staged, no barrier is taken, and the loads of all of a lane's members are in flight
// together. The threshold's sums, the support and the optimality test are reduced over the group
// with xor shuffles (every lane of a group ends with the same bits, so the group takes one path).
template <int G>
__device__ __forceinline__ unsigned group_mask(int lane) {
    return G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
}
template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned m) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(m, v, o);
    return v;
}
template <int G>
__device__ __forceinline__ uint32_t group_or(uint32_t v, unsigned m) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v |= __shfl_xor_sync(m, v, o);
    return v;
}

template <class T, int N, int G>
__global__ void __launch_bounds__(256, G >= 4 ? 4 : 2) prox_lanes_kernel(ProxTileArgs<T> P) {
    pdl_grid_sync();                                       // launched by launch_pdl
    if (P.active && !P.active[blockIdx.y]) return;         // a retired slot (uniform per CTA)
    const ll boff = (ll)blockIdx.y * P.bstride;
    const T *X = P.x + boff;
    T *X2 = P.x2 + boff, *Z = P.z + boff;
    const T *XH = P.xhat + boff;
    const ll Nloc = P.Nloc;
    const int lane = threadIdx.x & 31, gl = lane & (G - 1);
    const unsigned gm = group_mask<G>(lane);
    const uint32_t S = (uint32_t)(((ll)blockIdx.x * blockDim.x + threadIdx.x) / G);
    constexpr int J = (N + G - 1) / G;                      // member slots per lane
    const int k = __popc(S);
    const uint32_t wb = P.menu_obs[S];
    const bool mixed = wb != 0 && wb != S;
    const T one = (T)1, two = (T)2;
    const double cw = (double)P.b2 + 2.0, cu = (double)P.b2, icw = 1.0 / cw, icu = 1.0 / cu;
    T val[J], q[J];
    uint32_t A0 = 0;
    double s1 = 0.0, s2 = 0.0, f1 = 0.0, f2 = 0.0;
    // pass 1 (as the tile form): xo, v, q = z - b2 xo; val = the value the threshold works on
    // (the equal-curvature value, or v for a menu with observed and unobserved members)
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const int i = j * G + gl;
        val[j] = (T)0;
        q[j] = (T)0;
        if (i < N && ((S >> i) & 1u)) {
            const ll g = (ll)i * Nloc + (ll)cb32(S, i);
            const T x2o = X2[g];
            const T xo = P.alpha * X[g] + (one - P.alpha) * x2o;
            const T zz = Z[g];
            const T v = xo - P.ib2 * zz;
            q[j] = zz - P.b2 * xo;
            const bool w = (wb >> i) & 1u;
            const T xh = w ? XH[g] : (T)0;
            double ti, ic = 1.0;
            if (mixed) {
                val[j] = v;
                ti = (double)P.b2 * (double)v + (w ? 2.0 * (double)xh : 0.0);
                ic = w ? icw : icu;
            } else {
                val[j] = (P.b2 * v + two * (w ? one : (T)0) * xh) * (w ? P.inv_c1 : P.inv_c0);
                ti = (double)val[j];
            }
            f1 += mixed ? ti * ic : ti;
            f2 += ic;
            if (x2o > (T)0) {
                A0 |= 1u << i;
                s1 += mixed ? ti * ic : ti;
                s2 += ic;
            }
        }
    }
    auto t_of = [&](int j, int i) -> double {
        double ti = (double)val[j];
        if (mixed) ti = (double)P.b2 * ti + (((wb >> i) & 1u) ? 2.0 * (double)XH[(ll)i * Nloc + (ll)cb32(S, i)] : 0.0);
        return ti;
    };
    A0 = group_or<G>(A0, gm);
    s1 = group_sum<G>(s1, gm);
    s2 = group_sum<G>(s2, gm);
    double tau = 0.0;
    bool ok = false;
    if (k > 1 && A0 != 0) {
        tau = (s1 - 1.0) / s2;
        uint32_t bad = 0;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int i = j * G + gl;
            if (i < N && ((S >> i) & 1u)) {
                const bool in = (A0 >> i) & 1u;
                if (in != (t_of(j, i) > tau)) bad = 1;
            }
        }
        ok = group_or<G>(bad, gm) == 0;
    }
    if (k > 1 && !ok) {
        // Michelot's iteration from the full set (the active set only shrinks)
        f1 = group_sum<G>(f1, gm);
        f2 = group_sum<G>(f2, gm);
        uint32_t A = S;
        tau = (f1 - 1.0) / f2;
        for (int round = 0; round < 32; ++round) {
            uint32_t A2 = 0;
            double a1 = 0.0, a2 = 0.0;
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int i = j * G + gl;
                if (i < N && ((A >> i) & 1u)) {
                    const double ti = t_of(j, i);
                    const double ic = mixed ? (((wb >> i) & 1u) ? icw : icu) : 1.0;
                    if (ti > tau) {
                        A2 |= 1u << i;
                        a1 += mixed ? ti * ic : ti;
                        a2 += ic;
                    }
                }
            }
            A2 = group_or<G>(A2, gm);
            a1 = group_sum<G>(a1, gm);
            a2 = group_sum<G>(a2, gm);
            if (A2 == A) break;
            A = A2;
            tau = (a1 - 1.0) / a2;
        }
    }
    // pass 2: u = the projection, x2' = u, z' = q + b2 u
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const int i = j * G + gl;
        if (i < N && ((S >> i) & 1u)) {
            const ll g = (ll)i * Nloc + (ll)cb32(S, i);
            T u;
            if (k == 1) {
                u = one;
            } else if (mixed) {
                const bool w = (wb >> i) & 1u;
                const double yv = (t_of(j, i) - tau) / (w ? cw : cu);
                u = yv > 0.0 ? (T)yv : (T)0;
            } else {
                const double yv = (double)val[j] - tau;
                u = yv > 0.0 ? (T)yv : (T)0;
            }
            X2[g] = u;
            Z[g] = q[j] + P.b2 * u;
        }
    }
}

// ---------------------------------------------------------------- launchers
template <class T, int N>
static void launch_tile_n(const ProxTileArgs<T> &P, cudaStream_t st, int slots) {
    static std::atomic<unsigned long long> optin{0};   // the opt-in above 48 KB, per device
    const size_t smem = prox_tile_smem<T>(N);
    smem_optin(prox_tile_kernel<T, N>, (int)smem, optin);
    dim3 grid((unsigned)(1LL << (N - PT_M)), (unsigned)slots);
    launch_pdl(prox_tile_kernel<T, N>, grid, dim3(PT_THREADS), smem, st, P);
    RUMB_LAUNCH("prox_tile_kernel");
}

template <class T, int N>
static void launch_tau_n(const ProxTileArgs<T> &P, cudaStream_t st, int slots) {
    static std::atomic<unsigned long long> optin{0};   // the opt-in above 48 KB, per device
    const size_t smem = prox_tile_smem<T>(N);
    smem_optin(prox_tau_kernel<T, N>, (int)smem, optin);
    dim3 grid((unsigned)(1LL << (N - PT_M)), (unsigned)slots);
    launch_pdl(prox_tau_kernel<T, N>, grid, dim3(PT_THREADS), smem, st, P);
    RUMB_LAUNCH("prox_tau_kernel");
}

template <class T, int N, int TPM = 1>
static void launch_tau2_n(const ProxTileArgs<T> &P, cudaStream_t st, int slots) {
    static std::atomic<unsigned long long> optin{0};   // the opt-in above 48 KB, per device
    constexpr int E_max = (int)prox_tile_elems(N), VEC = 16 / (int)sizeof(T);
    const size_t smem = 256 + 2 * (size_t)E_max * sizeof(T) + (size_t)((E_max / VEC + 31) / 32) * VEC * 4;
    smem_optin(prox_tau2_kernel<T, N, TPM>, (int)smem, optin);
    dim3 grid((unsigned)(1LL << (N - PT_M)), (unsigned)slots);
    launch_pdl(prox_tau2_kernel<T, N, TPM>, grid, dim3(PT_THREADS * TPM), smem, st, P);
    RUMB_LAUNCH("prox_tau2_kernel");
}

template <class T, int N, int G>
static void launch_lanes_n(const ProxTileArgs<T> &P, cudaStream_t st, int slots) {
    dim3 grid((unsigned)(((1LL << N) * G) / 256), (unsigned)slots);
    launch_pdl(prox_lanes_kernel<T, N, G>, grid, dim3(256), 0, st, P);
    RUMB_LAUNCH("prox_lanes_kernel");
}

template <class T, int N>
static void launch_form_n(const ProxTileArgs<T> &P, cudaStream_t st, int slots, int form) {
    switch (form) {
        case PROX_LANES2: launch_lanes_n<T, N, 2>(P, st, slots); return;
        case PROX_LANES4: launch_lanes_n<T, N, 4>(P, st, slots); return;
        case PROX_LANES8: launch_lanes_n<T, N, 8>(P, st, slots); return;
        case PROX_TAU: launch_tau_n<T, N>(P, st, slots); return;
        case PROX_TAU2: launch_tau2_n<T, N>(P, st, slots); return;
        case PROX_PAIR: launch_tau2_n<T, N, 2>(P, st, slots); return;
        default: launch_tile_n<T, N>(P, st, slots); return;
    }
}

template <class T>
void launch_prox_tile(const ProxTileArgs<T> &P, cudaStream_t st, int slots, int form) {
    if (P.n > PROX_LANES_MAX_N && form != PROX_TAU && form != PROX_TAU2 && form != PROX_PAIR) form = PROX_TILE;
    switch (P.n) {
#define RUMB_PT_CASE(NN) \
    case NN: launch_form_n<T, NN>(P, st, slots, form); return;
        RUMB_PT_CASE(8) RUMB_PT_CASE(9) RUMB_PT_CASE(10) RUMB_PT_CASE(11) RUMB_PT_CASE(12) RUMB_PT_CASE(13)
        RUMB_PT_CASE(14) RUMB_PT_CASE(15) RUMB_PT_CASE(16) RUMB_PT_CASE(17) RUMB_PT_CASE(18) RUMB_PT_CASE(19)
        RUMB_PT_CASE(20) RUMB_PT_CASE(21) RUMB_PT_CASE(22)
#undef RUMB_PT_CASE
#define RUMB_PT_CASE(NN) \
    case NN:                                                                                                      \
        if (form == PROX_TAU) launch_tau_n<T, NN>(P, st, slots);                                                  \
        else if (form == PROX_TAU2) launch_tau2_n<T, NN>(P, st, slots);                                           \
        else if (form == PROX_PAIR) launch_tau2_n<T, NN, 2>(P, st, slots);                                        \
        else launch_tile_n<T, NN>(P, st, slots);                                                                  \
        return;
        RUMB_PT_CASE(23) RUMB_PT_CASE(24) RUMB_PT_CASE(25)
        RUMB_PT_CASE(26) RUMB_PT_CASE(27) RUMB_PT_CASE(28) RUMB_PT_CASE(29) RUMB_PT_CASE(30)
#undef RUMB_PT_CASE
    default: break;
    }
    fail(RUMB_E_INVAL, "prox: 8 <= n <= 30");
}

template void launch_prox_tile<float>(const ProxTileArgs<float> &, cudaStream_t, int, int);
template void launch_prox_tile<double>(const ProxTileArgs<double> &, cudaStream_t, int, int);

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
