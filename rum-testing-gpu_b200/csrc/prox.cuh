// The fused per-menu prox of the BM-ADMM iteration as a tile kernel (sm_100a).
//
// A CTA owns 2^m consecutive menu masks S = base | low (low < 2^m, one thread per menu). The
// slab entries of those menus form one contiguous, aligned run per alternative i:
//   i <  m: the 2^(m-1) rests base/2 + compress(low, i) over the lows that contain i
//   i >= m: the 2^m rests compress(base, i) + low, present only when base contains i
// so the tile's x, x2 and z values arrive as a handful of 1-D TMA bulk copies
// (cp.async.bulk, completion counted on one mbarrier) into shared memory, the projection runs
// out of shared memory with a small register footprint, and x2 and z leave as bulk stores.
//
// Per menu (the reference's fuse_xk, prox_all and fuse_z, solver/bm_admm/solver.py:37-46,66-139):
//   xo = alpha x + (1 - alpha) x2,  v = xo - z / b2
//   u  = simplex prox of v with curvature b2 (unobserved) or b2 + 2 (observed, pulled to p_hat)
//   z' = z - b2 (xo - u),  x2' = u
// The threshold comes from Michelot's active-set iteration (the active set only shrinks, at
// most |S| rounds), which gives the reference's sort-based threshold without a sort.
//
// Bounded waits: the mbarrier wait gives up after ~2^32 cycles, records an error word and skips
// the tile (the host turns the word into RUMB_E_TIMEOUT at the next check).
#pragma once
#include "common.cuh"

namespace rumb {

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tma_store_1d(void *dst, const void *src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tma_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void tma_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Bounded wait on phase `parity` of bar; false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
    long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1LL << 32)) return false;
    }
    return true;
}

constexpr int PT_M = 7;                 // 128 menus per tile
constexpr int PT_THREADS = 1 << PT_M;

template <class T>
struct ProxTileArgs {
    int n;
    ll Nloc;
    const T *x;
    T *x2, *z;
    const T *xhat;
    const uint32_t *menu_obs;   // per menu mask: its observed members (bit i = alternative i)
    T alpha, b2, ib2;
    T inv_c0, inv_c1;           // 1 / b2 and 1 / (b2 + 2): the curvatures of unobserved / observed
    unsigned int *err;
    ll bstride;                 // batched draws: elements between draws' slabs (grid.y = slot)
    const int *active;          // batched draws: slot flags (nullptr: every slot runs)
};

// Largest tile (elements per array): m 2^(m-1) + (n - m) 2^m.
__host__ __device__ inline ll prox_tile_elems(int n) {
    return (ll)PT_M * (1LL << (PT_M - 1)) + (ll)(n - PT_M) * (1LL << PT_M);
}

template <class T>
inline size_t prox_tile_smem(int n) {
    return 256 + 3 * (size_t)prox_tile_elems(n) * sizeof(T);
}

// run of alternative i in the tile: smem offset (elements), length and global start
__device__ __forceinline__ int pt_roff(uint32_t base, int i) {
    int lo = i < PT_M ? i : PT_M;
    uint32_t hm = base & ((1u << i) - 1u) & ~((1u << PT_M) - 1u);
    return lo * (1 << (PT_M - 1)) + __popc(hm) * (1 << PT_M);
}
__device__ __forceinline__ int pt_rlen(uint32_t base, int i) {
    return i < PT_M ? (1 << (PT_M - 1)) : (((base >> i) & 1u) ? (1 << PT_M) : 0);
}
__device__ __forceinline__ ll pt_rstart(uint32_t base, int i, ll Nloc) {
    ll rest0 = (i < PT_M) ? (ll)(base >> 1) : (ll)compress_bit(base & ~(1u << i), i);
    return (ll)i * Nloc + rest0;
}

template <class T, int N>
__global__ void __launch_bounds__(PT_THREADS, 5) prox_tile_kernel(ProxTileArgs<T> P) {
    extern __shared__ __align__(128) unsigned char pt_smem[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(pt_smem);
    int *roff = reinterpret_cast<int *>(pt_smem + 16);     // run offsets (elements), n <= 30
    if (P.active && !P.active[blockIdx.y]) return;         // a retired slot (uniform per CTA)
    {
        const ll boff = (ll)blockIdx.y * P.bstride;
        P.x += boff;
        P.x2 += boff;
        P.z += boff;
        P.xhat += boff;
    }
    const int n = P.n, tid = threadIdx.x, lane = tid & 31;
    const ll Nloc = P.Nloc;
    const ll E_max = prox_tile_elems(n);
    T *sx = reinterpret_cast<T *>(pt_smem + 256);
    T *sx2 = sx + E_max;
    T *sz = sx2 + E_max;
    const uint32_t base = (uint32_t)blockIdx.x << PT_M;
    if (tid == 0) {
        mbar_init(mbar, 1);
        fence_mbar_init();
    }
    if (tid < n) roff[tid] = pt_roff(base, tid);
    __syncthreads();
    if (tid < 32) {
        // lane i issues alternative i's three copies; lane 0 first announces the byte count
        if (lane == 0) {
            unsigned elems = (unsigned)(PT_M * (1 << (PT_M - 1)) + __popc(base >> PT_M) * (1 << PT_M));
            mbar_expect_tx(mbar, (unsigned)(3u * elems * sizeof(T)));
        }
        __syncwarp();
        if (lane < n) {
            int len = pt_rlen(base, lane);
            if (len) {
                int off = roff[lane];
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
    // The previous iterate's support {i : x2_i > 0} is almost always this iteration's: the
    // threshold is computed on it first and accepted when it satisfies the projection's
    // optimality conditions (active t_i > tau, inactive t_i <= tau), which make tau unique;
    // otherwise Michelot's iteration runs from the full set.
    uint32_t A0 = 0;
    double s1 = 0.0, s2 = 0.0, f1 = 0.0, f2 = 0.0;
    // pass 1 over the members (set bits of S): xo, v, q = z - b2 xo (kept in sz); the value the
    // threshold works on goes to sx: the equal-curvature value (b2 v + 2 w xh) / (b2 + 2 w) in the
    // state dtype, or v itself for a menu with observed and unobserved members (then t is
    // b2 v + 2 xh, rebuilt in double where it is read); sums over the previous support (s) and
    // over all members (f)
    for (uint32_t SS = S; SS; SS &= SS - 1) {
        const int i = __ffs(SS) - 1;
        const int e = roff[i] + (int)((i < PT_M) ? compress_bit(low, i) : low);
        T x2o = sx2[e];
        T xo = P.alpha * sx[e] + (one - P.alpha) * x2o;
        T zz = sz[e];
        T v = xo - P.ib2 * zz;
        sz[e] = zz - P.b2 * xo;
        const bool w = (wb >> i) & 1u;
        T xh = (T)0;
        if (w) xh = P.xhat[(ll)i * Nloc + (ll)compress_bit(S ^ (1u << i), i)];
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
    double tau = 0.0;
    bool ok = false;
    if (k > 1 && A0 != 0) {
        tau = (s1 - 1.0) / s2;
        ok = true;
        for (uint32_t SS = S; SS; SS &= SS - 1) {
            const int i = __ffs(SS) - 1;
            const int e = roff[i] + (int)((i < PT_M) ? compress_bit(low, i) : low);
            double ti = (double)sx[e];
            if (mixed) {
                const bool w = (wb >> i) & 1u;
                ti = (double)P.b2 * ti +
                     (w ? 2.0 * (double)P.xhat[(ll)i * Nloc + (ll)compress_bit(S ^ (1u << i), i)] : 0.0);
            }
            const bool in = (A0 >> i) & 1u;
            if (in ? !(ti > tau) : (ti > tau)) { ok = false; break; }
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
                const int e = roff[i] + (int)((i < PT_M) ? compress_bit(low, i) : low);
                double ti = (double)sx[e];
                double ic = 1.0;
                if (mixed) {
                    const bool w = (wb >> i) & 1u;
                    if (w) ti = (double)P.b2 * ti + 2.0 * (double)P.xhat[(ll)i * Nloc + (ll)compress_bit(S ^ (1u << i), i)];
                    else ti = (double)P.b2 * ti;
                    ic = w ? icw : icu;
                }
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
    for (uint32_t SS = S; SS; SS &= SS - 1) {
        const int i = __ffs(SS) - 1;
        const int e = roff[i] + (int)((i < PT_M) ? compress_bit(low, i) : low);
        T u;
        if (k == 1) {
            u = one;
        } else if (mixed) {
            const bool w = (wb >> i) & 1u;
            double ti = (double)P.b2 * (double)sx[e] +
                        (w ? 2.0 * (double)P.xhat[(ll)i * Nloc + (ll)compress_bit(S ^ (1u << i), i)] : 0.0);
            double yv = (ti - tau) / (w ? cw : cu);
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
    if (tid < 32 && lane < n) {
        int len = pt_rlen(base, lane);
        if (len) {
            int off = roff[lane];
            ll g = pt_rstart(base, lane, Nloc);
            unsigned b = (unsigned)(len * sizeof(T));
            tma_store_1d(P.x2 + g, sx2 + off, b);
            tma_store_1d(P.z + g, sz + off, b);
            tma_commit();
            tma_wait_read();
        }
    }
}

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

}  // namespace rumb
