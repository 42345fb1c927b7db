// Generalized 2x2 butterflies over the rest bits of every alternative block (sm_100a).
//
// The transform applies, for every rest bit j ascending, the map (lo, hi) -> (a*lo + b*hi,
// c*lo + d*hi) to each pair (l, l | 2^j) of an alternative's 2^(n-1) block -- the reference's
// Bfly2 / butterfly_fast (solver/bm_admm/butterfly2.py:72-102, solver/common/butterfly.py:304-363).
// Bits are always applied in ascending order, so every pass plan gives the same result.
//
// B200 design. One pass covers a window of B consecutive bits [s, s+B) for a tile of 2^B rows:
//   s == 0: the tile is 2^B contiguous values, laid out as rows of 32 lanes. The 5 lowest bits
//           are lane bits, done with warp shuffles straight after the coalesced load; the
//           remaining B-5 bits are row bits.
//   s >= 5: the tile is 2^B rows of 32 contiguous values (a 128/256-byte segment per row); all B
//           bits are row bits.
// Row bits are done in groups of up to 4 bits from shared memory: a thread loads the 2^r values
// of one column, applies r stages in registers and stores them back, so each group costs one
// shared-memory round trip instead of r. Lanes index consecutive 32-bit banks, so the column
// accesses are conflict-free. Prologue / epilogue functors fuse the elementwise ADMM steps into
// the first load and the last store of a transform.
#pragma once
#include <cstdio>

#include "common.cuh"

namespace rumb {

constexpr int BF_THREADS = 256;
constexpr int BF_MAX_TILE_LOG = 13;  // 8192 values per tile (64 KB in float64)

// ---------------------------------------------------------------- load / store modes
enum BfPro { PRO_PLAIN = 0, PRO_W = 1 };       // PRO_W: v = y - k0 * s (two inputs)
enum BfEpi { EPI_PLAIN = 0, EPI_RHS = 1, EPI_DIAG = 2 };
// EPI_RHS: out = (z + k1 * x2 - v) * k2;  EPI_DIAG: out = v * diag[popcount(rest)]

template <class T, class TI>
struct BfArgs {
    const TI *in;
    T *out;
    const T *p0, *p1;     // PRO_W: y, s
    const T *q0, *q1;     // EPI_RHS: z, x2
    T k0, k1, k2;         // PRO_W: k0 = beta1;  EPI_RHS: k1 = beta2, k2 = 1/beta1
    const T *diag;        // EPI_DIAG: n entries indexed by popcount of the rest index
    T a, b, c, d;
    ll Nloc;
    int nb;               // n - 1 rest bits
    int s, B;             // window
    int pro, epi;
};

template <class T, class TI>
__device__ __forceinline__ T bf_load(const BfArgs<T, TI> &A, ll g) {
    if (A.pro == PRO_W) return A.p0[g] - A.k0 * A.p1[g];
    return (T)A.in[g];
}

template <class T, class TI>
__device__ __forceinline__ void bf_store(const BfArgs<T, TI> &A, ll g, T v) {
    if (A.epi == EPI_RHS) {
        v = (A.q0[g] + A.k1 * A.q1[g] - v) * A.k2;
    } else if (A.epi == EPI_DIAG) {
        ll rest = g & (A.Nloc - 1);
        v = v * A.diag[__popcll((ull)rest)];
    }
    A.out[g] = v;
}

template <class T>
__device__ __forceinline__ void bf_pair(T &X, T &Y, T a, T b, T c, T d) {
    T lo = a * X + b * Y;
    T hi = c * X + d * Y;
    X = lo;
    Y = hi;
}

// r stages (ascending) on 2^R register values, local bit j pairs (i, i | 2^j)
template <class T, int R>
__device__ __forceinline__ void bf_reg_stages(T (&v)[1 << R], int r, T a, T b, T c, T d) {
#pragma unroll
    for (int j = 0; j < R; ++j) {
        if (j < r) {
#pragma unroll
            for (int i = 0; i < (1 << R); ++i)
                if (!(i & (1 << j))) bf_pair(v[i], v[i | (1 << j)], a, b, c, d);
        }
    }
}

// Row-bit groups on a tile in shared memory: rows = 2^nrb rows of 32 lanes.
template <class T>
__device__ __forceinline__ void bf_row_groups(T *sm, int nrb, T a, T b, T c, T d) {
    for (int gb = 0; gb < nrb; gb += 4) {
        int r = nrb - gb < 4 ? nrb - gb : 4;
        int cols = ((1 << nrb) >> r) * 32;
        for (int col = threadIdx.x; col < cols; col += blockDim.x) {
            int lane = col & 31;
            int rb = col >> 5;                                     // row index with r bits removed
            int row0 = ((rb >> gb) << (gb + r)) | (rb & ((1 << gb) - 1));
            T v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (i < (1 << r)) v[i] = sm[((row0 | (i << gb)) << 5) + lane];
            bf_reg_stages<T, 4>(v, r, a, b, c, d);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (i < (1 << r)) sm[((row0 | (i << gb)) << 5) + lane] = v[i];
        }
        __syncthreads();
    }
}

// One pass over the window [s, s+B). Grid: one CTA per (alternative, tile).
template <class T, class TI>
__global__ void __launch_bounds__(BF_THREADS) bfly_pass(BfArgs<T, TI> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sm = reinterpret_cast<T *>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int s = A.s, B = A.B;
    ll tiles_per_block = A.Nloc >> (s == 0 ? B : B + 5);
    ll x = blockIdx.x / tiles_per_block;
    ll t = blockIdx.x - x * tiles_per_block;
    ll blockbase = x * A.Nloc;
    if (s == 0) {
        // 2^B contiguous values; lane bits 0..4 by shuffles
        const int rows = 1 << (B - 5);
        ll base = blockbase + (t << B);
        for (int row = warp; row < rows; row += nwarps) {
            ll g = base + ((ll)row << 5) + lane;
            T v = bf_load(A, g);
#pragma unroll
            for (int j = 0; j < 5; ++j) {
                T o = __shfl_xor_sync(0xffffffffu, v, 1 << j);
                if (lane & (1 << j)) v = A.c * o + A.d * v;      // hi' = c*lo + d*hi
                else v = A.a * v + A.b * o;                      // lo' = a*lo + b*hi
            }
            sm[(row << 5) + lane] = v;
        }
        __syncthreads();
        bf_row_groups(sm, B - 5, A.a, A.b, A.c, A.d);
        for (int row = warp; row < rows; row += nwarps) {
            ll g = base + ((ll)row << 5) + lane;
            bf_store(A, g, sm[(row << 5) + lane]);
        }
    } else {
        // 2^B rows of 32 contiguous values: rest = high | (row << s) | (lowblk*32 + lane)
        const int rows = 1 << B;
        ll nlow = (1LL << s) >> 5;
        ll lowblk = t % nlow, hi = t / nlow;
        ll base = blockbase + (hi << (s + B)) + (lowblk << 5);
        for (int row = warp; row < rows; row += nwarps) {
            ll g = base + ((ll)row << s) + lane;
            sm[(row << 5) + lane] = bf_load(A, g);
        }
        __syncthreads();
        bf_row_groups(sm, B, A.a, A.b, A.c, A.d);
        for (int row = warp; row < rows; row += nwarps) {
            ll g = base + ((ll)row << s) + lane;
            bf_store(A, g, sm[(row << 5) + lane]);
        }
    }
}

// Blocks narrower than 32 values (n <= 5): one thread per alternative block, all in registers.
template <class T, class TI>
__global__ void bfly_small(BfArgs<T, TI> A, int nalt) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nalt) return;
    T v[16];
    int N = (int)A.Nloc;
    ll base = (ll)x * A.Nloc;
    for (int i = 0; i < N; ++i) v[i] = bf_load(A, base + i);
    for (int j = 0; j < A.nb; ++j)
        for (int i = 0; i < N; ++i)
            if (!(i & (1 << j))) bf_pair(v[i], v[i | (1 << j)], A.a, A.b, A.c, A.d);
    for (int i = 0; i < N; ++i) bf_store(A, base + i, v[i]);
}

// ---------------------------------------------------------------- pass plan (host)
struct BfPass {
    int s, B;
};

// Windows covering bits [0, nb): the first pass takes up to 12 low bits as one contiguous
// tile, later passes take up to 8 bits as 2^B rows x 32 lanes (both <= 8192 values).
inline std::vector<BfPass> bf_plan(int nb) {
    std::vector<BfPass> plan;
    if (nb < 5) {
        plan.push_back({0, nb});
        return plan;
    }
    int first = nb <= BF_MAX_TILE_LOG ? nb : 12;
    plan.push_back({0, first});
    int s = first;
    while (s < nb) {
        int rem = nb - s;
        int B = rem <= 8 ? rem : (rem - 8 < 3 ? rem - 3 : 8);
        plan.push_back({s, B});
        s += B;
    }
    return plan;
}

template <class T, class TI>
inline void bf_launch_pass(const BfArgs<T, TI> &A, int n, cudaStream_t st) {
    if (A.nb < 5) {
        bfly_small<T, TI><<<grid_for(n, 64), 64, 0, st>>>(A, n);
        RUMB_LAUNCH("bfly_small");
        return;
    }
    static std::atomic<unsigned long long> optin{0};
    smem_optin(bfly_pass<T, TI>, (int)(sizeof(T) << BF_MAX_TILE_LOG), optin);
    ll tiles = A.Nloc >> (A.s == 0 ? A.B : A.B + 5);
    size_t smem = (size_t)sizeof(T) << (A.s == 0 ? A.B : A.B + 5);
    if (g_prof) {
        double S = (double)A.Nloc * n;
        double bytes = S * (sizeof(TI) + sizeof(T));
        if (A.pro == PRO_W) bytes += S * sizeof(T);              // two inputs instead of one
        if (A.epi == EPI_RHS) bytes += 2.0 * S * sizeof(T);
        char nm[64];
        snprintf(nm, sizeof nm, "bfly_pass<%s>[s=%d,B=%d]", sizeof(T) == 8 ? "f64" : "f32", A.s, A.B);
        prof_begin(nm, bytes, st);
    }
    bfly_pass<T, TI><<<(unsigned)(tiles * n), BF_THREADS, smem, st>>>(A);
    RUMB_LAUNCH("bfly_pass");
    prof_end(st);
}

// Full transform in -> out. pro applies to the first pass's load, epi to the last pass's store;
// intermediate passes run in place on `out`. `in` may equal `out`.
template <class T, class TI>
inline void bf_transform(int n, const TI *in, T *out, T a, T b, T c, T d, cudaStream_t st,
                         int pro = PRO_PLAIN, const T *p0 = nullptr, const T *p1 = nullptr, T k0 = 0,
                         int epi = EPI_PLAIN, const T *q0 = nullptr, const T *q1 = nullptr, T k1 = 0,
                         T k2 = 0, const T *diag = nullptr) {
    int nb = n - 1;
    ll Nloc = 1LL << nb;
    std::vector<BfPass> plan = bf_plan(nb);
    for (size_t i = 0; i < plan.size(); ++i) {
        bool first = i == 0, last = i + 1 == plan.size();
        if (first) {
            BfArgs<T, TI> A{};
            A.in = in; A.out = out; A.Nloc = Nloc; A.nb = nb; A.s = plan[i].s; A.B = plan[i].B;
            A.a = a; A.b = b; A.c = c; A.d = d;
            A.pro = pro; A.p0 = p0; A.p1 = p1; A.k0 = k0;
            A.epi = EPI_PLAIN;
            if (last) { A.epi = epi; A.q0 = q0; A.q1 = q1; A.k1 = k1; A.k2 = k2; A.diag = diag; }
            bf_launch_pass<T, TI>(A, n, st);
        } else {
            BfArgs<T, T> A{};
            A.in = out; A.out = out; A.Nloc = Nloc; A.nb = nb; A.s = plan[i].s; A.B = plan[i].B;
            A.a = a; A.b = b; A.c = c; A.d = d;
            A.pro = PRO_PLAIN; A.epi = EPI_PLAIN;
            if (last) { A.epi = epi; A.q0 = q0; A.q1 = q1; A.k1 = k1; A.k2 = k2; A.diag = diag; }
            bf_launch_pass<T, T>(A, n, st);
        }
    }
}

}  // namespace rumb
