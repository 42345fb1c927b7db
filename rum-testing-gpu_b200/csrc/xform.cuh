// Register-tiled butterfly passes for the BM-ADMM iteration (sm_100a).
//
// A pass covers the window of rest bits [s, s+B) of every alternative block. Its tile is 2^B
// values arranged as rows of 32 lanes: for s == 0 the tile is 2^B contiguous values and the 5
// lowest bits are lane bits (warp shuffles); for s >= 5 the tile is 2^B rows of 32 contiguous
// values and every bit is a row bit. Row bits split into RB register bits and WB warp bits
// (RB >= WB), and a thread holds R = 2^RB values in one of two layouts:
//   layout A: register j = row bits 0..RB-1, warp = row bits RB..RB+WB-1
//   layout B: register j = (jh, jl): jh = row bits RB..RB+WB-1, jl = row bits WB..RB-1,
//             warp = row bits 0..WB-1
// A "forward" phase runs lane stages, the layout-A register stages, one shared-memory transpose
// and the layout-B register stages (ending in layout B); a "backward" phase runs them in the
// opposite order (ending in layout A). Loads and stores are coalesced rows of 32 lanes in either
// layout, and every load of a pass is issued before the first stage, so each warp keeps 2^RB
// (times the number of input streams) loads in flight.
//
// The four iteration passes fuse the elementwise ADMM steps of the reference's one_iter
// (solver/bm_admm/solver.py:240-254) into the transforms:
//   K_P1   (low bits)  w = y - b1 s;  A' forward                              -> T1
//   K_P2   (high bits) A' forward;  rhs = (z + b2 x2 - v) / b1;  Q^T backward -> T2
//   K_P3   (low bits)  Q^T forward;  v *= 1/(gamma + lambda(rest));  Q backward -> T3, and
//                      A backward on a copy of T3 -> T4 (= (A Q) on the low window)
//   K_P4   (high bits) Q forward on T3 -> x;  (A Q) forward on T4 -> A x, then the s/y update
//                      a = -alpha Ax - (1-alpha) s; s' = max(y/b1 - a, 0); y -= b1 (a + s')
//   K_FULL (all bits, n <= 13) P1..P4 in one pass
//   K_DUAL (middle high bits, n >= 21) Q and (A Q) forward on two streams, in place
//   K_P4A  K_P4, then the next iteration's w = y - b1 s and its A' on the same window -> T1
// With two windows an iteration sequence alternates the windows: iteration i runs P2 on window Y,
// P3 on the other window and P4A on Y, where Y is the high window for even i and the low window
// for odd i; the sequence starts with P1 on the low window and ends with a plain P4, so an
// iteration costs three passes instead of four (every pass is written window-agnostic).
// The tensor factors of a transform act on different bits and commute, so applying a
// transform's high bits before its low bits (P2 / P3) changes only the rounding.
#pragma once
#include "common.cuh"

namespace rumb {

template <class T>
struct Co {
    T a, b, c, d;
};

// Pair forms (MODE): 0 general (a, b, c, d); 1 A' = (1, 0, -1, p): lo' = lo, hi' = p hi - lo
// (one operation per pair); 2 A = (1, -1, 0, p): lo' = lo - hi, hi' = p hi (two operations);
// 3 a reflection scaled to unit diagonal, (1, b, c, -1): lo' = lo + b hi, hi' = c lo - hi (two
// fused multiply-adds per pair; the eigenvector matrix Q = q00 (1, t, t, -1) is applied this way and
// its scale q00 per stage is folded into the eigen-space diagonal)
constexpr int XF_GEN = 0, XF_APRIME = 1, XF_A = 2, XF_UNIT = 3;

template <class T, int MODE>
__device__ __forceinline__ void xf_pair(T &X, T &Y, const Co<T> &k) {
    if (MODE == XF_APRIME) {
        Y = k.d * Y - X;
        return;
    }
    if (MODE == XF_A) {
        X = X - Y;
        Y = k.d * Y;
        return;
    }
    if (MODE == XF_UNIT) {
        T lo = X + k.b * Y;
        T hi = k.c * X - Y;
        X = lo;
        Y = hi;
        return;
    }
    T lo = k.a * X + k.b * Y;
    T hi = k.c * X + k.d * Y;
    X = lo;
    Y = hi;
}

// stages on register-index bits [B0, B0+NB), ascending
template <class T, int R, int B0, int NB, int AP>
__device__ __forceinline__ void xf_regs(T (&v)[R], const Co<T> &k) {
#pragma unroll
    for (int j = B0; j < B0 + NB; ++j) {
#pragma unroll
        for (int i = 0; i < R; ++i)
            if (!(i & (1 << j))) xf_pair<T, AP>(v[i], v[i | (1 << j)], k);
    }
}

// the 5 lane-bit stages on every register value; the per-lane coefficients are picked once per
// stage (lo lane: a, b; hi lane: d, c), so each value costs one multiply and one fma
template <class T, int R, int AP>
__device__ __forceinline__ void xf_lanes(T (&v)[R], int lane, const Co<T> &k) {
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        const bool hi = (lane >> j) & 1;
        const T c0 = hi ? k.d : k.a, c1 = hi ? k.c : k.b;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            T o = __shfl_xor_sync(0xffffffffu, v[i], 1 << j);
            if (AP == XF_APRIME) {
                if (hi) v[i] = k.d * v[i] - o;
            } else if (AP == XF_UNIT) {
                v[i] = c1 * o + (hi ? -v[i] : v[i]);
            } else if (AP == XF_A) {
                v[i] = hi ? k.d * v[i] : v[i] - o;
            } else {
                v[i] = c0 * v[i] + c1 * o;
            }
        }
    }
}

template <int RB, int WB>
__device__ __forceinline__ int row_A(int w, int j) { return (w << RB) | j; }

template <int RB, int WB>
__device__ __forceinline__ int row_B(int w, int j) {
    constexpr int JL = RB - WB;
    int jh = j >> JL, jl = j & ((1 << JL) - 1);
    return (jh << RB) | (jl << WB) | w;
}

// shared-memory transposes between the layouts (sm holds 2^(RB+WB) rows of 32)
template <class T, int RB, int WB>
__device__ __forceinline__ void xf_A_to_B(T (&v)[1 << RB], T *sm, int w, int lane) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) sm[(row_A<RB, WB>(w, j) << 5) + lane] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) v[j] = sm[(row_B<RB, WB>(w, j) << 5) + lane];
    __syncthreads();
}

template <class T, int RB, int WB>
__device__ __forceinline__ void xf_B_to_A(T (&v)[1 << RB], T *sm, int w, int lane) {
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) sm[(row_B<RB, WB>(w, j) << 5) + lane] = v[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < (1 << RB); ++j) v[j] = sm[(row_A<RB, WB>(w, j) << 5) + lane];
    __syncthreads();
}

// forward: (lanes) -> A regs -> transpose -> B regs;   starts in A, ends in B
template <class T, int L, int RB, int WB, int AP = XF_GEN>
__device__ __forceinline__ void xf_forward(T (&v)[1 << RB], T *sm, int w, int lane, const Co<T> &k) {
    if (L) xf_lanes<T, 1 << RB, AP>(v, lane, k);
    xf_regs<T, 1 << RB, 0, RB, AP>(v, k);
    if (WB) {
        xf_A_to_B<T, RB, WB>(v, sm, w, lane);
        xf_regs<T, 1 << RB, RB - WB, WB, AP>(v, k);
    }
}

// backward: B regs -> transpose -> A regs -> (lanes);   starts in B, ends in A
template <class T, int L, int RB, int WB, int AP = XF_GEN>
__device__ __forceinline__ void xf_backward(T (&v)[1 << RB], T *sm, int w, int lane, const Co<T> &k) {
    if (WB) {
        xf_regs<T, 1 << RB, RB - WB, WB, AP>(v, k);
        xf_B_to_A<T, RB, WB>(v, sm, w, lane);
    }
    xf_regs<T, 1 << RB, 0, RB, AP>(v, k);
    if (L) xf_lanes<T, 1 << RB, AP>(v, lane, k);
}

enum XfKind { K_PLAIN = 0, K_P1 = 1, K_P2 = 2, K_P3 = 3, K_P4 = 4, K_FULL = 5, K_DUAL = 6, K_P4A = 7 };

template <class T, class TI>
struct XfArgs {
    const TI *in;       // K_PLAIN / K_P2 / K_P3 input; K_P4 / K_DUAL first stream
    const T *in2;       // K_P4 / K_DUAL second stream
    T *out, *out2;
    const T *y, *s;     // K_P1 / K_FULL inputs
    T *s_io, *y_io;     // K_P4 / K_FULL state
    const T *z, *x2;    // K_P2 / K_FULL
    const T *diag;      // K_P3: by popcount of the rest index
    Co<T> k1, k2, k3, k4;  // phase coefficients: see each kind (K_FULL: A', Q^T, Q, A Q)
    T b1, b2, ib1, alpha;
    ll Nloc;
    int s0, B;          // window
    ll bstride;         // batched draws: elements between consecutive draws' slabs (grid.y = draw slot)
    const int *active;  // batched draws: slot flags (nullptr: every slot runs)
};

template <class T, int L, int RB, int WB>
__device__ __forceinline__ ll xf_index(int s0, int B, ll Nloc, ll tile, int row, int lane) {
    // tile -> (alternative, position); returns the slab index of (row, lane)
    if (L) {
        ll tiles_per = Nloc >> B;
        ll x = tile / tiles_per, t = tile - x * tiles_per;
        return x * Nloc + (t << B) + ((ll)row << 5) + lane;
    }
    ll tiles_per = Nloc >> (B + 5);
    ll x = tile / tiles_per, t = tile - x * tiles_per;
    ll nlow = (1LL << s0) >> 5;
    ll lowblk = t % nlow, hi = t / nlow;
    return x * Nloc + (hi << (s0 + B)) + ((ll)row << s0) + (lowblk << 5) + lane;
}

// CTAs kept resident per SM: the four-stream kinds with 8 values a thread and 256 threads are held
// to 128 registers so that two CTAs fit an SM (85, three CTAs, on the low window)
template <int L, int RB, int WB, int KIND>
constexpr int xf_min_blocks() {
    return ((KIND == K_P4 || KIND == K_P4A) && RB <= 3 && WB == 3) ? (L ? 3 : 2) : 1;
}

template <class T, class TI, int L, int RB, int WB, int KIND>
__global__ void __launch_bounds__(32 << WB, xf_min_blocks<L, RB, WB, KIND>()) xform_pass(XfArgs<T, TI> A) {
    pdl_grid_sync();                                        // launched by launch_pdl: nothing read before
    extern __shared__ __align__(16) unsigned char xf_smem[];
    T *sm = reinterpret_cast<T *>(xf_smem);
    constexpr int R = 1 << RB;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const ll tile = blockIdx.x;
    const int s0 = A.s0, B = A.B;
    const ll Nloc = A.Nloc;
    if (A.active && !A.active[blockIdx.y]) return;          // a retired slot (uniform per CTA)
    const ll boff = (ll)blockIdx.y * A.bstride;
    T v[R];
    if constexpr (KIND == K_P4 || KIND == K_P4A || KIND == K_DUAL) {
        constexpr bool SY = KIND == K_P4 || KIND == K_P4A;
        T u[R], ss[SY ? R : 1], yy[SY ? R : 1];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row_A<RB, WB>(w, j), lane);
            v[j] = (T)A.in[g];
            u[j] = A.in2[g];
        }
        if constexpr (SY) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                int row = WB ? row_B<RB, WB>(w, j) : row_A<RB, WB>(w, j);
                ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row, lane);
                ss[j] = A.s_io[g];
                yy[j] = A.y_io[g];
            }
        }
        xf_forward<T, L, RB, WB, XF_UNIT>(v, sm, w, lane, A.k1);          // Q (unit form)
        xf_forward<T, L, RB, WB>(u, sm, w, lane, A.k3);                   // A Q (scaled)
#pragma unroll
        for (int j = 0; j < R; ++j) {
            int row = WB ? row_B<RB, WB>(w, j) : row_A<RB, WB>(w, j);
            ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row, lane);
            A.out[g] = v[j];
            if constexpr (!SY) {
                A.out2[g] = u[j];
            } else {
                T ax = u[j], sv = ss[j], yv = yy[j];
                T one = (T)1;
                T axor = -A.alpha * ax - (one - A.alpha) * sv;
                T sn = A.ib1 * yv - axor;
                sn = sn > (T)0 ? sn : (T)0;
                const T yn = yv - A.b1 * (axor + sn);
                A.y_io[g] = yn;
                A.s_io[g] = sn;
                ss[j] = yn - A.b1 * sn;                  // K_P4A: the next iteration's w
            }
        }
        if constexpr (KIND == K_P4A) {
            // the next iteration's A' on this window, from layout B back to layout A
            xf_backward<T, L, RB, WB, XF_APRIME>(ss, sm, w, lane, A.k4);
#pragma unroll
            for (int j = 0; j < R; ++j)
                A.out2[boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row_A<RB, WB>(w, j), lane)] = ss[j];
        }
        return;
    } else {
        // single input stream; the layout-B side inputs (z, x2) are loaded up front as well
        T zz[(KIND == K_P2 || KIND == K_FULL) ? R : 1], xx[(KIND == K_P2 || KIND == K_FULL) ? R : 1];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row_A<RB, WB>(w, j), lane);
            if (KIND == K_P1 || KIND == K_FULL) v[j] = A.y[g] - A.b1 * A.s[g];
            else v[j] = (T)A.in[g];
        }
        if (KIND == K_P2 || KIND == K_FULL) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                int row = WB ? row_B<RB, WB>(w, j) : row_A<RB, WB>(w, j);
                ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row, lane);
                zz[j] = A.z[g];
                xx[j] = A.x2[g];
            }
        }
        if (KIND == K_P1 || KIND == K_P2 || KIND == K_FULL) xf_forward<T, L, RB, WB, XF_APRIME>(v, sm, w, lane, A.k1);
        else if (KIND == K_P3) xf_forward<T, L, RB, WB, XF_UNIT>(v, sm, w, lane, A.k1);   // Q^T (unit form)
        else xf_forward<T, L, RB, WB, XF_GEN>(v, sm, w, lane, A.k1);
        // now in layout B (layout A when WB == 0)
        if constexpr (KIND == K_PLAIN || KIND == K_P1) {
#pragma unroll
            for (int j = 0; j < R; ++j) {
                int row = WB ? row_B<RB, WB>(w, j) : row_A<RB, WB>(w, j);
                A.out[boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row, lane)] = v[j];
            }
            return;
        }
        if constexpr (KIND == K_P2 || KIND == K_FULL) {
#pragma unroll
            for (int j = 0; j < R; ++j) v[j] = (zz[j] + A.b2 * xx[j] - v[j]) * A.ib1;
            xf_backward<T, L, RB, WB, XF_UNIT>(v, sm, w, lane, A.k2);        // Q^T (unit form)
            if (KIND == K_P2) {
#pragma unroll
                for (int j = 0; j < R; ++j)
                    A.out[boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row_A<RB, WB>(w, j), lane)] = v[j];
                return;
            }
            // K_FULL: diag, then Q and (A Q) forward, x and the s/y update (layout A -> B)
            T u[R];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row_A<RB, WB>(w, j), lane);
                v[j] = v[j] * A.diag[__popcll((ull)(g & (Nloc - 1)))];
                u[j] = v[j];
            }
            xf_forward<T, L, RB, WB, XF_UNIT>(v, sm, w, lane, A.k3);      // Q (unit form)
            xf_forward<T, L, RB, WB>(u, sm, w, lane, A.k4);               // A Q (scaled)
#pragma unroll
            for (int j = 0; j < R; ++j) {
                int row = WB ? row_B<RB, WB>(w, j) : row_A<RB, WB>(w, j);
                ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row, lane);
                A.out[g] = v[j];
                T ax = u[j], sv = A.s_io[g], yv = A.y_io[g];
                T one = (T)1;
                T axor = -A.alpha * ax - (one - A.alpha) * sv;
                T sn = A.ib1 * yv - axor;
                sn = sn > (T)0 ? sn : (T)0;
                A.y_io[g] = yv - A.b1 * (axor + sn);
                A.s_io[g] = sn;
            }
            return;
        }
        if constexpr (KIND == K_P3) {
            // (A Q) on the low window is A applied after Q: the fork copies Q's result (layout A) and
            // runs the two-operation A form (k4 = (1, -1, 0, p)) forward from layout A to layout B
            // instead of a second general transform; the factors of A commute, so the stage order
            // does not matter
            T u[R];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                int row = WB ? row_B<RB, WB>(w, j) : row_A<RB, WB>(w, j);
                ll g = boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row, lane);
                v[j] = v[j] * A.diag[__popcll((ull)(g & (Nloc - 1)))];
            }
            xf_backward<T, L, RB, WB, XF_UNIT>(v, sm, w, lane, A.k2);         // Q (unit form)
#pragma unroll
            for (int j = 0; j < R; ++j) {
                u[j] = v[j];
                A.out[boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row_A<RB, WB>(w, j), lane)] = v[j];
            }
            xf_forward<T, L, RB, WB, XF_A>(u, sm, w, lane, A.k4);
#pragma unroll
            for (int j = 0; j < R; ++j) {
                int row = WB ? row_B<RB, WB>(w, j) : row_A<RB, WB>(w, j);
                A.out2[boff + xf_index<T, L, RB, WB>(s0, B, Nloc, tile, row, lane)] = u[j];
            }
        }
    }
}

// ---------------------------------------------------------------- host side
struct XfShape {
    int s0, B, L, RB, WB;
};

// Window split of nb rest bits: a low pass (s0 = 0) of up to lo_bits (<= 12) bits, then high
// passes of up to 7 bits. Returns (L, RB, WB) per pass with RB >= WB, RB <= 4. The split is a
// tuning knob (rumb picks lo_bits per GPU, n and dtype by timing the candidates).
inline std::vector<XfShape> xf_plan(int nb, int lo_bits = 12) {
    std::vector<XfShape> plan;
    if (lo_bits > 12) lo_bits = 12;
    if (lo_bits < 5) lo_bits = 5;
    int first = nb < lo_bits ? nb : lo_bits;
    {
        int rw = first - 5;
        int wb = rw / 2 < 3 ? rw / 2 : 3;
        plan.push_back({0, first, 1, rw - wb, wb});
    }
    int s = first;
    while (s < nb) {
        int rem = nb - s;
        int B = rem <= 7 ? rem : (rem - 7 < 3 ? rem - 3 : 7);
        int wb = B / 2 < 3 ? B / 2 : 3;
        plan.push_back({s, B, 0, B - wb, wb});
        s += B;
    }
    return plan;
}

template <class T, class TI, int L, int RB, int WB, int KIND>
inline void xf_launch_one(const XfArgs<T, TI> &A, int n, cudaStream_t st, int slots = 1) {
    static std::atomic<unsigned long long> optin{0};
    size_t smem = (size_t)sizeof(T) << (RB + WB + 5);
    smem_optin(xform_pass<T, TI, L, RB, WB, KIND>, (int)smem, optin);
    ll tiles = (A.Nloc >> (L ? A.B : A.B + 5)) * n;
    if (g_prof) {
        double S = (double)A.Nloc * n * slots, e = sizeof(T), ei = sizeof(TI);
        double bytes = S * e;                                          // one output
        switch (KIND) {
            case K_PLAIN: bytes += S * ei; break;
            case K_P1: bytes += 2 * S * e; break;
            case K_P2: bytes += 3 * S * e; break;
            case K_P3: bytes += 2 * S * e; break;
            case K_DUAL: bytes += 3 * S * e; break;
            case K_P4: bytes += 6 * S * e; break;
            case K_P4A: bytes += 7 * S * e; break;
            case K_FULL: bytes += 7 * S * e; break;
        }
        const char *kn[] = {"plain", "P1", "P2", "P3", "P4", "full", "dual", "P4A"};
        char nm[64];
        snprintf(nm, sizeof nm, "xform<%s,%s>[s=%d,B=%d]", sizeof(T) == 8 ? "f64" : "f32", kn[KIND], A.s0, A.B);
        prof_begin(nm, bytes, st);
    }
    launch_pdl(xform_pass<T, TI, L, RB, WB, KIND>, dim3((unsigned)tiles, (unsigned)slots), dim3(32u << WB), smem, st, A);
    RUMB_LAUNCH("xform_pass");
    prof_end(st);
}

template <class T, class TI, int KIND>
inline void xf_launch(const XfArgs<T, TI> &A, const XfShape &sh, int n, cudaStream_t st, int slots = 1) {
#define XF_CASE(LL, RBB, WBB)                                                     \
    if (sh.L == LL && sh.RB == RBB && sh.WB == WBB) {                             \
        xf_launch_one<T, TI, LL, RBB, WBB, KIND>(A, n, st, slots);                 \
        return;                                                                   \
    }
    XF_CASE(1, 0, 0) XF_CASE(1, 1, 0) XF_CASE(1, 1, 1) XF_CASE(1, 2, 1) XF_CASE(1, 2, 2) XF_CASE(1, 3, 2)
    XF_CASE(1, 3, 3) XF_CASE(1, 4, 3)
    XF_CASE(0, 1, 0) XF_CASE(0, 1, 1) XF_CASE(0, 2, 1) XF_CASE(0, 2, 2) XF_CASE(0, 3, 2) XF_CASE(0, 3, 3)
    XF_CASE(0, 4, 3)
#undef XF_CASE
    fail(RUMB_E_INTERNAL, "xform: no kernel for this window");
}

}  // namespace rumb
