// Flow-CG pricing on the GPU (sm_100a): the Bellman-Ford longest path over the subset lattice,
//     V[D] = max over x in D of V[D \ {x}] + w(x, D),  w(x, D) = sum of the scores of x's rows whose
//     menu is a subset of D (a sequential float32 sum in row order),
// and the ranking it picks, bit for bit as the reference computes them.
//
// Reference behaviour (mingxiz/rum-testing-gpu):
//   stream sweep   solver/flow_cg/pricing_stream.py:61-182 (BODY, f32/u16/u24 storage), :302-345
//   backtrace      solver/flow_cg/pricing_stream.py:348-405 (pred layers, sub-lattice mask DP)
//   mask sweep     solver/flow_cg/bf_pricing.py:8-47, solver/flow_cg/solver.py:169-200
//
// What must match exactly, and how it is kept:
//   * w(x, D) adds x's rows in their x-major order, one float32 add at a time.
//   * stream: candidates over x descending with `>=` (ties -> lowest x); mask: x ascending with
//     `>` (ties -> lowest x). Both are computed here as one warp-uniform loop over x so that all
//     lanes read the same row at the same time (a broadcast), with the lane's own predicate.
//   * quantization blocks are 1024 consecutive ranks: one CTA of 1024 threads per block, block
//     min / max (exact, order-free), step = (max - min) / levels and q = rintf((v - min) / step)
//     (the values themselves come from a separate launch over 256-rank tiles, see below)
//     with IEEE division; the previous layer is decoded as fma(q, step, min) (fma_decode = 1,
//     the contraction the reference's JIT compiler applies to m + q * e) or as a rounded multiply
//     then add (fma_decode = 0).
//   * the sub-lattice DP after the descent uses the original menus and row order restricted to
//     the node reached, which is what the reference's relabelled sub-problem adds up.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "ctx.cuh"
#include "pricer.cuh"

namespace rumb {

constexpr int PB = 1024;       // ranks per quantization block = threads per CTA
constexpr int MAXN_PR = 40;

struct PricerArgs {
    int n, k;
    ull count;                 // ranks in this layer
    const ull *binom;          // C(b, t) at b*(n+1)+t
    const ull *menus;          // x-major rows
    const float *scores;
    const ll *offsets;         // n+1
    int mode;                  // 1 f32, 2 u16, 3 u24
    int fma_decode;
    // previous layer
    const float *vprev_f;
    const uint16_t *vprev_h;
    const uint8_t *lprev;
    const float *mprev, *eprev;
    const float *vprev_dec;    // the previous layer already decoded to float32 (or nullptr)
    // current layer
    float *vcur_f;
    uint16_t *vcur_h;
    uint8_t *lcur;
    float *mcur, *ecur;
    uint8_t *pred;             // nullptr when this layer keeps no predecessors
    unsigned int *layer_step;  // float bits, atomicMax (steps are >= 0)
    // mask mode: the layer's nodes, values and predecessors indexed by the mask
    const int *nodes;
    float *vmask;
    uint8_t *pmask;
    // w(x, D): row scan or cover lists (W_SCAN / W_LIST16 / W_LIST32)
    int wmode;
    const unsigned *loffs;
    const void *lent;
    ull lbase;                 // this layer's first pair index
};

__device__ ull colex_rank_dev(ull mask, const ull *binom, int n) {
    ull r = 0;
    int t = 0;
    for (int b = 0; b < n; ++b)
        if ((mask >> b) & 1ULL) {
            ++t;
            r += binom[b * (n + 1) + t];
        }
    return r;
}

// The binomial table C(b, t) at b*(n+1)+t, staged into shared memory by the whole CTA (the
// unranking and ranking below walk it with dependent lookups).
constexpr int BIN_MAX = (MAXN_PR + 1) * (MAXN_PR + 1);
__device__ __forceinline__ void stage_binom(ull *sbin, const ull *binom, int n) {
    for (int i = threadIdx.x; i < (n + 1) * (n + 1); i += blockDim.x) sbin[i] = binom[i];
}

// Colex unranking of r into a k-subset of [0, n) (elements ascending).
__device__ __forceinline__ ull colex_unrank(ull r, int k, int n, const ull *bin) {
    ull D = 0;
    int b = n - 1;
    for (int t = k; t >= 1; --t) {
        while (bin[b * (n + 1) + t] > r) --b;
        D |= 1ULL << b;
        r -= bin[b * (n + 1) + t];
        --b;
    }
    return D;
}

// Colex rank of D \ {x} from r = rank of D: with D's elements d_0 < ... and x = d_j (j = the
// number of elements below x), sum_{i<j} C(d_i, i+1) + sum_{i>j} C(d_i, i)
// = r - sum_{i>=j} C(d_i, i+1) + sum_{i>j} C(d_i, i).
__device__ __forceinline__ ull colex_rank_without(ull r, ull D, int x, int j, int n, const ull *bin) {
    int i = j;
    ull sub = 0, add = 0;
    for (ull E = D & ~((1ULL << x) - 1ULL); E; E &= E - 1ULL, ++i) {
        const int d = __ffsll((long long)E) - 1;
        sub += bin[d * (n + 1) + (i + 1)];
        if (i > j) add += bin[d * (n + 1) + i];
    }
    return r - sub + add;
}

__device__ __forceinline__ float decode_prev(const PricerArgs &A, ull rp) {
    if (A.vprev_dec) return A.vprev_dec[rp];
    if (A.mode == 1) return A.vprev_f[rp];
    unsigned int q = A.vprev_h[rp];
    if (A.mode == 3) q = (q << 8) | (unsigned int)A.lprev[rp];
    float qf = (float)q, m = A.mprev[rp / PB], e = A.eprev[rp / PB];
    if (A.fma_decode) return __fmaf_rn(qf, e, m);
    return __fadd_rn(m, __fmul_rn(qf, e));
}

// Cover lists. Only a small share of the (D, x, row) tests of a sweep succeed (a row of menu m
// qualifies for 2^(n - |m|) of the 2^(n-1) subsets D containing its alternative), and the menus do
// not change between sweeps of one pricer. So the pricer builds, once, for every pair (D, x in D)
// the list of x's rows whose menu is a subset of D, in row order, as indices local to x's rows;
// a sweep then adds exactly those rows' scores in that order, which is the same float32 sum as the
// row scan. Pair (D, x) of layer k = |D|, colex rank r of D and position j of x among D's elements
// (ascending) has index layer_base[k] + r k + j, with layer_base[k] = sum_{i<k} C(n, i) i, so a
// layer's lists are contiguous. offs[p]..offs[p+1] delimit pair p's entries (uint32 offsets);
// entries are uint16 when every alternative has <= 65536 rows, else uint32.
enum { W_SCAN = 0, W_LIST16 = 1, W_LIST32 = 2 };

// w(x, D) by scanning x's rows: a warp-uniform row loop (broadcast loads) with the lane's own
// subset test; every lane of the warp must call it.
__device__ __forceinline__ float w_scan(const ull *menus, const float *scores, ll lo, ll hi, ull D, bool in) {
    float w = 0.0f;
    if (__any_sync(0xffffffffu, in)) {
        for (ll i = lo; i < hi; ++i) {
            ull Dp = __ldg(menus + i);
            float sc = __ldg(scores + i);
            if (in && (Dp & D) == Dp) w = __fadd_rn(w, sc);
        }
    }
    return w;
}

// w(x, D) from pair p's cover list (sx = x's first score).
template <class IT>
__device__ __forceinline__ float w_list(const unsigned *offs, const IT *ent, ull p, const float *sx) {
    const unsigned b = __ldg(offs + p), e = __ldg(offs + p + 1);
    float w = 0.0f;
#pragma unroll 4
    for (unsigned i = b; i < e; ++i) w = __fadd_rn(w, __ldg(sx + __ldg(ent + i)));
    return w;
}

__device__ __forceinline__ float w_of(const PricerArgs &A, int x, ull D, bool in, ull p) {
    const ll lo = A.offsets[x];
    if (A.wmode == W_SCAN) return w_scan(A.menus, A.scores, lo, A.offsets[x + 1], D, in);
    if (!in) return 0.0f;
    if (A.wmode == W_LIST16) return w_list(A.loffs, (const uint16_t *)A.lent, p, A.scores + lo);
    return w_list(A.loffs, (const uint32_t *)A.lent, p, A.scores + lo);
}

// One popcount layer k of the sweep.
//
// layer_eval_kernel: a CTA of 1024 threads covers PE_R = 128 consecutive ranks (32 ranks and 256
// threads for the layers too small to give every SM two such CTAs) with PE_G = 8
// groups of alternatives (warp w: ranks 32 (w mod 4) .., group w / 4 = the x with x mod 8 equal to
// it), so a layer of C ranks spreads over C / 128 CTAs. Each thread walks its group's x from high
// to low, keeps the candidate with `>=` (ties -> lowest x); the eight group winners of a rank are
// merged the same way (the larger value, on a tie the lower x). That is the winner of the
// reference's loops in both modes: x descending with `>=` (stream) and x ascending with `>`
// (mask) both keep the lowest x among equal values.
//   MASK: the subset of rank r is the layer table's node r (ascending masks of popcount k, i.e.
//         colex order), values and predecessors are indexed by the mask and updated in place.
//   stream: D is the colex unranking of r; the value of D \ {x} is read from the previous layer's
//         storage at its colex rank; output: the float32 value (f32 mode, and the predecessor
//         byte) or the value for stream_quant_kernel to quantize (u16 / u24).
// stream_quant_kernel: one CTA per quantization block of 1024 ranks, as the number format asks:
// block min / max, step, rintf quantization of every value (u16 / u24 modes).
constexpr int PE_R = 128, PE_G = 8;
static_assert((PE_R / 32) * PE_G == 32 && (PE_G & (PE_G - 1)) == 0, "32 warps; PE_G a power of two");
// Layers whose 128-rank CTAs would not give every SM two of them run 32 ranks per CTA (8 warps).
constexpr int PE_R_SMALL = 32;

template <bool MASK, int PR>
__global__ void __launch_bounds__(PR * PE_G) layer_eval_kernel(PricerArgs A, float *vals) {
    pdl_grid_sync();                                       // launched by launch_pdl
    static_assert(PR % 32 == 0 && (PR / 32) * PE_G <= 32, "at most 32 warps");
    __shared__ float pbest[PE_G][PR];
    __shared__ signed char pbx[PE_G][PR];
    __shared__ ull sbin[MASK ? 1 : BIN_MAX];
    const int n = A.n, k = A.k;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rg = w % (PR / 32), xg = w / (PR / 32);
    const int loc = rg * 32 + lane;
    const ull r = (ull)blockIdx.x * PR + loc;
    const bool valid = r < A.count;
    if (!MASK) {
        stage_binom(sbin, A.binom, n);
        __syncthreads();
    }
    ull D = 0;
    if (valid) D = MASK ? (ull)(unsigned)A.nodes[r] : colex_unrank(r, k, n, sbin);
    const ull pbase = A.lbase + r * (ull)k;
    float best = 0.0f;
    int bestx = -1;
    for (int x = n - 1; x >= 0; --x) {
        if ((x & (PE_G - 1)) != xg) continue;            // uniform per warp
        const bool in = valid && ((D >> x) & 1ULL);
        const int j = __popcll(D & ((1ULL << x) - 1ULL));
        const float wsum = w_of(A, x, D, in, pbase + j);
        if (in) {
            float prev;
            if (MASK) prev = A.vmask[D ^ (1ULL << x)];
            else prev = decode_prev(A, colex_rank_without(r, D, x, j, n, sbin));
            const float cand = __fadd_rn(prev, wsum);
            if (bestx < 0 || cand >= best) { best = cand; bestx = x; }
        }
    }
    pbest[xg][loc] = best;
    pbx[xg][loc] = (signed char)bestx;
    __syncthreads();
    if (xg != 0 || !valid) return;
    float b = pbest[0][loc];
    int bx = pbx[0][loc];
    for (int g = 1; g < PE_G; ++g) {
        const float c = pbest[g][loc];
        const int cx = pbx[g][loc];
        if (cx < 0) continue;
        if (bx < 0 || c > b || (c == b && cx < bx)) { b = c; bx = cx; }
    }
    if (MASK) {
        A.vmask[D] = b;
        A.pmask[D] = (uint8_t)bx;
        return;
    }
    if (A.pred) A.pred[r] = (uint8_t)bx;
    if (A.mode == 1) A.vcur_f[r] = b;
    else vals[r] = b;
}

// The float64 max sweep (sweep_max64, the Frank-Wolfe bound's longest path when the float64 slab
// does not fit): the same layer mapping with float64 scores and values, only the maximum kept. Each
// w(x, D) is a sequential float64 sum over the same rows in row order (cover lists or the row scan)
// and the maximum is exact, so V[full] is the reference kernel's bit for bit.
template <int PR>
__global__ void __launch_bounds__(PR * PE_G) max64_layer_kernel(PricerArgs A, const double *scores,
                                                                 const double *vprev, double *vcur) {
    pdl_grid_sync();                                       // launched by launch_pdl
    static_assert(PR % 32 == 0 && (PR / 32) * PE_G <= 32, "at most 32 warps");
    __shared__ double pbest[PE_G][PR];
    __shared__ signed char pok[PE_G][PR];
    __shared__ ull sbin[BIN_MAX];
    const int n = A.n, k = A.k;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rg = w % (PR / 32), xg = w / (PR / 32);
    const int loc = rg * 32 + lane;
    const ull r = (ull)blockIdx.x * PR + loc;
    const bool valid = r < A.count;
    stage_binom(sbin, A.binom, n);
    __syncthreads();
    const ull D = valid ? colex_unrank(r, k, n, sbin) : 0ULL;
    const ull pbase = A.lbase + r * (ull)k;
    double best = 0.0;
    bool seen = false;
    for (int x = n - 1; x >= 0; --x) {
        if ((x & (PE_G - 1)) != xg) continue;            // uniform per warp
        const bool in = valid && ((D >> x) & 1ULL);
        const int j = __popcll(D & ((1ULL << x) - 1ULL));
        const ll lo = A.offsets[x];
        double wsum = 0.0;
        if (A.wmode == W_SCAN) {
            if (__any_sync(0xffffffffu, in)) {
                for (ll i = lo; i < A.offsets[x + 1]; ++i) {
                    const ull Dp = __ldg(A.menus + i);
                    const double sc = __ldg(scores + i);
                    if (in && (Dp & D) == Dp) wsum = __dadd_rn(wsum, sc);
                }
            }
        } else if (in) {
            const unsigned b = __ldg(A.loffs + pbase + j), e = __ldg(A.loffs + pbase + j + 1);
            if (A.wmode == W_LIST16) {
                const uint16_t *ent = (const uint16_t *)A.lent;
                for (unsigned i = b; i < e; ++i) wsum = __dadd_rn(wsum, __ldg(scores + lo + __ldg(ent + i)));
            } else {
                const uint32_t *ent = (const uint32_t *)A.lent;
                for (unsigned i = b; i < e; ++i) wsum = __dadd_rn(wsum, __ldg(scores + lo + __ldg(ent + i)));
            }
        }
        if (in) {
            const double cand = __dadd_rn(vprev[colex_rank_without(r, D, x, j, n, sbin)], wsum);
            if (!seen || cand > best) { best = cand; seen = true; }
        }
    }
    pbest[xg][loc] = best;
    pok[xg][loc] = seen ? 1 : 0;
    __syncthreads();
    if (xg != 0 || !valid) return;
    double b = 0.0;
    bool any = false;
    for (int g = 0; g < PE_G; ++g) {
        if (!pok[g][loc]) continue;
        if (!any || pbest[g][loc] > b) { b = pbest[g][loc]; any = true; }
    }
    vcur[r] = b;
}

// The same layer for long lists (the top layers, where a subset's lists hold up to all of x's
// rows): one CTA per rank, warp w takes the alternatives x = w, w + NW, ... in D. The warp walks
// pair (D, x)'s list 32 entries at a time (coalesced index loads, 32 score gathers in flight, the
// next chunk loaded while this one is added) and adds the chunk's scores in list order through
// shuffles, so each sum is the same sequence of float32 additions as one thread's loop. The
// candidates then merge in x order with `>` (ties -> lowest x).
template <bool MASK, class IT>
__global__ void __launch_bounds__(1024) layer_wide_kernel(PricerArgs A, float *vals) {
    pdl_grid_sync();                                       // launched by launch_pdl
    __shared__ ull sbin[MASK ? 1 : BIN_MAX];
    __shared__ float cv[MAXN_PR];
    __shared__ ull sD;
    const int n = A.n, k = A.k;
    const ull r = blockIdx.x;
    const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (!MASK) stage_binom(sbin, A.binom, n);
    __syncthreads();
    if (threadIdx.x == 0) sD = MASK ? (ull)(unsigned)A.nodes[r] : colex_unrank(r, k, n, sbin);
    __syncthreads();
    const ull D = sD;
    const ull pbase = A.lbase + r * (ull)k;
    const IT *ent = (const IT *)A.lent;
    for (int x = w; x < n; x += nw) {
        if (!((D >> x) & 1ULL)) continue;                 // uniform per warp
        const int j = __popcll(D & ((1ULL << x) - 1ULL));
        const unsigned b = __ldg(A.loffs + pbase + j), e = __ldg(A.loffs + pbase + j + 1);
        const float *sx = A.scores + A.offsets[x];
        float wsum = 0.0f;
        float v = (b + lane < e) ? __ldg(sx + __ldg(ent + b + lane)) : 0.0f;
        for (unsigned c = b; c < e; c += 32) {
            const unsigned nx = c + 32 + lane;
            const float vn = nx < e ? __ldg(sx + __ldg(ent + nx)) : 0.0f;
            const int m = (e - c) < 32u ? (int)(e - c) : 32;
            for (int u = 0; u < m; ++u) wsum = __fadd_rn(wsum, __shfl_sync(0xffffffffu, v, u));
            v = vn;
        }
        if (lane == 0) {
            const float prev = MASK ? A.vmask[D ^ (1ULL << x)]
                                    : decode_prev(A, colex_rank_without(r, D, x, j, n, sbin));
            cv[x] = __fadd_rn(prev, wsum);
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    float best = 0.0f;
    int bx = -1;
    for (int x = 0; x < n; ++x) {
        if (!((D >> x) & 1ULL)) continue;
        if (bx < 0 || cv[x] > best) { best = cv[x]; bx = x; }
    }
    if (MASK) {
        A.vmask[D] = best;
        A.pmask[D] = (uint8_t)bx;
        return;
    }
    if (A.pred) A.pred[r] = (uint8_t)bx;
    if (A.mode == 1) A.vcur_f[r] = best;
    else vals[r] = best;
}

// Cover-list construction, once per pricer: thread per subset D (mask order, all layers in one
// launch); the warp walks the alternatives in order and scans x's rows for its lanes with x in D
// (broadcast loads). COUNT: offs[pair] = the number of rows; else the rows' local indices are
// written from offs[pair] on (offs then holds the exclusive prefix sums).
template <bool COUNT, class IT>
__global__ void cover_build_kernel(int n, ull nD, const ull *binom, const ull *layer_base, const ull *menus,
                                   const ll *offsets, unsigned *offs, IT *ent) {
    const ull D = blockIdx.x * (ull)blockDim.x + threadIdx.x;
    const bool valid = D < nD && D != 0;
    ull p = 0;
    if (valid) {
        const int k = __popcll(D);
        p = layer_base[k] + colex_rank_dev(D, binom, n) * (ull)k;
    }
    for (int x = 0; x < n; ++x) {
        const bool in = valid && ((D >> x) & 1ULL);
        if (__any_sync(0xffffffffu, in)) {
            const ll lo = offsets[x], hi = offsets[x + 1];
            unsigned c = 0;
            const unsigned o = (!COUNT && in) ? offs[p] : 0u;
            for (ll i = lo; i < hi; ++i) {
                const ull Dp = __ldg(menus + i);
                if (in && (Dp & D) == Dp) {
                    if (!COUNT) ent[o + c] = (IT)(i - lo);
                    ++c;
                }
            }
            if (COUNT && in) offs[p] = c;
        }
        if (in) ++p;
    }
}

// The previous layer's quantized values decoded once to float32 (decode_prev's arithmetic, so the
// same floats), for the group sweep: a rank reads k predecessors, each a value, an offset and a step.
__global__ void stream_decode_kernel(PricerArgs A, ull count_prev, float *dec) {
    pdl_grid_sync();                                       // launched by launch_pdl
    const ull r = blockIdx.x * (ull)blockDim.x + threadIdx.x;
    if (r < count_prev) dec[r] = decode_prev(A, r);
}

__global__ void __launch_bounds__(PB) stream_quant_kernel(PricerArgs A, const float *vals) {
    pdl_grid_sync();                                       // launched by launch_pdl
    __shared__ float smin[PB / 32], smax[PB / 32];
    const ull r = (ull)blockIdx.x * PB + threadIdx.x;
    const bool valid = r < A.count;
    const float best = valid ? vals[r] : 0.0f;
    float tmin = valid ? best : 3.0e38f, tmax = valid ? best : -3.0e38f;
    for (int o = 16; o > 0; o >>= 1) {
        tmin = fminf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
        tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
    }
    if ((threadIdx.x & 31) == 0) { smin[threadIdx.x >> 5] = tmin; smax[threadIdx.x >> 5] = tmax; }
    __syncthreads();
    float bmin = smin[0], bmax = smax[0];
    for (int i = 1; i < PB / 32; ++i) { bmin = fminf(bmin, smin[i]); bmax = fmaxf(bmax, smax[i]); }
    const float levels = A.mode == 2 ? 65535.0f : 16777215.0f;
    float step = __fdiv_rn(__fsub_rn(bmax, bmin), levels);
    if (threadIdx.x == 0) {
        A.mcur[blockIdx.x] = bmin;
        A.ecur[blockIdx.x] = step;
        atomicMax(A.layer_step, __float_as_uint(step));
    }
    if (!valid) return;
    float q = (step > 0.0f) ? rintf(__fdiv_rn(__fsub_rn(best, bmin), step)) : 0.0f;
    q = fminf(fmaxf(q, 0.0f), levels);
    unsigned int qi = (unsigned int)q;
    if (A.mode == 2) {
        A.vcur_h[r] = (uint16_t)qi;
    } else {
        A.vcur_h[r] = (uint16_t)(qi >> 8);
        A.lcur[r] = (uint8_t)(qi & 255u);
    }
}

// Result block written by the device backtrace (one small D2H copy per price call).
struct PriceOut {
    float vtop;            // f32 value at the full set (f32 / mask modes)
    float mtop, etop;      // u16 / u24: offset and step of the top block
    unsigned int qtop;     // u16 / u24: quantized top value
    int rank_pos[MAXN_PR];
    int error;
    int pos;               // descent only: elements placed by the descent
    ull node;              // descent only: the node reached at layer k_pred
};

// Descent through the stored predecessor layers (stream modes), then the mask DP on the
// sub-lattice of the node reached; one CTA. V/pred scratch: 2^K entries (K = k_pred); Ws: the
// 2^K K sub-lattice sums. descend_only: stop after the descent and leave the node and the number
// of placed elements in *out (the larger sub-lattices run as a tile sweep of their own).
__global__ void backtrace_kernel(int n, int k_pred, const ull *binom, uint8_t *const *preds, const ull *menus,
                                 const float *scores, const ll *offsets, float *Vs, uint8_t *Ps, PriceOut *out,
                                 const float *vtop_f, const uint16_t *vtop_h, const uint8_t *ltop, const float *mtop,
                                 const float *etop, int mode, int wmode, const unsigned *loffs, const void *lent,
                                 const ull *layer_base, float *Ws, int descend_only) {
    __shared__ ull sD;
    __shared__ int elems[MAXN_PR];
    __shared__ int spos;
    __shared__ ull sbin[BIN_MAX];
    stage_binom(sbin, binom, n);
    __syncthreads();
    if (threadIdx.x == 0) {
        ull D = (n >= 64) ? ~0ULL : ((1ULL << n) - 1ULL);
        int pos = 0;
        for (int k = n; k > k_pred; --k) {
            ull r = colex_rank_dev(D, sbin, n);
            int x = preds[k][r];
            out->rank_pos[x] = pos++;
            D ^= 1ULL << x;
        }
        int K = 0;
        for (int b = 0; b < n; ++b)
            if ((D >> b) & 1ULL) elems[K++] = b;
        sD = D;
        spos = pos;
        if (mode == 1) out->vtop = vtop_f[0];
        else if (mode >= 2) {
            unsigned int q = vtop_h[0];
            if (mode == 3) q = (q << 8) | ltop[0];
            out->qtop = q;
            out->mtop = mtop[0];
            out->etop = etop[0];
        }
    }
    __syncthreads();
    if (descend_only) {                 // the sub-lattice is solved by the tile sweep
        if (threadIdx.x == 0) {
            out->node = sD;
            out->pos = spos;
            out->error = 0;
        }
        return;
    }
    const ull D = sD;
    const int K = __popcll(D);
    const ull Nsub = 1ULL << K;
    for (ull s = threadIdx.x; s < Nsub; s += blockDim.x) { Vs[s] = 0.0f; Ps[s] = 0; }
    // w(x_j, D(s)) for every sub-lattice node s and member j: independent of the DP, so all of them
    // at once (Ws[s K + j]), then the layers only add and compare
    for (ull t = threadIdx.x; t < Nsub * (ull)K; t += blockDim.x) {
        const ull s = t / (ull)K;
        const int j = (int)(t - s * (ull)K);
        if (!((s >> j) & 1ULL)) continue;
        ull Dorig = 0;
        for (int i = 0; i < K; ++i)
            if ((s >> i) & 1ULL) Dorig |= 1ULL << elems[i];
        const int x = elems[j];
        float w = 0.0f;
        if (wmode == W_SCAN) {
            for (ll i = offsets[x]; i < offsets[x + 1]; ++i) {
                ull Dp = menus[i];
                if ((Dp & Dorig) == Dp) w = __fadd_rn(w, scores[i]);
            }
        } else {
            const int c = __popcll(s);
            const ull p = layer_base[c] + colex_rank_dev(Dorig, sbin, n) * (ull)c +
                          __popcll(Dorig & ((1ULL << x) - 1ULL));
            w = wmode == W_LIST16 ? w_list(loffs, (const uint16_t *)lent, p, scores + offsets[x])
                                  : w_list(loffs, (const uint32_t *)lent, p, scores + offsets[x]);
        }
        Ws[t] = w;
    }
    __syncthreads();
    for (int c = 1; c <= K; ++c) {
        for (ull s = threadIdx.x; s < Nsub; s += blockDim.x) {
            if (__popcll(s) != c) continue;
            float best = 0.0f;
            bool seen = false;
            int bj = 0;
            for (int j = 0; j < K; ++j) {
                if (!((s >> j) & 1ULL)) continue;
                float cand = __fadd_rn(Vs[s ^ (1ULL << j)], Ws[s * (ull)K + j]);
                if (!seen || cand > best) { best = cand; seen = true; bj = j; }
            }
            Vs[s] = best;
            Ps[s] = (uint8_t)bj;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ull Dm = Nsub - 1;
        int pos = spos;
        for (int i = 0; i < K; ++i) {
            int j = Ps[Dm];
            out->rank_pos[elems[j]] = pos + i;
            Dm ^= 1ULL << j;
        }
        if (mode == 0) out->vtop = Vs[Nsub - 1];
        out->error = 0;
    }
}

// Mask mode: the whole lattice is solved; descend pred from the full set.
__global__ void mask_readout_kernel(int n, const float *V, const uint8_t *pred, PriceOut *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ull D = (1ULL << n) - 1ULL;
    out->vtop = V[D];
    for (int i = 0; i < n; ++i) {
        int x = pred[D];
        out->rank_pos[x] = i;
        D ^= 1ULL << x;
    }
    out->error = 0;
}

// Mask storage by tiles. The lattice V[D] (D < 2^n, float32, indexed by the mask) splits into tiles
// of MT_TILE = 256 consecutive masks: tile H holds D = H * 256 + L, L < 256 (alternatives 0..7 are
// the tile's low bits, L = lane + 32 j: bits 0-4 the lane, bits 5-7 the thread's register j). One
// warp computes one tile; one launch covers the tiles whose high part H has popcount t, for
// t = 0 .. n - 8, so every tile H ^ {x} a tile reads was written by the launch before. Per tile:
//   w(x, D) for every x in D: one pass over x's rows for the whole tile. A row whose menu's high
//     part is not a subset of H fails for all 256 masks (a warp-uniform skip); otherwise the lane
//     test (menu bits 0-4 within the lane's) gives the lane's addend (the score or +0, which leaves
//     a sum unchanged: a sum that starts at +0 is never -0) and a warp-uniform switch on the menu's
//     bits 5-7 adds it to the registers j that contain them, in row order;
//   high x in H: V[D \ {x}] is the same L of tile H ^ {x} (coalesced loads), merged at once;
//   low x in L: V[D \ {x}] is a mask of the same tile, so the tile's values and w(x, D) go to
//     shared memory and the low candidates are merged by popcount rounds of L (the masks of
//     popcount q are final once round q ends; a round's masks read only rounds before it).
// Sums add x's qualifying rows in row order, one float32 add at a time (the row scan's and the
// cover lists' sums), and candidates merge with the larger value winning and, on equal values,
// the lower x: V and the predecessor bytes are the layer kernels' bit for bit. The lattice is read
// once per (D, x in D) at 4 bytes over coalesced lines and written once, with no layer table.
// Scores are finite (a +0 addend and a skipped row are then the same).
constexpr int MT_LOW = 8, MT_TILE = 1 << MT_LOW, MT_WARPS = 4, MT_REGS = MT_TILE / 32;
constexpr int MASK_MIN_N_TILE = MT_LOW + 1;
constexpr int MASK_MAX_N = 34;

struct MaskTileArgs {
    int n, h, t;
    ull count;                 // tiles in this launch: C(h, t)
    const ull *binom;          // C(b, k) at b*bstride+k
    int bstride;
    const int4 *rows;          // x-major rows {menu >> 8, menu & 31, score bits, (menu >> 5) & 7}
    const ll *offsets;
    float *V;
    uint8_t *P;
};

// Row records for the tile and group sweeps, rebuilt with each call's scores:
// {menu >> shift, menu & ymask, score bits, (menu >> 5) & 7}; idx (may be NULL) maps record i to the
// row whose score it carries (the restricted rows of a sub-lattice).
__global__ void rows_kernel(ll mp, const ull *menus, const float *scores, const int *idx, int shift, unsigned ymask,
                            int4 *rows) {
    const ll i = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (i >= mp) return;
    const ull m = menus[i];
    const float sc = scores[idx ? (ll)idx[i] : i];
    rows[i] = make_int4((int)(unsigned)(m >> shift), (int)((unsigned)m & ymask), __float_as_int(sc),
                        (int)(unsigned)((m >> 5) & 7ULL));
}

// Row records are read ROW_PF at a time ahead of their use; ROW_NONE pads the last batch (its high
// part has every bit set, so no tile or group takes it: their high parts have at most 29 bits).
constexpr int ROW_PF = 4;
#define ROW_NONE make_int4(-1, 0, 0, 0)

// Row records of the float64 max sweep's group form: {menu >> shift, menu & ymask, score low and
// high words}.
__global__ void rows64_kernel(ll mp, const ull *menus, const double *scores, int shift, unsigned ymask, int4 *rows) {
    const ll i = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (i >= mp) return;
    const ull m = menus[i];
    const double sc = scores[i];
    rows[i] = make_int4((int)(unsigned)(m >> shift), (int)((unsigned)m & ymask), __double2loint(sc), __double2hiint(sc));
}

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

template <class T>
__device__ __forceinline__ void mt_merge(T &v, int &b, T c, int x) {
    if (b < 0 || c > v || (c == v && x < b)) {
        v = c;
        b = x;
    }
}

// acc[j] += s for the registers j that contain mr (j's bits 5-7 of L; mr warp-uniform).
__device__ __forceinline__ void mt_add(float (&acc)[MT_REGS], int mr, float s) {
#define MT_A(j) acc[j] = __fadd_rn(acc[j], s)
    switch (mr) {
        case 0: MT_A(0); MT_A(1); MT_A(2); MT_A(3); MT_A(4); MT_A(5); MT_A(6); MT_A(7); break;
        case 1: MT_A(1); MT_A(3); MT_A(5); MT_A(7); break;
        case 2: MT_A(2); MT_A(3); MT_A(6); MT_A(7); break;
        case 3: MT_A(3); MT_A(7); break;
        case 4: MT_A(4); MT_A(5); MT_A(6); MT_A(7); break;
        case 5: MT_A(5); MT_A(7); break;
        case 6: MT_A(6); MT_A(7); break;
        default: MT_A(7); break;
    }
#undef MT_A
}

// The 256 low masks ordered by popcount (ascending masks within one popcount), and where each
// popcount starts.
struct MtOrder {
    uint8_t order[MT_TILE];
    int qoff[MT_LOW + 2];
};
static MtOrder mt_order_host() {
    MtOrder o{};
    int k = 0;
    for (int q = 0; q <= MT_LOW; ++q) {
        o.qoff[q] = k;
        for (int L = 0; L < MT_TILE; ++L)
            if (__builtin_popcount(L) == q) o.order[k++] = (uint8_t)L;
    }
    o.qoff[MT_LOW + 1] = k;
    return o;
}

// Index of a low mask L that contains x among the 128 that do: L without bit x.
__device__ __forceinline__ int mt_half(int L, int x) { return ((L >> (x + 1)) << x) | (L & ((1 << x) - 1)); }

__global__ void __launch_bounds__(32 * MT_WARPS) mask_tile_kernel(MaskTileArgs A, MtOrder ord) {
    pdl_grid_sync();                                       // launched by launch_pdl
    __shared__ float wl[MT_WARPS][MT_LOW][MT_TILE / 2];   // w(x, D) for low x, at mt_half(L, x) (x in L)
    __shared__ float vt[MT_WARPS][MT_TILE];
    __shared__ uint8_t bt[MT_WARPS][MT_TILE];
    __shared__ unsigned sbin[(MASK_MAX_N - MT_LOW + 1) * (MASK_MAX_N - MT_LOW + 1)];   // C(b, k), b, k <= h
    __shared__ uint8_t sord[MT_TILE];
    const int n = A.n, h = A.h;
    for (int i = threadIdx.x; i < (h + 1) * (h + 1); i += blockDim.x)
        sbin[i] = (unsigned)A.binom[(i / (h + 1)) * A.bstride + i % (h + 1)];
    for (int i = threadIdx.x; i < MT_TILE; i += blockDim.x) sord[i] = ord.order[i];
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const ull tile = (ull)blockIdx.x * MT_WARPS + w;
    if (tile >= A.count) return;                          // whole warps leave
    unsigned H = 0;                                       // colex unranking of the tile in [0, h)
    {
        unsigned r = (unsigned)tile;
        int b = h - 1;
        for (int k = A.t; k >= 1; --k) {
            while (sbin[b * (h + 1) + k] > r) --b;
            H |= 1u << b;
            r -= sbin[b * (h + 1) + k];
            --b;
        }
    }
    const unsigned nH = ~H, nlane = ~(unsigned)lane;
    const ull base = (ull)H << MT_LOW;
    float best[MT_REGS];
    int bx[MT_REGS];
#pragma unroll
    for (int j = 0; j < MT_REGS; ++j) {
        best[j] = 0.0f;
        bx[j] = -1;
    }
    for (int x = 0; x < n; ++x) {
        const bool high = x >= MT_LOW;
        if (high && !((H >> (x - MT_LOW)) & 1u)) continue;      // uniform per warp
        float prev[MT_REGS];
        if (high) {
            const float *pv = A.V + (base ^ (1ULL << x)) + lane;
#pragma unroll
            for (int j = 0; j < MT_REGS; ++j) prev[j] = pv[32 * j];
        }
        float acc[MT_REGS];
#pragma unroll
        for (int j = 0; j < MT_REGS; ++j) acc[j] = 0.0f;
        const int lo = (int)A.offsets[x], hi = (int)A.offsets[x + 1];
        for (int i0 = lo; i0 < hi; i0 += ROW_PF) {
            int4 R[ROW_PF];                                     // loaded ahead: the skips depend on them
#pragma unroll
            for (int u = 0; u < ROW_PF; ++u) R[u] = i0 + u < hi ? __ldg(A.rows + i0 + u) : ROW_NONE;
#pragma unroll
            for (int u = 0; u < ROW_PF; ++u) {
                if ((unsigned)R[u].x & nH) continue;            // uniform: fails for the whole tile
                const float s = ((unsigned)R[u].y & nlane) ? 0.0f : __int_as_float(R[u].z);
                mt_add(acc, R[u].w, s);
            }
        }
        if (high) {
#pragma unroll
            for (int j = 0; j < MT_REGS; ++j) mt_merge(best[j], bx[j], __fadd_rn(prev[j], acc[j]), x);
        } else {
#pragma unroll
            for (int j = 0; j < MT_REGS; ++j) {
                const int L = lane + 32 * j;
                if ((L >> x) & 1) wl[w][x][mt_half(L, x)] = acc[j];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < MT_REGS; ++j) {
        vt[w][lane + 32 * j] = best[j];
        bt[w][lane + 32 * j] = (uint8_t)(bx[j] < 0 ? 255 : bx[j]);
    }
    __syncwarp();
    // low candidates, popcount round by popcount round (the round's masks share their popcount q,
    // so every lane walks q bits)
    for (int q = 1; q <= MT_LOW; ++q) {
        for (int idx = ord.qoff[q] + lane; idx < ord.qoff[q + 1]; idx += 32) {
            const int L = sord[idx];
            float v = vt[w][L];
            int b = bt[w][L] == 255 ? -1 : (int)bt[w][L];
            for (unsigned m = (unsigned)L; m; m &= m - 1u) {
                const int x = __ffs((int)m) - 1;
                mt_merge(v, b, __fadd_rn(vt[w][L ^ (1 << x)], wl[w][x][mt_half(L, x)]), x);
            }
            vt[w][L] = v;
            bt[w][L] = (uint8_t)(b < 0 ? 255 : b);
        }
        __syncwarp();
    }
#pragma unroll
    for (int j = 0; j < MT_REGS; ++j) {
        const int L = lane + 32 * j;
        A.V[base + L] = vt[w][L];
        A.P[base + L] = bt[w][L] == 255 ? (uint8_t)0 : bt[w][L];
    }
}

// The tile sweep's form for launches with few tiles (small n, the first and last popcounts): one
// CTA of MT_SPLIT warps per tile, warp w taking the alternatives x = w (mod MT_SPLIT) through the
// same row pass as mask_tile_kernel, the warps' high candidates merged through shared memory, and
// the low candidates' popcount rounds spread over the CTA's threads. A launch then waits for an
// eighth of a tile's row pass instead of all of it. The candidates, their sums and the merge rule
// are mask_tile_kernel's, so V and the predecessor bytes are the same bits.
constexpr int MT_SPLIT = 8;
__global__ void __launch_bounds__(32 * MT_SPLIT) mask_tile_split_kernel(MaskTileArgs A, MtOrder ord) {
    pdl_grid_sync();                                       // launched by launch_pdl
    __shared__ float wl[MT_LOW][MT_TILE / 2];
    __shared__ float pv[MT_SPLIT][MT_TILE];
    __shared__ signed char pb[MT_SPLIT][MT_TILE];
    __shared__ float vt[MT_TILE];
    __shared__ uint8_t bt[MT_TILE];
    __shared__ unsigned sbin[(MASK_MAX_N - MT_LOW + 1) * (MASK_MAX_N - MT_LOW + 1)];
    __shared__ uint8_t sord[MT_TILE];
    const int n = A.n, h = A.h;
    for (int i = threadIdx.x; i < (h + 1) * (h + 1); i += blockDim.x)
        sbin[i] = (unsigned)A.binom[(i / (h + 1)) * A.bstride + i % (h + 1)];
    for (int i = threadIdx.x; i < MT_TILE; i += blockDim.x) sord[i] = ord.order[i];
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned H = 0;
    {
        unsigned r = (unsigned)blockIdx.x;
        int b = h - 1;
        for (int k = A.t; k >= 1; --k) {
            while (sbin[b * (h + 1) + k] > r) --b;
            H |= 1u << b;
            r -= sbin[b * (h + 1) + k];
            --b;
        }
    }
    const unsigned nH = ~H, nlane = ~(unsigned)lane;
    const ull base = (ull)H << MT_LOW;
    float best[MT_REGS];
    int bx[MT_REGS];
#pragma unroll
    for (int j = 0; j < MT_REGS; ++j) {
        best[j] = 0.0f;
        bx[j] = -1;
    }
    for (int x = w; x < n; x += MT_SPLIT) {
        const bool high = x >= MT_LOW;
        if (high && !((H >> (x - MT_LOW)) & 1u)) continue;      // uniform per warp
        float prev[MT_REGS];
        if (high) {
            const float *pvp = A.V + (base ^ (1ULL << x)) + lane;
#pragma unroll
            for (int j = 0; j < MT_REGS; ++j) prev[j] = pvp[32 * j];
        }
        float acc[MT_REGS];
#pragma unroll
        for (int j = 0; j < MT_REGS; ++j) acc[j] = 0.0f;
        const int lo = (int)A.offsets[x], hi = (int)A.offsets[x + 1];
        for (int i0 = lo; i0 < hi; i0 += ROW_PF) {
            int4 R[ROW_PF];
#pragma unroll
            for (int u = 0; u < ROW_PF; ++u) R[u] = i0 + u < hi ? __ldg(A.rows + i0 + u) : ROW_NONE;
#pragma unroll
            for (int u = 0; u < ROW_PF; ++u) {
                if ((unsigned)R[u].x & nH) continue;
                const float sc = ((unsigned)R[u].y & nlane) ? 0.0f : __int_as_float(R[u].z);
                mt_add(acc, R[u].w, sc);
            }
        }
        if (high) {
#pragma unroll
            for (int j = 0; j < MT_REGS; ++j) mt_merge(best[j], bx[j], __fadd_rn(prev[j], acc[j]), x);
        } else {
#pragma unroll
            for (int j = 0; j < MT_REGS; ++j) {
                const int L = lane + 32 * j;
                if ((L >> x) & 1) wl[x][mt_half(L, x)] = acc[j];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < MT_REGS; ++j) {
        pv[w][lane + 32 * j] = best[j];
        pb[w][lane + 32 * j] = (signed char)bx[j];
    }
    __syncthreads();
    for (int L = threadIdx.x; L < MT_TILE; L += blockDim.x) {     // the warps' high candidates merged
        float v = 0.0f;
        int b = -1;
        for (int q = 0; q < MT_SPLIT; ++q)
            if (pb[q][L] >= 0) mt_merge(v, b, pv[q][L], pb[q][L]);
        vt[L] = v;
        bt[L] = (uint8_t)(b < 0 ? 255 : b);
    }
    __syncthreads();
    for (int q = 1; q <= MT_LOW; ++q) {                         // low candidates, popcount rounds
        for (int idx = ord.qoff[q] + (int)threadIdx.x; idx < ord.qoff[q + 1]; idx += blockDim.x) {
            const int L = sord[idx];
            float v = vt[L];
            int b = bt[L] == 255 ? -1 : (int)bt[L];
            for (unsigned m = (unsigned)L; m; m &= m - 1u) {
                const int x = __ffs((int)m) - 1;
                mt_merge(v, b, __fadd_rn(vt[L ^ (1 << x)], wl[x][mt_half(L, x)]), x);
            }
            vt[L] = v;
            bt[L] = (uint8_t)(b < 0 ? 255 : b);
        }
        __syncthreads();
    }
    for (int L = threadIdx.x; L < MT_TILE; L += blockDim.x) {
        A.V[base + L] = vt[L];
        A.P[base + L] = bt[L] == 255 ? (uint8_t)0 : bt[L];
    }
}

// The sub-lattice ranking after a tile sweep over the K elements left by the descent: positions
// pos .. pos + K - 1 in the order the sub-lattice's predecessors give (element j of the sub-problem
// is alternative elems[j]).
struct SubElems {
    int e[MAXN_PR];
};
__global__ void sub_readout_kernel(int K, const float *V, const uint8_t *pred, SubElems el, int mode, PriceOut *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ull D = (1ULL << K) - 1ULL;
    const int pos = out->pos;
    if (mode == 0) out->vtop = V[D];
    for (int i = 0; i < K; ++i) {
        const int j = pred[D];
        out->rank_pos[el.e[j]] = pos + i;
        D ^= 1ULL << j;
    }
    out->error = 0;
}

// Stream storage by groups (layers whose w(x, D) scans rows). The subsets of layer k whose elements
// >= SG_LOW agree (the high part H, t = |H| elements) and whose low part L has l = k - t elements
// take consecutive colex ranks: with H's elements a_0 < a_1 < ..., rank(L u H) = rank_l(L) +
// base(H, l), base(H, l) = sum_i C(a_i, l + i + 1), rank_l(L) = L's rank among the l-subsets of
// [0, SG_LOW) (ascending masks). One warp computes one group: slot s = lane + 32 j holds the l-subset
// of rank s (C(SG_LOW, l) <= 252 slots). Per group and alternative x in D:
//   x in H: D \ {x} is (L, H \ {x}) in layer k - 1, rank base(H \ {x}, l) + s (coalesced);
//   x in L: D \ {x} is (L \ {x}, H), rank base(H, l - 1) + rank_{l-1}(L \ {x});
//   w(x, D): one pass over x's rows for the group; a row whose menu's high part is not within H
//   fails for every slot (a warp-uniform skip), the others are tested on the low part per slot.
// Values are decoded from the previous layer's storage (in quantized storage once per layer by
// stream_decode_kernel when the float32 copy fits) and candidates merge with the larger value
// winning and, on equal values, the lower x (the row scan's x descending with `>=`): the layer is
// the layer kernels' bit for bit, and stream_quant_kernel quantizes it as before.
constexpr int SG_LOW = 10, SG_REGS = 8, SG_WARPS = 4, SG_PF = 4;   // SG_PF: rows read ahead
constexpr int SG_MIN_N = SG_LOW + 2;

struct StreamGroupArgs {
    int lmin, lmax;
    ull cum[SG_LOW + 2];       // groups before low popcount lmin + i
    int loff[SG_LOW + 2];      // first index of popcount l in the low-mask order
    const int4 *rows;          // {menu >> SG_LOW, menu & (2^SG_LOW - 1), score bits (float: .z, double: .z/.w)}
    const uint16_t *lowtab;    // low masks by (popcount, value); each mask's rank; the 9-bit masks by (popcount, value)
    const double *vprev64;     // the float64 max sweep: previous and current layer
    double *vcur64;
};

// One group's slots, NR registers per lane (NR * 32 >= the group's C(SG_LOW, l) slots).
// T = float: the pricing sweep (values decoded from the previous layer, predecessors, lowest x on
// ties); T = double: the float64 max sweep (previous layer G.vprev64, scores as double bits in the
// row records, only the maximum kept, G.vcur64 out).
template <int NR, int NRC, class T>
__device__ __forceinline__ void sg_group(const PricerArgs &A, const StreamGroupArgs &G, float *vals, const ull *sbin,
                                         const uint16_t *sord, const uint16_t *srk, const uint16_t *sord9,
                                         const int *off9, T *cbuf, int lane, int l, unsigned H, ull base, ull tsum,
                                         int nsl) {
    const int n = A.n;
    auto read_prev = [&](ull rp) -> T {
        if constexpr (sizeof(T) == 8) return G.vprev64[rp];
        else return decode_prev(A, rp);
    };
    unsigned Lj[NR], nLj[NR];
    T best[NR];
    int bx[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        const int sl = lane + 32 * j;
        Lj[j] = sl < nsl ? (unsigned)sord[G.loff[l] + sl] : 0u;
        nLj[j] = ~Lj[j];
        best[j] = (T)0;
        bx[j] = -1;
    }
    const unsigned nH = ~H;
    ull pre = 0, cle = 0;                                 // sums over the elements of H below x
    int ih = 0;
    for (int x = 0; x < n; ++x) {
        const bool high = x >= SG_LOW;
        ull hbase = 0;
        if (high) {
            if (!((H >> (x - SG_LOW)) & 1u)) continue;    // uniform per warp
            const ull c1 = sbin[x * (n + 1) + l + ih + 1], c0 = sbin[x * (n + 1) + l + ih];
            hbase = pre + (tsum - cle - c0);              // base(H \ {x}, l)
            pre += c1;
            cle += c0;
            ++ih;
        }
        if (!high && l == 0) continue;                    // no slot holds a low alternative
        if constexpr (NRC < NR) {
            if (!high) {
                // only the slots that contain x: the (l-1)-subsets of the other 9 low bits, expanded
                // around x (NRC registers instead of NR); each one's candidate goes to its slot
                // through shared memory
                const int c9 = (int)sbin[9 * (n + 1) + (l - 1)];
                unsigned Lc[NRC], nLc[NRC];
                T prevc[NRC], accc[NRC];
#pragma unroll
                for (int jc = 0; jc < NRC; ++jc) {
                    const int cs = lane + 32 * jc;
                    const unsigned m9 = cs < c9 ? (unsigned)sord9[off9[l - 1] + cs] : 0u;
                    Lc[jc] = ((m9 >> x) << (x + 1)) | (1u << x) | (m9 & ((1u << x) - 1u));
                    nLc[jc] = ~Lc[jc];
                    prevc[jc] = cs < c9 ? read_prev(tsum + (ull)srk[Lc[jc] ^ (1u << x)]) : (T)0;
                    accc[jc] = (T)0;
                }
                const int lo = (int)A.offsets[x], hi = (int)A.offsets[x + 1];
                for (int i0 = lo; i0 < hi; i0 += SG_PF) {
                    int4 R[SG_PF];
#pragma unroll
                    for (int u = 0; u < SG_PF; ++u) R[u] = i0 + u < hi ? __ldg(G.rows + i0 + u) : ROW_NONE;
#pragma unroll
                    for (int u = 0; u < SG_PF; ++u) {
                        if ((unsigned)R[u].x & nH) continue;        // uniform: fails for the whole group
                        const unsigned ml = (unsigned)R[u].y;
                        T sc;
                        if constexpr (sizeof(T) == 8) sc = __hiloint2double(R[u].w, R[u].z);
                        else sc = __int_as_float(R[u].z);
#pragma unroll
                        for (int jc = 0; jc < NRC; ++jc)
                            if (!(ml & nLc[jc])) accc[jc] = add_rn(accc[jc], sc);
                    }
                }
#pragma unroll
                for (int jc = 0; jc < NRC; ++jc)
                    if (lane + 32 * jc < c9) cbuf[srk[Lc[jc]]] = add_rn(prevc[jc], accc[jc]);
                __syncwarp();
#pragma unroll
                for (int j = 0; j < NR; ++j) {
                    const int sl = lane + 32 * j;
                    if (sl < nsl && ((Lj[j] >> x) & 1u)) mt_merge(best[j], bx[j], cbuf[sl], x);
                }
                __syncwarp();
                continue;
            }
        }
        T prev[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            const int sl = lane + 32 * j;
            const bool use = sl < nsl && (high || ((Lj[j] >> x) & 1u));
            const ull rp = high ? hbase + (ull)sl : tsum + (ull)srk[Lj[j] ^ (1u << x)];
            prev[j] = use ? read_prev(rp) : (T)0;
        }
        T acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = (T)0;
        const int lo = (int)A.offsets[x], hi = (int)A.offsets[x + 1];
        for (int i0 = lo; i0 < hi; i0 += SG_PF) {
            int4 R[SG_PF];
#pragma unroll
            for (int u = 0; u < SG_PF; ++u) R[u] = i0 + u < hi ? __ldg(G.rows + i0 + u) : ROW_NONE;
#pragma unroll
            for (int u = 0; u < SG_PF; ++u) {
                if ((unsigned)R[u].x & nH) continue;            // uniform: fails for the whole group
                const unsigned ml = (unsigned)R[u].y;
                T sc;
                if constexpr (sizeof(T) == 8) sc = __hiloint2double(R[u].w, R[u].z);
                else sc = __int_as_float(R[u].z);
                if (ml == 0u) {                                 // uniform: a menu within H fits every slot
#pragma unroll
                    for (int j = 0; j < NR; ++j) acc[j] = add_rn(acc[j], sc);
                } else {
#pragma unroll
                    for (int j = 0; j < NR; ++j)
                        if (!(ml & nLj[j])) acc[j] = add_rn(acc[j], sc);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            const int sl = lane + 32 * j;
            if (sl < nsl && (high || ((Lj[j] >> x) & 1u))) mt_merge(best[j], bx[j], add_rn(prev[j], acc[j]), x);
        }
    }
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        const int sl = lane + 32 * j;
        if (sl >= nsl) continue;
        const ull r = base + (ull)sl;
        if constexpr (sizeof(T) == 8) {
            G.vcur64[r] = best[j];
        } else {
            if (A.pred) A.pred[r] = (uint8_t)bx[j];
            if (A.mode == 1) A.vcur_f[r] = best[j];
            else vals[r] = best[j];
        }
    }
}

template <class T>
__global__ void __launch_bounds__(32 * SG_WARPS) stream_group_kernel(PricerArgs A, StreamGroupArgs G, float *vals) {
    pdl_grid_sync();                                       // launched by launch_pdl
    __shared__ ull sbin[BIN_MAX];
    __shared__ uint16_t sord[1 << SG_LOW], srk[1 << SG_LOW], sord9[1 << (SG_LOW - 1)];
    __shared__ int off9[SG_LOW + 1];
    __shared__ T cbuf[SG_WARPS][SG_REGS * 32];
    const int n = A.n, k = A.k, hb = n - SG_LOW;
    stage_binom(sbin, A.binom, n);
    for (int i = threadIdx.x; i < (1 << SG_LOW); i += blockDim.x) {
        sord[i] = G.lowtab[i];
        srk[i] = G.lowtab[(1 << SG_LOW) + i];
    }
    for (int i = threadIdx.x; i < (1 << (SG_LOW - 1)); i += blockDim.x) sord9[i] = G.lowtab[(2 << SG_LOW) + i];
    if (threadIdx.x == 0)
        for (int q = 0, o = 0; q <= SG_LOW; ++q) {
            off9[q] = o;
            o += q <= SG_LOW - 1 ? (int)A.binom[(SG_LOW - 1) * (n + 1) + q] : 0;
        }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const ull g = (ull)blockIdx.x * SG_WARPS + w;
    if (g >= G.cum[G.lmax - G.lmin + 1]) return;          // whole warps leave
    int l = G.lmin;
    while (g >= G.cum[l - G.lmin + 1]) ++l;
    const int t = k - l;
    unsigned H = 0;                                       // colex unranking among the t-subsets of [0, hb)
    {
        ull r = g - G.cum[l - G.lmin];
        int b = hb - 1;
        for (int kk = t; kk >= 1; --kk) {
            while (sbin[b * (n + 1) + kk] > r) --b;
            H |= 1u << b;
            r -= sbin[b * (n + 1) + kk];
            --b;
        }
    }
    ull base = 0, tsum = 0;                               // base(H, l) and base(H, l - 1)
    {
        int i = 0;
        for (unsigned m = H; m; m &= m - 1u, ++i) {
            const int a = SG_LOW + __ffs((int)m) - 1;
            base += sbin[a * (n + 1) + l + i + 1];
            tsum += sbin[a * (n + 1) + l + i];
        }
    }
    // registers per lane for all slots (C(SG_LOW, l)) and for the slots holding one low alternative
    // (C(SG_LOW - 1, l - 1)); the compact pass runs where it needs fewer
    const int nsl = (int)sbin[SG_LOW * (n + 1) + l];
    const int nc = l >= 1 ? (int)sbin[(SG_LOW - 1) * (n + 1) + (l - 1)] : 0;
    const int rc = (nc + 31) / 32;
    T *cb = cbuf[w];
#define SG_CALL(NR, NRC) sg_group<NR, NRC, T>(A, G, vals, sbin, sord, srk, sord9, off9, cb, lane, l, H, base, tsum, nsl)
    if (nsl <= 32) SG_CALL(1, 1);
    else if (nsl <= 64) { if (rc <= 1) SG_CALL(2, 1); else SG_CALL(2, 2); }
    else if (nsl <= 128) { if (rc <= 2) SG_CALL(4, 2); else if (rc == 3) SG_CALL(4, 3); else SG_CALL(4, 4); }
    else { if (rc <= 3) SG_CALL(SG_REGS, 3); else SG_CALL(SG_REGS, 4); }
#undef SG_CALL
}

// ----------------------------------------------------------------- host object
struct Pricer {
    Ctx *c = nullptr;
    int n = 0, mode = 0, k_pred = 0, fma_decode = 1;
    ll mp = 0;
    std::vector<ull> counts;
    DevBuf menus, scores, offsets, binom;
    DevBuf v[2], l[2], m[2], e[2];          // stream layers
    std::vector<std::unique_ptr<DevBuf>> pred;   // per layer >= k_pred
    DevBuf pred_ptrs;                       // device array of pred pointers (n+1)
    DevBuf layer_step;                      // n+1 uints (float bits)
    DevBuf Vs, Ps;                          // sub-lattice / mask scratch
    DevBuf Ws;                              // sub-lattice sums w(x_j, D(s)): 2^k_pred * k_pred floats
    DevBuf vals;                            // a layer's float32 values before quantization
    DevBuf dec;                             // the group sweep's decoded previous layer (quantized storage)
    DevBuf out;                             // PriceOut
    std::vector<ll> host_offsets;
    // cover lists (wmode != W_SCAN)
    int wmode = W_SCAN;
    ull list_entries = 0;
    size_t list_bytes = 0;
    std::vector<ull> lbase;                 // first pair index per layer (n+2)
    DevBuf lbase_dev, loffs, lent;
    std::vector<char> wide;                 // per layer: layer_wide_kernel (1) or layer_eval_kernel (0)
    DevBuf d64[2], s64;                     // the float64 max sweep's two layers and scores (on first use)
    DevBuf rows64;                          // its group form's row records
    // mask storage: the tile sweep (mask_tile_kernel) or the layer kernels over the layer table
    bool by_mask = false;                   // the lattice is stored by mask (mask storage, or float32 routed)
    bool mask_tile = false;
    DevBuf rows;                            // row records of the tile and group sweeps (int4 per row)
    // stream storage: the group sweep (stream_group_kernel) or the layer kernels
    bool stream_group = false;
    DevBuf lowtab;                          // the group sweep's low-mask order and ranks (uint16)
    // sub-lattices solved by the tile sweep (k_pred >= SUB_TILE_MIN)
    std::vector<ull> host_menus;
    DevBuf sub_menus, sub_idx, sub_offsets, sub_rows;
};

// The sub-lattice left by the descent is solved by the tile sweep from this many elements on (one
// CTA below it).
constexpr int SUB_TILE_MIN = 12;

// Mean cover-list length from which a layer runs layer_wide_kernel (measured at n = 18: a mean of
// 82 entries takes 68 us with a thread per pair and 13 us with a warp per pair; 41 entries, 41 and
// 49 us).
constexpr double WIDE_MIN_LIST = 64.0;

static std::vector<ull> binom_host(int n) {
    std::vector<ull> t((size_t)(n + 1) * (n + 1), 0);
    for (int b = 0; b <= n; ++b) {
        t[b * (n + 1)] = 1;
        for (int k = 1; k <= b; ++k)
            t[b * (n + 1) + k] = t[(b - 1) * (n + 1) + k - 1] + (k <= b - 1 ? t[(b - 1) * (n + 1) + k] : 0);
    }
    return t;
}

// Builds the cover lists when they fit: n <= 26, fewer than 2^32 entries and at most a quarter of
// the device's free memory; otherwise the sweeps scan x's rows.
static void build_cover_lists(Pricer &P, const uint64_t *menus_host) {
    const int n = P.n;
    if (P.mp == 0 || n > 26) return;
    const ull pairs = (ull)n << (n - 1);
    // a row of menu m qualifies for the 2^(n - |m|) subsets containing m (exact in a double)
    double entries = 0.0;
    for (ll i = 0; i < P.mp; ++i) entries += std::ldexp(1.0, n - __builtin_popcountll(menus_host[i]));
    ll maxrows = 0;
    for (int x = 0; x < n; ++x) maxrows = std::max(maxrows, P.host_offsets[x + 1] - P.host_offsets[x]);
    const bool idx16 = maxrows <= 65536;
    const double bytes = (double)(pairs + 1) * 4.0 + entries * (idx16 ? 2.0 : 4.0);
    size_t free_b = 0, total_b = 0;
    RUMB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (entries >= 4294967295.0 - 64.0 || bytes > 0.25 * (double)free_b) return;
    cudaStream_t st = P.c->own;
    std::vector<ull> bt = binom_host(n);
    P.lbase.assign(n + 2, 0);
    for (int k = 0; k <= n; ++k) P.lbase[k + 1] = P.lbase[k] + bt[n * (n + 1) + k] * (ull)k;
    P.lbase_dev.ensure((size_t)(n + 2) * 8);
    RUMB_CUDA(cudaMemcpyAsync(P.lbase_dev.ptr, P.lbase.data(), (size_t)(n + 2) * 8, cudaMemcpyHostToDevice, st));
    P.loffs.ensure((size_t)(pairs + 1) * 4);
    RUMB_CUDA(cudaMemsetAsync(P.loffs.ptr, 0, (size_t)(pairs + 1) * 4, st));
    const ull nD = 1ULL << n;
    unsigned *offs = P.loffs.as<unsigned>();
    cover_build_kernel<true, uint32_t><<<grid_for((ll)nD, 256), 256, 0, st>>>(
        n, nD, P.binom.as<ull>(), P.lbase_dev.as<ull>(), P.menus.as<ull>(), P.offsets.as<ll>(), offs, nullptr);
    RUMB_LAUNCH("cover_build_kernel<count>");
    size_t tmp_bytes = 0;
    RUMB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, offs, offs, (ll)(pairs + 1), st));
    DevBuf tmp;
    tmp.ensure(std::max<size_t>(tmp_bytes, 16));
    RUMB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tmp_bytes, offs, offs, (ll)(pairs + 1), st));
    unsigned total = 0;
    RUMB_CUDA(cudaMemcpyAsync(&total, offs + pairs, 4, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    if ((double)total != entries) fail(RUMB_E_INTERNAL, "cover lists: entry count does not match the menus");
    P.lent.ensure((size_t)total * (idx16 ? 2 : 4) + 16);
    if (idx16)
        cover_build_kernel<false, uint16_t><<<grid_for((ll)nD, 256), 256, 0, st>>>(
            n, nD, P.binom.as<ull>(), P.lbase_dev.as<ull>(), P.menus.as<ull>(), P.offsets.as<ll>(), offs,
            P.lent.as<uint16_t>());
    else
        cover_build_kernel<false, uint32_t><<<grid_for((ll)nD, 256), 256, 0, st>>>(
            n, nD, P.binom.as<ull>(), P.lbase_dev.as<ull>(), P.menus.as<ull>(), P.offsets.as<ll>(), offs,
            P.lent.as<uint32_t>());
    RUMB_LAUNCH("cover_build_kernel<fill>");
    RUMB_CUDA(cudaStreamSynchronize(st));
    P.wmode = idx16 ? W_LIST16 : W_LIST32;
    P.list_entries = total;
    P.list_bytes = (size_t)bytes;
    // each layer's kernel from its mean list length (both kernels give the same bits): one thread per
    // pair while lists are short, a warp per pair from WIDE_MIN_LIST entries on
    std::vector<unsigned> at(n + 2, 0);
    for (int k = 1; k <= n + 1; ++k)
        RUMB_CUDA(cudaMemcpy(&at[k], offs + P.lbase[k], 4, cudaMemcpyDeviceToHost));
    for (int k = 1; k <= n; ++k) {
        const double pairs_k = (double)(P.lbase[k + 1] - P.lbase[k]);
        P.wide[k] = pairs_k > 0 && (double)(at[k + 1] - at[k]) >= WIDE_MIN_LIST * pairs_k ? 1 : 0;
    }
}

static void run_sweep(Pricer *P, const float *scores);

// One tile sweep over an n-element lattice whose x-major rows are menus[0..mp) (offsets[n+1] on the
// device, idx: each record's score index or NULL), into V and pred (2^n entries each).
static void tile_sweep(cudaStream_t st, int n, ll mp, const ull *menus, const float *scores, const int *idx,
                       const ll *offsets, const ull *binom, int bstride, int4 *rows, float *V, uint8_t *pred) {
    static const MtOrder order = mt_order_host();
    if (mp) {
        rows_kernel<<<grid_for(mp, 256), 256, 0, st>>>(mp, menus, scores, idx, MT_LOW, 31u, rows);
        RUMB_LAUNCH("rows_kernel");
    }
    const int h = n - MT_LOW;
    std::vector<ull> bt = binom_host(h);
    int dev = 0;
    RUMB_CUDA(cudaGetDevice(&dev));
    const ull split_below = (ull)num_sms(dev) * 16;
    for (int t = 0; t <= h; ++t) {
        MaskTileArgs A{};
        A.n = n;
        A.h = h;
        A.t = t;
        A.count = bt[h * (h + 1) + t];
        A.binom = binom;
        A.bstride = bstride;
        A.rows = rows;
        A.offsets = offsets;
        A.V = V;
        A.P = pred;
        if (A.count < split_below) {                    // too few tiles to fill the GPU: split each tile
            launch_pdl(mask_tile_split_kernel, dim3((unsigned)A.count), dim3(32 * MT_SPLIT), 0, st, A, order);
            RUMB_LAUNCH("mask_tile_split_kernel");
        } else {
            launch_pdl(mask_tile_kernel, dim3((unsigned)((A.count + MT_WARPS - 1) / MT_WARPS)), dim3(32 * MT_WARPS), 0, st, A, order);
            RUMB_LAUNCH("mask_tile_kernel");
        }
    }
}

// After a descend-only backtrace: the rows of the K elements left whose menus lie within the node
// (in their order, relabelled to the node's elements, as the reference's sub-problem builds them),
// solved by a tile sweep, and the ranking completed from its predecessors.
static void sublattice_tile(Pricer &P, const float *scores) {
    cudaStream_t st = P.c->own;
    PriceOut h;
    RUMB_CUDA(cudaMemcpyAsync(&h, P.out.ptr, sizeof(PriceOut), cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    const ull node = h.node;
    SubElems el{};
    int K = 0;
    for (int b = 0; b < P.n; ++b)
        if ((node >> b) & 1ULL) el.e[K++] = b;
    std::vector<ull> sm;
    std::vector<int> si;
    std::vector<ll> so(K + 1, 0);
    for (int j = 0; j < K; ++j) {
        const int x = el.e[j];
        for (ll i = P.host_offsets[x]; i < P.host_offsets[x + 1]; ++i) {
            const ull m = P.host_menus[i];
            if (m & ~node) continue;
            ull c = 0;
            for (int q = 0; q < K; ++q) c |= ((m >> el.e[q]) & 1ULL) << q;
            sm.push_back(c);
            si.push_back((int)i);
        }
        so[j + 1] = (ll)sm.size();
    }
    const ll smp = (ll)sm.size();
    P.sub_menus.ensure((size_t)std::max<ll>(smp, 1) * 8);
    P.sub_idx.ensure((size_t)std::max<ll>(smp, 1) * 4);
    P.sub_offsets.ensure((size_t)(K + 1) * 8);
    P.sub_rows.ensure((size_t)std::max<ll>(smp, 1) * sizeof(int4));
    if (smp) {
        RUMB_CUDA(cudaMemcpyAsync(P.sub_menus.ptr, sm.data(), (size_t)smp * 8, cudaMemcpyHostToDevice, st));
        RUMB_CUDA(cudaMemcpyAsync(P.sub_idx.ptr, si.data(), (size_t)smp * 4, cudaMemcpyHostToDevice, st));
    }
    RUMB_CUDA(cudaMemcpyAsync(P.sub_offsets.ptr, so.data(), (size_t)(K + 1) * 8, cudaMemcpyHostToDevice, st));
    tile_sweep(st, K, smp, P.sub_menus.as<ull>(), scores, P.sub_idx.as<int>(), P.sub_offsets.as<ll>(),
               P.binom.as<ull>(), P.n + 1, P.sub_rows.as<int4>(), P.Vs.as<float>(), P.Ps.as<uint8_t>());
    sub_readout_kernel<<<1, 32, 0, st>>>(K, P.Vs.as<float>(), P.Ps.as<uint8_t>(), el, P.mode, P.out.as<PriceOut>());
    RUMB_LAUNCH("sub_readout_kernel");
    // the sub-problem's buffers go back to the stream before the host vectors above are freed
    RUMB_CUDA(cudaStreamSynchronize(st));
}

// Times one sweep in each of two forms (the form flag set by `set`) and keeps the faster; both give
// the same bits.
template <class F>
static bool faster_second(Pricer &P, F set) {
    cudaStream_t st = P.c->own;
    if (P.mp) RUMB_CUDA(cudaMemsetAsync(P.scores.ptr, 0, (size_t)P.mp * 4, st));
    cudaEvent_t e[2];
    for (auto &ev : e) RUMB_CUDA(cudaEventCreate(&ev));
    float ms[2] = {0.0f, 0.0f};
    for (int f = 0; f < 2; ++f) {
        set(f == 1);
        run_sweep(&P, P.scores.as<float>());                 // warm (the layer table is built once)
        RUMB_CUDA(cudaEventRecord(e[0], st));
        run_sweep(&P, P.scores.as<float>());
        RUMB_CUDA(cudaEventRecord(e[1], st));
        RUMB_CUDA(cudaEventSynchronize(e[1]));
        RUMB_CUDA(cudaEventElapsedTime(&ms[f], e[0], e[1]));
    }
    for (auto &ev : e) cudaEventDestroy(ev);
    return ms[1] <= ms[0];
}

// Up to this n a pricer times one sweep of each form at creation and keeps the faster (a layer-kernel
// sweep is cheap there; the tile and group forms lose where a layer has few tiles or groups and every
// alternative many rows); above it the tile / group forms are taken (the layer kernels scan every
// row of every alternative per rank and the cover lists are not built).
constexpr int TIMED_FORMS_MAX_N = 26;

// Mask storage: the tile sweep from n = 9 on (the layer kernels below that, and above n = 30 the
// layer table would not fit). Up to TIMED_FORMS_MAX_N one sweep of each on zero scores picks the
// faster (both give the same bits); above it the tile sweep is taken. RUMB_MASK_FORM = "tile" or
// "layer" pins the form where it can run.
static void choose_mask_form(Pricer &P) {
    const int n = P.n;
    const bool tile_ok = n >= MASK_MIN_N_TILE, layer_ok = n <= 30;
    if (tile_ok) P.rows.ensure((size_t)std::max<ll>(P.mp, 1) * sizeof(int4));
    const char *env = getenv("RUMB_MASK_FORM");
    if (env && std::strcmp(env, "tile") == 0 && tile_ok) { P.mask_tile = true; return; }
    if (env && std::strcmp(env, "layer") == 0 && layer_ok) { P.mask_tile = false; return; }
    if (!tile_ok || !layer_ok) { P.mask_tile = tile_ok; return; }
    if (n > TIMED_FORMS_MAX_N) { P.mask_tile = true; return; }
    P.mask_tile = faster_second(P, [&](bool second) { P.mask_tile = second; });
}

// The group sweep's low-mask table: the 2^SG_LOW masks by (popcount, value), then each mask's rank
// among those of its popcount (once per pricer).
static void ensure_lowtab(Pricer &P) {
    if (P.lowtab.ptr) return;
    std::vector<uint16_t> tab((2 << SG_LOW) + (1 << (SG_LOW - 1)));
    int k = 0;
    std::vector<int> rk(SG_LOW + 1, 0);
    for (int q = 0; q <= SG_LOW; ++q)
        for (int L = 0; L < (1 << SG_LOW); ++L)
            if (__builtin_popcount(L) == q) {
                tab[k++] = (uint16_t)L;
                tab[(1 << SG_LOW) + L] = (uint16_t)rk[q]++;
            }
    k = 2 << SG_LOW;                                      // then the (SG_LOW - 1)-bit masks by (popcount, value)
    for (int q = 0; q < SG_LOW; ++q)
        for (int L = 0; L < (1 << (SG_LOW - 1)); ++L)
            if (__builtin_popcount(L) == q) tab[k++] = (uint16_t)L;
    P.lowtab.ensure(tab.size() * 2);
    RUMB_CUDA(cudaMemcpy(P.lowtab.ptr, tab.data(), tab.size() * 2, cudaMemcpyHostToDevice));
}

// Stream storage: the group sweep from n = 12 on. Up to TIMED_FORMS_MAX_N one sweep of each form on
// zero scores picks the faster; above it the group sweep is taken. RUMB_STREAM_FORM = "group" or
// "layer" pins the form where it can run.
static void choose_stream_form(Pricer &P) {
    const int n = P.n;
    const bool group_ok = n >= SG_MIN_N;
    if (group_ok) {
        P.rows.ensure((size_t)std::max<ll>(P.mp, 1) * sizeof(int4));
        ensure_lowtab(P);
    }
    const char *env = getenv("RUMB_STREAM_FORM");
    if (env && std::strcmp(env, "layer") == 0) { P.stream_group = false; return; }
    if (!group_ok) { P.stream_group = false; return; }
    // quantized storage: each layer decoded once for the group sweep while it fits a quarter of the
    // free memory (one float32 per rank of the largest layer)
    if (P.mode >= 2) {
        ull cap = 0;
        for (ull v : P.counts) cap = v > cap ? v : cap;
        size_t free_b = 0, total_b = 0;
        RUMB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        if ((double)cap * 4.0 <= 0.25 * (double)free_b) P.dec.ensure((size_t)cap * 4);
    }
    if (n > TIMED_FORMS_MAX_N || (env && std::strcmp(env, "group") == 0)) P.stream_group = true;
    else P.stream_group = faster_second(P, [&](bool second) { P.stream_group = second; });
    if (!P.stream_group) P.dec.release();
}

// Float32 storage keeps the same float32 value for every subset whether it is stored by colex rank
// (two live layers) or by mask, and the readout from the full set walks the same predecessors as
// the layer descent and sub-lattice DP, so the priced value and ranking are the same bits. The
// float32 pricer therefore stores the lattice by mask and runs the tile sweep when 5 * 2^n bytes
// are at most half the free device memory (n <= 34), unless RUMB_PRICE_STREAM asks for the
// two-layer storage.
static bool f32_by_mask(int n, size_t free_b) {
    return n >= MASK_MIN_N_TILE && n <= MASK_MAX_N && std::ldexp(5.0, n) <= 0.5 * (double)free_b;
}

Pricer *pricer_create(Ctx &c, int n, ll mp, const uint64_t *menus, const int64_t *offsets, int mode, int k_pred,
                      int fma_decode) {
    const bool scan = (mode & RUMB_PRICE_SCAN) != 0, keep_stream = (mode & RUMB_PRICE_STREAM) != 0;
    mode &= ~(RUMB_PRICE_SCAN | RUMB_PRICE_STREAM);
    if (mode < 0 || mode > 3) fail(RUMB_E_INVAL, "pricer mode must be 0 (mask), 1 (f32), 2 (u16) or 3 (u24)");
    if (n < 1 || n > 39) fail(RUMB_E_INVAL, "pricing handles 1 <= n <= 39");
    if (mode == 0 && n > MASK_MAX_N) fail(RUMB_E_INVAL, "mask pricing handles n <= 34");
    if (mp < 0 || (mp > 0 && !menus) || !offsets) fail(RUMB_E_INVAL, "menus / offsets must not be NULL");
    std::vector<ll> off(offsets, offsets + n + 1);
    if (off[0] != 0 || off[n] != mp) fail(RUMB_E_INVAL, "offsets must run from 0 to mp");
    for (int x = 0; x < n; ++x) {
        if (off[x + 1] < off[x]) fail(RUMB_E_INVAL, "offsets must be nondecreasing");
        for (ll i = off[x]; i < off[x + 1]; ++i)
            if (!((menus[i] >> x) & 1ULL) || (n < 64 && (menus[i] >> n) != 0))
                fail(RUMB_E_INVAL, "row's menu does not contain its alternative or exceeds n");
    }
    std::unique_ptr<Pricer> P(new Pricer());
    P->c = &c;
    P->n = n;
    P->mp = mp;
    P->mode = mode;
    P->fma_decode = fma_decode ? 1 : 0;
    int kp = k_pred > 0 ? k_pred : n - 10;
    P->k_pred = kp < 1 ? 1 : (kp > n ? n : kp);
    P->host_offsets = off;
    std::vector<ull> bt = binom_host(n);
    for (int k = 0; k <= n; ++k) P->counts.push_back(bt[n * (n + 1) + k]);
    cudaStream_t st = c.own;
    P->menus.ensure((size_t)std::max<ll>(mp, 1) * 8);
    P->scores.ensure((size_t)std::max<ll>(mp, 1) * 4);
    P->offsets.ensure((size_t)(n + 1) * 8);
    P->binom.ensure(bt.size() * 8);
    if (mp) RUMB_CUDA(cudaMemcpyAsync(P->menus.ptr, menus, (size_t)mp * 8, cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(P->offsets.ptr, off.data(), (size_t)(n + 1) * 8, cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(P->binom.ptr, bt.data(), bt.size() * 8, cudaMemcpyHostToDevice, st));
    P->out.ensure(sizeof(PriceOut));
    P->layer_step.ensure((size_t)(n + 1) * 4);
    size_t free_b = 0, total_b = 0;
    RUMB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    P->by_mask = mode == 0 || (mode == 1 && !keep_stream && f32_by_mask(n, free_b));
    if (P->by_mask) {
        ull N = 1ULL << n;
        if ((double)N * 5.0 > 0.9 * (double)free_b)
            fail(RUMB_E_OOM, "mask pricing needs 5 * 2^n bytes of device memory");
        P->Vs.ensure((size_t)N * 4);
        P->Ps.ensure((size_t)N);
    } else {
        if (P->k_pred > MASK_MAX_N) fail(RUMB_E_INVAL, "k_pred must be <= 34");
        ull cap = 0;
        for (ull v : P->counts) cap = v > cap ? v : cap;
        ull nblk = (cap + PB - 1) / PB;
        P->vals.ensure((size_t)cap * 4);
        for (int i = 0; i < 2; ++i) {
            P->v[i].ensure((size_t)cap * (mode == 1 ? 4 : 2));
            if (mode == 3) P->l[i].ensure((size_t)cap);
            P->m[i].ensure((size_t)nblk * 4);
            P->e[i].ensure((size_t)nblk * 4);
        }
        std::vector<uint8_t *> ptrs(n + 1, nullptr);
        P->pred.resize(n + 1);
        for (int k = P->k_pred; k <= n; ++k) {
            P->pred[k].reset(new DevBuf());
            P->pred[k]->ensure((size_t)P->counts[k]);
            ptrs[k] = P->pred[k]->as<uint8_t>();
        }
        P->pred_ptrs.ensure((size_t)(n + 1) * sizeof(void *));
        RUMB_CUDA(cudaMemcpyAsync(P->pred_ptrs.ptr, ptrs.data(), (size_t)(n + 1) * sizeof(void *),
                                  cudaMemcpyHostToDevice, st));
        ull Nsub = 1ULL << P->k_pred;
        P->Vs.ensure((size_t)Nsub * 4);
        P->Ps.ensure((size_t)Nsub);
        if (P->k_pred < SUB_TILE_MIN) P->Ws.ensure((size_t)Nsub * P->k_pred * 4);
        else P->host_menus.assign(menus, menus + mp);
    }
    RUMB_CUDA(cudaStreamSynchronize(st));
    P->wide.assign(n + 1, 0);
    if (!scan) build_cover_lists(*P, menus);
    if (P->by_mask) choose_mask_form(*P);
    else choose_stream_form(*P);
    return P.release();
}

void pricer_max64(Pricer *P, const double *scores_host, double *vmax) {
    Ctx &c = *P->c;
    cudaStream_t st = c.own;
    const int n = P->n;
    ull cap = 0;
    for (ull v : P->counts) cap = v > cap ? v : cap;
    P->s64.ensure((size_t)std::max<ll>(P->mp, 1) * 8);
    for (int i = 0; i < 2; ++i) P->d64[i].ensure((size_t)cap * 8);
    if (P->mp) RUMB_CUDA(cudaMemcpyAsync(P->s64.ptr, scores_host, (size_t)P->mp * 8, cudaMemcpyHostToDevice, st));
    // the group form (rows scanned per group of ranks) above TIMED_FORMS_MAX_N where no cover lists
    // were built, or where RUMB_STREAM_FORM = "group" asks for it
    const char *env = getenv("RUMB_STREAM_FORM");
    const bool group = n >= SG_MIN_N && !(env && std::strcmp(env, "layer") == 0) &&
                       ((P->wmode == W_SCAN && n > TIMED_FORMS_MAX_N) || (env && std::strcmp(env, "group") == 0));
    std::vector<ull> bh, b10;
    if (group) {
        ensure_lowtab(*P);
        P->rows64.ensure((size_t)std::max<ll>(P->mp, 1) * sizeof(int4));
        if (P->mp) {
            rows64_kernel<<<grid_for(P->mp, 256), 256, 0, st>>>(P->mp, P->menus.as<ull>(), P->s64.as<double>(), SG_LOW,
                                                               (1u << SG_LOW) - 1u, P->rows64.as<int4>());
            RUMB_LAUNCH("rows64_kernel");
        }
        bh = binom_host(n - SG_LOW);
        b10 = binom_host(SG_LOW);
    }
    int cur = 0, prev = 1;
    RUMB_CUDA(cudaMemsetAsync(P->d64[prev].ptr, 0, 8, st));     // layer 0: V[empty set] = 0
    for (int k = 1; k <= n; ++k) {
        PricerArgs A{};
        A.n = n;
        A.k = k;
        A.count = P->counts[k];
        A.binom = P->binom.as<ull>();
        A.menus = P->menus.as<ull>();
        A.offsets = P->offsets.as<ll>();
        A.wmode = P->wmode;
        A.loffs = P->loffs.as<unsigned>();
        A.lent = P->lent.ptr;
        A.lbase = P->wmode == W_SCAN ? 0 : P->lbase[k];
        const double *vp = P->d64[prev].as<double>();
        double *vc = P->d64[cur].as<double>();
        if (group) {
            const int hb = n - SG_LOW;
            StreamGroupArgs G{};
            G.lmin = std::max(0, k - hb);
            G.lmax = std::min(SG_LOW, k);
            for (int l = G.lmin; l <= G.lmax; ++l) G.cum[l - G.lmin + 1] = G.cum[l - G.lmin] + bh[hb * (hb + 1) + (k - l)];
            for (int l = 0, o = 0; l <= SG_LOW; ++l) {
                G.loff[l] = o;
                o += (int)b10[SG_LOW * (SG_LOW + 1) + l];
            }
            G.rows = P->rows64.as<int4>();
            G.lowtab = P->lowtab.as<uint16_t>();
            G.vprev64 = vp;
            G.vcur64 = vc;
            const ull groups = G.cum[G.lmax - G.lmin + 1];
            launch_pdl(stream_group_kernel<double>, dim3((unsigned)((groups + SG_WARPS - 1) / SG_WARPS)), dim3(32 * SG_WARPS), 0, st, A, G, nullptr);
            RUMB_LAUNCH("stream_group_kernel<f64>");
        } else if ((long long)A.count < 2LL * num_sms(c.device) * PE_R) {
            launch_pdl(max64_layer_kernel<PE_R_SMALL>, dim3((unsigned)((A.count + PE_R_SMALL - 1) / PE_R_SMALL)), dim3(PE_R_SMALL * PE_G), 0, st, A, P->s64.as<double>(), vp, vc);
        } else {
            launch_pdl(max64_layer_kernel<PE_R>, dim3((unsigned)((A.count + PE_R - 1) / PE_R)), dim3(PE_R * PE_G), 0, st, A, P->s64.as<double>(), vp, vc);
        }
        RUMB_LAUNCH("max64_layer_kernel");
        std::swap(cur, prev);
    }
    RUMB_CUDA(cudaMemcpyAsync(vmax, P->d64[prev].ptr, 8, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
}

void pricer_info(const Pricer *P, long long *list_entries, long long *list_bytes) {
    if (list_entries) *list_entries = P->wmode == W_SCAN ? -1 : (long long)P->list_entries;
    if (list_bytes) *list_bytes = P->wmode == W_SCAN ? 0 : (long long)P->list_bytes;
}

void pricer_destroy(Pricer *P) { delete P; }

int pricer_device(const Pricer *P) { return P->c->device; }
Ctx &pricer_ctx(const Pricer *P) { return *P->c; }
int pricer_n(const Pricer *P) { return P->n; }
ll pricer_rows(const Pricer *P) { return P->mp; }
const ull *pricer_menus(const Pricer *P) { return P->menus.as<ull>(); }

// One sweep over the lattice on the context's stream, ending with the backtrace (stream storage)
// or the readout (mask storage) into P->out.
static void run_sweep(Pricer *P, const float *scores) {
    Ctx &c = *P->c;
    cudaStream_t st = c.own;
    const int n = P->n;
    const ull *menus = P->menus.as<ull>();
    const ll *offs = P->offsets.as<ll>();
    auto layer = [&](PricerArgs &A, bool mask, float *vals) {
        auto thread_kernel = [&]() {
            if ((long long)A.count < 2LL * num_sms(c.device) * PE_R) {
                constexpr int PR = PE_R_SMALL;
                const unsigned grid = (unsigned)((A.count + PR - 1) / PR);
                if (mask) launch_pdl(layer_eval_kernel<true, PR>, dim3(grid), dim3(PR * PE_G), 0, st, A, vals);
                else launch_pdl(layer_eval_kernel<false, PR>, dim3(grid), dim3(PR * PE_G), 0, st, A, vals);
            } else {
                const unsigned grid = (unsigned)((A.count + PE_R - 1) / PE_R);
                if (mask) launch_pdl(layer_eval_kernel<true, PE_R>, dim3(grid), dim3(PE_R * PE_G), 0, st, A, vals);
                else launch_pdl(layer_eval_kernel<false, PE_R>, dim3(grid), dim3(PE_R * PE_G), 0, st, A, vals);
            }
            RUMB_LAUNCH("layer_eval_kernel");
        };
        auto wide_kernel = [&]() {
            const unsigned threads = 32u * (unsigned)std::min(n, 32), grid = (unsigned)A.count;
            if (mask && P->wmode == W_LIST16) launch_pdl(layer_wide_kernel<true, uint16_t>, dim3(grid), dim3(threads), 0, st, A, vals);
            else if (mask) launch_pdl(layer_wide_kernel<true, uint32_t>, dim3(grid), dim3(threads), 0, st, A, vals);
            else if (P->wmode == W_LIST16) launch_pdl(layer_wide_kernel<false, uint16_t>, dim3(grid), dim3(threads), 0, st, A, vals);
            else launch_pdl(layer_wide_kernel<false, uint32_t>, dim3(grid), dim3(threads), 0, st, A, vals);
            RUMB_LAUNCH("layer_wide_kernel");
        };
        if (P->wmode != W_SCAN && P->wide[A.k]) wide_kernel();
        else thread_kernel();
    };
    RUMB_CUDA(cudaMemsetAsync(P->layer_step.ptr, 0, (size_t)(n + 1) * 4, st));
    auto args = [&](int k) {
        PricerArgs A{};
        A.n = n;
        A.k = k;
        A.count = P->counts[k];
        A.binom = P->binom.as<ull>();
        A.menus = menus;
        A.scores = scores;
        A.offsets = offs;
        A.mode = P->mode;
        A.fma_decode = P->fma_decode;
        A.wmode = P->wmode;
        A.loffs = P->loffs.as<unsigned>();
        A.lent = P->lent.ptr;
        A.lbase = P->wmode == W_SCAN ? 0 : P->lbase[k];
        return A;
    };
    const unsigned *loffs = P->loffs.as<unsigned>();
    const ull *lbase = P->lbase_dev.as<ull>();
    if (P->by_mask && P->mask_tile) {
        tile_sweep(st, n, P->mp, menus, scores, nullptr, offs, P->binom.as<ull>(), n + 1, P->rows.as<int4>(),
                   P->Vs.as<float>(), P->Ps.as<uint8_t>());
        mask_readout_kernel<<<1, 32, 0, st>>>(n, P->Vs.as<float>(), P->Ps.as<uint8_t>(), P->out.as<PriceOut>());
        RUMB_LAUNCH("mask_readout_kernel");
    } else if (P->by_mask) {
        RUMB_CUDA(cudaMemsetAsync(P->Vs.ptr, 0, ((size_t)1 << n) * 4, st));
        RUMB_CUDA(cudaMemsetAsync(P->Ps.ptr, 0, (size_t)1 << n, st));
        std::vector<ll> bounds;
        const int *nodes = c.layer_table(n, bounds);
        for (int k = 1; k <= n; ++k) {
            PricerArgs A = args(k);
            A.nodes = nodes + bounds[k];
            A.vmask = P->Vs.as<float>();
            A.pmask = P->Ps.as<uint8_t>();
            layer(A, true, nullptr);
        }
        mask_readout_kernel<<<1, 32, 0, st>>>(n, P->Vs.as<float>(), P->Ps.as<uint8_t>(), P->out.as<PriceOut>());
        RUMB_LAUNCH("mask_readout_kernel");
    } else {
        int cur = 0, prev = 1;
        // layer 0: V = 0 (offset 0, step 0, q 0)
        RUMB_CUDA(cudaMemsetAsync(P->v[prev].ptr, 0, P->mode == 1 ? 4 : 2, st));
        if (P->mode == 3) RUMB_CUDA(cudaMemsetAsync(P->l[prev].ptr, 0, 1, st));
        RUMB_CUDA(cudaMemsetAsync(P->m[prev].ptr, 0, 4, st));
        RUMB_CUDA(cudaMemsetAsync(P->e[prev].ptr, 0, 4, st));
        std::vector<ull> bh, b10;
        if (P->stream_group) {
            b10 = binom_host(SG_LOW);
            if (P->mp) {
                rows_kernel<<<grid_for(P->mp, 256), 256, 0, st>>>(P->mp, menus, scores, nullptr, SG_LOW,
                                                                  (1u << SG_LOW) - 1u, P->rows.as<int4>());
                RUMB_LAUNCH("rows_kernel");
            }
            bh = binom_host(n - SG_LOW);
        }
        for (int k = 1; k <= n; ++k) {
            PricerArgs A = args(k);
            A.vprev_f = P->v[prev].as<float>();
            A.vprev_h = P->v[prev].as<uint16_t>();
            A.lprev = P->l[prev].as<uint8_t>();
            A.mprev = P->m[prev].as<float>();
            A.eprev = P->e[prev].as<float>();
            A.vcur_f = P->v[cur].as<float>();
            A.vcur_h = P->v[cur].as<uint16_t>();
            A.lcur = P->l[cur].as<uint8_t>();
            A.mcur = P->m[cur].as<float>();
            A.ecur = P->e[cur].as<float>();
            A.pred = k >= P->k_pred ? P->pred[k]->as<uint8_t>() : nullptr;
            A.layer_step = P->layer_step.as<unsigned int>() + k;
            if (P->stream_group) {
                const int hb = n - SG_LOW;
                StreamGroupArgs G{};
                G.lmin = std::max(0, k - hb);
                G.lmax = std::min(SG_LOW, k);
                for (int l = G.lmin; l <= G.lmax; ++l) G.cum[l - G.lmin + 1] = G.cum[l - G.lmin] + bh[hb * (hb + 1) + (k - l)];
                for (int l = 0, o = 0; l <= SG_LOW; ++l) {
                    G.loff[l] = o;
                    o += (int)b10[SG_LOW * (SG_LOW + 1) + l];
                }
                G.rows = P->rows.as<int4>();
                G.lowtab = P->lowtab.as<uint16_t>();
                if (P->dec.ptr && A.mode >= 2) {
                    const ull cprev = P->counts[k - 1];
                    launch_pdl(stream_decode_kernel, dim3(grid_for((ll)cprev, 256)), dim3(256), 0, st, A, cprev, P->dec.as<float>());
                    RUMB_LAUNCH("stream_decode_kernel");
                    A.vprev_dec = P->dec.as<float>();
                } else if (A.mode == 1) {
                    A.vprev_dec = A.vprev_f;                    // float32 storage is its own decoded copy
                }
                const ull groups = G.cum[G.lmax - G.lmin + 1];
                launch_pdl(stream_group_kernel<float>, dim3((unsigned)((groups + SG_WARPS - 1) / SG_WARPS)), dim3(32 * SG_WARPS), 0, st, A, G, P->vals.as<float>());
                RUMB_LAUNCH("stream_group_kernel");
            } else {
                layer(A, false, P->vals.as<float>());
            }
            if (A.mode != 1) {
                launch_pdl(stream_quant_kernel, dim3((unsigned)((A.count + PB - 1) / PB)), dim3(PB), 0, st, A, P->vals.as<float>());
                RUMB_LAUNCH("stream_quant_kernel");
            }
            std::swap(cur, prev);
        }
        backtrace_kernel<<<1, 1024, 0, st>>>(n, P->k_pred, P->binom.as<ull>(), P->pred_ptrs.as<uint8_t *>(), menus,
                                             scores, offs, P->Vs.as<float>(), P->Ps.as<uint8_t>(),
                                             P->out.as<PriceOut>(), P->v[prev].as<float>(), P->v[prev].as<uint16_t>(),
                                             P->l[prev].as<uint8_t>(), P->m[prev].as<float>(), P->e[prev].as<float>(),
                                             P->mode, P->wmode, loffs, P->lent.ptr, lbase, P->Ws.as<float>(),
                                             P->k_pred >= SUB_TILE_MIN ? 1 : 0);
        RUMB_LAUNCH("backtrace_kernel");
        if (P->k_pred >= SUB_TILE_MIN) sublattice_tile(*P, scores);
    }
}

void pricer_price(Pricer *P, const float *scores_host, int on_device, double *vmax, int32_t *rank_pos, double *margin,
                  float *layer_step_out) {
    Ctx &c = *P->c;
    cudaStream_t st = c.own;
    int n = P->n;
    const float *scores = scores_host;
    if (!on_device) {
        if (P->mp) RUMB_CUDA(cudaMemcpyAsync(P->scores.ptr, scores_host, (size_t)P->mp * 4, cudaMemcpyHostToDevice, st));
        scores = P->scores.as<float>();
    }
    run_sweep(P, scores);
    PriceOut h;
    std::vector<unsigned int> steps(n + 1);
    RUMB_CUDA(cudaMemcpyAsync(&h, P->out.ptr, sizeof(PriceOut), cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaMemcpyAsync(steps.data(), P->layer_step.ptr, (size_t)(n + 1) * 4, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    double ms = 0.0;
    for (int k = 1; k <= n; ++k) {
        float f;
        std::memcpy(&f, &steps[k], 4);
        ms += (double)f;
        if (layer_step_out) layer_step_out[k] = f;
    }
    if (layer_step_out) layer_step_out[0] = 0.0f;
    for (int x = 0; x < n; ++x) rank_pos[x] = h.rank_pos[x];
    if (P->mode <= 1) {
        *vmax = (double)h.vtop;
        *margin = 0.0;
    } else {
        *vmax = (double)h.mtop + (double)h.qtop * (double)h.etop;
        *margin = P->mode == 2 ? 0.5 * ms : ms;
    }
}

}  // namespace rumb
