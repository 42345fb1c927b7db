// The fused per-menu prox of the BM-ADMM iteration as a tile kernel (sm_100a).
//
// A CTA owns 2^m consecutive menu masks S = base | low (low < 2^m, one thread per menu). The
// slab entries of those menus form one contiguous, aligned run per alternative i:
//   i <  m: the 2^(m-1) rests base/2 + compress(low, i) over the lows that contain i
//   i >= m: the 2^m rests compress(base, i) + low, present only when base contains i
// so the tile's x, x2 and z values are staged in shared memory as a few contiguous runs, the
// projection runs out of shared memory with a small register footprint, and x2 and z go back the
// same way (csrc/prox.cu).
//
// Per menu (the reference's fuse_xk, prox_all and fuse_z, solver/bm_admm/solver.py:37-46,66-139):
//   xo = alpha x + (1 - alpha) x2,  v = xo - z / b2
//   u  = simplex prox of v with curvature b2 (unobserved) or b2 + 2 (observed, pulled to p_hat)
//   z' = z - b2 (xo - u),  x2' = u
// The threshold comes from Michelot's active-set iteration (the active set only shrinks, at
// most |S| rounds), which gives the reference's sort-based threshold without a sort.
//
// The mbarrier / bulk-copy helpers below serve the tensor-core GEMM (csrc/mlp.cu); their waits
// are bounded (~2^32 cycles) and report failure instead of spinning on.
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
__host__ __device__ constexpr ll prox_tile_elems(int n) {
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

// The forms of the prox kernel (csrc/prox.cu): the shared-memory tile; the tile with one pass over
// each menu's members (the menu's threshold kept in shared memory, the projection and the write-back
// done element by element; x, x2, z staged, or the relaxed point and z with a support bit); or G
// lanes per menu reading the slab straight into registers
// (n <= PROX_LANES_MAX_N). Picked per GPU, n and dtype by timing (the iteration's autotuner).
constexpr int PROX_TILE = 0, PROX_LANES2 = 1, PROX_LANES4 = 2, PROX_LANES8 = 3, PROX_TAU = 4, PROX_TAU2 = 5,
              PROX_PAIR = 6, PROX_FORMS = 7;
constexpr int PROX_LANES_MAX_N = 22;

// The prox for one dtype (csrc/prox.cu; grid.y = batched draws' slots).
template <class T>
void launch_prox_tile(const ProxTileArgs<T> &P, cudaStream_t st, int slots = 1, int form = PROX_TILE);

// menu_obs[S] = the observed members of menu S, from the slab's observation bits.
void launch_menu_obs(const uint32_t *obsbits, int n, ll Nloc, uint32_t *menu_obs, cudaStream_t st);

}  // namespace rumb
