// BF16 tensor-core GEMM for sm_100a (tcgen05 MMA with the accumulator in tensor memory, operands
// staged by TMA) and the warm-start MLP trained with it.
//
// GEMM: C[M x N] = A[M x K] . B[N x K]^T, A and B bf16 row-major (K contiguous), f32 accumulate.
// One CTA of 128 threads per 128 x 128 output tile:
//   thread 0   TMA producer: 128 x 64 tiles of A and B into a 4-stage ring of 128-byte-swizzled
//              shared-memory buffers (cp.async.bulk.tensor.2d, completion on a "full" mbarrier)
//   thread 32  MMA issuer: 4 tcgen05.mma (K = 16 each) per stage into a 128 x 128 f32 accumulator
//              in tensor memory; tcgen05.commit frees the stage ("empty" mbarrier) and, after the
//              last stage, signals the epilogue
//   all warps  epilogue: warp w reads accumulator lanes 32w..32w+31 (tcgen05.ld 32x32b), applies the
//              fused epilogue (bias, GELU, GELU derivative) and stores f32 / bf16 rows and, where
//              asked, the bf16 transpose (coalesced: a warp's lanes are 32 consecutive rows)
// Every mbarrier wait is bounded (~2^32 cycles); on expiry the kernel records an error word, stops
// issuing work and still frees its tensor memory; the host turns the word into RUMB_E_TIMEOUT.
// M and N are multiples of 128 and K of 64 (callers pad); nothing reads outside the operands.
//
// MLP: dims d_0 -> d_1 -> ... -> d_L, GELU after every layer but the last, BF16 weights and
// activations, FP32 accumulate and master weights, MSE loss, Adam. Forward, backward and the
// optimizer step are this file's kernels; every matrix product is the GEMM above:
//   forward   Z_l = H_{l-1} W_l^T + b_l,  H_l = gelu(Z_l)          (epilogue: bias + GELU)
//   backward  dW_l = dZ_l^T H_{l-1}  (A = dZ_l^T, B = H_{l-1}^T)   (epilogue: f32 store)
//             dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1})  (B = W_l^T)  (epilogue: GELU derivative)
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "ctx.cuh"
#include "mlp.cuh"
#include "prox.cuh"

namespace rumb {

typedef __nv_bfloat16 bf16;

constexpr int GM_BM = 128, GM_BN = 128, GM_BK = 64, GM_STAGES = 4, GM_THREADS = 128;
constexpr uint32_t GM_TILE_BYTES = GM_BM * GM_BK * 2;                  // one 128 x 64 bf16 tile
constexpr size_t GM_SMEM = 1024 + (size_t)GM_STAGES * 2 * GM_TILE_BYTES + 256;

enum GemmEpi { EPI_F32 = 0, EPI_BIAS_F32 = 1, EPI_BIAS_GELU = 2, EPI_DGELU = 3 };

struct GemmArgs {
    int M, N, K;
    int epi;
    float *C;            // f32 out [M x N] (EPI_F32, EPI_BIAS_F32); pre-activation out (EPI_BIAS_GELU)
    bf16 *H;             // bf16 out [M x N] (EPI_BIAS_GELU, EPI_DGELU; may be null)
    bf16 *Ht;            // bf16 transposed out [N x M] (may be null)
    const float *bias;   // [N]
    const float *Z;      // EPI_DGELU: pre-activation [M x N]
    unsigned int *err;
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(tm), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// shared-memory matrix descriptor of a K-major 128-byte-swizzled tile (rows of 64 bf16, 8-row
// groups 1024 bytes apart): start address, leading offset 16 B, stride offset 1024 B, version 1,
// layout SWIZZLE_128B; the tile must start on a 1024-byte boundary
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// instruction descriptor: kind::f16 with bf16 A and B (K-major), f32 accumulator, M x N
__host__ __device__ constexpr uint32_t bf16_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\ntcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ---------------------------------------------------------------- the GEMM kernel
__global__ void __launch_bounds__(GM_THREADS, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char gm_raw[];
    // 1024-byte aligned ring of stages: [A_0 B_0 A_1 B_1 ...], then the barriers
    const uint32_t raw = smem_u32(gm_raw);
    unsigned char *base = gm_raw + ((1024u - (raw & 1023u)) & 1023u);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + GM_STAGES * 2 * GM_TILE_BYTES);
    uint64_t *empty = full + GM_STAGES;
    uint64_t *accum = empty + GM_STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(accum + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GM_BM, n0 = blockIdx.x * GM_BN;
    const int KT = g.K / GM_BK;
    if (tid == 0) {
        for (int s = 0; s < GM_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accum, 1);
        fence_mbar_init();
    }
    if (warp == 1) {   // the accumulator: 128 lanes x 128 f32 columns of tensor memory
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(GM_BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool failed = false;
    int issued = 0;                     // k-tiles whose loads the producer issued

    if (tid == 0) {
        // producer
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % GM_STAGES;
            if (kt >= GM_STAGES && !mbar_wait_bounded(&empty[s], (unsigned)((kt / GM_STAGES - 1) & 1))) {
                failed = true;
                break;
            }
            unsigned char *sa = base + (size_t)s * 2 * GM_TILE_BYTES;
            mbar_expect_tx(&full[s], 2 * GM_TILE_BYTES);
            tma_load_2d(sa, &tmA, kt * GM_BK, m0, &full[s]);
            tma_load_2d(sa + GM_TILE_BYTES, &tmB, kt * GM_BK, n0, &full[s]);
            issued = kt + 1;
        }
    } else if (tid == 32) {
        // MMA issuer
        const uint32_t idesc = bf16_idesc(GM_BM, GM_BN);
        for (int kt = 0; kt < KT; ++kt) {
            const int s = kt % GM_STAGES;
            if (!mbar_wait_bounded(&full[s], (unsigned)((kt / GM_STAGES) & 1))) {
                failed = true;
                break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(base + (size_t)s * 2 * GM_TILE_BYTES);
            const uint64_t da = sw128_desc(sa), db = sw128_desc(sa + GM_TILE_BYTES);
#pragma unroll
            for (int k = 0; k < GM_BK / 16; ++k)      // +32 bytes along K per MMA: +2 in the address field
                umma_bf16(tmem, da + 2 * k, db + 2 * k, idesc, (kt > 0 || k > 0) ? 1u : 0u);
            umma_commit(&empty[s]);
        }
        umma_commit(accum);   // also after a failure: the epilogue's wait ends either way
    }
    if (failed) atomicOr(g.err, 1u);

    // epilogue (tcgen05.ld is warp-collective: the decision is made per warp)
    const bool ready = mbar_wait_bounded(accum, 0);
    __syncwarp();
    const bool go = __all_sync(0xffffffffu, ready);
    if (!go && lane == 0) atomicOr(g.err, 2u);
    tc_fence_after();
    if (go) {
        const int row = m0 + warp * 32 + lane;
        for (int c = 0; c < GM_BN / 32; ++c) {
            uint32_t r[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32), r);
            const int col0 = n0 + c * 32;
            float v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
            if (g.epi == EPI_BIAS_F32 || g.epi == EPI_BIAS_GELU) {
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] += g.bias[col0 + j];
            }
            if (g.epi == EPI_F32 || g.epi == EPI_BIAS_F32 || g.epi == EPI_BIAS_GELU) {
                float4 *dst = reinterpret_cast<float4 *>(g.C + (size_t)row * g.N + col0);
#pragma unroll
                for (int j = 0; j < 8; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            }
            if (g.epi == EPI_BIAS_GELU || g.epi == EPI_DGELU) {
                if (g.epi == EPI_BIAS_GELU) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = gelu_f(v[j]);
                } else {
                    const float4 *zp = reinterpret_cast<const float4 *>(g.Z + (size_t)row * g.N + col0);
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        float4 z = zp[j];
                        v[4 * j] *= gelu_grad(z.x);
                        v[4 * j + 1] *= gelu_grad(z.y);
                        v[4 * j + 2] *= gelu_grad(z.z);
                        v[4 * j + 3] *= gelu_grad(z.w);
                    }
                }
                bf16 hb[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) hb[j] = __float2bfloat16_rn(v[j]);
                if (g.H) {
                    uint4 *dst = reinterpret_cast<uint4 *>(g.H + (size_t)row * g.N + col0);
                    const uint4 *src = reinterpret_cast<const uint4 *>(hb);
#pragma unroll
                    for (int j = 0; j < 4; ++j) dst[j] = src[j];
                }
                if (g.Ht) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) g.Ht[(size_t)(col0 + j) * g.M + row] = hb[j];
                }
            }
        }
    }
    if (tid == 0) {
        // the last load of each stage has landed before the CTA's shared memory goes away (at once
        // in a normal run; bounded after a failure)
        for (int kt = std::max(0, issued - GM_STAGES); kt < issued; ++kt)
            mbar_wait_bounded(&full[kt % GM_STAGES], (unsigned)((kt / GM_STAGES) & 1));
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GM_BN) : "memory");
    }
}

// ---------------------------------------------------------------- host side of the GEMM
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        RUMB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) fail(RUMB_E_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 2-D map of a row-major bf16 matrix [rows x cols], boxes of 128 rows x 64 columns, 128B swizzle
static CUtensorMap bf16_map(const bf16 *ptr, ll rows, ll cols) {
    if (cols % GM_BK || rows % GM_BM || (reinterpret_cast<uintptr_t>(ptr) & 15))
        fail(RUMB_E_INTERNAL, "GEMM operand shape or alignment");
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    cuuint64_t gdim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)GM_BK, (cuuint32_t)GM_BM};
    cuuint32_t es[2] = {1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(ptr), gdim, gstride, box, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(RUMB_E_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

static void gemm(const bf16 *A, const bf16 *B, GemmArgs g, cudaStream_t st) {
    if (g.M % GM_BM || g.N % GM_BN || g.K % GM_BK || g.M <= 0 || g.N <= 0 || g.K <= 0)
        fail(RUMB_E_INVAL, "GEMM: M and N multiples of 128, K a multiple of 64");
    static std::atomic<unsigned long long> optin{0};
    smem_optin(umma_gemm_kernel, (int)GM_SMEM, optin);
    CUtensorMap ta = bf16_map(A, g.M, g.K), tb = bf16_map(B, g.N, g.K);
    dim3 grid((unsigned)(g.N / GM_BN), (unsigned)(g.M / GM_BM));
    if (g_prof) prof_begin("umma_gemm", 2.0 * ((double)g.M * g.K + (double)g.N * g.K) + 4.0 * g.M * g.N, st);
    umma_gemm_kernel<<<grid, GM_THREADS, GM_SMEM, st>>>(ta, tb, g);
    RUMB_LAUNCH("umma_gemm_kernel");
    prof_end(st);
}

static void check_err(const DevBuf &err, cudaStream_t st) {
    unsigned int h = 0;
    RUMB_CUDA(cudaMemcpyAsync(&h, err.ptr, 4, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    if (h) fail(RUMB_E_TIMEOUT, "a tensor-core GEMM's bounded wait gave up");
}

int gemm_bf16_host(Ctx &c, int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C) {
    if (!A || !B || !C) fail(RUMB_E_INVAL, "gemm: NULL buffer");
    if (M <= 0 || N <= 0 || K <= 0 || M % GM_BM || N % GM_BN || K % GM_BK)
        fail(RUMB_E_INVAL, "gemm: M and N multiples of 128, K a multiple of 64");
    cudaStream_t st = c.own;
    c.join_in();
    DevBuf dA, dB, dC, err;
    dA.ensure((size_t)M * K * 2);
    dB.ensure((size_t)N * K * 2);
    dC.ensure((size_t)M * N * 4);
    err.ensure(4);
    RUMB_CUDA(cudaMemsetAsync(err.ptr, 0, 4, st));
    RUMB_CUDA(cudaMemcpyAsync(dA.ptr, A, (size_t)M * K * 2, cudaMemcpyHostToDevice, st));
    RUMB_CUDA(cudaMemcpyAsync(dB.ptr, B, (size_t)N * K * 2, cudaMemcpyHostToDevice, st));
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.epi = EPI_F32;
    g.C = dC.as<float>();
    g.err = err.as<unsigned int>();
    gemm(dA.as<bf16>(), dB.as<bf16>(), g, st);
    RUMB_CUDA(cudaMemcpyAsync(C, dC.ptr, (size_t)M * N * 4, cudaMemcpyDeviceToHost, st));
    check_err(err, st);
    c.join_out();
    return RUMB_OK;
}

// ---------------------------------------------------------------- elementwise kernels of the MLP
// rows idx[r] of X (f32, [m x d] real) -> bf16 batch [Mb x dp] and its transpose [dp x Mb], zero padded
__global__ void gather_in_kernel(const float *X, const int *idx, int nrows, int d, int dp, int Mb, bf16 *out,
                                 bf16 *outT) {
    ll t = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (t >= (ll)Mb * dp) return;
    int r = (int)(t / dp), j = (int)(t % dp);
    float v = 0.f;
    if (r < nrows && j < d) v = X[(ll)idx[r] * d + j];
    bf16 b = __float2bfloat16_rn(v);
    out[t] = b;
    outT[(ll)j * Mb + r] = b;
}

// loss terms and dOut = 2 (out - T) / count on the real rows and columns (bf16, and transposed)
__global__ void mse_grad_kernel(const float *out, const float *T, const int *idx, int nrows, int d, int dp, int Mb,
                                float scale, bf16 *dout, bf16 *doutT, double *loss_parts) {
    ll t = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    double sq = 0.0;
    if (t < (ll)Mb * dp) {
        int r = (int)(t / dp), j = (int)(t % dp);
        float g = 0.f;
        if (r < nrows && j < d) {
            float e = out[t] - T[(ll)idx[r] * d + j];
            sq = (double)e * (double)e;
            g = 2.0f * e * scale;
        }
        bf16 b = __float2bfloat16_rn(g);
        dout[t] = b;
        doutT[(ll)j * Mb + r] = b;
    }
    // block sum of the squared errors
    __shared__ double red[256];
    red[threadIdx.x] = sq;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_parts[blockIdx.x] = red[0];
}

// db[n] = sum over rows of the bf16 gradient G [Mb x N] (one thread per column, fixed row order)
__global__ void colsum_kernel(const bf16 *G, int Mb, int N, float *db) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int r = 0; r < Mb; ++r) s += __bfloat162float(G[(ll)r * N + n]);
    db[n] = s;
}

// Adam on f32 master weights; writes the bf16 copy [R x Cc] and its transpose [Cc x R]
__global__ void adam_kernel(float *w, const float *gr, float *m, float *v, ll count, int R, int Cc, float lr,
                            float b1, float b2, float c1, float c2, float eps, bf16 *wb, bf16 *wbT) {
    ll t = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (t >= count) return;
    float g = gr[t];
    float mm = b1 * m[t] + (1.f - b1) * g;
    float vv = b2 * v[t] + (1.f - b2) * g * g;
    m[t] = mm;
    v[t] = vv;
    float x = w[t] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    w[t] = x;
    if (wb) {
        bf16 b = __float2bfloat16_rn(x);
        wb[t] = b;
        int r = (int)(t / Cc), cc = (int)(t % Cc);
        wbT[(ll)cc * R + r] = b;
    }
}

// bf16 copy [R x Cc] and transpose of f32 weights
__global__ void to_bf16_kernel(const float *w, ll count, int R, int Cc, bf16 *wb, bf16 *wbT) {
    ll t = blockIdx.x * (ll)blockDim.x + threadIdx.x;
    if (t >= count) return;
    bf16 b = __float2bfloat16_rn(w[t]);
    wb[t] = b;
    int r = (int)(t / Cc), cc = (int)(t % Cc);
    wbT[(ll)cc * R + r] = b;
}

// ---------------------------------------------------------------- the MLP object
static int pad_to(int x, int q) { return (x + q - 1) / q * q; }

struct MlpLayer {
    int in = 0, out = 0, inp = 0, outp = 0;     // real and padded (128) widths
    DevBuf W, b, Wb, WbT, gW, gb, mW, vW, mb, vb;
};

struct Mlp {
    Ctx *c = nullptr;
    std::vector<MlpLayer> L;
    int Mb = 0;                                   // batch rows the activations hold
    std::vector<DevBuf> X, XT;                    // X[l]: layer l's input (bf16) [Mb x inp], XT transposed
    std::vector<DevBuf> Z;                        // pre-activations (f32) [Mb x outp]
    DevBuf out, dA, dAT, dB, dBT, idx, err, loss_parts, Xall, Tall;
    ll n_rows_all = 0;
    long long t = 0;                              // Adam steps

    int d_in() const { return L.front().in; }
    int d_out() const { return L.back().out; }

    void ensure_batch(int mb) {
        if (mb <= Mb) return;
        Mb = mb;
        size_t n = L.size();
        X.clear();
        XT.clear();
        Z.clear();
        X.resize(n);
        XT.resize(n);
        Z.resize(n);
        int wmax = 0;
        for (size_t l = 0; l < n; ++l) {
            X[l].ensure((size_t)Mb * L[l].inp * 2);
            XT[l].ensure((size_t)Mb * L[l].inp * 2);
            Z[l].ensure((size_t)Mb * L[l].outp * 4);
            wmax = std::max(wmax, std::max(L[l].inp, L[l].outp));
        }
        out.ensure((size_t)Mb * L.back().outp * 4);
        dA.ensure((size_t)Mb * wmax * 2);
        dAT.ensure((size_t)Mb * wmax * 2);
        dB.ensure((size_t)Mb * wmax * 2);
        dBT.ensure((size_t)Mb * wmax * 2);
        idx.ensure((size_t)Mb * 4);
        loss_parts.ensure((size_t)grid_for((ll)Mb * L.back().outp, 256) * 8);
    }
};

static void refresh_bf16(MlpLayer &l, cudaStream_t st) {
    ll cnt = (ll)l.outp * l.inp;
    to_bf16_kernel<<<grid_for(cnt, 256), 256, 0, st>>>(l.W.as<float>(), cnt, l.outp, l.inp, l.Wb.as<bf16>(),
                                                       l.WbT.as<bf16>());
    RUMB_LAUNCH("to_bf16_kernel");
}

Mlp *mlp_create(Ctx &c, int n_layers, const int *dims, unsigned long long seed) {
    if (n_layers < 1 || n_layers > 16 || !dims) fail(RUMB_E_INVAL, "mlp: 1 to 16 layers");
    for (int l = 0; l <= n_layers; ++l)
        if (dims[l] < 1 || dims[l] > 16384) fail(RUMB_E_INVAL, "mlp: widths 1 .. 16384");
    std::unique_ptr<Mlp> m(new Mlp());
    m->c = &c;
    m->L.resize(n_layers);
    std::mt19937_64 rng(seed);
    cudaStream_t st = c.own;
    for (int l = 0; l < n_layers; ++l) {
        MlpLayer &y = m->L[l];
        y.in = dims[l];
        y.out = dims[l + 1];
        y.inp = pad_to(y.in, 128);
        y.outp = pad_to(y.out, 128);
        size_t cnt = (size_t)y.outp * y.inp;
        // uniform(-1/sqrt(in), 1/sqrt(in)) on the real block, zero in the padding
        std::vector<float> w(cnt, 0.f), b((size_t)y.outp, 0.f);
        std::uniform_real_distribution<float> U(-1.0f / std::sqrt((float)y.in), 1.0f / std::sqrt((float)y.in));
        for (int r = 0; r < y.out; ++r)
            for (int k = 0; k < y.in; ++k) w[(size_t)r * y.inp + k] = U(rng);
        for (int r = 0; r < y.out; ++r) b[r] = U(rng);
        for (DevBuf *d : {&y.W, &y.gW, &y.mW, &y.vW}) d->ensure(cnt * 4);
        for (DevBuf *d : {&y.b, &y.gb, &y.mb, &y.vb}) d->ensure((size_t)y.outp * 4);
        y.Wb.ensure(cnt * 2);
        y.WbT.ensure(cnt * 2);
        RUMB_CUDA(cudaMemcpyAsync(y.W.ptr, w.data(), cnt * 4, cudaMemcpyHostToDevice, st));
        RUMB_CUDA(cudaMemcpyAsync(y.b.ptr, b.data(), (size_t)y.outp * 4, cudaMemcpyHostToDevice, st));
        for (DevBuf *d : {&y.mW, &y.vW, &y.gW}) RUMB_CUDA(cudaMemsetAsync(d->ptr, 0, cnt * 4, st));
        for (DevBuf *d : {&y.mb, &y.vb, &y.gb}) RUMB_CUDA(cudaMemsetAsync(d->ptr, 0, (size_t)y.outp * 4, st));
        refresh_bf16(y, st);
    }
    m->err.ensure(4);
    RUMB_CUDA(cudaMemsetAsync(m->err.ptr, 0, 4, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    return m.release();
}

void mlp_destroy(Mlp *m) { delete m; }

ll mlp_num_params(const Mlp &m) {
    ll n = 0;
    for (auto &y : m.L) n += (ll)y.out * y.in + y.out;
    return n;
}

// params <-> flat host vector: per layer W (out x in, row-major) then b (out)
void mlp_get_params(Mlp &m, float *buf, bool grads) {
    cudaStream_t st = m.c->own;
    ll off = 0;
    for (auto &y : m.L) {
        std::vector<float> w((size_t)y.outp * y.inp), b((size_t)y.outp);
        RUMB_CUDA(cudaMemcpyAsync(w.data(), (grads ? y.gW : y.W).ptr, w.size() * 4, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaMemcpyAsync(b.data(), (grads ? y.gb : y.b).ptr, b.size() * 4, cudaMemcpyDeviceToHost, st));
        RUMB_CUDA(cudaStreamSynchronize(st));
        for (int r = 0; r < y.out; ++r)
            std::memcpy(buf + off + (ll)r * y.in, w.data() + (size_t)r * y.inp, (size_t)y.in * 4);
        off += (ll)y.out * y.in;
        std::memcpy(buf + off, b.data(), (size_t)y.out * 4);
        off += y.out;
    }
}

void mlp_set_params(Mlp &m, const float *buf) {
    cudaStream_t st = m.c->own;
    ll off = 0;
    for (auto &y : m.L) {
        std::vector<float> w((size_t)y.outp * y.inp, 0.f), b((size_t)y.outp, 0.f);
        for (int r = 0; r < y.out; ++r)
            std::memcpy(w.data() + (size_t)r * y.inp, buf + off + (ll)r * y.in, (size_t)y.in * 4);
        off += (ll)y.out * y.in;
        std::memcpy(b.data(), buf + off, (size_t)y.out * 4);
        off += y.out;
        RUMB_CUDA(cudaMemcpyAsync(y.W.ptr, w.data(), w.size() * 4, cudaMemcpyHostToDevice, st));
        RUMB_CUDA(cudaMemcpyAsync(y.b.ptr, b.data(), b.size() * 4, cudaMemcpyHostToDevice, st));
        refresh_bf16(y, st);
        RUMB_CUDA(cudaStreamSynchronize(st));
    }
    m.t = 0;
    for (auto &y : m.L) {
        RUMB_CUDA(cudaMemsetAsync(y.mW.ptr, 0, y.mW.bytes, st));
        RUMB_CUDA(cudaMemsetAsync(y.vW.ptr, 0, y.vW.bytes, st));
        RUMB_CUDA(cudaMemsetAsync(y.mb.ptr, 0, y.mb.bytes, st));
        RUMB_CUDA(cudaMemsetAsync(y.vb.ptr, 0, y.vb.bytes, st));
    }
}

// forward over a batch already gathered into X[0] (Mb rows); output f32 in m.out [Mb x outp_last]
static void forward(Mlp &m, cudaStream_t st) {
    size_t n = m.L.size();
    for (size_t l = 0; l < n; ++l) {
        MlpLayer &y = m.L[l];
        GemmArgs g{};
        g.M = m.Mb;
        g.N = y.outp;
        g.K = y.inp;
        g.bias = y.b.as<float>();
        g.err = m.err.as<unsigned int>();
        if (l + 1 < n) {
            g.epi = EPI_BIAS_GELU;
            g.C = m.Z[l].as<float>();
            g.H = m.X[l + 1].as<bf16>();
            g.Ht = m.XT[l + 1].as<bf16>();
        } else {
            g.epi = EPI_BIAS_F32;
            g.C = m.out.as<float>();
        }
        gemm(m.X[l].as<bf16>(), y.Wb.as<bf16>(), g, st);
    }
}

// backward from dOut (in m.dA / m.dAT) into every layer's gW, gb
static void backward(Mlp &m, cudaStream_t st) {
    int n = (int)m.L.size();
    DevBuf *G = &m.dA, *GT = &m.dAT, *G2 = &m.dB, *G2T = &m.dBT;
    for (int l = n - 1; l >= 0; --l) {
        MlpLayer &y = m.L[l];
        // dW_l = G^T X_l : A = G^T [outp x Mb], B = X_l^T [inp x Mb]
        GemmArgs g{};
        g.M = y.outp;
        g.N = y.inp;
        g.K = m.Mb;
        g.epi = EPI_F32;
        g.C = y.gW.as<float>();
        g.err = m.err.as<unsigned int>();
        gemm(GT->as<bf16>(), m.XT[l].as<bf16>(), g, st);
        colsum_kernel<<<grid_for(y.outp, 128), 128, 0, st>>>(G->as<bf16>(), m.Mb, y.outp, y.gb.as<float>());
        RUMB_LAUNCH("colsum_kernel");
        if (l == 0) break;
        // G_{l-1} = (G W_l) * gelu'(Z_{l-1}) : A = G [Mb x outp], B = W_l^T [inp x outp]
        GemmArgs h{};
        h.M = m.Mb;
        h.N = y.inp;
        h.K = y.outp;
        h.epi = EPI_DGELU;
        h.Z = m.Z[l - 1].as<float>();
        h.H = G2->as<bf16>();
        h.Ht = G2T->as<bf16>();
        h.err = m.err.as<unsigned int>();
        gemm(G->as<bf16>(), y.WbT.as<bf16>(), h, st);
        std::swap(G, G2);
        std::swap(GT, G2T);
    }
}

static void upload_rows(Mlp &m, const float *X, const float *T, ll rows, cudaStream_t st) {
    m.Xall.ensure((size_t)rows * m.d_in() * 4);
    RUMB_CUDA(cudaMemcpyAsync(m.Xall.ptr, X, (size_t)rows * m.d_in() * 4, cudaMemcpyHostToDevice, st));
    if (T) {
        m.Tall.ensure((size_t)rows * m.d_out() * 4);
        RUMB_CUDA(cudaMemcpyAsync(m.Tall.ptr, T, (size_t)rows * m.d_out() * 4, cudaMemcpyHostToDevice, st));
    }
    m.n_rows_all = rows;
}

static void gather(Mlp &m, const int *idx_host, int nrows, cudaStream_t st) {
    RUMB_CUDA(cudaMemcpyAsync(m.idx.ptr, idx_host, (size_t)nrows * 4, cudaMemcpyHostToDevice, st));
    MlpLayer &y = m.L[0];
    gather_in_kernel<<<grid_for((ll)m.Mb * y.inp, 256), 256, 0, st>>>(
        m.Xall.as<float>(), m.idx.as<int>(), nrows, y.in, y.inp, m.Mb, m.X[0].as<bf16>(), m.XT[0].as<bf16>());
    RUMB_LAUNCH("gather_in_kernel");
}

// loss over the gathered rows (mean over nrows x d_out) and dOut into dA/dAT
static double loss_and_dout(Mlp &m, int nrows, cudaStream_t st) {
    MlpLayer &y = m.L.back();
    ll total = (ll)m.Mb * y.outp;
    unsigned blocks = grid_for(total, 256);
    float scale = 1.0f / ((float)nrows * (float)y.out);
    mse_grad_kernel<<<blocks, 256, 0, st>>>(m.out.as<float>(), m.Tall.as<float>(), m.idx.as<int>(), nrows, y.out,
                                            y.outp, m.Mb, scale, m.dA.as<bf16>(), m.dAT.as<bf16>(),
                                            m.loss_parts.as<double>());
    RUMB_LAUNCH("mse_grad_kernel");
    std::vector<double> parts(blocks);
    RUMB_CUDA(cudaMemcpyAsync(parts.data(), m.loss_parts.ptr, blocks * 8, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    double s = 0.0;
    for (double p : parts) s += p;
    return s / ((double)nrows * y.out);
}

static void adam_step(Mlp &m, float lr, cudaStream_t st) {
    m.t++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float c1 = 1.f - std::pow(b1, (float)m.t), c2 = 1.f - std::pow(b2, (float)m.t);
    for (auto &y : m.L) {
        ll cnt = (ll)y.outp * y.inp;
        adam_kernel<<<grid_for(cnt, 256), 256, 0, st>>>(y.W.as<float>(), y.gW.as<float>(), y.mW.as<float>(),
                                                        y.vW.as<float>(), cnt, y.outp, y.inp, lr, b1, b2, c1, c2, eps,
                                                        y.Wb.as<bf16>(), y.WbT.as<bf16>());
        RUMB_LAUNCH("adam_kernel");
        adam_kernel<<<grid_for(y.outp, 256), 256, 0, st>>>(y.b.as<float>(), y.gb.as<float>(), y.mb.as<float>(),
                                                           y.vb.as<float>(), y.outp, 1, y.outp, lr, b1, b2, c1, c2,
                                                           eps, nullptr, nullptr);
        RUMB_LAUNCH("adam_kernel");
    }
}

static void read_out(Mlp &m, int nrows, float *Y, cudaStream_t st) {
    MlpLayer &y = m.L.back();
    std::vector<float> o((size_t)m.Mb * y.outp);
    RUMB_CUDA(cudaMemcpyAsync(o.data(), m.out.ptr, o.size() * 4, cudaMemcpyDeviceToHost, st));
    RUMB_CUDA(cudaStreamSynchronize(st));
    for (int r = 0; r < nrows; ++r) std::memcpy(Y + (ll)r * y.out, o.data() + (size_t)r * y.outp, (size_t)y.out * 4);
}

void mlp_forward(Mlp &m, const float *X, ll rows, float *Y) {
    if (!X || !Y || rows < 1) fail(RUMB_E_INVAL, "mlp forward: X, Y and rows >= 1");
    cudaStream_t st = m.c->own;
    RUMB_CUDA(cudaMemsetAsync(m.err.ptr, 0, 4, st));
    upload_rows(m, X, nullptr, rows, st);
    const int chunk = 1024;
    m.ensure_batch((int)std::min<ll>(pad_to((int)std::min<ll>(rows, chunk), 128), chunk));
    std::vector<int> idx(m.Mb);
    for (ll r0 = 0; r0 < rows; r0 += m.Mb) {
        int nr = (int)std::min<ll>(m.Mb, rows - r0);
        for (int i = 0; i < nr; ++i) idx[i] = (int)(r0 + i);
        gather(m, idx.data(), nr, st);
        forward(m, st);
        read_out(m, nr, Y + r0 * m.d_out(), st);
    }
    check_err(m.err, st);
}

double mlp_loss_grad(Mlp &m, const float *X, const float *T, ll rows, float *grad) {
    if (!X || !T || rows < 1 || rows > 16384) fail(RUMB_E_INVAL, "mlp grad: X, T and 1 <= rows <= 16384");
    cudaStream_t st = m.c->own;
    RUMB_CUDA(cudaMemsetAsync(m.err.ptr, 0, 4, st));
    upload_rows(m, X, T, rows, st);
    m.ensure_batch(pad_to((int)rows, 128));
    std::vector<int> idx((size_t)rows);
    for (ll i = 0; i < rows; ++i) idx[(size_t)i] = (int)i;
    gather(m, idx.data(), (int)rows, st);
    forward(m, st);
    double loss = loss_and_dout(m, (int)rows, st);
    backward(m, st);
    check_err(m.err, st);
    if (grad) mlp_get_params(m, grad, true);
    return loss;
}

double mlp_train(Mlp &m, const float *X, const float *T, ll rows, int epochs, int batch, double lr,
                 unsigned long long seed) {
    if (!X || !T || rows < 1 || epochs < 1 || batch < 1) fail(RUMB_E_INVAL, "mlp train: X, T, rows, epochs, batch");
    cudaStream_t st = m.c->own;
    RUMB_CUDA(cudaMemsetAsync(m.err.ptr, 0, 4, st));
    upload_rows(m, X, T, rows, st);
    int bs = (int)std::min<ll>(batch, rows);
    m.ensure_batch(pad_to(bs, 128));
    std::vector<int> order((size_t)rows);
    for (ll i = 0; i < rows; ++i) order[(size_t)i] = (int)i;
    std::mt19937_64 rng(seed);
    double last = 0.0;
    for (int e = 0; e < epochs; ++e) {
        std::shuffle(order.begin(), order.end(), rng);
        double tot = 0.0;
        ll seen = 0;
        for (ll r0 = 0; r0 < rows; r0 += bs) {
            int nr = (int)std::min<ll>(bs, rows - r0);
            gather(m, order.data() + r0, nr, st);
            forward(m, st);
            tot += loss_and_dout(m, nr, st) * nr;
            seen += nr;
            backward(m, st);
            adam_step(m, (float)lr, st);
        }
        last = tot / (double)seen;
    }
    check_err(m.err, st);
    return last;
}

}  // namespace rumb
