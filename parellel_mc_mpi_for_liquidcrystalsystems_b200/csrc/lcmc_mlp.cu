// lcmc_mlp.cu - the volume-move surrogate: a 4097 -> 128 -> 128 -> 1 MLP with
// BF16 weights/activations and FP32 accumulation, trained and evaluated on the
// GPU by this file's kernels.  The matrix products run on the 5th-generation
// tensor cores (tcgen05.mma, accumulators in TMEM); bias, activation, loss and
// Adam are small FP32 CUDA-core kernels.  (No reference counterpart: the
// reference has no NPT move at all, MCnptColloid.c:3978.)
#include <cuda.h> // CUtensorMap and its enums (the encoder is taken from the driver at run time)
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/lcmc.h"
#include "lcmc_rng.cuh"
#include "lcmc_tc.cuh"

namespace lcmc {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------
// C[M x N] (FP32, row-major) (+)= A[M x K] * B[N x K]^T; A, B BF16 row-major
// with K contiguous (lda, ldb in elements, multiples of 8), K a multiple of 64.
// CTA = 128 threads per 128 x BN output tile (BN = 128, or 64 when 128-wide
// tiles would leave most SMs idle).  The K loop runs over 64-wide slices
// through a GT_STAGES-deep ring of shared-memory stages filled by cp.async
// (16-byte copies, zero-filled beyond M and N) in the K-major core-matrix
// layout (8 rows x 16 bytes per core matrix, K halves 128 B apart, 8-row
// groups 1024 B apart).  One elected thread issues the slice's four
// 128 x BN x 16 tcgen05 MMAs and commits them to the stage's mbarrier; a stage
// is refilled once the MMAs that read it have completed, so GT_STAGES - 1
// slices of loads are in flight while the tensor core works.  The accumulator
// lives in BN TMEM columns and is read back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31 = rows).  Waits are bounded: on a timeout the tile sets
// *err, lets its copies and MMAs in flight finish and frees its TMEM.
// ---------------------------------------------------------------------------
constexpr int GT_M = 128, GT_K = 64, GT_STAGES = 4;
// mbarrier tries before a wait gives up (lcmc_set_wait_limit lowers it for tests)
constexpr uint32_t kWaitIters = 1u << 24;
static uint32_t g_wait_iters = kWaitIters;

template <int BN> struct GemmShape {
    static constexpr int A_BYTES = GT_M * GT_K * 2, B_BYTES = BN * GT_K * 2, STAGE = A_BYTES + B_BYTES;
    static constexpr int SMEM = GT_STAGES * STAGE;
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_u32(smem)), "l"(gmem),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Slice kt of A (128 rows from m0) and B (BN rows from n0) into one stage (sA, sB).
template <int BN>
__device__ __forceinline__ void gemm_load_slice(unsigned char *sA, unsigned char *sB, const bf16 *__restrict__ A,
                                                int lda, const bf16 *__restrict__ B, int ldb, int M, int N, int m0,
                                                int n0, int kt, int t)
{
    const int k0 = kt * GT_K;
#pragma unroll
    for (int i = 0; i < GT_M * 8 / 128; i++) {
        const int v = t + 128 * i;
        const int row = v >> 3, ch = v & 7;
        const int off = ((row >> 3) * 8 + ch) * 128 + (row & 7) * 16;
        const int gm = m0 + row;
        const bool in = gm < M;
        cp_async16(sA + off, in ? (const void *)(A + (size_t)gm * lda + k0 + ch * 8) : (const void *)A, in ? 16 : 0);
    }
#pragma unroll
    for (int i = 0; i < BN * 8 / 128; i++) {
        const int v = t + 128 * i;
        const int row = v >> 3, ch = v & 7;
        const int off = ((row >> 3) * 8 + ch) * 128 + (row & 7) * 16;
        const int gn = n0 + row;
        const bool in = gn < N;
        cp_async16(sB + off, in ? (const void *)(B + (size_t)gn * ldb + k0 + ch * 8) : (const void *)B, in ? 16 : 0);
    }
}

template <int BN>
__global__ void __launch_bounds__(128) k_gemm_tc(const bf16 *__restrict__ A, int lda, const bf16 *__restrict__ B,
                                                 int ldb, float *__restrict__ C, int ldc, int M, int N, int K,
                                                 int accumulate, int *err, uint32_t wait_iters)
{
    using G = GemmShape<BN>;
    constexpr int S = GT_STAGES;
    extern __shared__ __align__(1024) unsigned char gsm[];
    __shared__ __align__(8) uint64_t bar[S];
    __shared__ uint32_t tmem_base;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int m0 = blockIdx.x * GT_M, n0 = blockIdx.y * BN;
    const int nk = K / GT_K;
    if (w == 0) {
        tc::tmem_alloc(&tmem_base, BN);
        tc::tmem_relinquish();
    }
    if (t == 0) {
        for (int i = 0; i < S; i++) tc::mbar_init(&bar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // prologue: slices 0 .. S-2 in flight (one commit group per slice; empty groups past the end)
#pragma unroll
    for (int st = 0; st < S - 1; st++) {
        if (st < nk)
            gemm_load_slice<BN>(gsm + st * G::STAGE, gsm + st * G::STAGE + G::A_BYTES, A, lda, B, ldb, M, N, m0, n0,
                                st, t);
        cp_async_commit();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmem_base;
    const uint32_t idesc = tc::idesc_bf16_f32(GT_M, BN);
    bool ok = true;
    int issued = -1; // last slice whose MMAs were committed
    for (int i = 0; i < nk; i++) {
        cp_async_wait<S - 2>();            // this thread's copies of slice i have landed
        tc::fence_proxy_async_smem();      // ... and are visible to the tensor core
        if (__syncthreads_or(!ok)) break;  // every thread's copies of slice i, unless a wait gave up
        const int st = i % S;
        if (t == 0) {
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_u32(gsm + st * G::STAGE), b0 = a0 + G::A_BYTES;
#pragma unroll
            for (int s = 0; s < GT_K / 16; s++) {
                const uint64_t ad = tc::smem_desc_kmajor(a0 + 256u * s, 128u, 1024u);
                const uint64_t bd = tc::smem_desc_kmajor(b0 + 256u * s, 128u, 1024u);
                tc::mma_bf16(tbase, ad, bd, idesc, (i > 0 || s > 0) ? 1u : 0u);
            }
            tc::mma_commit(&bar[st]);
        }
        issued = i;
        // slice i + S - 1 goes into the stage that slice i - 1 used: wait for those MMAs first
        const int nxt = i + S - 1;
        if (nxt < nk) {
            if (i >= 1 && !tc::mbar_wait_bounded(&bar[(i - 1) % S], (uint32_t)((i - 1) / S) & 1u, wait_iters))
                ok = false;
            if (ok)
                gemm_load_slice<BN>(gsm + (nxt % S) * G::STAGE, gsm + (nxt % S) * G::STAGE + G::A_BYTES, A, lda, B,
                                    ldb, M, N, m0, n0, nxt, t);
        }
        cp_async_commit();
    }
    // the last commit covers every MMA issued before it
    if (ok && issued == nk - 1 && nk > 0 &&
        !tc::mbar_wait_bounded(&bar[issued % S], (uint32_t)(issued / S) & 1u, wait_iters))
        ok = false;
    const bool failed = __syncthreads_or(!ok) != 0;
    cp_async_wait_all();
    tc::fence_after_sync();
    if (!failed) {
        const int row = m0 + 32 * w + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tbase + ((uint32_t)(32 * w) << 16) + (uint32_t)c0, v);
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int col = n0 + c0 + j;
                    if (col < N) {
                        float *p = C + (size_t)row * ldc + col;
                        *p = accumulate ? *p + v[j] : v[j];
                    }
                }
            }
        }
    } else {
        if (t == 0) atomicOr(err, 1);
        // the MMAs in flight finish before their TMEM is freed (full bound)
        if (issued >= 0) tc::mbar_wait_bounded(&bar[issued % S], (uint32_t)(issued / S) & 1u, kWaitIters);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (w == 0) tc::tmem_dealloc(tbase, BN);
}

// ---------------------------------------------------------------------------
// The same product with TMA tile loads (used when A and B are 16-byte aligned
// with 16-byte row strides): one thread streams 64-wide K slices of A
// (128 rows) and B (BN rows) through GT_TMA_STAGES shared-memory stages with
// cp.async.bulk.tensor (128-byte swizzle, rows beyond M or N filled with
// zeros), each stage's loads completing on its "full" mbarrier; the same
// thread issues the slice's four MMAs once the stage is full and commits them
// to the stage's "empty" mbarrier, and refills the stage the previous slice
// used as soon as that slice's MMAs have completed, so the loads of the next
// GT_TMA_STAGES - 1 slices are in flight while the tensor core works.  The
// other threads wait at a block barrier for the epilogue.  Every wait is
// bounded; on a timeout the tile sets *err, waits (with the full bound) for its
// loads and MMAs in flight and frees its TMEM.
// ---------------------------------------------------------------------------
constexpr int GT_TMA_STAGES = 4;
template <int BN> struct TmaShape {
    static constexpr int A_BYTES = GT_M * GT_K * 2, B_BYTES = BN * GT_K * 2, STAGE = A_BYTES + B_BYTES;
    static constexpr int SMEM = GT_TMA_STAGES * STAGE + 1024; // + slack to align the stages to 1024 bytes
};

// K slice j of A (128 rows from m0) and B (rows from n0) into one stage, on its full barrier.
__device__ __forceinline__ void tma_stage_load(unsigned char *dst, int a_bytes, uint32_t stage_bytes,
                                               const CUtensorMap *ta, const CUtensorMap *tb, int j, int m0, int n0,
                                               uint64_t *full)
{
    tc::mbar_arrive_expect_tx(full, stage_bytes);
    tc::tma_load_2d(dst, ta, j * GT_K, m0, full);
    tc::tma_load_2d(dst + a_bytes, tb, j * GT_K, n0, full);
}

template <int BN>
__global__ void __launch_bounds__(128) k_gemm_tma(const __grid_constant__ CUtensorMap ta,
                                                  const __grid_constant__ CUtensorMap tb, float *__restrict__ C,
                                                  int ldc, int M, int N, int K, int accumulate, int *err,
                                                  uint32_t wait_iters)
{
    using G = TmaShape<BN>;
    constexpr int S = GT_TMA_STAGES;
    extern __shared__ unsigned char gsm_raw[];
    __shared__ __align__(8) uint64_t full[S], empty[S];
    __shared__ uint32_t tmem_base;
    __shared__ int bad;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int m0 = blockIdx.x * GT_M, n0 = blockIdx.y * BN;
    const int nk = K / GT_K;
    const uint32_t raw = tc::smem_u32(gsm_raw);
    unsigned char *gsm = gsm_raw + (((raw + 1023u) & ~1023u) - raw);
    if (w == 0) {
        tc::tmem_alloc(&tmem_base, BN);
        tc::tmem_relinquish();
    }
    if (t == 0) {
        for (int i = 0; i < S; i++) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmem_base;
    if (t == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32(GT_M, BN);
        int last_load[S]; // last slice loaded into each stage (-1: none)
#pragma unroll
        for (int i = 0; i < S; i++) last_load[i] = -1;
        for (int j = 0; j < S && j < nk; j++) {
            tma_stage_load(gsm + j * G::STAGE, G::A_BYTES, (uint32_t)G::STAGE, &ta, &tb, j, m0, n0, &full[j]);
            last_load[j] = j;
        }
        bool ok = true;
        int issued = -1; // last slice whose MMAs were committed
        for (int i = 0; i < nk; i++) {
            const int st = i % S;
            if (!tc::mbar_wait_bounded(&full[st], (uint32_t)(i / S) & 1u, wait_iters)) {
                ok = false;
                break;
            }
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_u32(gsm + st * G::STAGE), b0 = a0 + G::A_BYTES;
#pragma unroll
            for (int s = 0; s < GT_K / 16; s++)
                tc::mma_bf16(tbase, tc::smem_desc_sw128(a0 + 32u * s), tc::smem_desc_sw128(b0 + 32u * s), idesc,
                             (i > 0 || s > 0) ? 1u : 0u);
            tc::mma_commit(&empty[st]);
            issued = i;
            // refill the stage that slice i - 1 used once its MMAs have completed
            const int j = i - 1 + S;
            if (i >= 1 && j < nk) {
                const int ps = (i - 1) % S;
                if (!tc::mbar_wait_bounded(&empty[ps], (uint32_t)((i - 1) / S) & 1u, wait_iters)) {
                    ok = false;
                    break;
                }
                tma_stage_load(gsm + ps * G::STAGE, G::A_BYTES, (uint32_t)G::STAGE, &ta, &tb, j, m0, n0,
                               &full[ps]);
                last_load[ps] = j;
            }
        }
        // the last commit covers every MMA issued before it
        if (ok && issued >= 0 &&
            !tc::mbar_wait_bounded(&empty[issued % S], (uint32_t)(issued / S) & 1u, wait_iters))
            ok = false;
        if (!ok || issued != nk - 1) {
            bad = 1;
            atomicOr(err, 1);
            // loads and MMAs in flight finish before the block leaves (full bound)
            for (int st = 0; st < S; st++)
                if (last_load[st] >= 0)
                    tc::mbar_wait_bounded(&full[st], (uint32_t)(last_load[st] / S) & 1u, kWaitIters);
            if (issued >= 0) tc::mbar_wait_bounded(&empty[issued % S], (uint32_t)(issued / S) & 1u, kWaitIters);
        }
    }
    __syncthreads();
    tc::fence_after_sync();
    if (!bad) {
        const int row = m0 + 32 * w + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tbase + ((uint32_t)(32 * w) << 16) + (uint32_t)c0, v);
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int col = n0 + c0 + j;
                    if (col < N) {
                        float *p = C + (size_t)row * ldc + col;
                        *p = accumulate ? *p + v[j] : v[j];
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (w == 0) tc::tmem_dealloc(tbase, BN);
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static int g_encode_state = 0; // 0 unknown, 1 available, -1 not available

static bool tma_available()
{
    if (g_encode_state == 0) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && fn) {
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
            g_encode_state = 1;
        } else {
            cudaGetLastError();
            g_encode_state = -1;
        }
    }
    return g_encode_state == 1;
}

// rows x K BF16 matrix with row stride ld elements, tiles of box_rows x 64
static bool make_tile_map(CUtensorMap *m, const bf16 *p, int rows, int K, int ld, int box_rows)
{
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2u};
    const cuuint32_t box[2] = {(cuuint32_t)GT_K, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1u, 1u};
    return g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(p), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static bool g_gemm_attr = false;

void gemm_tc(const bf16 *A, int lda, const bf16 *B, int ldb, float *C, int ldc, int M, int N, int K, int accumulate,
             int *err, cudaStream_t s)
{
    if (!g_gemm_attr) {
        cudaFuncSetAttribute(k_gemm_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmShape<128>::SMEM);
        cudaFuncSetAttribute(k_gemm_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmShape<64>::SMEM);
        cudaFuncSetAttribute(k_gemm_tma<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, TmaShape<128>::SMEM);
        cudaFuncSetAttribute(k_gemm_tma<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, TmaShape<64>::SMEM);
        g_gemm_attr = true;
    }
    const int mt = (M + GT_M - 1) / GT_M;
    // 128-wide tiles when they give at least two tiles per SM, else 64-wide (twice the CTAs)
    const bool wide = (long long)mt * ((N + 127) / 128) >= 2 * 148;
    if (K >= GT_K && tma_available() && ((uintptr_t)A & 15u) == 0 && ((uintptr_t)B & 15u) == 0 && lda % 8 == 0 &&
        ldb % 8 == 0) {
        CUtensorMap ta, tb;
        if (make_tile_map(&ta, A, M, K, lda, GT_M) && make_tile_map(&tb, B, N, K, ldb, wide ? 128 : 64)) {
            if (wide) {
                dim3 g(mt, (N + 127) / 128);
                k_gemm_tma<128><<<g, 128, TmaShape<128>::SMEM, s>>>(ta, tb, C, ldc, M, N, K, accumulate, err,
                                                                    g_wait_iters);
            } else {
                dim3 g(mt, (N + 63) / 64);
                k_gemm_tma<64><<<g, 128, TmaShape<64>::SMEM, s>>>(ta, tb, C, ldc, M, N, K, accumulate, err,
                                                                  g_wait_iters);
            }
            return;
        }
    }
    if (wide) {
        dim3 g(mt, (N + 127) / 128);
        k_gemm_tc<128><<<g, 128, GemmShape<128>::SMEM, s>>>(A, lda, B, ldb, C, ldc, M, N, K, accumulate, err,
                                                            g_wait_iters);
    } else {
        dim3 g(mt, (N + 63) / 64);
        k_gemm_tc<64><<<g, 128, GemmShape<64>::SMEM, s>>>(A, lda, B, ldb, C, ldc, M, N, K, accumulate, err,
                                                          g_wait_iters);
    }
}

} // namespace lcmc

// Limit of the tensor-core kernels' bounded mbarrier waits, in tries, for
// launches made from now on (0 restores the default).  A wait that runs out
// sets the kernel's error flag, drains the MMAs in flight with the full bound,
// frees its TMEM and returns; the call reports LCMC_ETIMEOUT.  For tests of
// that path: a limit of 1 makes the first wait give up.
extern "C" int lcmc_set_wait_limit(unsigned int tries)
{
    lcmc::g_wait_iters = tries ? (uint32_t)tries : lcmc::kWaitIters;
    return LCMC_OK;
}

namespace lcmc {

// ---------------------------------------------------------------------------
// MLP kernels (FP32 CUDA cores)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z)
{
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Z += bias; H = silu(Z) (BF16, row-major B x H) and its transpose (H x B)
__global__ void k_bias_act(float *Z, const float *bias, bf16 *Hb, bf16 *HbT, float *Hf, int Bn, int Hn)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Bn * Hn; i += gridDim.x * blockDim.x) {
        const int b = i / Hn, h = i % Hn;
        const float z = Z[i] + bias[h];
        Z[i] = z;
        const float a = silu(z);
        const bf16 ab = __float2bfloat16(a);
        Hb[i] = ab;
        if (HbT) HbT[(size_t)h * Bn + b] = ab;
        if (Hf) Hf[i] = a;
    }
}

// y = A2 . w3 + b3 (warp per row); optionally dy = 2 (y - t) / n_valid for rows < n_valid
__global__ void k_out_layer(const float *A2, const float *w3, const float *b3, float *y, const float *target,
                            float *dy, float *loss, int Bn, int Hn, int n_valid)
{
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < Bn; r += (gridDim.x * blockDim.x) >> 5) {
        float s = 0.0f;
        for (int h = lane; h < Hn; h += 32) s += A2[(size_t)r * Hn + h] * w3[h];
        for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const float v = s + b3[0];
            y[r] = v;
            if (target) {
                const float e = r < n_valid ? v - target[r] : 0.0f;
                dy[r] = 2.0f * e / (float)n_valid;
                atomicAdd(loss, e * e / (float)n_valid);
            }
        }
    }
}

// dZ2 = (dy w3) * silu'(Z2); also dw3 += dy A2 (atomics), db3 += dy; writes dZ2 (B x H) and dZ2^T (H x B) in BF16
__global__ void k_back_out(const float *dy, const float *w3, const float *Z2, const float *A2, float *gw3, float *gb3,
                           bf16 *dZ2b, bf16 *dZ2bT, float *dZ2f, int Bn, int Hn)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Bn * Hn; i += gridDim.x * blockDim.x) {
        const int b = i / Hn, h = i % Hn;
        const float g = dy[b] * w3[h] * dsilu(Z2[i]);
        const bf16 gb = __float2bfloat16(g);
        dZ2b[i] = gb;
        dZ2bT[(size_t)h * Bn + b] = gb;
        dZ2f[i] = g;
        atomicAdd(&gw3[h], dy[b] * A2[i]);
        if (h == 0) atomicAdd(gb3, dy[b]);
    }
}

// dZ1 = dH1 * silu'(Z1) -> dZ1^T (H x B) in BF16; db1 accumulated
__global__ void k_back_hidden(const float *dH, const float *Z, bf16 *dZbT, float *gbias, int Bn, int Hn)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Bn * Hn; i += gridDim.x * blockDim.x) {
        const int b = i / Hn, h = i % Hn;
        const float g = dH[i] * dsilu(Z[i]);
        dZbT[(size_t)h * Bn + b] = __float2bfloat16(g);
        atomicAdd(&gbias[h], g);
    }
}

__global__ void k_colsum(const float *X, float *out, int Bn, int Hn)
{
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < Hn; h += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int b = 0; b < Bn; b++) s += X[(size_t)b * Hn + h];
        out[h] += s;
    }
}

// B x K (row-major BF16) -> K x B
__global__ void k_transpose_bf16(const bf16 *X, bf16 *XT, int Bn, int Kn)
{
    __shared__ bf16 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        if (r < Bn && c < Kn) tile[j][threadIdx.x] = X[(size_t)r * Kn + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = bx + j, c = by + threadIdx.x; // r: K index, c: B index
        if (r < Kn && c < Bn) XT[(size_t)r * Bn + c] = tile[threadIdx.x][j];
    }
}

__global__ void k_f32_to_bf16(const float *x, bf16 *y, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = __float2bfloat16(x[i]);
}

// W (rows x cols FP32) -> BF16 copy and BF16 transpose
__global__ void k_weights_bf16(const float *W, bf16 *Wb, bf16 *WbT, int rows, int cols)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * cols; i += gridDim.x * blockDim.x) {
        const int r = i / cols, c = i % cols;
        const bf16 v = __float2bfloat16(W[i]);
        Wb[i] = v;
        if (WbT) WbT[(size_t)c * rows + r] = v;
    }
}

// Adam (Kingma & Ba 2015), FP32 master weights
__global__ void k_adam(float *w, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

} // namespace lcmc

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace lcmc;

struct lcmc_mlp {
    int n_in = 0, k1 = 0, hid = 0, bmax = 0;
    cudaStream_t s = nullptr;
    // FP32 masters, Adam moments and gradients, in one block each
    float *W1 = nullptr, *b1 = nullptr, *W2 = nullptr, *b2 = nullptr, *w3 = nullptr, *b3 = nullptr;
    float *P = nullptr, *G = nullptr, *Mm = nullptr, *Vv = nullptr; // parameter / grad / moment blocks
    size_t np = 0;
    bf16 *W1b = nullptr, *W2b = nullptr, *W2bT = nullptr;
    // activations (bmax rows)
    bf16 *X = nullptr, *XT = nullptr, *H1 = nullptr, *H1T = nullptr, *H2 = nullptr, *dZ2 = nullptr, *dZ2T = nullptr,
         *dZ1T = nullptr;
    float *Xf = nullptr, *Z1 = nullptr, *Z2 = nullptr, *A2 = nullptr, *y = nullptr, *t = nullptr, *dy = nullptr,
          *dZ2f = nullptr, *dH1 = nullptr, *loss = nullptr;
    int *err = nullptr;
    long long step = 0;
    std::string msg;
};

static int mlp_fail(lcmc_mlp *m, const char *what, cudaError_t e)
{
    if (m) m->msg = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? LCMC_ENOMEM : LCMC_ECUDA;
}

extern "C" int lcmc_mlp_destroy(lcmc_mlp *m)
{
    if (!m) return LCMC_EINVAL;
    if (m->s) cudaStreamSynchronize(m->s);
    void *ptrs[] = {m->P, m->G, m->Mm, m->Vv, m->W1b, m->W2b, m->W2bT, m->X, m->XT, m->H1, m->H1T, m->H2, m->dZ2,
                    m->dZ2T, m->dZ1T, m->Xf, m->Z1, m->Z2, m->A2, m->y, m->t, m->dy, m->dZ2f, m->dH1, m->loss,
                    m->err};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
    return LCMC_OK;
}

// Weights: uniform(-a, a) with a = sqrt(6 / (fan_in + fan_out)) (Glorot & Bengio
// 2010), from Philox so that a seed fixes the network.
extern "C" int lcmc_mlp_create(int n_in, int hidden, int max_batch, uint64_t seed, lcmc_mlp **out)
{
    if (!out || n_in <= 0 || hidden != 128 || max_batch <= 0) return LCMC_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return LCMC_ENODEV;
    }
    lcmc_mlp *m = new lcmc_mlp();
    m->n_in = n_in;
    m->k1 = (n_in + 127) / 128 * 128;
    m->hid = hidden;
    m->bmax = (max_batch + 127) / 128 * 128;
    const int H = hidden, K1 = m->k1, B = m->bmax;
    m->np = (size_t)H * K1 + H + (size_t)H * H + H + H + 1;
    cudaError_t e = cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        lcmc_mlp_destroy(m);
        return LCMC_ECUDA;
    }
#define MA(ptr, bytes)                                                                                                \
    do {                                                                                                              \
        if ((e = cudaMalloc((void **)&(ptr), (bytes))) != cudaSuccess) {                                              \
            lcmc_mlp_destroy(m);                                                                                      \
            return LCMC_ENOMEM;                                                                                       \
        }                                                                                                             \
    } while (0)
    MA(m->P, m->np * 4);
    MA(m->G, m->np * 4);
    MA(m->Mm, m->np * 4);
    MA(m->Vv, m->np * 4);
    MA(m->W1b, (size_t)H * K1 * 2);
    MA(m->W2b, (size_t)H * H * 2);
    MA(m->W2bT, (size_t)H * H * 2);
    MA(m->X, (size_t)B * K1 * 2);
    MA(m->XT, (size_t)B * K1 * 2);
    MA(m->H1, (size_t)B * H * 2);
    MA(m->H1T, (size_t)B * H * 2);
    MA(m->H2, (size_t)B * H * 2);
    MA(m->dZ2, (size_t)B * H * 2);
    MA(m->dZ2T, (size_t)B * H * 2);
    MA(m->dZ1T, (size_t)B * H * 2);
    MA(m->Xf, (size_t)B * K1 * 4);
    MA(m->Z1, (size_t)B * H * 4);
    MA(m->Z2, (size_t)B * H * 4);
    MA(m->A2, (size_t)B * H * 4);
    MA(m->y, (size_t)B * 4);
    MA(m->t, (size_t)B * 4);
    MA(m->dy, (size_t)B * 4);
    MA(m->dZ2f, (size_t)B * H * 4);
    MA(m->dH1, (size_t)B * H * 4);
    MA(m->loss, 4);
    MA(m->err, 4);
#undef MA
    m->W1 = m->P;
    m->b1 = m->W1 + (size_t)H * K1;
    m->W2 = m->b1 + H;
    m->b2 = m->W2 + (size_t)H * H;
    m->w3 = m->b2 + H;
    m->b3 = m->w3 + H;
    std::vector<float> host(m->np, 0.0f);
    uint32_t key[2];
    seed_key(seed, key);
    auto uni = [&](size_t i, float a) {
        U4 o = draw(key, (uint32_t)(i & 0xFFFFFFFFu), 0xABCD0000ull + (i >> 32), 0x300u);
        return (float)((2.0 * u01(o.x) - 1.0) * a);
    };
    const float a1 = sqrtf(6.0f / (n_in + H)), a2 = sqrtf(6.0f / (2 * H)), a3 = sqrtf(6.0f / (H + 1));
    for (int h = 0; h < H; h++)
        for (int k = 0; k < n_in; k++) host[(size_t)h * K1 + k] = uni((size_t)h * K1 + k, a1); // padding stays 0
    const size_t o2 = (size_t)H * K1 + H;
    for (size_t i = 0; i < (size_t)H * H; i++) host[o2 + i] = uni(o2 + i, a2);
    const size_t o3 = o2 + (size_t)H * H + H;
    for (int h = 0; h < H; h++) host[o3 + h] = uni(o3 + h, a3);
    cudaMemcpy(m->P, host.data(), m->np * 4, cudaMemcpyHostToDevice);
    cudaMemsetAsync(m->Mm, 0, m->np * 4, m->s);
    cudaMemsetAsync(m->Vv, 0, m->np * 4, m->s);
    cudaMemsetAsync(m->X, 0, (size_t)B * K1 * 2, m->s);
    cudaMemsetAsync(m->Xf, 0, (size_t)B * K1 * 4, m->s);
    cudaMemsetAsync(m->err, 0, 4, m->s);
    k_weights_bf16<<<256, 256, 0, m->s>>>(m->W1, m->W1b, nullptr, H, K1);
    k_weights_bf16<<<64, 256, 0, m->s>>>(m->W2, m->W2b, m->W2bT, H, H);
    e = cudaStreamSynchronize(m->s);
    if (e != cudaSuccess) {
        lcmc_mlp_destroy(m);
        return LCMC_ECUDA;
    }
    *out = m;
    return LCMC_OK;
}

// forward on the B (multiple of 128) rows of m->X -> activations A2
static void mlp_forward_s(lcmc_mlp *m, int B, cudaStream_t s)
{
    const int H = m->hid, K1 = m->k1;
    gemm_tc(m->X, K1, m->W1b, K1, m->Z1, H, B, H, K1, 0, m->err, s);
    k_bias_act<<<(B * H + 255) / 256, 256, 0, s>>>(m->Z1, m->b1, m->H1, m->H1T, nullptr, B, H);
    gemm_tc(m->H1, H, m->W2b, H, m->Z2, H, B, H, H, 0, m->err, s);
    k_bias_act<<<(B * H + 255) / 256, 256, 0, s>>>(m->Z2, m->b2, m->H2, nullptr, m->A2, B, H);
}
static void mlp_forward(lcmc_mlp *m, int B) { mlp_forward_s(m, B, m->s); }

namespace lcmc {
// In-sweep inference: the sweep's kernels write the BF16 input rows into
// mlp_input() (leading dimension mlp_ld()), then the forward pass and the
// output layer run on the sweep's stream; returns the device output vector.
void *mlp_input(lcmc_mlp *m) { return m->X; }
int mlp_ld(lcmc_mlp *m) { return m->k1; }
int mlp_bmax(lcmc_mlp *m) { return m->bmax; }
int mlp_n_in(lcmc_mlp *m) { return m->n_in; }
const float *mlp_forward_device(lcmc_mlp *m, int B, cudaStream_t s)
{
    mlp_forward_s(m, B, s);
    k_out_layer<<<(B * 32 + 255) / 256, 256, 0, s>>>(m->A2, m->w3, m->b3, m->y, nullptr, nullptr, nullptr, B, m->hid,
                                                     B);
    return m->y;
}
int *mlp_err(lcmc_mlp *m) { return m->err; }
} // namespace lcmc

// rows of host features (n x n_in, FP32) -> m->X (BF16, padded to k1 columns, B rows)
static void load_batch(lcmc_mlp *m, const float *x, int n, int B)
{
    const int K1 = m->k1;
    cudaMemset2DAsync(m->Xf, (size_t)K1 * 4, 0, (size_t)K1 * 4, B, m->s);
    cudaMemcpy2DAsync(m->Xf, (size_t)K1 * 4, x, (size_t)m->n_in * 4, (size_t)m->n_in * 4, n, cudaMemcpyHostToDevice,
                      m->s);
    k_f32_to_bf16<<<512, 256, 0, m->s>>>(m->Xf, m->X, B * K1);
}

extern "C" int lcmc_mlp_predict(lcmc_mlp *m, const float *x, int n, float *y)
{
    if (!m || !x || !y || n < 0) return LCMC_EINVAL;
    for (int off = 0; off < n; off += m->bmax) {
        const int nb = n - off < m->bmax ? n - off : m->bmax;
        const int B = (nb + 127) / 128 * 128;
        load_batch(m, x + (size_t)off * m->n_in, nb, B);
        mlp_forward(m, B);
        k_out_layer<<<(B * 32 + 255) / 256, 256, 0, m->s>>>(m->A2, m->w3, m->b3, m->y, nullptr, nullptr, nullptr, B,
                                                             m->hid, nb);
        cudaMemcpyAsync(y + off, m->y, (size_t)nb * 4, cudaMemcpyDeviceToHost, m->s);
    }
    cudaError_t e = cudaStreamSynchronize(m->s);
    if (e != cudaSuccess) return mlp_fail(m, "predict", e);
    int err = 0;
    cudaMemcpy(&err, m->err, 4, cudaMemcpyDeviceToHost);
    return err ? LCMC_ETIMEOUT : LCMC_OK;
}

// Forward + backward on rows [0, n) of a host batch: gradients in m->G, MSE in m->loss.
static void mlp_backward(lcmc_mlp *m, const float *x, const float *t, int n);

// One Adam step on rows [0, n) of the given host batch; returns the batch MSE.
static int mlp_step(lcmc_mlp *m, const float *x, const float *t, int n, float lr, float *loss_out)
{
    const int H = m->hid, K1 = m->k1;
    mlp_backward(m, x, t, n);
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)m->step), c2 = 1.0f - powf(b2, (float)m->step);
    k_adam<<<512, 256, 0, m->s>>>(m->P, m->G, m->Mm, m->Vv, (int)m->np, lr, b1, b2, 1e-8f, c1, c2);
    // padding columns of W1 stay exactly zero: their gradient is zero (zero inputs)
    k_weights_bf16<<<256, 256, 0, m->s>>>(m->W1, m->W1b, nullptr, H, K1);
    k_weights_bf16<<<64, 256, 0, m->s>>>(m->W2, m->W2b, m->W2bT, H, H);
    if (loss_out) cudaMemcpyAsync(loss_out, m->loss, 4, cudaMemcpyDeviceToHost, m->s);
    return LCMC_OK;
}

static void mlp_backward(lcmc_mlp *m, const float *x, const float *t, int n)
{
    const int H = m->hid, K1 = m->k1;
    const int B = (n + 127) / 128 * 128;
    load_batch(m, x, n, B);
    cudaMemsetAsync(m->t, 0, (size_t)B * 4, m->s);
    cudaMemcpyAsync(m->t, t, (size_t)n * 4, cudaMemcpyHostToDevice, m->s);
    cudaMemsetAsync(m->G, 0, m->np * 4, m->s);
    cudaMemsetAsync(m->loss, 0, 4, m->s);
    mlp_forward(m, B);
    float *gW1 = m->G, *gb1 = gW1 + (size_t)H * K1, *gW2 = gb1 + H, *gb2 = gW2 + (size_t)H * H, *gw3 = gb2 + H,
          *gb3 = gw3 + H;
    k_out_layer<<<(B * 32 + 255) / 256, 256, 0, m->s>>>(m->A2, m->w3, m->b3, m->y, m->t, m->dy, m->loss, B, H, n);
    k_back_out<<<(B * H + 255) / 256, 256, 0, m->s>>>(m->dy, m->w3, m->Z2, m->A2, gw3, gb3, m->dZ2, m->dZ2T, m->dZ2f,
                                                      B, H);
    k_colsum<<<1, 128, 0, m->s>>>(m->dZ2f, gb2, B, H);
    // dW2 = dZ2^T H1: (H x B) . (H x B)^T
    gemm_tc(m->dZ2T, B, m->H1T, B, gW2, H, H, H, B, 0, m->err, m->s);
    // dH1 = dZ2 W2: (B x H) . (W2^T)^T
    gemm_tc(m->dZ2, H, m->W2bT, H, m->dH1, H, B, H, H, 0, m->err, m->s);
    k_back_hidden<<<(B * H + 255) / 256, 256, 0, m->s>>>(m->dH1, m->Z1, m->dZ1T, gb1, B, H);
    // dW1 = dZ1^T X: (H x B) . (X^T)^T with X^T = K1 x B
    dim3 tg((K1 + 31) / 32, (B + 31) / 32), tb(32, 8);
    k_transpose_bf16<<<tg, tb, 0, m->s>>>(m->X, m->XT, B, K1);
    gemm_tc(m->dZ1T, B, m->XT, B, gW1, K1, H, K1, B, 0, m->err, m->s);
}

extern "C" int lcmc_mlp_num_params(const lcmc_mlp *m) { return m ? (int)m->np : 0; }

extern "C" int lcmc_mlp_gradients(lcmc_mlp *m, const float *x, const float *t, int n, float *grad, float *loss)
{
    if (!m || !x || !t || !grad || n <= 0 || n > m->bmax) return LCMC_EINVAL;
    mlp_backward(m, x, t, n);
    cudaMemcpyAsync(grad, m->G, m->np * 4, cudaMemcpyDeviceToHost, m->s);
    if (loss) cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->s);
    cudaError_t e = cudaStreamSynchronize(m->s);
    if (e != cudaSuccess) return mlp_fail(m, "gradients", e);
    int err = 0;
    cudaMemcpy(&err, m->err, 4, cudaMemcpyDeviceToHost);
    return err ? LCMC_ETIMEOUT : LCMC_OK;
}

extern "C" int lcmc_mlp_get_params(lcmc_mlp *m, float *params)
{
    if (!m || !params) return LCMC_EINVAL;
    cudaError_t e = cudaMemcpy(params, m->P, m->np * 4, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LCMC_OK : mlp_fail(m, "get_params", e);
}

extern "C" int lcmc_mlp_set_params(lcmc_mlp *m, const float *params)
{
    if (!m || !params) return LCMC_EINVAL;
    cudaError_t e = cudaMemcpy(m->P, params, m->np * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return mlp_fail(m, "set_params", e);
    k_weights_bf16<<<256, 256, 0, m->s>>>(m->W1, m->W1b, nullptr, m->hid, m->k1);
    k_weights_bf16<<<64, 256, 0, m->s>>>(m->W2, m->W2b, m->W2bT, m->hid, m->hid);
    e = cudaStreamSynchronize(m->s);
    return e == cudaSuccess ? LCMC_OK : mlp_fail(m, "set_params", e);
}

extern "C" int lcmc_mlp_train(lcmc_mlp *m, const float *x, const float *t, int n, int epochs, int batch, float lr,
                              uint64_t seed, float *final_loss)
{
    if (!m || !x || !t || n <= 0 || epochs <= 0 || batch <= 0 || batch > m->bmax) return LCMC_EINVAL;
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::vector<float> bx((size_t)batch * m->n_in), bt(batch);
    uint32_t key[2];
    seed_key(seed, key);
    float last = 0.0f;
    for (int ep = 0; ep < epochs; ep++) {
        for (int i = n - 1; i > 0; i--) { // shuffle
            U4 o = draw(key, (uint32_t)i, (uint64_t)ep, 0x301u);
            int j = (int)(o.x % (uint32_t)(i + 1));
            int tmp = idx[i];
            idx[i] = idx[j];
            idx[j] = tmp;
        }
        double acc = 0.0;
        int nb = 0;
        for (int off = 0; off + batch <= n; off += batch) {
            for (int r = 0; r < batch; r++) {
                memcpy(&bx[(size_t)r * m->n_in], x + (size_t)idx[off + r] * m->n_in, sizeof(float) * m->n_in);
                bt[r] = t[idx[off + r]];
            }
            float l = 0.0f;
            mlp_step(m, bx.data(), bt.data(), batch, lr, &l);
            cudaError_t e = cudaStreamSynchronize(m->s);
            if (e != cudaSuccess) return mlp_fail(m, "train", e);
            acc += l;
            nb++;
        }
        last = nb ? (float)(acc / nb) : 0.0f;
    }
    int err = 0;
    cudaMemcpy(&err, m->err, 4, cudaMemcpyDeviceToHost);
    if (final_loss) *final_loss = last;
    return err ? LCMC_ETIMEOUT : LCMC_OK;
}

// C[M x N] = A[M x K] B[N x K]^T on the tensor cores, host arrays (test hook).
extern "C" int lcmc_gemm_bf16(const float *A, const float *B, float *C, int M, int N, int K)
{
    if (!A || !B || !C || M <= 0 || N <= 0 || K <= 0 || K % 64) return LCMC_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return LCMC_ENODEV;
    }
    float *fa, *fb, *fc;
    bf16 *ba, *bb;
    int *err;
    if (cudaMalloc(&fa, (size_t)M * K * 4) || cudaMalloc(&fb, (size_t)N * K * 4) ||
        cudaMalloc(&fc, (size_t)M * N * 4) || cudaMalloc(&ba, (size_t)M * K * 2) ||
        cudaMalloc(&bb, (size_t)N * K * 2) || cudaMalloc(&err, 4))
        return LCMC_ENOMEM;
    cudaMemcpy(fa, A, (size_t)M * K * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(fb, B, (size_t)N * K * 4, cudaMemcpyHostToDevice);
    cudaMemset(err, 0, 4);
    k_f32_to_bf16<<<256, 256>>>(fa, ba, M * K);
    k_f32_to_bf16<<<256, 256>>>(fb, bb, N * K);
    gemm_tc(ba, K, bb, K, fc, N, M, N, K, 0, err, 0);
    cudaError_t e = cudaMemcpy(C, fc, (size_t)M * N * 4, cudaMemcpyDeviceToHost);
    int herr = 0;
    cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    cudaFree(fa);
    cudaFree(fb);
    cudaFree(fc);
    cudaFree(ba);
    cudaFree(bb);
    cudaFree(err);
    if (e != cudaSuccess) return LCMC_ECUDA;
    return herr ? LCMC_ETIMEOUT : LCMC_OK;
}
