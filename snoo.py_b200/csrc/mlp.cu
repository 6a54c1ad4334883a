// Dense kernels of the warm-start surrogate (an MLP on POD coefficients): a BF16 GEMM on the
// 5th-generation tensor cores (tcgen05.mma, FP32 accumulator in tensor memory) with a fused
// bias / GELU epilogue, and the element-wise kernels of its training step.
//
// GEMM  C[M,N] = A[M,K] . B[N,K]^T  (+ bias[N]),  A and B row-major BF16 with K contiguous.
// One CTA of 128 threads computes a 128 x NT tile (NT <= 256, a multiple of 16): K is walked
// in chunks of 64; each chunk of A (128 x 64) and B (NT x 64) is copied into shared memory in
// the no-swizzle K-major layout the MMA reads (8-row x 16-byte core matrices: element (r, k)
// of a chunk at ((k / 8) * (rows / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2 bytes), then
// one thread issues four 128 x NT x 16 MMAs and commits them to an mbarrier that every thread
// waits on.  The epilogue reads the accumulator back with tcgen05.ld (warp w owns TMEM lanes
// 32w .. 32w+31 = tile rows) and writes FP32 C and/or BF16 act(C).
//
// Every wait on the mbarrier is bounded: after kMaxSpin polls the CTA records an error in
// *err (a device flag the caller reads when it synchronises), stops issuing work, frees its
// tensor memory and returns.  The kernel asks for more
// than half of an SM's shared memory, so one CTA (holding 256 TMEM columns) runs per SM and
// the allocation never waits on another CTA.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>

#include "snp_common.cuh"
#include "snp_internal.cuh"

namespace snp {

namespace {

constexpr int kGemmThreads = 128;
constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr int kMaxNT = 256;
constexpr int kTmemCols = 256;
constexpr size_t kGemmSmem = 120 * 1024;  // > half of the SM: one CTA per SM
constexpr long long kMaxSpin = 1ll << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: no swizzle, K-major canonical layout.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int m, int n) {
    return (1u << 4)                      // accumulator F32
           | (1u << 7)                    // A BF16
           | (1u << 10)                   // B BF16
           | ((uint32_t)(n >> 3) << 17)   // N / 8
           | ((uint32_t)(m >> 4) << 24);  // M / 16
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kMaxSpin; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

// Copy rows [r0, r0 + rows) x K-chunk [k0, k0 + 64) of a row-major BF16 matrix (ld elements,
// rows_total x k_total) into the canonical layout; out-of-range elements become zero.
__device__ __forceinline__ void load_chunk(uint8_t *dst, const __nv_bfloat16 *src, int ld, int r0, int rows,
                                           int rows_total, int k0, int k_total) {
    const int vecs = rows * (kChunkK / 8);
    for (int v = threadIdx.x; v < vecs; v += kGemmThreads) {
        const int r = v / (kChunkK / 8);
        const int kc = v - r * (kChunkK / 8);
        const int gr = r0 + r, gk = k0 + 8 * kc;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (gr < rows_total && gk < k_total)  // k_total is a multiple of 8 (checked on the host)
            val = *reinterpret_cast<const uint4 *>(src + (int64_t)gr * ld + gk);
        *reinterpret_cast<uint4 *>(dst + (kc * (rows / 8) + r / 8) * 128 + (r % 8) * 16) = val;
    }
}

// C (float32) and H (BF16) rows accept whole 16-byte stores: both 16-byte aligned, ldc a multiple
// of 4 floats, ldh a multiple of 8 BF16 (every row then starts on a 16-byte boundary).
__device__ __forceinline__ bool vector_stores_ok(const float *C, int ldc, const __nv_bfloat16 *H, int ldh) {
    return (C == nullptr || ((reinterpret_cast<uintptr_t>(C) & 15) == 0 && (ldc & 3) == 0)) &&
           (H == nullptr || ((reinterpret_cast<uintptr_t>(H) & 15) == 0 && (ldh & 7) == 0));
}

// Epilogue of eight accumulator columns col0 .. col0 + 7 of one row: z = acc + bias, C = z,
// H = BF16(GELU(z)) (act 1) or BF16(z); one thread's eight values as two 16-byte stores into C
// and one into H when the row allows it (every 32-byte sector written whole), else one by one.
__device__ __forceinline__ void store_row8(const uint32_t (&v)[8], int row, int col0, int N, const float *bias,
                                           int act, float *C, int ldc, __nv_bfloat16 *H, int ldh, bool vec_ok) {
    float z[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        z[j] = __uint_as_float(v[j]);
        if (bias && col0 + j < N) z[j] += bias[col0 + j];
    }
    if (vec_ok && col0 + 8 <= N && (col0 & 7) == 0) {
        if (C) {
            float4 *cp = reinterpret_cast<float4 *>(C + (int64_t)row * ldc + col0);
            cp[0] = make_float4(z[0], z[1], z[2], z[3]);
            cp[1] = make_float4(z[4], z[5], z[6], z[7]);
        }
        if (H) {
            uint32_t hw[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat16 lo = __float2bfloat16_rn(act == 1 ? gelu(z[2 * j]) : z[2 * j]);
                const __nv_bfloat16 hi = __float2bfloat16_rn(act == 1 ? gelu(z[2 * j + 1]) : z[2 * j + 1]);
                hw[j] = (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
            }
            *reinterpret_cast<uint4 *>(H + (int64_t)row * ldh + col0) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int col = col0 + j;
        if (col < N) {
            if (C) C[(int64_t)row * ldc + col] = z[j];
            if (H) H[(int64_t)row * ldh + col] = __float2bfloat16_rn(act == 1 ? gelu(z[j]) : z[j]);
        }
    }
}

__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_bf16(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, int lda,
                const __nv_bfloat16 *__restrict__ B, int ldb, const float *__restrict__ bias, int act,
                float *__restrict__ C, int ldc, __nv_bfloat16 *__restrict__ H, int ldh, int nt, int *err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base_slot;
    __shared__ int failed;
    uint8_t *sa = smem;                                  // 128 x 64 BF16 = 16 KiB
    uint8_t *sb = smem + kTileM * kChunkK * 2;           // nt x 64 BF16 <= 32 KiB
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * nt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
        failed = 0;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_slot;
    const uint32_t idesc = instr_desc_bf16(kTileM, nt);
    const uint32_t bar_addr = smem_u32(&bar);
    const int n_chunks = (K + kChunkK - 1) / kChunkK;

    for (int c = 0; c < n_chunks; ++c) {
        load_chunk(sa, A, lda, m0, kTileM, M, c * kChunkK, K);
        load_chunk(sb, B, ldb, n0, nt, N, c * kChunkK, K);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int s = 0; s < kChunkK / 16; ++s) {
                // MMA step s covers k-chunks 2s and 2s+1 of 8 elements each
                const uint64_t da = smem_desc(a0 + 2 * s * (kTileM / 8) * 128, (kTileM / 8) * 128, 128);
                const uint64_t db = smem_desc(b0 + 2 * s * (nt / 8) * 128, (nt / 8) * 128, 128);
                const uint32_t accumulate = (c > 0 || s > 0) ? 1u : 0u;
                const uint32_t no_mask = 0u;  // disable-output-lane mask: every lane written
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(no_mask));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_addr)
                         : "memory");
        }
        // every thread waits for the chunk's MMAs before the buffers are refilled
        if (!mbar_wait(bar_addr, (uint32_t)(c & 1))) atomicExch(&failed, 1);
        __syncthreads();
        if (failed) break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");

    if (!failed) {
        const int row = m0 + 32 * warp + lane;
        const bool vec_ok = vector_stores_ok(C, ldc, H, ldh);
        for (int c8 = 0; c8 < nt / 8; ++c8) {
            uint32_t v[8];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(8 * c8);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) store_row8(v, row, n0 + 8 * c8, N, bias, act, C, ldc, H, ldh, vec_ok);
        }
    } else if (threadIdx.x == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// The same GEMM with its operands brought in by the Tensor Memory Accelerator and two
// shared-memory stages: thread 0 issues, per 64-wide K chunk, eight 2-D TMA tile loads for A
// (box 8 x 128: one 16-byte K group of 128 rows, which lands exactly as one K group of the
// no-swizzle K-major layout) and eight for B (box 8 x nt), all completing on the stage's
// mbarrier (expect-tx bytes); the MMAs of chunk c run while chunk c + 1 is in flight, and the
// stage is refilled with chunk c + 2 once the commit of chunk c's MMAs has arrived.  Rows or K
// columns beyond the matrix are zero-filled by the TMA unit.  Every wait is bounded; after a
// timeout the CTA records the error, waits (bounded) for the copies and MMAs it issued, frees
// its tensor memory and returns.  The tensor maps cover this GPU's own memory only and no load
// uses multicast.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_bf16_tma(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, int M, int N,
                    int K, const float *__restrict__ bias, int act, float *__restrict__ C, int ldc,
                    __nv_bfloat16 *__restrict__ H, int ldh, int nt, int *err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[2], mma_done[2];
    __shared__ uint32_t tmem_base_slot;
    __shared__ int failed;
    const int stage_a = kTileM * kChunkK * 2;  // 16 KiB
    const int stage_b = kMaxNT * kChunkK * 2;  // 32 KiB (nt rows used)
    // stage s: A at s * (stage_a + stage_b), B right after it
    const uint32_t s_base = smem_u32(smem);
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * nt;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tx_bytes = (uint32_t)(kTileM + nt) * kChunkK * 2;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mma_done[s])), "r"(1));
        }
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
        failed = 0;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_slot;
    const uint32_t idesc = instr_desc_bf16(kTileM, nt);
    const int n_chunks = (K + kChunkK - 1) / kChunkK;

    // chunk c -> stage c % 2: eight K groups of A and of B
    auto issue = [&](int c) {
        const int s = c & 1;
        const uint32_t bar = smem_u32(&full[s]);
        mbar_expect_tx(bar, tx_bytes);
#pragma unroll
        for (int kc = 0; kc < kChunkK / 8; ++kc) {
            const int x = c * kChunkK + 8 * kc;  // a multiple of 8 BF16 elements (16 bytes)
            const uint32_t a_s = s_base + (uint32_t)(s * (stage_a + stage_b));
            tma_load_2d(a_s + kc * kTileM * 16, &map_a, x, m0, bar);
            tma_load_2d(a_s + stage_a + kc * nt * 16, &map_b, x, n0, bar);
        }
    };
    int issued = 0, mma_issued = 0;  // (thread 0's counts)
    if (threadIdx.x == 0) {
        for (; issued < 2 && issued < n_chunks; ++issued) issue(issued);
    }
    for (int c = 0; c < n_chunks; ++c) {
        const int s = c & 1;
        const uint32_t ph = (uint32_t)((c >> 1) & 1);
        if (threadIdx.x == 0) {
            bool ok = mbar_wait(smem_u32(&full[s]), ph);
            if (ok) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t a0 = s_base + (uint32_t)(s * (stage_a + stage_b)), b0 = a0 + stage_a;
#pragma unroll
                for (int st = 0; st < kChunkK / 16; ++st) {
                    const uint64_t da = smem_desc(a0 + 2 * st * (kTileM / 8) * 128, (kTileM / 8) * 128, 128);
                    const uint64_t db = smem_desc(b0 + 2 * st * (nt / 8) * 128, (nt / 8) * 128, 128);
                    const uint32_t accumulate = (c > 0 || st > 0) ? 1u : 0u;
                    const uint32_t no_mask = 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(no_mask));
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                        smem_u32(&mma_done[s]))
                    : "memory");
                mma_issued = c + 1;
                // refill this stage with chunk c + 2 once these MMAs have read it
                if (c + 2 < n_chunks) {
                    ok = mbar_wait(smem_u32(&mma_done[s]), ph);
                    if (ok) {
                        issue(c + 2);
                        issued = c + 3;
                    }
                }
            }
            if (!ok) failed = 1;
        }
        __syncthreads();
        if (failed) break;
    }
    // the last chunk's MMAs (commits arrive in order, so the last one covers all)
    if (!failed && threadIdx.x == 0) {
        const int c = n_chunks - 1;
        if (!mbar_wait(smem_u32(&mma_done[c & 1]), (uint32_t)((c >> 1) & 1))) failed = 1;
    }
    __syncthreads();
    if (failed && threadIdx.x == 0) {
        // bounded drain of what this CTA still has in flight before the memory goes away
        for (int c = 0; c < issued; ++c)
            if (c >= mma_issued) mbar_wait(smem_u32(&full[c & 1]), (uint32_t)((c >> 1) & 1));
        if (mma_issued > 0) {
            const int c = mma_issued - 1;
            mbar_wait(smem_u32(&mma_done[c & 1]), (uint32_t)((c >> 1) & 1));
        }
        atomicExch(err, 1);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!failed) {
        const int row = m0 + 32 * warp + lane;
        const bool vec_ok = vector_stores_ok(C, ldc, H, ldh);
        for (int c8 = 0; c8 < nt / 8; ++c8) {
            uint32_t v[8];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(8 * c8);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) store_row8(v, row, n0 + 8 * c8, N, bias, act, C, ldc, H, ldh, vec_ok);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// dZ = dH * GELU'(Z) (FP32 in, BF16 out for the next GEMMs, FP32 copy optional)
__global__ void k_gelu_backward(int64_t count, const float *__restrict__ dH, const float *__restrict__ Z,
                                __nv_bfloat16 *__restrict__ dZb, float *__restrict__ dZf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const float z = Z[i];
        const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
        const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
        const float g = dH[i] * (cdf + z * pdf);
        if (dZb) dZb[i] = __float2bfloat16_rn(g);
        if (dZf) dZf[i] = g;
    }
}

// out[c, r] = in[r, c] (BF16, rows x cols -> cols x rows, ld = row length)
__global__ void k_transpose_bf16(int rows, int cols, const __nv_bfloat16 *__restrict__ in, int ldi,
                                 __nv_bfloat16 *__restrict__ out, int ldo) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = r0 + j, c = c0 + threadIdx.x;
        tile[j][threadIdx.x] = (r < rows && c < cols) ? in[(int64_t)r * ldi + c] : __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = c0 + j, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[(int64_t)c * ldo + r] = tile[threadIdx.x][j];
    }
}

// column sums of a rows x cols FP32 matrix (bias gradients), one block per column group
__global__ void k_col_sum(int rows, int cols, const float *__restrict__ in, int ld, float *__restrict__ out) {
    __shared__ float sh[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float s = 0.f;
    if (c < cols)
        for (int r = threadIdx.y; r < rows; r += blockDim.y) s += in[(int64_t)r * ld + c];
    sh[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float t = 0.f;
        for (int j = 0; j < (int)blockDim.y; ++j) t += sh[j][threadIdx.x];
        out[c] = t;
    }
}

// Adam step on FP32 master weights, refreshing their BF16 copy.
__global__ void k_adam(int64_t count, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, __nv_bfloat16 *__restrict__ wb, float lr, float b1, float b2, float eps,
                       float bc1, float bc2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

// Mean-squared-error gradient dY = scale * (Y - T) with a BF16 copy (the next GEMMs' input).
__global__ void k_mse_grad(int64_t count, const float *__restrict__ Y, const float *__restrict__ T, float scale,
                           float *__restrict__ dY, __nv_bfloat16 *__restrict__ dYb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const float g = scale * (Y[i] - T[i]);
        dY[i] = g;
        if (dYb) dYb[i] = __float2bfloat16_rn(g);
    }
}

__global__ void k_f32_to_bf16(int64_t count, const float *__restrict__ a, __nv_bfloat16 *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16_rn(a[i]);
}

}  // namespace

}  // namespace snp

// out[p][i] = mean[i] + sum_c V[i][c] coef[p][c]: one warp per row i of V (lanes over the m
// columns, the row read once for all P vectors), float64 products and a fixed shuffle tree;
// the coefficients of all P vectors staged in shared memory.
namespace snp {

// Tensor map of a row-major BF16 matrix [rows][ld] with K contiguous, read in boxes of one
// 16-byte K group (8 elements) by box_rows rows: the K-major no-swizzle group layout of the
// tcgen05 operands.  Out-of-range boxes are zero-filled.  cuTensorMapEncodeTiled comes from
// the driver through the runtime's entry-point query (no link to libcuda).
int encode_kmajor_map(CUtensorMap *map, const void *base, int K, int rows, int ld, int box_rows) {
    using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeFn encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SNP_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        SNP_REQUIRE(q == cudaDriverEntryPointSuccess && fn, "cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<EncodeFn>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {8u, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    SNP_REQUIRE(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return SNP_OK;
}

namespace {
constexpr int kCombineMaxM = 128;
constexpr int kCombineMaxP = 32;
__global__ void __launch_bounds__(256)
    k_basis_combine(int32_t n, const float *__restrict__ V, int m, int64_t ldv, const double *__restrict__ coef,
                    int P, const double *__restrict__ mean, double *__restrict__ out, int64_t ldo) {
    __shared__ double sc[kCombineMaxP * kCombineMaxM];
    for (int t = threadIdx.x; t < P * m; t += blockDim.x) sc[t] = coef[t];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        double v[kCombineMaxM / 32];
#pragma unroll
        for (int k = 0; k < kCombineMaxM / 32; ++k) {
            const int c = lane + 32 * k;
            v[k] = c < m ? (double)__ldcs(V + i * ldv + c) : 0.0;
        }
        const double base = mean ? mean[i] : 0.0;
        for (int p = 0; p < P; ++p) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < kCombineMaxM / 32; ++k) {
                const int c = lane + 32 * k;
                if (c < m) acc = fma(v[k], sc[p * m + c], acc);
            }
            acc = warp_sum(acc);
            if (lane == 0) out[(int64_t)p * ldo + i] = base + acc;
        }
    }
}
}  // namespace
}  // namespace snp

extern "C" {

// Reconstruction of P vectors from coefficients in a basis (the POD reconstruction of the
// warm start): out[p][i] = mean[i] + sum_c V[i][c] coef[p][c].
int snp_basis_combine(int32_t n, const float *V, int32_t m, int64_t ldv, const double *coef, int32_t P,
                      const double *mean, double *out, int64_t ldo, void *stream) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(n >= 0 && m >= 1 && m <= kCombineMaxM && P >= 1 && P <= kCombineMaxP && ldv >= m && ldo >= n,
                "snp_basis_combine: need 1 <= m <= %d, 1 <= P <= %d, ldv >= m, ldo >= n", kCombineMaxM, kCombineMaxP);
    SNP_REQUIRE(V && coef && out, "snp_basis_combine: NULL argument");
    if (n == 0) return SNP_OK;
    cudaStream_t st = as_stream(stream);
    k_basis_combine<<<stride_grid(32 * (int64_t)n, 256, 8), 256, 0, st>>>(n, V, m, ldv, coef, P, mean, out, ldo);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_gemm_bf16(int32_t M, int32_t N, int32_t K, const void *A, int32_t lda, const void *B, int32_t ldb,
                  const float *bias, int32_t act, float *C, int32_t ldc, void *H, int32_t ldh, int32_t *err,
                  void *stream) {
    snp::clear_error();
    SNP_REQUIRE(M >= 0 && N >= 0 && K >= 0, "snp_gemm_bf16: negative size");
    if (M == 0 || N == 0) return SNP_OK;
    SNP_REQUIRE(A && B && err, "snp_gemm_bf16: A, B or err is NULL");
    SNP_REQUIRE(C || H, "snp_gemm_bf16: no output (C and H are NULL)");
    SNP_REQUIRE(K % 8 == 0 && K > 0, "snp_gemm_bf16: K = %d must be a positive multiple of 8 (pad with zeros)", K);
    SNP_REQUIRE(lda % 8 == 0 && ldb % 8 == 0 && lda >= K && ldb >= K,
                "snp_gemm_bf16: lda/ldb must be multiples of 8 and >= K");
    SNP_REQUIRE(((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0, "snp_gemm_bf16: A and B must be 16-byte aligned");
    SNP_REQUIRE(!C || ldc >= N, "snp_gemm_bf16: ldc < N");
    SNP_REQUIRE(!H || ldh >= N, "snp_gemm_bf16: ldh < N");
    SNP_REQUIRE(act == 0 || act == 1, "snp_gemm_bf16: act must be 0 (none) or 1 (GELU)");
    // N tile: the whole N when it fits, else 256-wide tiles (both multiples of 16)
    const int nt = N <= snp::kMaxNT ? ((N + 15) / 16) * 16 : snp::kMaxNT;
    cudaStream_t s = snp::as_stream(stream);
    dim3 grid((M + snp::kTileM - 1) / snp::kTileM, (N + nt - 1) / nt);
    const char *env = getenv("SNP_GEMM_TMA");
    if (!(env && env[0] == '0')) {
        CUtensorMap ma, mb;
        SNP_TRY(snp::encode_kmajor_map(&ma, A, K, M, lda, snp::kTileM));
        SNP_TRY(snp::encode_kmajor_map(&mb, B, K, N, ldb, nt));
        SNP_CUDA_TRY(cudaFuncSetAttribute(snp::k_gemm_bf16_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)snp::kGemmSmem));
        snp::k_gemm_bf16_tma<<<grid, snp::kGemmThreads, snp::kGemmSmem, s>>>(
            ma, mb, M, N, K, bias, act, C, ldc, static_cast<__nv_bfloat16 *>(H), ldh, nt, err);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }
    SNP_CUDA_TRY(cudaFuncSetAttribute(snp::k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)snp::kGemmSmem));
    snp::k_gemm_bf16<<<grid, snp::kGemmThreads, snp::kGemmSmem, s>>>(
        M, N, K, static_cast<const __nv_bfloat16 *>(A), lda, static_cast<const __nv_bfloat16 *>(B), ldb, bias, act, C,
        ldc, static_cast<__nv_bfloat16 *>(H), ldh, nt, err);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_gelu_backward(int64_t count, const float *dH, const float *Z, void *dZ_bf16, float *dZ_f32, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(count >= 0 && dH && Z && (dZ_bf16 || dZ_f32), "snp_gelu_backward: bad arguments");
    if (count == 0) return SNP_OK;
    snp::k_gelu_backward<<<snp::stride_grid(count, 256, 8), 256, 0, snp::as_stream(stream)>>>(
        count, dH, Z, static_cast<__nv_bfloat16 *>(dZ_bf16), dZ_f32);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_transpose_bf16(int32_t rows, int32_t cols, const void *in, int32_t ldi, void *out, int32_t ldo, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(rows >= 0 && cols >= 0 && in && out && ldi >= cols && ldo >= rows, "snp_transpose_bf16: bad arguments");
    if (rows == 0 || cols == 0) return SNP_OK;
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    snp::k_transpose_bf16<<<grid, block, 0, snp::as_stream(stream)>>>(
        rows, cols, static_cast<const __nv_bfloat16 *>(in), ldi, static_cast<__nv_bfloat16 *>(out), ldo);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_col_sum(int32_t rows, int32_t cols, const float *in, int32_t ld, float *out, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(rows >= 0 && cols >= 0 && in && out && ld >= cols, "snp_col_sum: bad arguments");
    if (cols == 0) return SNP_OK;
    dim3 grid((cols + 31) / 32), block(32, 8);
    snp::k_col_sum<<<grid, block, 0, snp::as_stream(stream)>>>(rows, cols, in, ld, out);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_adam_step(int64_t count, float *w, const float *g, float *m, float *v, void *w_bf16, float lr, float beta1,
                  float beta2, float eps, int32_t step, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(count >= 0 && w && g && m && v && step >= 1, "snp_adam_step: bad arguments");
    if (count == 0) return SNP_OK;
    const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
    snp::k_adam<<<snp::stride_grid(count, 256, 8), 256, 0, snp::as_stream(stream)>>>(
        count, w, g, m, v, static_cast<__nv_bfloat16 *>(w_bf16), lr, beta1, beta2, eps, bc1, bc2);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_mse_grad(int64_t count, const float *Y, const float *T, float scale, float *dY, void *dY_bf16, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(count >= 0 && Y && T && dY, "snp_mse_grad: bad arguments");
    if (count == 0) return SNP_OK;
    snp::k_mse_grad<<<snp::stride_grid(count, 256, 8), 256, 0, snp::as_stream(stream)>>>(
        count, Y, T, scale, dY, static_cast<__nv_bfloat16 *>(dY_bf16));
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_f32_to_bf16(int64_t count, const float *in, void *out, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(count >= 0 && in && out, "snp_f32_to_bf16: bad arguments");
    if (count == 0) return SNP_OK;
    snp::k_f32_to_bf16<<<snp::stride_grid(count, 256, 8), 256, 0, snp::as_stream(stream)>>>(
        count, in, static_cast<__nv_bfloat16 *>(out));
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

}  // extern "C"
