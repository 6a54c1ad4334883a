// Device arithmetic of the matrix-free Newton Jacobian shared by the single-problem solver
// (elem_krylov.cu) and the batched solver (batch.cu): the same rounded expressions wherever
// an element product, a CG direction or a block-Jacobi block is formed, so both give the
// same values for the same inputs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "snp_internal.cuh"
#include "snp_krylov.cuh"
#include "snp_reduce.cuh"

namespace snp {

constexpr uint32_t kSignBit = 0x80000000u;  // edof / incidence words: the edge function is negated
constexpr int kBjMax = kBlockJacobiMax;     // DoFs per block-Jacobi block
constexpr int kBjTile = 256;                // blocks never cross a multiple of this many DoFs

// p = z + beta p_old, rounded the same way wherever it is formed
__device__ __forceinline__ double pnext(double beta, double p_old, double z) { return __fma_rn(beta, p_old, z); }
__device__ __forceinline__ float pnext(float beta, float p_old, float z) { return __fmaf_rn(beta, p_old, z); }

// Edge term s chat_k . v of one element edge, rounded the same way wherever it is formed.
template <typename TT>
__device__ __forceinline__ TT edge_term(const TT *sc, int k, bool neg, TT v0, TT v1, TT v2) {
    TT c;
    if constexpr (sizeof(TT) == 8)
        c = __fma_rn(sc[3 * k + 2], v2, __fma_rn(sc[3 * k + 1], v1, __dmul_rn(sc[3 * k], v0)));
    else
        c = __fmaf_rn(sc[3 * k + 2], v2, __fmaf_rn(sc[3 * k + 1], v1, __fmul_rn(sc[3 * k], v0)));
    return neg ? -c : c;
}

// z_i = sum over DoF i's block of M_ij r_j, r of the tile in shared memory (t = DoF - tile base);
// a, b: DoF i's row of the block inverse, loaded before the tile's barrier
template <typename TT>
__device__ __forceinline__ TT bj_row(unsigned mt, float4 a, float4 b, const TT *s_r, int t) {
    const float m[kBjMax] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    const int size = (int)(mt >> 8);
    const TT *rb = s_r + (t - (int)(mt & 0xffu));
    TT z = TT(0);
#pragma unroll
    for (int c = 0; c < kBjMax; ++c)
        if (c < size) z = fma((TT)m[c], rb[c], z);
    return z;
}

// asks L1 for DoF i's block row ahead of the tile barrier, holding no registers
__device__ __forceinline__ void bj_prefetch(const float *__restrict__ binv, int64_t i) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(binv + i * kBjMax));
}

__device__ __forceinline__ void bj_load(const float *__restrict__ binv, int64_t i, float4 &a, float4 &b) {
    const float4 *p = reinterpret_cast<const float4 *>(binv + i * kBjMax);
    a = __ldg(p);
    b = __ldg(p + 1);
}

// DoF i's row of its block of J (block columns 0..size-1, the rest 0), summed over the DoF's
// incidence list in order: for each incident (element, edge k) the element block's entries
// J_e,k k2 = s_k s_k2 chat_k . S_e chat_k2 of the element's edges k2 inside the block.
// sc: the reference curls (orientation 0) in shared memory.
template <typename TT>
__device__ __forceinline__ void bj_entries_row(int64_t i, const int32_t *__restrict__ inc_ptr,
                                               const int32_t *__restrict__ inc, const int32_t *__restrict__ edof,
                                               const TT *__restrict__ T, const double *sc, unsigned mt,
                                               double (&row)[kBjMax]) {
    const int64_t b0 = i - (int64_t)(mt & 0xffu);
    const int size = (int)(mt >> 8);
    for (int t = inc_ptr[i]; t < inc_ptr[i + 1]; ++t) {
        const uint32_t u = (uint32_t)inc[t];
        const uint32_t ek = u & ~kSignBit;
        const int k = (int)(ek & 7u);
        const int64_t eb = eslot((int64_t)(ek >> 3), 0);
        double tt[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) tt[c] = (double)T[eb + 32 * c];
        const double c0 = sc[3 * k], c1 = sc[3 * k + 1], c2 = sc[3 * k + 2];
        const double v0 = tt[0] * c0 + tt[1] * c1 + tt[2] * c2;
        const double v1 = tt[1] * c0 + tt[3] * c1 + tt[4] * c2;
        const double v2 = tt[2] * c0 + tt[4] * c1 + tt[5] * c2;
#pragma unroll
        for (int k2 = 0; k2 < 6; ++k2) {
            const uint32_t d2 = (uint32_t)edof[eb + 32 * k2];
            const int64_t r = (int64_t)(d2 & ~kSignBit) - b0;
            if (r < 0 || r >= size) continue;
            double val = sc[3 * k2] * v0 + sc[3 * k2 + 1] * v1 + sc[3 * k2 + 2] * v2;
            if ((u ^ d2) & kSignBit) val = -val;
#pragma unroll
            for (int c = 0; c < kBjMax; ++c)
                if (c == r) row[c] += val;
        }
    }
}

// Inverse of the block that starts at DoF i (size DoFs, rows in bmat[i..i+size)[kBjMax]):
// Cholesky of the block (upper triangle of its rows), padded to 8 x 8 with the identity so that
// every loop unrolls with fixed indices (registers, no local arrays); the lower triangle of the
// inverse is written to both sides (symmetric by construction), rounded to float32.  Point
// Jacobi (and one count in *n_fallback) for a block whose pivot is not positive enough; fr:
// the block's first DoF is free.
__device__ __forceinline__ void bj_invert_block(int64_t i, int size, bool fr, const uint8_t *__restrict__ free_mask,
                                                const double *__restrict__ bmat, float *__restrict__ binv,
                                                int *n_fallback) {
    double L[kBjMax][kBjMax], d0[kBjMax], rl[kBjMax];
#pragma unroll
    for (int r = 0; r < kBjMax; ++r) {
#pragma unroll
        for (int c = 0; c < kBjMax; ++c) {
            double v = r == c ? 1.0 : 0.0;
            if (r < size && c < size) v = c >= r ? bmat[(i + r) * kBjMax + c] : bmat[(i + c) * kBjMax + r];
            L[r][c] = v;
        }
        d0[r] = L[r][r];
    }
    bool ok = fr;
#pragma unroll
    for (int j = 0; j < kBjMax; ++j) {
        double p = L[j][j];
#pragma unroll
        for (int k = 0; k < j; ++k) p -= L[j][k] * L[j][k];
        if (!(p > 1e-12 * d0[j]) || !isfinite(p)) {
            ok = false;
            p = 1.0;
        }
        const double ljj = sqrt(p);
        L[j][j] = ljj;
        rl[j] = 1.0 / ljj;
#pragma unroll
        for (int r = j + 1; r < kBjMax; ++r) {
            double t = L[r][j];
#pragma unroll
            for (int k = 0; k < j; ++k) t -= L[r][k] * L[j][k];
            L[r][j] = t * rl[j];
        }
    }
    if (ok) {
#pragma unroll
        for (int c = 0; c < kBjMax; ++c) {
            double y[kBjMax], x[kBjMax];
#pragma unroll
            for (int r = 0; r < kBjMax; ++r) {
                double t = r == c ? 1.0 : 0.0;
#pragma unroll
                for (int k = 0; k < r; ++k) t -= L[r][k] * y[k];
                y[r] = t * rl[r];
            }
#pragma unroll
            for (int r = kBjMax - 1; r >= 0; --r) {
                double t = y[r];
#pragma unroll
                for (int k = r + 1; k < kBjMax; ++k) t -= L[k][r] * x[k];
                x[r] = t * rl[r];
            }
#pragma unroll
            for (int r = 0; r < kBjMax; ++r) {
                if (r >= c && r < size && c < size) {
                    const float v = (float)x[r];
                    binv[(i + r) * kBjMax + c] = v;
                    binv[(i + c) * kBjMax + r] = v;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < kBjMax; ++r)
#pragma unroll
            for (int c = 0; c < kBjMax; ++c)
                if (r < size && c >= size) binv[(i + r) * kBjMax + c] = 0.0f;
    } else {
        if (fr) atomicAdd(n_fallback, 1);
#pragma unroll
        for (int r = 0; r < kBjMax; ++r) {
            if (r >= size) continue;
            const bool f = is_free(free_mask, i + r);
#pragma unroll
            for (int c = 0; c < kBjMax; ++c)
                binv[(i + r) * kBjMax + c] = (c == r && f && d0[r] > 0.0) ? (float)(1.0 / d0[r]) : 0.0f;
        }
    }
}

}  // namespace snp
