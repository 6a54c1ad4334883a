// Newton assembly of the P1 grad-grad (scalar potential / Laplace) operator.
//
// Element arithmetic of compute_K_dK (fem_c/ctools.c:730-919), one thread per element,
// scattered into a fixed CSR pattern through the slot map:
//   Jm = sum_i X_i (x) dphi_i, H = Jm^-T sum_i dphi_i x_i        (ctools.c:506-547)
//   mu, mu' = B-spline in log10|H| or constant                   (ctools.c:317-346)
//   K_ab  = sum_q mu det w_q (Jm^-T dphi_a . Jm^-T dphi_b)
//   dK_ab = sum_q [|H| >= 1e-14] mu' det w_q (g_a . H)(g_b . H) / |H|
// For linear tetrahedra the gradients are constant per element, so mu is evaluated once
// and the sums over q factor through sum_q w_q.
//
// By default the values are added deterministically: the element kernel stores each element's
// 10 upper-triangle values of K and of dK, then one thread per CSR entry adds the sum of the
// entry's couplings from this call's elements, taken in element order from the pattern's sorted
// coupling list, to K, dK and J (one add per entry and call, so the result does not depend on
// the launch).  SNP_ASSEMBLY=atomic, or a pattern without coupling lists, adds each element's
// contributions with float64 atomics instead.
#include <cstdlib>
#include <cstring>

#include "snp_common.cuh"
#include "snp_internal.cuh"

namespace snp {

namespace {

constexpr int kBlock = 128;

struct GradArgs {
    int64_t n_elems;
    const double *nodes;
    const int32_t *cells;
    const double *dphi0;
    const double *w;
    int32_t nq;
    const double *x;
    int32_t type, degree, n_ctrl;
    const double *knots, *ctrl;
    double H_min, mu_H_min;
    const int32_t *slots;
    double *K, *dK, *J;
    double *ET;        // store mode: element values, K block [10][et_stride] then dK block
    int64_t et_stride;
};

// upper-triangle index of the element pair (a, b), 4 nodes: row min, column max, row by row
__host__ __device__ __forceinline__ int tri4(int a, int b) {
    const int j = a < b ? a : b, k = a < b ? b : a;
    return j * 4 - (j * (j - 1)) / 2 + (k - j);
}

__global__ void __launch_bounds__(kBlock) k_gradgrad(GradArgs a) {
    extern __shared__ double sm[];
    const int n_t = a.type == 1 ? a.n_ctrl + a.degree + 1 : 0;
    double *s_dphi = sm;
    double *s_t = sm + 12;
    double *s_c = s_t + n_t;
    for (int t = threadIdx.x; t < 12; t += blockDim.x) s_dphi[t] = a.dphi0[t];
    for (int t = threadIdx.x; t < n_t; t += blockDim.x) s_t[t] = a.knots[t];
    for (int t = threadIdx.x; t < (a.type == 1 ? a.n_ctrl : 0); t += blockDim.x) s_c[t] = a.ctrl[t];
    __syncthreads();
    double wsum = 0.0;
    for (int q = 0; q < a.nq; ++q) wsum += __ldg(a.w + q);

    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.n_elems; e += (int64_t)gridDim.x * blockDim.x) {
        const int4 cv = __ldg(reinterpret_cast<const int4 *>(a.cells) + e);
        const int cidx[4] = {cv.x, cv.y, cv.z, cv.w};
        double Jm[9];
#pragma unroll
        for (int r = 0; r < 9; ++r) Jm[r] = 0.0;
        double gr[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double X0 = __ldg(a.nodes + 3 * (int64_t)cidx[i]);
            const double X1 = __ldg(a.nodes + 3 * (int64_t)cidx[i] + 1);
            const double X2 = __ldg(a.nodes + 3 * (int64_t)cidx[i] + 2);
            const double xi = __ldg(a.x + cidx[i]);
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                const double d = s_dphi[3 * i + l];
                Jm[0 + l] += X0 * d;
                Jm[3 + l] += X1 * d;
                Jm[6 + l] += X2 * d;
                gr[l] += d * xi;
            }
        }
        const double det = Jm[0] * (Jm[4] * Jm[8] - Jm[7] * Jm[5]) - Jm[1] * (Jm[3] * Jm[8] - Jm[5] * Jm[6]) +
                           Jm[2] * (Jm[3] * Jm[7] - Jm[4] * Jm[6]);
        const double id = 1.0 / det;
        double Ji[9];
        Ji[0] = (Jm[4] * Jm[8] - Jm[7] * Jm[5]) * id;
        Ji[1] = (Jm[2] * Jm[7] - Jm[1] * Jm[8]) * id;
        Ji[2] = (Jm[1] * Jm[5] - Jm[2] * Jm[4]) * id;
        Ji[3] = (Jm[5] * Jm[6] - Jm[3] * Jm[8]) * id;
        Ji[4] = (Jm[0] * Jm[8] - Jm[2] * Jm[6]) * id;
        Ji[5] = (Jm[3] * Jm[2] - Jm[0] * Jm[5]) * id;
        Ji[6] = (Jm[3] * Jm[7] - Jm[6] * Jm[4]) * id;
        Ji[7] = (Jm[6] * Jm[1] - Jm[0] * Jm[7]) * id;
        Ji[8] = (Jm[0] * Jm[4] - Jm[3] * Jm[1]) * id;
        // transposed map (mat_vec with transpose = 1, ctools.c:415-438)
        double H[3];
        H[0] = Ji[0] * gr[0] + Ji[3] * gr[1] + Ji[6] * gr[2];
        H[1] = Ji[1] * gr[0] + Ji[4] * gr[1] + Ji[7] * gr[2];
        H[2] = Ji[2] * gr[0] + Ji[5] * gr[1] + Ji[8] * gr[2];
        double gphi[4][3];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double d0 = s_dphi[3 * i], d1 = s_dphi[3 * i + 1], d2 = s_dphi[3 * i + 2];
            gphi[i][0] = Ji[0] * d0 + Ji[3] * d1 + Ji[6] * d2;
            gphi[i][1] = Ji[1] * d0 + Ji[4] * d1 + Ji[7] * d2;
            gphi[i][2] = Ji[2] * d0 + Ji[5] * d1 + Ji[8] * d2;
        }
        const double hm = sqrt(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
        double dmu;
        const double mu = bspline_mu(a.type, a.degree, a.n_ctrl, s_t, s_c, a.H_min, a.mu_H_min, hm, dmu);
        const double kf = mu * det * wsum;
        const double df = (hm >= 1e-14) ? dmu * det * wsum / hm : 0.0;
        double p[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) p[i] = gphi[i][0] * H[0] + gphi[i][1] * H[1] + gphi[i][2] * H[2];
        const int32_t *sl = a.slots + 16 * e;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
#pragma unroll
            for (int k = i; k < 4; ++k) {
                const double kv = kf * (gphi[i][0] * gphi[k][0] + gphi[i][1] * gphi[k][1] + gphi[i][2] * gphi[k][2]);
                const double dv = df * p[i] * p[k];
                if (a.ET) {
                    a.ET[(int64_t)tri4(i, k) * a.et_stride + e] = kv;
                    a.ET[(int64_t)(10 + tri4(i, k)) * a.et_stride + e] = dv;
                    continue;
                }
                const int s1 = __ldg(sl + 4 * i + k);
                if (a.K) atomicAdd(a.K + s1, kv);
                if (a.dK) atomicAdd(a.dK + s1, dv);
                if (a.J) atomicAdd(a.J + s1, kv + dv);
                if (k != i) {
                    const int s2 = __ldg(sl + 4 * k + i);
                    if (a.K) atomicAdd(a.K + s2, kv);
                    if (a.dK) atomicAdd(a.dK + s2, dv);
                    if (a.J) atomicAdd(a.J + s2, kv + dv);
                }
            }
        }
    }
}

// K_p += sum, over the couplings t = e * 16 + a * 4 + b of CSR entry p whose element lies in
// [e_lo, e_lo + n), in element order, of the stored K value of (e, a, b); dK likewise; J gets the
// two sums added.  Entries without such a coupling are left alone.
__global__ void __launch_bounds__(256)
    k_gg_entries(int64_t nnz, const int32_t *__restrict__ cptr, const int32_t *__restrict__ cid,
                 const double *__restrict__ ET, int64_t stride, int64_t e_lo, int64_t n, double *K, double *dK,
                 double *J) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
        double s0 = 0.0, s1 = 0.0;
        int cnt = 0;
        for (int c = __ldg(cptr + p); c < __ldg(cptr + p + 1); ++c) {
            const uint32_t t = (uint32_t)__ldg(cid + c);
            const int64_t e = (int64_t)(t >> 4) - e_lo;
            if (e < 0 || e >= n) continue;
            const int ab = (int)(t & 15u);
            const int q = tri4(ab >> 2, ab & 3);
            s0 += __ldg(ET + (int64_t)q * stride + e);
            s1 += __ldg(ET + (int64_t)(10 + q) * stride + e);
            ++cnt;
        }
        if (cnt == 0) continue;
        if (K) K[p] += s0;
        if (dK) dK[p] += s1;
        if (J) J[p] += s0 + s1;
    }
}

}  // namespace
}  // namespace snp

extern "C" int snp_gradgrad_assemble(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems, const double *nodes,
                                     const int32_t *cells, const double *d_phi, const double *w, int32_t n_quad,
                                     const double *x, int32_t perm_type, int32_t degree, int32_t n_ctrl,
                                     const double *knots, const double *ctrl, double H_min, double mu_H_min,
                                     double *K_vals, double *dK_vals, double *J_vals, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(pat != nullptr && pat->dpe == 4, "snp_gradgrad_assemble: pattern with 4 DoFs per element required");
    SNP_REQUIRE(n_elems >= 0 && elem_offset >= 0 && elem_offset + n_elems <= pat->n_elems,
                "snp_gradgrad_assemble: element range outside the pattern");
    SNP_REQUIRE(perm_type == 0 || perm_type == 1, "snp_gradgrad_assemble: permeability type must be 0 or 1");
    SNP_REQUIRE(n_quad >= 1, "snp_gradgrad_assemble: n_quad must be >= 1");
    if (perm_type == 1) {
        SNP_REQUIRE(degree >= 0 && degree <= snp::kMaxSplineDegree, "snp_gradgrad_assemble: spline degree %d unsupported", degree);
        SNP_REQUIRE(n_ctrl >= 1 && knots && ctrl, "snp_gradgrad_assemble: spline tables missing");
    }
    SNP_REQUIRE(n_elems == 0 || (nodes && cells && d_phi && w && x), "snp_gradgrad_assemble: NULL input");
    SNP_REQUIRE(((uintptr_t)cells & 15) == 0, "cells must be 16-byte aligned");
    if (n_elems == 0) return SNP_OK;
    snp::GradArgs a{};
    a.n_elems = n_elems;
    a.nodes = nodes;
    a.cells = cells;
    a.dphi0 = d_phi;
    a.w = w;
    a.nq = n_quad;
    a.x = x;
    a.type = perm_type;
    a.degree = degree;
    a.n_ctrl = n_ctrl;
    a.knots = knots;
    a.ctrl = ctrl;
    a.H_min = H_min;
    a.mu_H_min = mu_H_min;
    a.slots = pat->slots.p + 16 * elem_offset;
    a.K = K_vals;
    a.dK = dK_vals;
    a.J = J_vals;
    const int n_t = perm_type == 1 ? n_ctrl + degree + 1 : 0;
    const size_t smem = sizeof(double) * (12 + n_t + (perm_type == 1 ? n_ctrl : 0));
    SNP_REQUIRE(smem <= 200 * 1024, "snp_gradgrad_assemble: spline tables too large");
    if (smem > 48 * 1024)
        SNP_CUDA_TRY(cudaFuncSetAttribute(snp::k_gradgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaStream_t st = snp::as_stream(stream);
    const char *env = getenv("SNP_ASSEMBLY");
    const bool atomic = (env && std::strcmp(env, "atomic") == 0) || !pat->has_contrib;
    if (!atomic) {
        const size_t need = (size_t)20 * (size_t)n_elems;
        if (pat->gg_terms.n < need) SNP_TRY(pat->gg_terms.alloc(need));
        a.ET = pat->gg_terms.p;
        a.et_stride = n_elems;
    }
    snp::k_gradgrad<<<snp::stride_grid(n_elems, snp::kBlock, 16), snp::kBlock, smem, st>>>(a);
    SNP_LAUNCH_CHECK();
    if (!atomic) {
        snp::k_gg_entries<<<snp::stride_grid(pat->nnz, 256, 8), 256, 0, st>>>(
            pat->nnz, pat->cptr.p, pat->cid.p, pat->gg_terms.p, n_elems, elem_offset, n_elems, K_vals, dK_vals, J_vals);
        SNP_LAUNCH_CHECK();
    }
    return SNP_OK;
}
