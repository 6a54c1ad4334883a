// Persistent Newton solver for the (reduced) magnetic vector potential formulation.
//
// Mirrors the Newton loops of RedMVPSolver.solve (snoopy/red_mvp_solver.py:121-224) and
// MVPSolver.solve_nonlin (snoopy/mvp_solver.py:222-334) with every step on the device:
// assembly into the cached CSR pattern (the reference re-runs scipy's COO->CSR, the sparse
// adds and the Dirichlet fancy-indexing every step), the masked Jacobi-PCG, and the vector
// updates.  The host only reads a few scalars per Newton step.
//
// Mode 0 keeps the reference's semantics: b = J x - K x + rhs, zero-excitation exit when
// max|b| < 1e-14, x_{n+1} = CG(J_free, b_free, x0 = x_n, atol = tol, rtol = cg_rtol),
// stop when max|x_{n+1} - x_n| < tol * max|x_{n+1}|.
// Mode 1 is Newton on F(x) = K(x) x - rhs(x) until ||F_free|| <= tol * ||F_free(x0)||, each
// step J h = -F solved by CG to an Eisenstat-Walker forcing tolerance; with precision 1 the
// Jacobian values and the CG run in float32 while F, the update and the norms stay float64
// (the Newton loop is the iterative refinement of the float32 solves).
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "snp_common.cuh"
#include "snp_internal.cuh"
#include "snp_krylov.cuh"

namespace snp {
namespace {

constexpr int kVB = 256;

struct Material {
    int64_t offset = 0, count = 0;
    int32_t n_int = -1;
    DevBuf<int32_t> cells, gids, orient;
    DevBuf<double> relc, relx, Bs;
    bool has_bs = false;
    // diluted steel: nodal basis at the quadrature points [Q][4] and {c_num, m_num, c_den, m_den}
    DevBuf<double> phi;
    bool diluted = false;
    double dil[4] = {0.0, 0.0, 1.0, 0.0};
};

// c = -A^-1 g for a symmetric positive semi-definite m x m matrix A (row-major): Cholesky of
// the Jacobi-scaled matrix; a direction whose pivot falls below 1e-10 of its diagonal (a
// dependent basis column) is left out of the solve.  False when A has a non-positive or
// non-finite diagonal entry.
bool spd_solve(int m, const double *A, const double *g, double *c) {
    std::vector<double> L((size_t)m * m), d(m), y(m);
    for (int i = 0; i < m; ++i) {
        const double a = A[(size_t)i * m + i];
        if (!(a > 0.0) || !std::isfinite(a)) return false;
        d[i] = 1.0 / std::sqrt(a);
    }
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) L[(size_t)i * m + j] = A[(size_t)i * m + j] * d[i] * d[j];
    std::vector<char> keep(m, 1);
    for (int j = 0; j < m; ++j) {
        double p = L[(size_t)j * m + j];
        for (int k = 0; k < j; ++k) p -= L[(size_t)j * m + k] * L[(size_t)j * m + k];
        if (!(p > 1e-10)) {
            keep[j] = 0;
            for (int i = j; i < m; ++i) L[(size_t)i * m + j] = 0.0;
            continue;
        }
        const double ljj = std::sqrt(p);
        L[(size_t)j * m + j] = ljj;
        for (int i = j + 1; i < m; ++i) {
            double t = L[(size_t)i * m + j];
            for (int k = 0; k < j; ++k) t -= L[(size_t)i * m + k] * L[(size_t)j * m + k];
            L[(size_t)i * m + j] = t / ljj;
        }
    }
    for (int i = 0; i < m; ++i) {  // L y = -D g
        double t = -d[i] * g[i];
        for (int k = 0; k < i; ++k) t -= L[(size_t)i * m + k] * y[k];
        y[i] = keep[i] ? t / L[(size_t)i * m + i] : 0.0;
    }
    for (int i = m - 1; i >= 0; --i) {  // L^T z = y, c = D z
        double t = y[i];
        for (int k = i + 1; k < m; ++k) t -= L[(size_t)k * m + i] * c[k];
        c[i] = keep[i] ? t / L[(size_t)i * m + i] : 0.0;
    }
    for (int i = 0; i < m; ++i) {
        if (!std::isfinite(c[i])) return false;
    }
    for (int i = 0; i < m; ++i) c[i] *= d[i];
    return true;
}

// res[0] += sum over free i of v[i]^2 (deterministic last-block reduction)
// res[1]  = max over all i of |v[i]|; res[2] = max |v - w| and res[3] = max |v| (when w != null)
__global__ void k_vstats(int32_t n, const uint8_t *__restrict__ fm, const double *__restrict__ v,
                         const double *__restrict__ w, double *part, unsigned int *counter, double *res) {
    __shared__ double sh[32];
    double ss = 0.0, mx = 0.0, md = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double a = v[i];
        if (fm == nullptr || fm[i]) ss += a * a;
        mx = fmax(mx, fabs(a));
        if (w) md = fmax(md, fabs(a - w[i]));
    }
    // sum
    ss = block_sum(ss, sh);
    __syncthreads();
    // max via warp shuffles
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    }
    __shared__ double smx[32], smd[32];
    if ((threadIdx.x & 31) == 0) {
        smx[threadIdx.x >> 5] = mx;
        smd[threadIdx.x >> 5] = md;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            mx = fmax(mx, smx[k]);
            md = fmax(md, smd[k]);
        }
        part[3 * blockIdx.x] = ss;
        part[3 * blockIdx.x + 1] = mx;
        part[3 * blockIdx.x + 2] = md;
        __threadfence();
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) last = atomicInc(counter, gridDim.x - 1) == gridDim.x - 1;
    __syncthreads();
    if (last && threadIdx.x == 0) {
        double s = 0.0, m = 0.0, d = 0.0;
        for (unsigned int b = 0; b < gridDim.x; ++b) {
            s += __ldcg(part + 3 * b);
            m = fmax(m, __ldcg(part + 3 * b + 1));
            d = fmax(d, __ldcg(part + 3 * b + 2));
        }
        res[0] = s;
        res[1] = m;
        res[2] = d;
    }
}

__global__ void k_vdot(int32_t n, const uint8_t *__restrict__ fm, const double *__restrict__ a,
                       const double *__restrict__ b, double *part, unsigned int *counter, double *res) {
    __shared__ double sh[32];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (fm[i]) s += a[i] * b[i];
    s = block_sum(s, sh);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        __threadfence();
        last = atomicInc(counter, gridDim.x - 1) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        double t = 0.0;
        for (unsigned int k = 0; k < gridDim.x; ++k) t += __ldcg(part + k);
        res[0] = t;
    }
}

__global__ void k_sub(int32_t n, double *__restrict__ b, const double *__restrict__ F) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] -= F[i];
}

__global__ void k_neg_free(int32_t n, const uint8_t *__restrict__ fm, const double *__restrict__ F, double *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = fm[i] ? -F[i] : 0.0;
}

__global__ void k_neg_free_f32(int32_t n, const uint8_t *__restrict__ fm, const double *__restrict__ F, float *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = fm[i] ? (float)(-F[i]) : 0.0f;
}

__global__ void k_add_free(int32_t n, const uint8_t *__restrict__ fm, double *__restrict__ x, const double *__restrict__ h) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (fm[i]) x[i] += h[i];
}

__global__ void k_add_free_f32(int32_t n, const uint8_t *__restrict__ fm, double *__restrict__ x, const float *__restrict__ h) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (fm[i]) x[i] += (double)h[i];
}

// y = x + alpha h on free rows, y = x elsewhere
__global__ void k_axpy_free(int32_t n, const uint8_t *__restrict__ fm, const double *__restrict__ x,
                            const double *__restrict__ h, double alpha, double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = fm[i] ? x[i] + alpha * h[i] : x[i];
}

__global__ void k_f32_to_f64(int32_t n, const float *__restrict__ a, double *__restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

__global__ void k_zero_nonfree(int32_t n, const uint8_t *__restrict__ fm, double *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!fm[i]) x[i] = 0.0;
}

__global__ void k_count_free(int32_t n, const uint8_t *__restrict__ fm, unsigned long long *cnt) {
    unsigned long long c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) c += fm[i] ? 1 : 0;
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

}  // namespace
}  // namespace snp

struct snp_solver {
    int32_t n = 0;
    int64_t n_nodes = 0;
    int32_t nq = 0, n_orient = 0;
    int64_t n_free = 0;
    cudaStream_t stream = nullptr;
    snp::DevBuf<double> nodes, curls, dphi, w, rhs_extra;
    snp::DevBuf<uint8_t> free_mask;
    bool has_extra = false;
    std::vector<std::unique_ptr<snp::Material>> mats;
    snp_pattern *pat = nullptr;
    // storage of the Newton loop's Jacobian: element tensors (matrix-free), or an assembled
    // CSR / SELL-C-sigma matrix; reference-semantics solves and exports always use the CSR
    int layout = SNP_LAYOUT_CSR;
    snp::SellLayout sell;
    bool use_sell = false;
    snp::ElemTopology etop;
    snp::DevBuf<double> T64, Jdiag, Fe, De, rsys_scratch;
    // two-phase CSR assembly (element records, then one gather per row)
    bool rows_asm = false;
    snp::DevBuf<double> terms;
    // Krylov method of the residual-mode Newton steps (snp_solver_set_krylov): 0 CG, 1 GMRES(restart)
    int krylov = 0, krylov_restart = 30;
    snp::Gmres gmres;
    // Galerkin correction of a warm start (snp_solver_set_galerkin_basis): basis, its system
    // and coefficients on the device and in pinned memory, and a copy of x to fall back to
    const float *gal_V = nullptr;
    int32_t gal_m = 0, gal_steps = 0;
    int64_t gal_ldv = 0;
    snp::DevBuf<double> gal_sys, gal_x;
    snp::HostBuf<double> gal_host;
    // block Jacobi of the residual-mode Krylov solves (snp_solver_set_block_jacobi)
    bool bj_on = false;
    snp::DevBuf<uint16_t> bj_meta;
    snp::DevBuf<double> bj_mat;
    snp::DevBuf<float> bj_inv;
    snp::DevBuf<int> bj_fallback;

    // z = M r with the block Jacobi of the current element tensors (test and inspection entry)
    int precond_apply(bool f32, const double *r, double *z, int32_t *fallback_blocks) {
        SNP_CUDA_TRY(cudaMemsetAsync(bj_fallback.p, 0, sizeof(int), stream));
        SNP_TRY(build_block_jacobi(f32));
        SNP_TRY(snp::block_jacobi_apply(n, free_mask.p, bj_meta.p, bj_inv.p, r, z, stream));
        if (fallback_blocks) {
            int fb = 0;
            SNP_CUDA_TRY(cudaMemcpyAsync(&fb, bj_fallback.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
            SNP_CUDA_TRY(cudaStreamSynchronize(stream));
            *fallback_blocks = fb;
        }
        return SNP_OK;
    }

    int build_block_jacobi(bool f32) {
        if (f32)
            SNP_TRY(snp::block_jacobi_build(etop, T32.p, free_mask.p, bj_meta.p, bj_mat.p, bj_inv.p, bj_fallback.p,
                                            stream));
        else
            SNP_TRY(snp::block_jacobi_build(etop, T64.p, free_mask.p, bj_meta.p, bj_mat.p, bj_inv.p, bj_fallback.p,
                                            stream));
        launches += 2;
        return SNP_OK;
    }
    snp::DevBuf<float> T32;
    snp::ElemPcg<double> epcg64;
    snp::ElemPcg<float> epcg32;
    int j_valid[2] = {0, 0};  // the float64 / float32 Newton Jacobian is current
    bool finalized = false;
    snp::DevBuf<double> J, F, b, xw, h, part, res;
    snp::DevBuf<float> J32, b32, h32;
    snp::DevBuf<unsigned int> counter;
    snp::HostBuf<double> hres;
    snp::Pcg<double, double> pcg64;
    snp::Pcg<float, float> pcg32;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t launches = 0;  // kernels of this library launched by the current solve
    mutable std::vector<snp::SolverMaterialView> views;  // solver_view's material list

    ~snp_solver() {
        if (pat) snp_pattern_destroy(pat);
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
    }

    int64_t n_elems_total() const {
        int64_t t = 0;
        for (auto &m : mats) t += m->count;
        return t;
    }

    int vstats(const double *v, const double *w2, bool free_only, double out[3]) {
        const int grid = snp::stride_grid(n, snp::kVB, 4);
        snp::k_vstats<<<grid, snp::kVB, 0, stream>>>(n, free_only ? free_mask.p : nullptr, v, w2, part.p, counter.p, res.p);
        SNP_LAUNCH_CHECK();
        ++launches;
        SNP_CUDA_TRY(cudaMemcpyAsync(hres.p, res.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        SNP_CUDA_TRY(cudaStreamSynchronize(stream));
        for (int k = 0; k < 3; ++k) out[k] = hres.p[k];
        return SNP_OK;
    }

    // sum over free i of a[i] * b[i] (deterministic, read back)
    int vdot(const double *a, const double *bb, double *out) {
        const int grid = snp::stride_grid(n, snp::kVB, 4);
        snp::k_vdot<<<grid, snp::kVB, 0, stream>>>(n, free_mask.p, a, bb, part.p, counter.p, res.p);
        SNP_LAUNCH_CHECK();
        ++launches;
        SNP_CUDA_TRY(cudaMemcpyAsync(hres.p, res.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
        SNP_CUDA_TRY(cudaStreamSynchronize(stream));
        *out = hres.p[0];
        return SNP_OK;
    }

    // The Newton Jacobian's matrix view (SELL when use_sell) over values v.
    template <typename VT>
    snp::CsrView<VT> jacobian_view(const VT *v) const {
        snp::CsrView<VT> A{n, pat->nnz, pat->row_ptr.p, pat->col_idx.p, v};
        if (use_sell) {
            A.n_slices = sell.n_slices;
            A.sell_off = sell.slice_off.p;
            A.sell_row = sell.slice_row.p;
            A.sell_col = sell.col.p;
        }
        return A;
    }

    int apply_jacobian(int precision, const void *x, void *y, cudaStream_t st) {
        if (layout == SNP_LAYOUT_ELEM) {
            if (precision == 0)
                return epcg64.apply(etop, T64.p, free_mask.p, static_cast<const double *>(x), static_cast<double *>(y), st);
            return epcg32.apply(etop, T32.p, free_mask.p, static_cast<const float *>(x), static_cast<float *>(y), st);
        }
        if (precision == 0)
            return snp::spmv_f64(jacobian_view<double>(J.p), free_mask.p, static_cast<const double *>(x),
                                 static_cast<double *>(y), st);
        return snp::spmv_f32(jacobian_view<float>(J32.p), free_mask.p, static_cast<const float *>(x),
                             static_cast<float *>(y), st);
    }

    // Element tensors (float64 or float32), diag(J) and F = K x - rhs - rhs_extra at x.
    int assemble_elem(const double *x, bool f32, double *Fv) {
        j_valid[f32 ? 1 : 0] = 1;
        for (auto &m : mats) {
            snp::CurlArgs a{};
            a.n_elems = m->count;
            a.nodes = nodes.p;
            a.cells = m->cells.p;
            a.gids = m->gids.p;
            a.orient = m->orient.p;
            a.ctab = curls.p;
            a.n_orient = n_orient;
            a.dphi0 = dphi.p;
            a.w = w.p;
            a.nq = nq;
            a.x = x;
            a.Bs = m->has_bs ? m->Bs.p : nullptr;
            a.n_int = m->n_int;
            a.rel_c = m->relc.p;
            a.rel_x = m->relx.p;
            if (m->diluted && m->has_bs) {
                a.phi = m->phi.p;
                for (int i = 0; i < 4; ++i) a.dil[i] = m->dil[i];
            }
            a.T64 = f32 ? nullptr : T64.p;
            a.T32 = f32 ? T32.p : nullptr;
            a.t_offset = m->offset;
            a.Fe = Fe.p;
            a.De = De.p;
            SNP_TRY(snp::launch_curlcurl_tensor(a, stream));
            if (m->count) ++launches;
        }
        SNP_TRY(snp::elem_sum_to_dofs(etop, Fe.p, De.p, has_extra ? rhs_extra.p : nullptr, Fv, Jdiag.p, stream));
        ++launches;
        return SNP_OK;
    }

    // Newton-loop assembly at x in the solver's layout: Jacobian (precision f32 or not) and F.
    // One Galerkin Newton step from x in the span of the attached basis, with the Jacobian and
    // F of the last assembly at x: x += V c, (V^T J V) c = -V^T F.  *applied = false (x kept)
    // when the reduced system is not positive definite.
    int galerkin_step(double *x, bool f32, bool *applied) {
        *applied = false;
        const int m = gal_m;
        double *Jr = gal_sys.p, *g = gal_sys.p + (size_t)m * m, *c = g + m;
        if (f32)
            SNP_TRY(snp::elem_reduced_system(etop, T32.p, free_mask.p, gal_V, m, gal_ldv, F.p, Jr, g, rsys_scratch,
                                             stream));
        else
            SNP_TRY(snp::elem_reduced_system(etop, T64.p, free_mask.p, gal_V, m, gal_ldv, F.p, Jr, g, rsys_scratch,
                                             stream));
        launches += 4;
        SNP_CUDA_TRY(cudaMemcpyAsync(gal_host.p, gal_sys.p, sizeof(double) * ((size_t)m * m + m),
                                     cudaMemcpyDeviceToHost, stream));
        SNP_CUDA_TRY(cudaStreamSynchronize(stream));
        double *ch = gal_host.p + (size_t)m * m + m;
        if (!snp::spd_solve(m, gal_host.p, gal_host.p + (size_t)m * m, ch)) return SNP_OK;
        SNP_CUDA_TRY(cudaMemcpyAsync(c, ch, sizeof(double) * m, cudaMemcpyHostToDevice, stream));
        SNP_TRY(snp::basis_axpy(n, free_mask.p, gal_V, m, gal_ldv, c, x, stream));
        ++launches;
        *applied = true;
        return SNP_OK;
    }

    int assemble_newton(const double *x, bool f32) {
        if (layout == SNP_LAYOUT_ELEM) return assemble_elem(x, f32, F.p);
        return assemble(x, nullptr, f32 ? nullptr : J.p, f32 ? J32.p : nullptr, nullptr, F.p, true);
    }

    // J (f64 or f32), F = K x - rhs - rhs_extra; optional K and rhs.  With sell_order the
    // matrix outputs are written in the SELL layout (the Newton loop's Jacobian), else in CSR.
    int assemble(const double *x, double *Kv, double *Jv, float *J32v, double *rhsv, double *Fv,
                 bool sell_order = false) {
        const bool so = sell_order && use_sell;
        const int64_t nnz = so ? sell.total : pat->nnz;
        // the assembled Newton Jacobian is what jacobian_apply uses unless the layout is matrix-free
        const bool newton_j = sell_order && layout != SNP_LAYOUT_ELEM;
        if (Jv == J.p) j_valid[0] = newton_j;
        if (J32v == J32.p) j_valid[1] = newton_j;
        if (!so && rows_asm) return assemble_rows(x, Kv, Jv, J32v, rhsv, Fv);
        if (Kv) SNP_CUDA_TRY(cudaMemsetAsync(Kv, 0, sizeof(double) * nnz, stream));
        if (Jv) SNP_CUDA_TRY(cudaMemsetAsync(Jv, 0, sizeof(double) * nnz, stream));
        if (J32v) SNP_CUDA_TRY(cudaMemsetAsync(J32v, 0, sizeof(float) * nnz, stream));
        if (rhsv) SNP_CUDA_TRY(cudaMemsetAsync(rhsv, 0, sizeof(double) * n, stream));
        if (Fv) SNP_CUDA_TRY(cudaMemsetAsync(Fv, 0, sizeof(double) * n, stream));
        for (auto &m : mats) {
            snp::CurlArgs a{};
            a.n_elems = m->count;
            a.nodes = nodes.p;
            a.cells = m->cells.p;
            a.gids = m->gids.p;
            a.orient = m->orient.p;
            a.ctab = curls.p;
            a.n_orient = n_orient;
            a.dphi0 = dphi.p;
            a.w = w.p;
            a.nq = nq;
            a.x = x;
            a.Bs = m->has_bs ? m->Bs.p : nullptr;
            a.n_int = m->n_int;
            a.rel_c = m->relc.p;
            a.rel_x = m->relx.p;
            if (m->diluted && m->has_bs) {
                a.phi = m->phi.p;
                for (int i = 0; i < 4; ++i) a.dil[i] = m->dil[i];
            }
            a.slots = (so ? sell.slots.p : pat->slots.p) + 36 * m->offset;
            a.K = Kv;
            a.J = Jv;
            a.J32 = J32v;
            a.rhs = rhsv;
            a.F = Fv;
            SNP_TRY(snp::launch_curlcurl(a, stream));
            if (m->count) ++launches;
        }
        if (Fv && has_extra) {
            snp::k_sub<<<snp::stride_grid(n, snp::kVB, 4), snp::kVB, 0, stream>>>(n, Fv, rhs_extra.p);
            SNP_LAUNCH_CHECK();
            ++launches;
        }
        return SNP_OK;
    }

    // CSR assembly in two phases: each material's element values, then every CSR entry and
    // vector entry summed from its element contributions (bitwise repeatable; each output
    // overwritten once)
    int assemble_rows(const double *x, double *Kv, double *Jv, float *J32v, double *rhsv, double *Fv) {
        int parts = 0;
        if (Kv) parts |= SNP_TERMS_K | ((Jv || J32v) ? SNP_TERMS_DK : 0);
        else if (Jv || J32v) parts |= SNP_TERMS_J;
        if (Fv) parts |= SNP_TERMS_F;
        if (rhsv) parts |= SNP_TERMS_RHS;
        const snp::TermLayout L = snp::term_layout(parts);
        const size_t need = (size_t)pat->n_elems * (size_t)L.stride;
        if (terms.n < need) SNP_TRY(terms.alloc(need));
        for (auto &m : mats) {
            snp::CurlArgs a{};
            a.n_elems = m->count;
            a.nodes = nodes.p;
            a.cells = m->cells.p;
            a.gids = m->gids.p;
            a.orient = m->orient.p;
            a.ctab = curls.p;
            a.n_orient = n_orient;
            a.dphi0 = dphi.p;
            a.w = w.p;
            a.nq = nq;
            a.x = x;
            a.Bs = m->has_bs ? m->Bs.p : nullptr;
            a.n_int = m->n_int;
            a.rel_c = m->relc.p;
            a.rel_x = m->relx.p;
            if (m->diluted && m->has_bs) {
                a.phi = m->phi.p;
                for (int i = 0; i < 4; ++i) a.dil[i] = m->dil[i];
            }
            a.t_offset = m->offset;
            SNP_TRY(snp::launch_curlcurl_terms(a, L, terms.p, pat->n_elems, stream));
            if (m->count) ++launches;
        }
        SNP_TRY(snp::launch_curlcurl_rows(pat, terms.p, L, Kv, nullptr, Jv, J32v, rhsv, Fv, stream));
        ++launches;
        if (Fv && has_extra) {
            snp::k_sub<<<snp::stride_grid(n, snp::kVB, 4), snp::kVB, 0, stream>>>(n, Fv, rhs_extra.p);
            SNP_LAUNCH_CHECK();
            ++launches;
        }
        return SNP_OK;
    }

    float elapsed(int a, int b2) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[a], ev[b2]);
        return ms;
    }

    int solve(double *x, const snp_solve_opts &o, snp_solve_stats &S) {
        std::memset(&S, 0, sizeof(S));
        launches = 0;
        pcg64.launches = 0;
        pcg32.launches = 0;
        epcg64.launches = 0;
        epcg32.launches = 0;
        const int grid = snp::stride_grid(n, snp::kVB, 4);
        SNP_CUDA_TRY(cudaEventRecord(ev[2], stream));
        const snp::CsrView<double> A = jacobian_view(J.p);
        const snp::CsrView<float> A32 = jacobian_view(J32.p);
        const int32_t *diag = use_sell ? sell.diag.p : pat->diag_pos.p;
        const int64_t cg_maxit = o.cg_maxiter < 0 ? 10 * n_free : o.cg_maxiter;
        double st3[3];
        int status = SNP_OK;
        if (o.mode == 0) {
            SNP_REQUIRE(o.precision == 0, "mode 0 (reference semantics) runs in float64 only");
            for (int it = 0; it < o.max_newton; ++it) {
                SNP_CUDA_TRY(cudaEventRecord(ev[0], stream));
                SNP_TRY(assemble(x, nullptr, J.p, nullptr, nullptr, F.p, true));
                SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
                // b = J x - (K x - rhs)
                SNP_TRY(snp::spmv_f64(A, nullptr, x, b.p, stream));
                snp::k_sub<<<grid, snp::kVB, 0, stream>>>(n, b.p, F.p);
                SNP_LAUNCH_CHECK();
                launches += 2;  // with the SpMV above
                SNP_TRY(vstats(F.p, nullptr, true, st3));
                S.res = std::sqrt(st3[0]);
                if (it == 0) S.res0 = S.res;
                SNP_TRY(vstats(b.p, nullptr, false, st3));
                S.t_assemble_ms += elapsed(0, 1);
                S.newton_iterations = it + 1;
                if (st3[1] < 1e-14) {
                    SNP_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, stream));
                    if (o.verbose) printf("  zero excitation!\n");
                    break;
                }
                bool zp = false;
                SNP_TRY(pcg64.set_jacobi(A, diag, free_mask.p, stream, &zp));
                if (zp) return snp::fail(SNP_ZERO_PIVOT, "Newton step %d: zero Jacobian diagonal on a free DoF", it);
                SNP_CUDA_TRY(cudaMemcpyAsync(xw.p, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
                SNP_CUDA_TRY(cudaEventRecord(ev[0], stream));
                int64_t its = 0;
                double rn = 0.0;
                int st = SNP_OK;
                SNP_TRY(pcg64.solve(A, free_mask.p, b.p, xw.p, o.cg_rtol, o.tol, cg_maxit, false, stream, &its, &rn, &st));
                SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
                if (st == SNP_NAN_DETECTED) return snp::fail(st, "Newton step %d: non-finite CG residual", it);
                S.cg_iterations += its;
                SNP_TRY(vstats(xw.p, x, false, st3));  // st3[1] = max|x_new|, st3[2] = max|x_new - x|
                S.t_krylov_ms += elapsed(0, 1);
                SNP_CUDA_TRY(cudaMemcpyAsync(x, xw.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
                if (o.verbose)
                    printf("  step %d: max relative increment %.3e, cg its %lld\n", it,
                           st3[1] > 0 ? st3[2] / st3[1] : 0.0, (long long)its);
                if (st3[2] < o.tol * st3[1]) break;
            }
        } else if (o.mode == 1) {
            // Newton on F(x) = K(x) x - rhs(x).  Every assembly produces the Jacobian and F at
            // once, so an accepted (trial) point already carries the next step's system.
            double F0 = 0.0, fprev = 0.0, eta_prev = 0.0;
            double eta_max = o.cg_rtol > 0 ? o.cg_rtol : 0.1;
            if (eta_max > 0.5) eta_max = 0.5;
            const bool f32 = o.precision == 1;
            snp::k_zero_nonfree<<<grid, snp::kVB, 0, stream>>>(n, free_mask.p, x);
            SNP_LAUNCH_CHECK();
            ++launches;
            SNP_CUDA_TRY(cudaEventRecord(ev[0], stream));
            SNP_TRY(assemble_newton(x, f32));
            SNP_TRY(vstats(F.p, nullptr, true, st3));
            SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
            SNP_CUDA_TRY(cudaEventSynchronize(ev[1]));
            S.t_assemble_ms += elapsed(0, 1);
            double fn = std::sqrt(st3[0]);
            S.res0 = fn;
            // Galerkin correction of the start in the attached basis; a step that does not lower
            // ||F_free|| is undone.  The drop rule below applies to the corrected start.
            if (gal_V && gal_m > 0 && layout == SNP_LAYOUT_ELEM && fn > 0.0) {
                for (int gs = 0; gs < gal_steps; ++gs) {
                    SNP_CUDA_TRY(cudaEventRecord(ev[0], stream));
                    SNP_CUDA_TRY(cudaMemcpyAsync(gal_x.p, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
                    bool applied = false;
                    SNP_TRY(galerkin_step(x, f32, &applied));
                    if (!applied) break;
                    SNP_TRY(assemble_newton(x, f32));
                    SNP_TRY(vstats(F.p, nullptr, true, st3));
                    const double fg = std::sqrt(st3[0]);
                    if (!(fg < fn)) {
                        SNP_CUDA_TRY(cudaMemcpyAsync(x, gal_x.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
                        SNP_TRY(assemble_newton(x, f32));
                        SNP_TRY(vstats(F.p, nullptr, true, st3));
                        SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
                        SNP_CUDA_TRY(cudaEventSynchronize(ev[1]));
                        S.t_assemble_ms += elapsed(0, 1);
                        fn = std::sqrt(st3[0]);
                        break;
                    }
                    SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
                    SNP_CUDA_TRY(cudaEventSynchronize(ev[1]));
                    S.t_assemble_ms += elapsed(0, 1);
                    fn = fg;
                    S.galerkin_steps += 1;
                }
            }
            if (o.res_ref > 0.0 && !(fn <= o.res_ref * (1.0 + 1e-9))) {
                // a start worse than x = 0 (by the zero-start residual, up to rounding of the
                // two evaluations) is dropped for x = 0
                SNP_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, stream));
                SNP_CUDA_TRY(cudaEventRecord(ev[0], stream));
                SNP_TRY(assemble_newton(x, f32));
                SNP_TRY(vstats(F.p, nullptr, true, st3));
                SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
                SNP_CUDA_TRY(cudaEventSynchronize(ev[1]));
                S.t_assemble_ms += elapsed(0, 1);
                fn = std::sqrt(st3[0]);
                S.start_dropped = 1;
            }
            F0 = o.res_ref > 0.0 ? o.res_ref : S.res0;
            for (int it = 0;; ++it) {
                if (!(fn == fn)) return snp::fail(SNP_NAN_DETECTED, "Newton step %d: non-finite residual", it);
                S.res = fn;
                if (o.verbose) printf("  newton %d: |F| = %.6e (rel %.3e)\n", it, fn, F0 > 0 ? fn / F0 : 0.0);
                if (F0 == 0.0 || fn <= o.tol * F0) break;
                if (it == o.max_newton) {
                    status = SNP_NOT_CONVERGED;
                    break;
                }
                // Eisenstat-Walker forcing term (choice 2) with safeguards
                double eta = eta_max;
                if (it > 0) {
                    const double ratio = fn / fprev;
                    eta = 0.9 * ratio * ratio;
                    const double sg = 0.9 * eta_prev * eta_prev;
                    if (sg > 0.1 && sg > eta) eta = sg;
                    if (eta > eta_max) eta = eta_max;
                }
                const double floor_eta = 0.5 * o.tol * F0 / fn;
                if (eta < floor_eta) eta = floor_eta;
                if (f32 && eta < 1e-6) eta = 1e-6;
                if (eta > 0.5) eta = 0.5;
                fprev = fn;
                eta_prev = eta;
                int64_t its = 0;
                double rn = 0.0;
                int st = SNP_OK;
                bool zp = false;
                SNP_CUDA_TRY(cudaEventRecord(ev[0], stream));
                if (layout == SNP_LAYOUT_ELEM) {
                    if (bj_on) SNP_TRY(build_block_jacobi(f32));
                    const uint16_t *bm = bj_on ? bj_meta.p : nullptr;
                    const float *bi = bj_on ? bj_inv.p : nullptr;
                    int rc;
                    if (krylov == 1) {
                        if (f32) return snp::fail(SNP_BAD_ARG, "GMRES runs in float64 (solve with precision 0)");
                        SNP_TRY(gmres.reserve(n, krylov_restart));
                        gmres.launches = 0;
                        const snp::Gmres::Op opJ = [&](const double *xx, double *yy) {
                            launches += 2;
                            return epcg64.apply(etop, T64.p, free_mask.p, xx, yy, stream);
                        };
                        const snp::Gmres::Op opM = [&](const double *rr, double *zz) {
                            ++launches;
                            return bj_on ? snp::block_jacobi_apply(n, free_mask.p, bm, bi, rr, zz, stream)
                                         : snp::point_jacobi_apply(n, free_mask.p, Jdiag.p, rr, zz, stream);
                        };
                        rc = gmres.solve(opJ, opM, free_mask.p, F.p, -1.0, h.p, eta, 0.0, cg_maxit, stream, &its, &rn,
                                         &st);
                        launches += gmres.launches;
                    } else {
                        rc = f32 ? epcg32.solve(etop, T32.p, Jdiag.p, free_mask.p, F.p, -1.0, h.p, eta, 0.0, cg_maxit,
                                                stream, &its, &rn, &st, bm, bi)
                                 : epcg64.solve(etop, T64.p, Jdiag.p, free_mask.p, F.p, -1.0, h.p, eta, 0.0, cg_maxit,
                                                stream, &its, &rn, &st, bm, bi);
                    }
                    if (rc == SNP_ZERO_PIVOT)
                        return snp::fail(SNP_ZERO_PIVOT, "Newton step %d: zero Jacobian diagonal on a free DoF", it);
                    SNP_TRY(rc);
                } else if (f32) {
                    SNP_TRY(pcg32.set_jacobi(A32, diag, free_mask.p, stream, &zp));
                    if (zp) return snp::fail(SNP_ZERO_PIVOT, "Newton step %d: zero Jacobian diagonal on a free DoF", it);
                    snp::k_neg_free_f32<<<grid, snp::kVB, 0, stream>>>(n, free_mask.p, F.p, b32.p);
                    SNP_LAUNCH_CHECK();
                    SNP_TRY(pcg32.solve(A32, free_mask.p, b32.p, h32.p, eta, 0.0, cg_maxit, true, stream, &its, &rn, &st));
                    snp::k_f32_to_f64<<<grid, snp::kVB, 0, stream>>>(n, h32.p, h.p);
                    SNP_LAUNCH_CHECK();
                    launches += 2;
                } else {
                    SNP_TRY(pcg64.set_jacobi(A, diag, free_mask.p, stream, &zp));
                    if (zp) return snp::fail(SNP_ZERO_PIVOT, "Newton step %d: zero Jacobian diagonal on a free DoF", it);
                    snp::k_neg_free<<<grid, snp::kVB, 0, stream>>>(n, free_mask.p, F.p, b.p);
                    SNP_LAUNCH_CHECK();
                    SNP_TRY(pcg64.solve(A, free_mask.p, b.p, h.p, eta, 0.0, cg_maxit, true, stream, &its, &rn, &st));
                    launches += 1;
                }
                SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
                SNP_CUDA_TRY(cudaEventSynchronize(ev[1]));
                S.t_krylov_ms += elapsed(0, 1);
                if (st == SNP_NAN_DETECTED) return snp::fail(st, "Newton step %d: non-finite CG residual", it);
                S.cg_iterations += its;
                S.newton_iterations = it + 1;
                // step length: the full step, or (line search) the point along h where the
                // energy's slope phi'(a) = F(x + a h) . h has fallen to 0.5 |phi'(0)|; F is
                // the gradient of the magnetic energy, convex for a monotone B-H law, so
                // phi' increases along h and a safeguarded secant brackets the step
                double alpha = 1.0, g0 = 0.0, a_lo = 0.0, g_lo = 0.0, a_hi = 1.0, g_hi = 0.0;
                SNP_CUDA_TRY(cudaEventRecord(ev[0], stream));
                if (o.line_search) {
                    SNP_TRY(vdot(F.p, h.p, &g0));
                    g_lo = g0;
                }
                for (int ls = 0;; ++ls) {
                    snp::k_axpy_free<<<grid, snp::kVB, 0, stream>>>(n, free_mask.p, x, h.p, alpha, xw.p);
                    SNP_LAUNCH_CHECK();
                    ++launches;
                    SNP_TRY(assemble_newton(xw.p, f32));
                    if (ls > 0) S.residual_evals += 1;
                    if (!o.line_search) break;
                    double g = 0.0;
                    SNP_TRY(vdot(F.p, h.p, &g));
                    // the full step is kept unless it overshoots (slope above +0.5 |phi'(0)|);
                    // inside the bracket a trial must have |phi'| <= 0.5 |phi'(0)|, an undershoot
                    // raising the lower end and an overshoot lowering the upper end
                    const double c = 0.5 * std::fabs(g0);
                    if (!(g == g) || ls >= 11) break;
                    if (ls == 0 ? !(g > c) : std::fabs(g) <= c) break;
                    if (g < -c) {
                        a_lo = alpha;
                        g_lo = g;
                    } else {
                        a_hi = alpha;
                        g_hi = g;
                    }
                    const double a_new = a_lo - g_lo * (a_hi - a_lo) / (g_hi - g_lo);
                    const double width = a_hi - a_lo;
                    alpha = std::fmin(std::fmax(a_new, a_lo + 0.01 * width), a_hi - 0.01 * width);
                }
                SNP_CUDA_TRY(cudaMemcpyAsync(x, xw.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
                SNP_TRY(vstats(F.p, nullptr, true, st3));
                SNP_CUDA_TRY(cudaEventRecord(ev[1], stream));
                SNP_CUDA_TRY(cudaEventSynchronize(ev[1]));
                S.t_assemble_ms += elapsed(0, 1);
                fn = std::sqrt(st3[0]);
                if (o.verbose) printf("    cg: eta %.2e, %lld its, step %.3e\n", eta, (long long)its, alpha);
            }
        } else {
            return snp::fail(SNP_BAD_ARG, "unknown solve mode %d", o.mode);
        }
        SNP_CUDA_TRY(cudaEventRecord(ev[3], stream));
        SNP_CUDA_TRY(cudaEventSynchronize(ev[3]));
        S.t_total_ms = elapsed(2, 3);
        S.status = status;
        S.kernel_launches = launches + pcg64.launches + pcg32.launches + epcg64.launches + epcg32.launches;
        return status == SNP_OK ? SNP_OK : snp::fail(status, "Newton did not reach the tolerance in %d steps", o.max_newton);
    }
};

namespace snp {

int solver_view(const snp_solver *s, SolverView *v) {
    SNP_REQUIRE(s != nullptr && s->finalized, "solver missing or not finalized");
    v->n = s->n;
    v->n_free = s->n_free;
    v->n_nodes = s->n_nodes;
    v->n_elems = s->n_elems_total();
    v->nq = s->nq;
    v->n_orient = s->n_orient;
    v->nodes = s->nodes.p;
    v->curls = s->curls.p;
    v->dphi = s->dphi.p;
    v->w = s->w.p;
    v->rhs_extra = s->has_extra ? s->rhs_extra.p : nullptr;
    v->free_mask = s->free_mask.p;
    v->etop = s->layout == SNP_LAYOUT_ELEM ? &s->etop : nullptr;
    v->bj_meta = s->bj_on ? s->bj_meta.p : nullptr;
    s->views.clear();
    for (auto &m : s->mats) {
        SolverMaterialView mv{};
        mv.offset = m->offset;
        mv.count = m->count;
        mv.cells = m->cells.p;
        mv.gids = m->gids.p;
        mv.orient = m->orient.p;
        mv.Bs = m->has_bs ? m->Bs.p : nullptr;
        mv.n_int = m->n_int;
        mv.relc = m->relc.p;
        mv.relx = m->relx.p;
        mv.phi = (m->diluted && m->has_bs) ? m->phi.p : nullptr;
        for (int k = 0; k < 4; ++k) mv.dil[k] = m->dil[k];
        s->views.push_back(mv);
    }
    v->n_mats = (int)s->views.size();
    v->mats = s->views.data();
    return SNP_OK;
}

}  // namespace snp

extern "C" {

int snp_solver_create(int32_t n_dofs, const double *nodes, int64_t n_nodes, const double *curls, int32_t n_orient,
                      const double *d_phi, const double *w, int32_t n_quad, const uint8_t *free_mask, void *stream,
                      snp_solver **out) {
    snp::clear_error();
    SNP_REQUIRE(out != nullptr, "snp_solver_create: out is NULL");
    *out = nullptr;
    SNP_REQUIRE(n_dofs > 0 && n_nodes > 0 && n_orient > 0 && n_quad > 0, "snp_solver_create: sizes must be positive");
    SNP_REQUIRE(nodes && curls && d_phi && w && free_mask, "snp_solver_create: NULL argument");
    cudaStream_t st = snp::as_stream(stream);
    bool affine = false;
    SNP_TRY(snp::check_affine_tables(curls, n_orient, d_phi, n_quad, st, &affine));
    SNP_REQUIRE(affine, "snp_solver_create: d_phi/curls vary across quadrature points; only affine first-order tetrahedra are supported");
    auto S = std::make_unique<snp_solver>();
    S->n = n_dofs;
    S->n_nodes = n_nodes;
    S->nq = n_quad;
    S->n_orient = n_orient;
    S->stream = st;
    SNP_TRY(S->nodes.alloc(3 * n_nodes));
    SNP_TRY(S->curls.alloc((size_t)n_orient * n_quad * 18));
    SNP_TRY(S->dphi.alloc((size_t)n_quad * 12));
    SNP_TRY(S->w.alloc(n_quad));
    SNP_TRY(S->free_mask.alloc(n_dofs));
    SNP_CUDA_TRY(cudaMemcpyAsync(S->nodes.p, nodes, sizeof(double) * 3 * n_nodes, cudaMemcpyDeviceToDevice, st));
    SNP_CUDA_TRY(cudaMemcpyAsync(S->curls.p, curls, sizeof(double) * n_orient * n_quad * 18, cudaMemcpyDeviceToDevice, st));
    SNP_CUDA_TRY(cudaMemcpyAsync(S->dphi.p, d_phi, sizeof(double) * n_quad * 12, cudaMemcpyDeviceToDevice, st));
    SNP_CUDA_TRY(cudaMemcpyAsync(S->w.p, w, sizeof(double) * n_quad, cudaMemcpyDeviceToDevice, st));
    SNP_CUDA_TRY(cudaMemcpyAsync(S->free_mask.p, free_mask, n_dofs, cudaMemcpyDeviceToDevice, st));
    for (auto &e : S->ev) SNP_CUDA_TRY(cudaEventCreate(&e));
    *out = S.release();
    return SNP_OK;
}

int snp_solver_add_material(snp_solver *s, const int32_t *cells, const int32_t *glob_ids, const int32_t *orientations,
                            int64_t n_elems, int32_t n_int, const double *rel_c, const double *rel_x, const double *B_s) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr, "snp_solver_add_material: solver is NULL");
    SNP_REQUIRE(!s->finalized, "snp_solver_add_material: solver already finalized");
    SNP_REQUIRE(n_elems >= 0, "snp_solver_add_material: negative element count");
    SNP_REQUIRE(n_int == -1 || n_int >= 1, "snp_solver_add_material: n_int must be -1 or >= 1");
    SNP_REQUIRE(rel_c && (n_int < 0 || rel_x), "snp_solver_add_material: reluctance tables missing");
    SNP_REQUIRE(n_elems == 0 || (cells && glob_ids && orientations), "snp_solver_add_material: NULL mesh arrays");
    auto m = std::make_unique<snp::Material>();
    m->offset = s->n_elems_total();
    m->count = n_elems;
    m->n_int = n_int;
    cudaStream_t st = s->stream;
    SNP_TRY(m->cells.alloc(4 * n_elems));
    SNP_TRY(m->gids.alloc(6 * n_elems));
    SNP_TRY(m->orient.alloc(n_elems));
    if (n_elems) {
        SNP_CUDA_TRY(cudaMemcpyAsync(m->cells.p, cells, sizeof(int32_t) * 4 * n_elems, cudaMemcpyDeviceToDevice, st));
        SNP_CUDA_TRY(cudaMemcpyAsync(m->gids.p, glob_ids, sizeof(int32_t) * 6 * n_elems, cudaMemcpyDeviceToDevice, st));
        SNP_CUDA_TRY(cudaMemcpyAsync(m->orient.p, orientations, sizeof(int32_t) * n_elems, cudaMemcpyDeviceToDevice, st));
    }
    const int nc = n_int < 0 ? 1 : 4 * n_int, nx = n_int < 0 ? 1 : n_int + 1;
    SNP_TRY(m->relc.alloc(nc));
    SNP_TRY(m->relx.alloc(nx));
    SNP_CUDA_TRY(cudaMemcpyAsync(m->relc.p, rel_c, sizeof(double) * nc, cudaMemcpyDeviceToDevice, st));
    if (n_int >= 0) SNP_CUDA_TRY(cudaMemcpyAsync(m->relx.p, rel_x, sizeof(double) * nx, cudaMemcpyDeviceToDevice, st));
    else SNP_CUDA_TRY(cudaMemsetAsync(m->relx.p, 0, sizeof(double), st));
    if (B_s && n_elems) {
        m->has_bs = true;
        SNP_TRY(m->Bs.alloc((size_t)n_elems * s->nq * 3));
        SNP_CUDA_TRY(cudaMemcpyAsync(m->Bs.p, B_s, sizeof(double) * n_elems * s->nq * 3, cudaMemcpyDeviceToDevice, st));
    }
    s->mats.push_back(std::move(m));
    return SNP_OK;
}

int snp_solver_set_rhs(snp_solver *s, const double *rhs) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr, "snp_solver_set_rhs: solver is NULL");
    if (!rhs) {
        s->has_extra = false;
        return SNP_OK;
    }
    if (!s->rhs_extra.p) SNP_TRY(s->rhs_extra.alloc(s->n));
    SNP_CUDA_TRY(cudaMemcpyAsync(s->rhs_extra.p, rhs, sizeof(double) * s->n, cudaMemcpyDeviceToDevice, s->stream));
    s->has_extra = true;
    return SNP_OK;
}

int snp_solver_finalize(snp_solver *s) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr, "snp_solver_finalize: solver is NULL");
    SNP_REQUIRE(!s->finalized, "snp_solver_finalize: already finalized");
    SNP_REQUIRE(!s->mats.empty(), "snp_solver_finalize: no materials");
    const int64_t E = s->n_elems_total();
    cudaStream_t st = s->stream;
    snp::DevBuf<int32_t> all;
    SNP_TRY(all.alloc(6 * E));
    for (auto &m : s->mats)
        if (m->count)
            SNP_CUDA_TRY(cudaMemcpyAsync(all.p + 6 * m->offset, m->gids.p, sizeof(int32_t) * 6 * m->count,
                                         cudaMemcpyDeviceToDevice, st));
    SNP_TRY(snp::pattern_create(all.p, E, 6, s->n, st, &s->pat));
    int64_t nnz = s->pat->nnz;
    // CSR assembly: deterministic row gather (default) or element atomics (SNP_ASSEMBLY=atomic)
    {
        const char *ea = getenv("SNP_ASSEMBLY");
        s->rows_asm = snp::rows_supported(s->pat) && !(ea && std::string(ea) == "atomic");
    }
    // Newton-loop Jacobian layout: SNP_JACOBIAN = elem (default) | csr | sell
    const char *env = getenv("SNP_JACOBIAN");
    const std::string want = env ? env : "elem";
    s->layout = want == "csr" ? SNP_LAYOUT_CSR : want == "sell" ? SNP_LAYOUT_SELL : SNP_LAYOUT_ELEM;
    if (s->layout == SNP_LAYOUT_ELEM) {
        std::vector<double> ctab((size_t)s->n_orient * 18);
        for (int o = 0; o < s->n_orient; ++o)
            SNP_CUDA_TRY(cudaMemcpyAsync(ctab.data() + (size_t)o * 18, s->curls.p + (size_t)o * s->nq * 18,
                                         18 * sizeof(double), cudaMemcpyDeviceToHost, st));
        SNP_CUDA_TRY(cudaStreamSynchronize(st));
        std::vector<snp::ElemBlock> blocks;
        for (auto &m : s->mats) blocks.push_back(snp::ElemBlock{m->gids.p, m->orient.p, m->count, m->offset});
        bool usable = false;
        SNP_TRY(snp::build_elem_topology(s->etop, s->n, blocks.data(), (int)blocks.size(), ctab.data(), s->n_orient,
                                         st, &usable));
        if (usable) {
            SNP_TRY(s->T64.alloc(snp::eslots_size(E)));
            SNP_TRY(s->Fe.alloc(snp::eslots_size(E)));
            SNP_TRY(s->De.alloc(snp::eslots_size(E)));
            SNP_TRY(s->T32.alloc(snp::eslots_size(E)));
            SNP_TRY(s->Jdiag.alloc(s->n));
        } else {
            s->layout = SNP_LAYOUT_CSR;
        }
    }
    s->use_sell = s->layout == SNP_LAYOUT_SELL;
    if (s->use_sell) {
        SNP_TRY(snp::build_sell(s->pat, s->sell, st));
        if (s->sell.total > nnz) nnz = s->sell.total;
    }
    SNP_TRY(s->J.alloc(nnz));
    SNP_TRY(s->J32.alloc(nnz));
    SNP_TRY(s->F.alloc(s->n));
    SNP_TRY(s->b.alloc(s->n));
    SNP_TRY(s->xw.alloc(s->n));
    SNP_TRY(s->h.alloc(s->n));
    SNP_TRY(s->b32.alloc(s->n));
    SNP_TRY(s->h32.alloc(s->n));
    SNP_TRY(s->part.alloc(3 * (size_t)(snp::sm_count() * 4 + 1)));
    SNP_TRY(s->res.alloc(3));
    SNP_TRY(s->counter.alloc(1));
    SNP_TRY(s->hres.alloc(3));
    SNP_CUDA_TRY(cudaMemsetAsync(s->counter.p, 0, sizeof(unsigned int), st));
    snp::DevBuf<unsigned long long> cnt;
    SNP_TRY(cnt.alloc(1));
    SNP_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), st));
    snp::k_count_free<<<snp::stride_grid(s->n, snp::kVB, 4), snp::kVB, 0, st>>>(s->n, s->free_mask.p, cnt.p);
    SNP_LAUNCH_CHECK();
    unsigned long long hc = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&hc, cnt.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
    SNP_CUDA_TRY(cudaStreamSynchronize(st));
    s->n_free = (int64_t)hc;
    SNP_TRY(s->pcg64.reserve(s->n));
    SNP_TRY(s->pcg32.reserve(s->n));
    s->finalized = true;
    return SNP_OK;
}

int snp_solver_solve(snp_solver *s, double *x, const snp_solve_opts *opts, snp_solve_stats *stats) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_solve: solver missing or not finalized");
    SNP_REQUIRE(x && opts, "snp_solver_solve: NULL argument");
    SNP_REQUIRE(opts->max_newton >= 1, "snp_solver_solve: max_newton must be >= 1");
    SNP_REQUIRE(opts->tol > 0, "snp_solver_solve: tol must be positive");
    SNP_REQUIRE(opts->precision == 0 || opts->precision == 1, "snp_solver_solve: precision must be 0 or 1");
    snp_solve_stats tmp;
    snp_solve_stats &S = stats ? *stats : tmp;
    return s->solve(x, *opts, S);
}

int snp_solver_solve_many(snp_solver *const *solvers, int32_t count, double *const *x, const snp_solve_opts *opts,
                          snp_solve_stats *stats, int32_t n_threads, int32_t *status) {
    snp::clear_error();
    SNP_REQUIRE(count >= 0, "snp_solver_solve_many: negative count");
    if (count == 0) return SNP_OK;
    SNP_REQUIRE(solvers && x && opts, "snp_solver_solve_many: NULL argument");
    for (int32_t i = 0; i < count; ++i) {
        SNP_REQUIRE(solvers[i] && solvers[i]->finalized && x[i], "snp_solver_solve_many: instance %d missing", i);
        for (int32_t j = 0; j < i; ++j)
            SNP_REQUIRE(solvers[j] != solvers[i], "snp_solver_solve_many: instances %d and %d share a solver", j, i);
    }
    int dev = 0;
    SNP_CUDA_TRY(cudaGetDevice(&dev));
    const int32_t nt = (n_threads <= 0 || n_threads > count) ? count : n_threads;
    std::atomic<int32_t> next{0};
    std::vector<int> rc((size_t)count, SNP_OK);
    std::vector<std::string> msg((size_t)count);
    auto worker = [&]() {
        if (cudaSetDevice(dev) != cudaSuccess) cudaGetLastError();
        for (;;) {
            const int32_t i = next.fetch_add(1);
            if (i >= count) break;
            snp_solve_stats tmp;
            rc[i] = snp_solver_solve(solvers[i], x[i], &opts[i], stats ? &stats[i] : &tmp);
            if (rc[i] != SNP_OK) msg[i] = snp_last_error();
        }
    };
    // the persisting-L2 set-aside is one setting of the whole context: solves running at once
    // leave it alone (a solve alone raises it around each Krylov solve)
    for (int32_t i = 0; i < count; ++i) solvers[i]->epcg64.l2_hold = solvers[i]->epcg32.l2_hold = false;
    std::vector<std::thread> pool;
    for (int32_t t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto &th : pool) th.join();
    for (int32_t i = 0; i < count; ++i) solvers[i]->epcg64.l2_hold = solvers[i]->epcg32.l2_hold = true;
    int first = -1;
    for (int32_t i = 0; i < count; ++i) {
        if (status) status[i] = rc[i];
        if (rc[i] != SNP_OK && first < 0) first = i;
    }
    if (first >= 0) return snp::fail(rc[first], "instance %d: %s", first, msg[first].c_str());
    return SNP_OK;
}

int snp_solver_assemble(snp_solver *s, const double *x, double *K_vals, double *J_vals, double *rhs, double *F,
                        void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_assemble: solver missing or not finalized");
    SNP_REQUIRE(x != nullptr, "snp_solver_assemble: x is NULL");
    cudaStream_t keep = s->stream;
    if (stream) s->stream = snp::as_stream(stream);
    int rc = s->assemble(x, K_vals, J_vals, nullptr, rhs, F);
    s->stream = keep;
    return rc;
}

int snp_solver_assemble_tensors(snp_solver *s, const double *x, int precision, double *F, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_assemble_tensors: solver missing or not finalized");
    SNP_REQUIRE(s->layout == SNP_LAYOUT_ELEM, "snp_solver_assemble_tensors: the solver's Jacobian layout is not elem");
    SNP_REQUIRE(precision == 0 || precision == 1, "snp_solver_assemble_tensors: precision must be 0 or 1");
    SNP_REQUIRE(x != nullptr, "snp_solver_assemble_tensors: x is NULL");
    cudaStream_t keep = s->stream;
    if (stream) s->stream = snp::as_stream(stream);
    int rc = s->assemble_elem(x, precision == 1, F ? F : s->F.p);
    s->stream = keep;
    return rc;
}

int snp_solver_jacobian_apply(snp_solver *s, int precision, const void *x, void *y, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_jacobian_apply: solver missing or not finalized");
    SNP_REQUIRE(precision == 0 || precision == 1, "snp_solver_jacobian_apply: precision must be 0 or 1");
    SNP_REQUIRE(x != nullptr && y != nullptr, "snp_solver_jacobian_apply: x or y is NULL");
    SNP_REQUIRE(s->j_valid[precision], "snp_solver_jacobian_apply: no %s Newton Jacobian (run a solve first)",
                precision ? "float32" : "float64");
    return s->apply_jacobian(precision, x, y, stream ? snp::as_stream(stream) : s->stream);
}

int snp_solver_set_krylov(snp_solver *s, int32_t method, int32_t restart) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_set_krylov: solver missing or not finalized");
    SNP_REQUIRE(method == SNP_KRYLOV_CG || method == SNP_KRYLOV_GMRES, "snp_solver_set_krylov: unknown method %d",
                method);
    SNP_REQUIRE(method == SNP_KRYLOV_CG || s->layout == SNP_LAYOUT_ELEM,
                "snp_solver_set_krylov: GMRES needs the matrix-free (elem) Jacobian layout");
    SNP_REQUIRE(restart >= 1 && restart <= 200, "snp_solver_set_krylov: restart must be in [1, 200] (got %d)", restart);
    s->krylov = method;
    s->krylov_restart = restart;
    return SNP_OK;
}

int snp_solver_set_block_jacobi(snp_solver *s, const uint16_t *meta) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_set_block_jacobi: solver missing or not finalized");
    if (meta == nullptr) {
        s->bj_on = false;
        return SNP_OK;
    }
    SNP_REQUIRE(s->layout == SNP_LAYOUT_ELEM, "snp_solver_set_block_jacobi: the solver's Jacobian layout is not elem");
    const int32_t n = s->n;
    std::vector<uint8_t> fm((size_t)n);
    SNP_CUDA_TRY(cudaMemcpy(fm.data(), s->free_mask.p, (size_t)n, cudaMemcpyDeviceToHost));
    // every block: 1..8 consecutive DoFs inside one 256-DoF tile, offsets 0..size-1 in order,
    // free DoFs only unless it is a constrained DoF alone
    for (int32_t i = 0; i < n;) {
        const int off = meta[i] & 0xff, size = meta[i] >> 8;
        SNP_REQUIRE(off == 0 && size >= 1 && size <= snp::kBlockJacobiMax && i + size <= n &&
                        (i / 256) == ((i + size - 1) / 256),
                    "snp_solver_set_block_jacobi: bad block at DoF %d (offset %d, size %d)", i, off, size);
        for (int k = 0; k < size; ++k) {
            SNP_REQUIRE((meta[i + k] & 0xff) == k && (meta[i + k] >> 8) == size,
                        "snp_solver_set_block_jacobi: inconsistent block at DoF %d", i + k);
            SNP_REQUIRE(size == 1 || fm[i + k], "snp_solver_set_block_jacobi: constrained DoF %d inside a block", i + k);
        }
        i += size;
    }
    SNP_TRY(s->bj_meta.alloc(n));
    SNP_TRY(s->bj_mat.alloc((size_t)n * snp::kBlockJacobiMax));
    SNP_TRY(s->bj_inv.alloc((size_t)n * snp::kBlockJacobiMax));
    SNP_TRY(s->bj_fallback.alloc(1));
    SNP_CUDA_TRY(cudaMemcpy(s->bj_meta.p, meta, sizeof(uint16_t) * n, cudaMemcpyHostToDevice));
    SNP_CUDA_TRY(cudaMemset(s->bj_fallback.p, 0, sizeof(int)));
    s->bj_on = true;
    return SNP_OK;
}

int snp_solver_precond_apply(snp_solver *s, int precision, const double *r, double *z, int32_t *fallback_blocks,
                             void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_precond_apply: solver missing or not finalized");
    SNP_REQUIRE(s->layout == SNP_LAYOUT_ELEM && s->bj_on, "snp_solver_precond_apply: no block Jacobi on this solver");
    SNP_REQUIRE(precision == 0 || precision == 1, "snp_solver_precond_apply: precision must be 0 or 1");
    SNP_REQUIRE(s->j_valid[precision], "snp_solver_precond_apply: no %s Newton Jacobian (assemble first)",
                precision ? "float32" : "float64");
    SNP_REQUIRE(r != nullptr && z != nullptr, "snp_solver_precond_apply: r or z is NULL");
    cudaStream_t keep = s->stream;
    if (stream) s->stream = snp::as_stream(stream);
    const int rc = s->precond_apply(precision == 1, r, z, fallback_blocks);
    s->stream = keep;
    return rc;
}

int snp_solver_block_jacobi_export(snp_solver *s, int precision, double *bmat, float *binv, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized && s->bj_on, "snp_solver_block_jacobi_export: no block Jacobi");
    SNP_REQUIRE(precision == 0 || precision == 1, "snp_solver_block_jacobi_export: precision must be 0 or 1");
    SNP_REQUIRE(s->j_valid[precision], "snp_solver_block_jacobi_export: assemble first");
    cudaStream_t st = stream ? snp::as_stream(stream) : s->stream;
    cudaStream_t keep = s->stream;
    s->stream = st;
    int rc = s->build_block_jacobi(precision == 1);
    s->stream = keep;
    SNP_TRY(rc);
    const size_t m = (size_t)s->n * snp::kBlockJacobiMax;
    if (bmat) SNP_CUDA_TRY(cudaMemcpyAsync(bmat, s->bj_mat.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, st));
    if (binv) SNP_CUDA_TRY(cudaMemcpyAsync(binv, s->bj_inv.p, sizeof(float) * m, cudaMemcpyDeviceToDevice, st));
    return SNP_OK;
}

int snp_spd_solve(int32_t m, const double *A, const double *g, double *c) {
    snp::clear_error();
    SNP_REQUIRE(m >= 1 && A != nullptr && g != nullptr && c != nullptr, "snp_spd_solve: bad arguments");
    SNP_REQUIRE(snp::spd_solve(m, A, g, c), "snp_spd_solve: non-positive or non-finite diagonal, or non-finite solution");
    return SNP_OK;
}

int snp_solver_set_galerkin_basis(snp_solver *s, const float *V, int32_t m, int64_t ldv, int32_t steps) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_set_galerkin_basis: solver missing or not finalized");
    if (V == nullptr || m == 0 || steps == 0) {
        s->gal_V = nullptr;
        s->gal_m = s->gal_steps = 0;
        return SNP_OK;
    }
    SNP_REQUIRE(s->layout == SNP_LAYOUT_ELEM, "snp_solver_set_galerkin_basis: the solver's Jacobian layout is not elem");
    SNP_REQUIRE(m >= 1 && m <= 128 && ldv >= m && steps >= 1, "snp_solver_set_galerkin_basis: need 1 <= m <= 128, "
                "ldv >= m and steps >= 1");
    if (s->gal_sys.n < (size_t)m * m + 2 * (size_t)m) {
        SNP_TRY(s->gal_sys.alloc((size_t)m * m + 2 * (size_t)m));
        SNP_TRY(s->gal_host.alloc((size_t)m * m + 2 * (size_t)m));
    }
    if (s->gal_x.n < (size_t)s->n) SNP_TRY(s->gal_x.alloc(s->n));
    s->gal_V = V;
    s->gal_m = m;
    s->gal_ldv = ldv;
    s->gal_steps = steps;
    return SNP_OK;
}

int snp_solver_reduced_system(snp_solver *s, int precision, const float *V, int m, int64_t ldv, const double *F,
                              double *Jr, double *g, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && s->finalized, "snp_solver_reduced_system: solver missing or not finalized");
    SNP_REQUIRE(s->layout == SNP_LAYOUT_ELEM, "snp_solver_reduced_system: the solver's Jacobian layout is not elem");
    SNP_REQUIRE(precision == 0 || precision == 1, "snp_solver_reduced_system: precision must be 0 or 1");
    SNP_REQUIRE(s->j_valid[precision], "snp_solver_reduced_system: no %s Newton Jacobian (assemble first)",
                precision ? "float32" : "float64");
    cudaStream_t st = stream ? snp::as_stream(stream) : s->stream;
    if (precision == 0)
        return snp::elem_reduced_system(s->etop, s->T64.p, s->free_mask.p, V, m, ldv, F, Jr, g, s->rsys_scratch, st);
    return snp::elem_reduced_system(s->etop, s->T32.p, s->free_mask.p, V, m, ldv, F, Jr, g, s->rsys_scratch, st);
}

int snp_solver_jacobian_layout(const snp_solver *s, int *layout) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && layout != nullptr && s->finalized,
                "snp_solver_jacobian_layout: solver missing or not finalized");
    *layout = s->layout;
    return SNP_OK;
}

int snp_solver_set_nodes(snp_solver *s, const double *nodes, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && nodes != nullptr, "snp_solver_set_nodes: NULL argument");
    SNP_CUDA_TRY(cudaMemcpyAsync(s->nodes.p, nodes, sizeof(double) * 3 * s->n_nodes, cudaMemcpyDeviceToDevice,
                                 stream ? snp::as_stream(stream) : s->stream));
    s->j_valid[0] = s->j_valid[1] = 0;
    return SNP_OK;
}

int snp_solver_set_dilution(snp_solver *s, int32_t material, const double *phi, const double *dilution) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr, "snp_solver_set_dilution: solver is NULL");
    SNP_REQUIRE(material >= 0 && material < (int32_t)s->mats.size(), "snp_solver_set_dilution: no material %d", material);
    auto &m = *s->mats[material];
    if (dilution == nullptr) {
        m.diluted = false;
        return SNP_OK;
    }
    SNP_REQUIRE(phi != nullptr, "snp_solver_set_dilution: phi is NULL");
    SNP_REQUIRE(std::isfinite(dilution[0]) && std::isfinite(dilution[1]) && std::isfinite(dilution[2]) &&
                    std::isfinite(dilution[3]),
                "snp_solver_set_dilution: coefficients must be finite");
    if (!m.phi.p) SNP_TRY(m.phi.alloc((size_t)4 * s->nq));
    SNP_CUDA_TRY(cudaMemcpyAsync(m.phi.p, phi, sizeof(double) * 4 * s->nq, cudaMemcpyDeviceToDevice, s->stream));
    for (int i = 0; i < 4; ++i) m.dil[i] = dilution[i];
    m.diluted = true;
    return SNP_OK;
}

int snp_solver_set_source(snp_solver *s, int32_t material, const double *B_s, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(s != nullptr && B_s != nullptr, "snp_solver_set_source: NULL argument");
    SNP_REQUIRE(material >= 0 && material < (int32_t)s->mats.size(), "snp_solver_set_source: no material %d", material);
    snp::Material &m = *s->mats[material];
    SNP_REQUIRE(m.has_bs, "snp_solver_set_source: material %d was added without a source field", material);
    SNP_CUDA_TRY(cudaMemcpyAsync(m.Bs.p, B_s, sizeof(double) * m.count * s->nq * 3, cudaMemcpyDeviceToDevice,
                                 stream ? snp::as_stream(stream) : s->stream));
    s->j_valid[0] = s->j_valid[1] = 0;
    return SNP_OK;
}

int snp_solver_pattern(const snp_solver *s, const snp_pattern **pat) {
    SNP_REQUIRE(s != nullptr && pat != nullptr && s->finalized, "snp_solver_pattern: solver missing or not finalized");
    *pat = s->pat;
    return SNP_OK;
}

int snp_solver_destroy(snp_solver *s) {
    delete s;
    return SNP_OK;
}

}  // extern "C"
