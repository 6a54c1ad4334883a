// Restarted GMRES(m) with right preconditioning for the Newton step J h = b (b = b_scale F on the
// free DoFs, zero elsewhere), float64 vectors, for the residual-mode Newton loop
// (snp_solver_set_krylov).  The reference solves each Newton step with scipy's Jacobi-
// preconditioned cg (red_mvp_solver.py:199-203); GMRES is the Krylov method for Jacobians that are
// not symmetric positive definite on the free DoFs, with the same matrix-free operator and the
// same (block or point) Jacobi preconditioner as the CG.
//
// One Arnoldi step: z = M v_j, w = J z, classical Gram-Schmidt applied twice (h = V^T w,
// w -= V h, twice: orthogonality to rounding level with two fused passes over V), ||w||,
// v_{j+1} = w / ||w||.  Every dot product is deterministic: block partials summed in a fixed
// order by the last block.  The host reads the new Hessenberg column once per step, applies the
// Givens rotations and tracks |g_{j+1}| = ||b - J x_j||; at the end of a cycle (restart, or
// convergence) it solves the triangular system and x += M (V y).
#include <cmath>
#include <vector>

#include "snp_common.cuh"
#include "snp_internal.cuh"
#include "snp_krylov.cuh"
#include "snp_reduce.cuh"

namespace snp {

namespace {

constexpr int kGB = 256;
constexpr int kVB = 256;

// h[i] = V_i . w for i < k (V_i = V + i * ld); per-block partials, the last block sums them in
// block order
__global__ void __launch_bounds__(kGB) k_gm_mdot(int64_t n, const double *__restrict__ V, int64_t ld, int k,
                                                 const double *__restrict__ w, double *__restrict__ part,
                                                 double *__restrict__ h, unsigned int *counter) {
    __shared__ double sh[32];
    for (int i = 0; i < k; ++i) {
        double a = 0.0;
        const double *v = V + (int64_t)i * ld;
        for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
            a = fma(__ldg(v + r), __ldg(w + r), a);
        a = block_sum(a, sh);
        if (threadIdx.x == 0) part[(int64_t)i * gridDim.x + blockIdx.x] = a;
    }
    if (last_block(counter)) {
        for (int i = 0; i < k; ++i) {
            const double s = reduce_parts(part + (int64_t)i * gridDim.x, gridDim.x, 1, 0, sh);
            if (threadIdx.x == 0) h[i] = s;
        }
    }
}

// w -= sum_{i<k} h[i] V_i
__global__ void k_gm_update(int64_t n, const double *__restrict__ V, int64_t ld, int k, const double *__restrict__ h,
                            double *__restrict__ w) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double t = w[r];
        for (int i = 0; i < k; ++i) t = fma(-__ldg(h + i), __ldg(V + (int64_t)i * ld + r), t);
        w[r] = t;
    }
}

// out = w / sqrt(ss[0]) (out = 0 when the norm is 0)
__global__ void k_gm_scale(int64_t n, const double *__restrict__ w, const double *__restrict__ ss,
                           double *__restrict__ out) {
    const double s = ss[0];
    const double inv = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        out[r] = w[r] * inv;
}

// u = sum_{i<k} y[i] V_i
__global__ void k_gm_combine(int64_t n, const double *__restrict__ V, int64_t ld, int k, const double *__restrict__ y,
                             double *__restrict__ u) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int i = 0; i < k; ++i) t = fma(__ldg(y + i), __ldg(V + (int64_t)i * ld + r), t);
        u[r] = t;
    }
}

// r = b_scale b - Ax on the free DoFs (0 elsewhere); with Ax == nullptr r = b_scale b
__global__ void k_gm_resid(int64_t n, const uint8_t *__restrict__ fm, const double *__restrict__ b, double b_scale,
                           const double *__restrict__ Ax, double *__restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = is_free(fm, i) ? b_scale * b[i] - (Ax ? Ax[i] : 0.0) : 0.0;
}

__global__ void k_gm_add(int64_t n, const double *__restrict__ z, double *__restrict__ x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] += z[i];
}

__global__ void k_pj_apply(int64_t n, const uint8_t *__restrict__ fm, const double *__restrict__ diag,
                           const double *__restrict__ r, double *__restrict__ z) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z[i] = is_free(fm, i) ? r[i] / diag[i] : 0.0;
}

}  // namespace

int point_jacobi_apply(int32_t n, const uint8_t *free_mask, const double *diag, const double *r, double *z,
                       cudaStream_t s) {
    SNP_REQUIRE(diag && r && z && n > 0, "point Jacobi apply: bad arguments");
    k_pj_apply<<<stride_grid(n, kVB, 4), kVB, 0, s>>>(n, free_mask, diag, r, z);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int Gmres::reserve(int64_t n_, int m_) {
    if (n_ == n && m_ == m) return SNP_OK;
    n = n_;
    m = m_;
    blocks = stride_grid(n, kGB, 4);
    SNP_TRY(V.alloc((size_t)(m + 1) * (size_t)n));
    SNP_TRY(w.alloc(n));
    SNP_TRY(z.alloc(n));
    SNP_TRY(part.alloc((size_t)(m + 1) * blocks));
    SNP_TRY(hdev.alloc(2 * (size_t)(m + 1) + 2));
    SNP_TRY(counter.alloc(1));
    SNP_TRY(hhost.alloc(2 * (size_t)(m + 1) + 2));
    SNP_CUDA_TRY(cudaMemset(counter.p, 0, sizeof(unsigned int)));
    return SNP_OK;
}

int Gmres::solve(const Op &apply_J, const Op &apply_M, const uint8_t *free_mask, const double *b, double b_scale,
                 double *x, double rtol, double atol, int64_t maxit, cudaStream_t s, int64_t *its_out,
                 double *res_out, int *status) {
    *its_out = 0;
    *res_out = 0.0;
    *status = SNP_OK;
    const int grid = stride_grid(n, kVB, 4);
    double *hh = hhost.p;
    double *h1 = hdev.p, *h2 = hdev.p + (m + 1), *hn = hdev.p + 2 * (m + 1);
    auto mdot = [&](int k, const double *vec, double *out) -> int {
        k_gm_mdot<<<blocks, kGB, 0, s>>>(n, V.p, n, k, vec, part.p, out, counter.p);
        SNP_LAUNCH_CHECK();
        ++launches;
        return SNP_OK;
    };
    auto norm2 = [&](const double *vec, double *out) -> int {
        // ||vec||^2 with vec placed as the "basis" and itself as the vector
        k_gm_mdot<<<blocks, kGB, 0, s>>>(n, vec, n, 1, vec, part.p, out, counter.p);
        SNP_LAUNCH_CHECK();
        ++launches;
        return SNP_OK;
    };
    // x starts at 0: r = b_scale b
    SNP_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
    k_gm_resid<<<grid, kVB, 0, s>>>(n, free_mask, b, b_scale, nullptr, w.p);
    SNP_LAUNCH_CHECK();
    SNP_TRY(norm2(w.p, hn));
    SNP_CUDA_TRY(cudaMemcpyAsync(hh, hn, sizeof(double), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    const double bnorm = std::sqrt(hh[0]);
    const double tol = std::fmax(rtol * bnorm, atol);
    double beta = bnorm;
    int64_t its = 0;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    while (true) {
        if (!(beta == beta)) {
            *status = SNP_NAN_DETECTED;
            break;
        }
        if (beta <= tol || its >= maxit) break;
        // v_0 = r / beta
        k_gm_scale<<<grid, kVB, 0, s>>>(n, w.p, hn, V.p);
        SNP_LAUNCH_CHECK();
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int kdone = 0;
        double res = beta;
        for (int j = 0; j < m; ++j) {
            double *vj = V.p + (int64_t)j * n;
            SNP_TRY(apply_M(vj, z.p));
            SNP_TRY(apply_J(z.p, w.p));
            SNP_TRY(mdot(j + 1, w.p, h1));
            k_gm_update<<<grid, kVB, 0, s>>>(n, V.p, n, j + 1, h1, w.p);
            SNP_LAUNCH_CHECK();
            SNP_TRY(mdot(j + 1, w.p, h2));
            k_gm_update<<<grid, kVB, 0, s>>>(n, V.p, n, j + 1, h2, w.p);
            SNP_LAUNCH_CHECK();
            SNP_TRY(norm2(w.p, hn));
            k_gm_scale<<<grid, kVB, 0, s>>>(n, w.p, hn, V.p + (int64_t)(j + 1) * n);
            SNP_LAUNCH_CHECK();
            launches += 4;
            SNP_CUDA_TRY(cudaMemcpyAsync(hh, hdev.p, sizeof(double) * (2 * (size_t)(m + 1) + 1), cudaMemcpyDeviceToHost, s));
            SNP_CUDA_TRY(cudaStreamSynchronize(s));
            ++its;
            // Hessenberg column j: h1 + h2 (both passes), subdiagonal ||w||
            double *col = H.data() + (size_t)j * (m + 1);
            for (int i = 0; i <= j; ++i) col[i] = hh[i] + hh[(m + 1) + i];
            const double sub = std::sqrt(hh[2 * (m + 1)]);
            for (int i = 0; i < j; ++i) {
                const double t = cs[i] * col[i] + sn[i] * col[i + 1];
                col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1];
                col[i] = t;
            }
            const double d = std::hypot(col[j], sub);
            if (d > 0.0) {
                cs[j] = col[j] / d;
                sn[j] = sub / d;
            } else {
                cs[j] = 1.0;
                sn[j] = 0.0;
            }
            col[j] = d;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            res = std::fabs(g[j + 1]);
            kdone = j + 1;
            if (!(res == res)) {
                *status = SNP_NAN_DETECTED;
                break;
            }
            if (res <= tol || its >= maxit || !(sub > 0.0)) break;
        }
        if (*status != SNP_OK) break;
        // y = R^{-1} g, x += M (V y)
        for (int i = kdone - 1; i >= 0; --i) {
            double t = g[i];
            for (int c = i + 1; c < kdone; ++c) t -= H[(size_t)c * (m + 1) + i] * y[c];
            const double rii = H[(size_t)i * (m + 1) + i];
            y[i] = rii != 0.0 ? t / rii : 0.0;
        }
        std::copy(y.begin(), y.begin() + kdone, hh);
        SNP_CUDA_TRY(cudaMemcpyAsync(hdev.p, hh, sizeof(double) * kdone, cudaMemcpyHostToDevice, s));
        k_gm_combine<<<grid, kVB, 0, s>>>(n, V.p, n, kdone, hdev.p, w.p);
        SNP_LAUNCH_CHECK();
        SNP_TRY(apply_M(w.p, z.p));
        k_gm_add<<<grid, kVB, 0, s>>>(n, z.p, x);
        SNP_LAUNCH_CHECK();
        launches += 2;
        if (res <= tol || its >= maxit) {
            beta = res;
            break;
        }
        // restart: r = b_scale b - J x, beta = ||r||
        SNP_TRY(apply_J(x, z.p));
        k_gm_resid<<<grid, kVB, 0, s>>>(n, free_mask, b, b_scale, z.p, w.p);
        SNP_LAUNCH_CHECK();
        SNP_TRY(norm2(w.p, hn));
        SNP_CUDA_TRY(cudaMemcpyAsync(hh, hn, sizeof(double), cudaMemcpyDeviceToHost, s));
        SNP_CUDA_TRY(cudaStreamSynchronize(s));
        beta = std::sqrt(hh[0]);
        launches += 2;
    }
    *its_out = its;
    *res_out = beta;
    if (*status == SNP_OK && beta > tol) *status = SNP_NOT_CONVERGED;
    return SNP_OK;
}

}  // namespace snp
