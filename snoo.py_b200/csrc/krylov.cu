// Sparse linear algebra on the device: masked CSR SpMV and Jacobi-preconditioned CG.
//
// The reference extracts J_c = J[mask,:][:,mask], builds M = diags(1/diag(J_c)) and calls
// scipy.sparse.linalg.cg (snoopy/red_mvp_solver.py:195-203).  Here the Dirichlet mask is
// applied inside the kernels (rows and columns with free[i] == 0 are skipped), so J is
// never copied, and the CG iteration runs entirely on the device:
//
//   per iteration  k_spmv_dot : q = A p, last block reduces p.q  -> alpha
//                  k_update   : x += alpha p, r -= alpha q, z = dinv r, last block
//                               reduces r.z and r.r -> beta, convergence flag
//                  k_pupdate  : p = z + beta p
//
// Block partial sums are reduced by whichever block finishes last (one atomicInc ticket
// per launch, no waiting), in a fixed order, so results are deterministic.  The loop is a
// CUDA-graph conditional WHILE node whose body clears its condition once the flag is set;
// the flag is set at convergence, at `maxiter` and on a non-finite residual, so the loop
// always ends.  Stopping rule of scipy's cg: ||r|| < max(atol, rtol * ||b||).
#include <cstdio>
#include <cstdlib>

#include "snp_common.cuh"
#include "snp_internal.cuh"
#include "snp_krylov.cuh"
#include "snp_reduce.cuh"

namespace snp {

namespace {

constexpr int kVecBlock = 256;
constexpr int kSpmvBlock = 256;
constexpr int kSpmvUnroll = 4;  // matrix entries per lane and pass
constexpr int kVecIlp = 4;      // vector elements per thread and pass

// y = A x restricted to free rows/cols; TPR threads per row.  DOT: also p.y partial sums.
template <typename VT, typename XT, int TPR, bool MASKCOL, bool DOT>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmv(int32_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci, const VT *__restrict__ v,
           const uint8_t *__restrict__ free_mask, const XT *__restrict__ x, XT *__restrict__ y, PcgState *st,
           double *part) {
    __shared__ double sh[32];
    if (DOT && st->done) return;
    const int lane = threadIdx.x % TPR;
    const int group = threadIdx.x / TPR;
    const int groups_per_block = kSpmvBlock / TPR;
    double dot = 0.0;
    // the loop bound is uniform across the block, so every lane reaches the shuffles
    for (int64_t base = (int64_t)blockIdx.x * groups_per_block; base < n; base += (int64_t)gridDim.x * groups_per_block) {
        const int64_t row = base + group;
        const bool valid = row < n;
        double s = 0.0;
        const bool fr = valid && is_free(free_mask, row);
        if (fr) {
            const int b = __ldg(rp + row), e = __ldg(rp + row + 1);
            // kSpmvUnroll independent index/value loads per lane before any gather; the matrix
            // is streamed (evict-first) so the gathered vector stays in L2
            for (int k0 = b; k0 < e; k0 += TPR * kSpmvUnroll) {
                int c[kSpmvUnroll];
                VT a[kSpmvUnroll];
#pragma unroll
                for (int u = 0; u < kSpmvUnroll; ++u) {
                    const int k = k0 + lane + u * TPR;
                    if (k < e) {
                        c[u] = __ldcs(ci + k);
                        a[u] = __ldcs(v + k);
                    } else {
                        c[u] = -1;
                        a[u] = VT(0);
                    }
                }
#pragma unroll
                for (int u = 0; u < kSpmvUnroll; ++u)
                    if (c[u] >= 0 && (!MASKCOL || is_free(free_mask, c[u])))
                        s += (double)a[u] * (double)__ldg(x + c[u]);
            }
        }
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, TPR);
        if (lane == 0 && valid) {
            y[row] = fr ? (XT)s : (XT)0;
            if (DOT && fr) dot += (double)x[row] * s;
        }
    }
    if (DOT) {
        dot = block_sum(dot, sh);
        if (threadIdx.x == 0) part[blockIdx.x] = dot;
        if (last_block(&st->counter)) {
            const double pq = reduce_parts(part, gridDim.x, 1, 0, sh);
            if (threadIdx.x == 0) {
                st->pq = pq;
                st->alpha = st->rz / pq;
            }
        }
    }
}

// x += alpha p, r -= alpha q, z = dinv r on free rows; r.z and r.r reduced by the last block,
// which also forms beta and the convergence flag.  kVecIlp independent elements per thread.
template <typename XT>
__global__ void __launch_bounds__(kVecBlock)
    k_update(int32_t n, const uint8_t *__restrict__ free_mask, XT *__restrict__ x, XT *__restrict__ r,
             XT *__restrict__ z, const XT *__restrict__ p, const XT *__restrict__ q, const XT *__restrict__ dinv,
             PcgState *st, double *part, int use_cond, cudaGraphConditionalHandle cond) {
    __shared__ double sh2[2][32];
    if (st->done) {
        if (use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
        return;
    }
    const XT alpha = (XT)st->alpha;
    double rz = 0.0, rr = 0.0;
    for (int64_t base = (int64_t)blockIdx.x * kVecBlock * kVecIlp; base < n;
         base += (int64_t)gridDim.x * kVecBlock * kVecIlp) {
        XT pv[kVecIlp], rv[kVecIlp], qv[kVecIlp], dv[kVecIlp], xv[kVecIlp];
        bool f[kVecIlp];
#pragma unroll
        for (int j = 0; j < kVecIlp; ++j) {
            const int64_t i = base + threadIdx.x + (int64_t)j * kVecBlock;
            f[j] = i < n && is_free(free_mask, i);
            if (f[j]) {
                pv[j] = p[i];
                rv[j] = r[i];
                qv[j] = q[i];
                dv[j] = dinv[i];
                xv[j] = x[i];
            }
        }
#pragma unroll
        for (int j = 0; j < kVecIlp; ++j) {
            if (f[j]) {
                const int64_t i = base + threadIdx.x + (int64_t)j * kVecBlock;
                const XT ri = rv[j] - alpha * qv[j];
                const XT zi = dv[j] * ri;
                x[i] = xv[j] + alpha * pv[j];
                r[i] = ri;
                z[i] = zi;
                rz += (double)ri * (double)zi;
                rr += (double)ri * (double)ri;
            }
        }
    }
    block_sum2(rz, rr, sh2);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rz;
        part[2 * blockIdx.x + 1] = rr;
    }
    if (last_block(&st->counter)) {
        double a = 0.0, b = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            a += __ldcg(part + 2 * i);
            b += __ldcg(part + 2 * i + 1);
        }
        __syncthreads();
        block_sum2(a, b, sh2);
        if (threadIdx.x == 0) {
            const double rz_new = a, rr_new = b;
            st->beta = rz_new / st->rz;
            st->rz = rz_new;
            st->rr = rr_new;
            st->iter += 1;
            int done = 0;
            if (!(rr_new == rr_new) || isinf(rr_new)) done = 3;
            else if (sqrt(rr_new) < st->atol_eff) done = 1;
            else if (st->iter >= st->maxit) done = 2;
            st->done = done;
            if (use_cond && done) cudaGraphSetConditional(cond, 0);
        }
    }
}

// p = z + beta p on free rows, kVecIlp independent elements per thread.
template <typename XT>
__global__ void __launch_bounds__(kVecBlock)
    k_pupdate(int32_t n, const uint8_t *__restrict__ free_mask, XT *__restrict__ p, const XT *__restrict__ z,
              const PcgState *st) {
    if (st->done) return;
    const XT beta = (XT)st->beta;
    for (int64_t base = (int64_t)blockIdx.x * kVecBlock * kVecIlp; base < n;
         base += (int64_t)gridDim.x * kVecBlock * kVecIlp) {
        XT zv[kVecIlp], pv[kVecIlp];
        bool f[kVecIlp];
#pragma unroll
        for (int j = 0; j < kVecIlp; ++j) {
            const int64_t i = base + threadIdx.x + (int64_t)j * kVecBlock;
            f[j] = i < n && is_free(free_mask, i);
            if (f[j]) {
                zv[j] = z[i];
                pv[j] = p[i];
            }
        }
#pragma unroll
        for (int j = 0; j < kVecIlp; ++j) {
            const int64_t i = base + threadIdx.x + (int64_t)j * kVecBlock;
            if (f[j]) p[i] = zv[j] + beta * pv[j];
        }
    }
}

// r = b - q (free rows), z = dinv r, p = z; x = 0 on non-free rows; partials of r.z, r.r, b.b
template <typename XT>
__global__ void __launch_bounds__(kVecBlock)
    k_init(int32_t n, const uint8_t *__restrict__ free_mask, const XT *__restrict__ b, XT *__restrict__ x,
           XT *__restrict__ r, XT *__restrict__ z, XT *__restrict__ p, const XT *__restrict__ q,
           const XT *__restrict__ dinv, PcgState *st, double *part, double rtol, double atol, long long maxit,
           int zero_x) {
    __shared__ double sh[32];
    double rz = 0.0, rr = 0.0, bb = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (is_free(free_mask, i)) {
            const XT bi = b[i];
            const XT ri = zero_x ? bi : (XT)(bi - q[i]);
            const XT zi = dinv[i] * ri;
            if (zero_x) x[i] = (XT)0;
            r[i] = ri;
            z[i] = zi;
            p[i] = zi;
            rz += (double)ri * (double)zi;
            rr += (double)ri * (double)ri;
            bb += (double)bi * (double)bi;
        } else {
            x[i] = (XT)0;
            r[i] = (XT)0;
            z[i] = (XT)0;
            p[i] = (XT)0;
        }
    }
    const double a0 = block_sum(rz, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x] = a0;
    const double a1 = block_sum(rr, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x + 1] = a1;
    const double a2 = block_sum(bb, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x + 2] = a2;
    if (last_block(&st->counter)) {
        const double s_rz = reduce_parts(part, gridDim.x, 3, 0, sh);
        const double s_rr = reduce_parts(part, gridDim.x, 3, 1, sh);
        const double s_bb = reduce_parts(part, gridDim.x, 3, 2, sh);
        if (threadIdx.x == 0) {
            st->rz = s_rz;
            st->rr = s_rr;
            st->bnorm = sqrt(s_bb);
            st->atol_eff = fmax(atol, rtol * st->bnorm);
            st->iter = 0;
            st->maxit = maxit;
            st->alpha = 0.0;
            st->beta = 0.0;
            int done = 0;
            if (s_bb == 0.0) done = 4;
            else if (!(s_rr == s_rr) || isinf(s_rr)) done = 3;
            else if (sqrt(s_rr) < st->atol_eff) done = 1;
            else if (maxit <= 0) done = 2;
            st->done = done;
        }
    }
}

template <typename VT, typename XT>
__global__ void k_dinv(int32_t n, const int32_t *__restrict__ diag_pos, const VT *__restrict__ vals,
                       const uint8_t *__restrict__ free_mask, XT *__restrict__ dinv, int *bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (is_free(free_mask, i)) {
            const int d = diag_pos[i];
            const double v = d >= 0 ? (double)vals[d] : 0.0;
            if (v == 0.0 || !(v == v)) {
                atomicExch(bad, 1);
                dinv[i] = (XT)0;
            } else {
                dinv[i] = (XT)(1.0 / v);
            }
        } else {
            dinv[i] = (XT)0;
        }
    }
}

__global__ void k_find_diag(int32_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                            int32_t *__restrict__ diag) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int lo = rp[r], hi = rp[r + 1] - 1, pos = -1;
        while (lo <= hi) {
            const int mid = (lo + hi) >> 1;
            const int c = ci[mid];
            if (c == r) {
                pos = mid;
                break;
            }
            if (c < r) lo = mid + 1; else hi = mid - 1;
        }
        diag[r] = pos;
    }
}

}  // namespace

int find_diag(int32_t n, const int32_t *rp, const int32_t *ci, int32_t *diag, cudaStream_t s) {
    k_find_diag<<<stride_grid(n, kVecBlock, 8), kVecBlock, 0, s>>>(n, rp, ci, diag);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

// lanes per row: each lane takes kSpmvUnroll entries per pass, so rows of up to
// kSpmvUnroll * TPR entries finish in one pass
int choose_tpr(int64_t nnz, int32_t n) {
    const double avg = n > 0 ? (double)nnz / n : 0.0;
    if (avg > 96) return 32;
    if (avg > 48) return 16;
    if (avg > 24) return 8;
    return 4;
}

template <typename VT, typename XT, int TPR, bool MASKCOL, bool DOT>
static void spmv_launch(int32_t n, const int32_t *rp, const int32_t *ci, const VT *v, const uint8_t *fm, const XT *x,
                        XT *y, PcgState *st, double *part, cudaStream_t s) {
    const int64_t groups = kSpmvBlock / TPR;
    auto kern = k_spmv<VT, XT, TPR, MASKCOL, DOT>;
    const int grid = wave_grid(kern, (n + groups - 1) / groups * kSpmvBlock, kSpmvBlock);
    kern<<<grid, kSpmvBlock, 0, s>>>(n, rp, ci, v, fm, x, y, st, part);
}

template <typename VT, typename XT, bool MASKCOL, bool DOT>
static int spmv_dispatch(int tpr, int32_t n, const int32_t *rp, const int32_t *ci, const VT *v, const uint8_t *fm,
                         const XT *x, XT *y, PcgState *st, double *part, cudaStream_t s) {
    switch (tpr) {
        case 4: spmv_launch<VT, XT, 4, MASKCOL, DOT>(n, rp, ci, v, fm, x, y, st, part, s); break;
        case 8: spmv_launch<VT, XT, 8, MASKCOL, DOT>(n, rp, ci, v, fm, x, y, st, part, s); break;
        case 16: spmv_launch<VT, XT, 16, MASKCOL, DOT>(n, rp, ci, v, fm, x, y, st, part, s); break;
        default: spmv_launch<VT, XT, 32, MASKCOL, DOT>(n, rp, ci, v, fm, x, y, st, part, s); break;
    }
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

// y = A x with A in SELL-C-sigma order: one warp per 32-row slice, one thread per row, four
// independent coalesced (column, value) loads per thread before the gathers.  DOT as k_spmv.
template <typename VT, typename XT, bool MASKCOL, bool DOT>
__global__ void __launch_bounds__(kSpmvBlock)
    k_spmv_sell(int64_t n_slices, const int64_t *__restrict__ off, const int32_t *__restrict__ srow,
                const int32_t *__restrict__ col, const VT *__restrict__ v, const uint8_t *__restrict__ free_mask,
                const XT *__restrict__ x, XT *__restrict__ y, PcgState *st, double *part) {
    __shared__ double sh[32];
    if (DOT && st->done) return;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double dot = 0.0;
    for (int64_t sl = warp; sl < n_slices; sl += nwarps) {
        const int32_t row = __ldg(srow + sl * 32 + lane);
        if (row < 0) continue;
        const int64_t o = __ldg(off + sl);
        const int L = (int)((__ldg(off + sl + 1) - o) >> 5);
        const bool fr = is_free(free_mask, row);
        double sum = 0.0;
        if (fr) {
            const VT *vp = v + o + lane;
            const int32_t *cp = col + o + lane;
            int k = 0;
            for (; k + kSpmvUnroll <= L; k += kSpmvUnroll) {
                int c[kSpmvUnroll];
                VT a[kSpmvUnroll];
#pragma unroll
                for (int u = 0; u < kSpmvUnroll; ++u) {
                    c[u] = __ldcs(cp + (int64_t)(k + u) * 32);
                    a[u] = __ldcs(vp + (int64_t)(k + u) * 32);
                }
#pragma unroll
                for (int u = 0; u < kSpmvUnroll; ++u)
                    if (!MASKCOL || is_free(free_mask, c[u])) sum += (double)a[u] * (double)__ldg(x + c[u]);
            }
            for (; k < L; ++k) {
                const int c = __ldcs(cp + (int64_t)k * 32);
                if (!MASKCOL || is_free(free_mask, c)) sum += (double)__ldcs(vp + (int64_t)k * 32) * (double)__ldg(x + c);
            }
        }
        y[row] = fr ? (XT)sum : (XT)0;
        if (DOT && fr) dot += (double)x[row] * sum;
    }
    if (DOT) {
        dot = block_sum(dot, sh);
        if (threadIdx.x == 0) part[blockIdx.x] = dot;
        if (last_block(&st->counter)) {
            const double pq = reduce_parts(part, gridDim.x, 1, 0, sh);
            if (threadIdx.x == 0) {
                st->pq = pq;
                st->alpha = st->rz / pq;
            }
        }
    }
}

// Launch the SpMV for A's layout (SELL when present, else CSR with TPR lanes per row).
template <typename VT, typename XT, bool MASKCOL, bool DOT>
static int spmv_run(const CsrView<VT> &A, const uint8_t *fm, const XT *x, XT *y, PcgState *st, double *part,
                    cudaStream_t s) {
    if (A.sell_off) {
        auto kern = k_spmv_sell<VT, XT, MASKCOL, DOT>;
        const int grid = wave_grid(kern, A.n_slices * 32, kSpmvBlock);
        kern<<<grid, kSpmvBlock, 0, s>>>(A.n_slices, A.sell_off, A.sell_row, A.sell_col, A.v, fm, x, y, st, part);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }
    const int tpr = choose_tpr(A.nnz, A.n);
    return spmv_dispatch<VT, XT, MASKCOL, DOT>(tpr, A.n, A.rp, A.ci, A.v, fm, x, y, st, part, s);
}

int spmv_f64(const CsrView<double> &A, const uint8_t *free_mask, const double *x, double *y, cudaStream_t s) {
    if (free_mask)
        return spmv_run<double, double, true, false>(A, free_mask, x, y, nullptr, nullptr, s);
    return spmv_run<double, double, false, false>(A, nullptr, x, y, nullptr, nullptr, s);
}

int spmv_f32(const CsrView<float> &A, const uint8_t *free_mask, const float *x, float *y, cudaStream_t s) {
    if (free_mask)
        return spmv_run<float, float, true, false>(A, free_mask, x, y, nullptr, nullptr, s);
    return spmv_run<float, float, false, false>(A, nullptr, x, y, nullptr, nullptr, s);
}

// float32 matrix applied to a float64 vector with float64 accumulation (refinement residuals)
int spmv_f32_f64(const CsrView<float> &A, const uint8_t *free_mask, const double *x, double *y, cudaStream_t s) {
    if (free_mask)
        return spmv_run<float, double, true, false>(A, free_mask, x, y, nullptr, nullptr, s);
    return spmv_run<float, double, false, false>(A, nullptr, x, y, nullptr, nullptr, s);
}

// ------------------------------------------------------------------ PCG engine

template <typename VT, typename XT>
Pcg<VT, XT>::~Pcg() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
}

template <typename VT, typename XT>
int Pcg<VT, XT>::reserve(int32_t n_) {
    if (n_ <= cap) {
        n = n_;
        return SNP_OK;
    }
    drop_graph();
    n = cap = n_;
    SNP_TRY(r.alloc(n));
    SNP_TRY(z.alloc(n));
    SNP_TRY(p.alloc(n));
    SNP_TRY(q.alloc(n));
    SNP_TRY(dinv.alloc(n));
    const int gmax = sm_count() * 8 + 1;
    SNP_TRY(part.alloc(3 * (size_t)gmax));
    SNP_TRY(st.alloc(1));
    SNP_TRY(hst.alloc(1));
    SNP_TRY(bad.alloc(1));
    SNP_CUDA_TRY(cudaMemset(st.p, 0, sizeof(PcgState)));
    return SNP_OK;
}

template <typename VT, typename XT>
void Pcg<VT, XT>::drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
}

template <typename VT, typename XT>
int Pcg<VT, XT>::set_jacobi(const CsrView<VT> &A, const int32_t *diag_pos, const uint8_t *free_mask, cudaStream_t s,
                            bool *zero_pivot) {
    SNP_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    k_dinv<VT, XT><<<stride_grid(A.n, kVecBlock, 8), kVecBlock, 0, s>>>(A.n, diag_pos, A.v, free_mask, dinv.p, bad.p);
    SNP_LAUNCH_CHECK();
    launches += 1;
    int h = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    *zero_pivot = h != 0;
    return SNP_OK;
}

template <typename VT, typename XT>
int Pcg<VT, XT>::launch_iteration(const CsrView<VT> &A, const uint8_t *free_mask, XT *x, cudaStream_t s, int use_cond,
                                  cudaGraphConditionalHandle cond) {
    if (free_mask) SNP_TRY((spmv_run<VT, XT, false, true>(A, free_mask, p.p, q.p, st.p, part.p, s)));
    else SNP_TRY((spmv_run<VT, XT, false, true>(A, nullptr, p.p, q.p, st.p, part.p, s)));
    const int64_t nt = (A.n + kVecIlp - 1) / kVecIlp;
    k_update<XT><<<wave_grid(k_update<XT>, nt, kVecBlock), kVecBlock, 0, s>>>(A.n, free_mask, x, r.p, z.p, p.p, q.p,
                                                                             dinv.p, st.p, part.p, use_cond, cond);
    SNP_LAUNCH_CHECK();
    k_pupdate<XT><<<wave_grid(k_pupdate<XT>, nt, kVecBlock), kVecBlock, 0, s>>>(A.n, free_mask, p.p, z.p, st.p);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

template <typename VT, typename XT>
int Pcg<VT, XT>::build_graph(const CsrView<VT> &A, const uint8_t *free_mask, XT *x, cudaStream_t s) {
    drop_graph();
    const char *env = getenv("SNP_PCG_GRAPH");
    if (env && env[0] == '0') return SNP_OK;
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) {
        cudaGetLastError();
        return SNP_OK;
    }
    cudaGraphConditionalHandle h;
    cudaGraphNode_t node;
    cudaGraphNodeParams cp = {};
    bool ok = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&node, g, nullptr, 0, &cp) == cudaSuccess;
    }
    cudaStream_t cs = nullptr;
    if (ok) ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            const int unroll = pcg_body_unroll();
            int rc = SNP_OK;
            for (int u = 0; u < unroll && rc == SNP_OK; ++u) rc = launch_iteration(A, free_mask, x, cs, 1, h);
            cudaGraph_t out = nullptr;
            cudaError_t e = cudaStreamEndCapture(cs, &out);
            ok = (rc == SNP_OK) && e == cudaSuccess;
        }
    }
    if (ok) ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
    if (cs) cudaStreamDestroy(cs);
    if (!ok) {
        cudaGetLastError();
        clear_error();
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        cudaGraphDestroy(g);
        return SNP_OK;
    }
    graph = g;
    key_rp = A.rp;
    key_v = A.v;
    key_fm = free_mask;
    key_x = x;
    key_n = A.n;
    (void)s;
    return SNP_OK;
}

template <typename VT, typename XT>
int Pcg<VT, XT>::solve(const CsrView<VT> &A, const uint8_t *free_mask, const XT *b, XT *x, double rtol, double atol,
                       int64_t maxit, bool zero_x, cudaStream_t s, int64_t *its, double *res, int *status) {
    SNP_TRY(reserve(A.n));
    if (maxit < 0) maxit = 10 * (int64_t)A.n;  // scipy's default uses n_free; A.n bounds it
    // initial residual
    const int g = stride_grid(A.n, kVecBlock, 8);
    if (!zero_x) {
        if (free_mask)
            SNP_TRY((spmv_run<VT, XT, true, false>(A, free_mask, x, q.p, nullptr, nullptr, s)));
        else
            SNP_TRY((spmv_run<VT, XT, false, false>(A, nullptr, x, q.p, nullptr, nullptr, s)));
        launches += 1;
    }
    k_init<XT><<<g, kVecBlock, 0, s>>>(A.n, free_mask, b, x, r.p, z.p, p.p, q.p, dinv.p, st.p, part.p, rtol, atol,
                                       (long long)maxit, zero_x ? 1 : 0);
    SNP_LAUNCH_CHECK();
    launches += 1;
    int64_t chunk_launches = -1;
    // iterate
    const bool same = exec && key_rp == A.rp && key_v == A.v && key_fm == free_mask && key_x == x && key_n == A.n;
    if (!same) SNP_TRY(build_graph(A, free_mask, x, s));
    if (exec) {
        SNP_CUDA_TRY(cudaGraphLaunch(exec, s));
    } else {
        // chunked host loop: launch a batch, then check the flag
        const int chunk = 32;
        int64_t launched = 0;
        while (true) {
            for (int k = 0; k < chunk; ++k) SNP_TRY(launch_iteration(A, free_mask, x, s, 0, 0));
            launched += chunk;
            SNP_CUDA_TRY(cudaMemcpyAsync(hst.p, st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
            SNP_CUDA_TRY(cudaStreamSynchronize(s));
            if (hst.p->done || launched > maxit + chunk) break;
        }
        chunk_launches = 3 * launched;
    }
    SNP_CUDA_TRY(cudaMemcpyAsync(hst.p, st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    const PcgState &H = *hst.p;
    // the WHILE body runs once per iteration (once if the initial residual already passes)
    launches += chunk_launches >= 0 ? chunk_launches : 3 * (H.iter > 0 ? H.iter : 1);
    if (its) *its = H.iter;
    if (res) *res = sqrt(H.rr);
    int stt = SNP_OK;
    if (H.done == 2) stt = SNP_NOT_CONVERGED;
    else if (H.done == 3) stt = SNP_NAN_DETECTED;
    if (status) *status = stt;
    last_bnorm = H.bnorm;
    return SNP_OK;
}

template struct Pcg<double, double>;
template struct Pcg<float, float>;

int pcg_on_buffers(const CsrView<double> &A, const uint8_t *free_mask, const double *b, double *x, double rtol,
                   double atol, int64_t maxit, const PcgBuffers &B, cudaStream_t s, int64_t *its, double *res,
                   int *status) {
    if (maxit < 0) maxit = 10 * (int64_t)A.n;
    // the state (with its reduction ticket) and the pivot flag must start at zero
    SNP_CUDA_TRY(cudaMemsetAsync(B.st, 0, sizeof(PcgState), s));
    SNP_CUDA_TRY(cudaMemsetAsync(B.bad, 0, sizeof(int), s));
    SNP_TRY(find_diag(A.n, A.rp, A.ci, B.diag, s));
    const int gv = stride_grid(A.n, kVecBlock, 8);
    const int64_t nt = (A.n + kVecIlp - 1) / kVecIlp;
    const int gu = wave_grid(k_update<double>, nt, kVecBlock);
    const int gp = wave_grid(k_pupdate<double>, nt, kVecBlock);
    // every grid below (k_dinv, k_init, the SpMV with its dot product, k_update, k_pupdate) is
    // sized by stride_grid(..., 8) or wave_grid, so at most 8 blocks per SM index the partials
    SNP_REQUIRE((int64_t)sm_count() * 8 <= B.max_blocks && gv <= B.max_blocks && gu <= B.max_blocks &&
                    gp <= B.max_blocks,
                "pcg: %d SMs x 8 blocks exceed the %d partial-sum slots", sm_count(), B.max_blocks);
    k_dinv<double, double><<<gv, kVecBlock, 0, s>>>(A.n, B.diag, A.v, free_mask, B.dinv, B.bad);
    SNP_LAUNCH_CHECK();
    int hbad = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&hbad, B.bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    if (hbad) return fail(SNP_ZERO_PIVOT, "pcg: zero or missing diagonal entry on a free row");

    if (free_mask)
        SNP_TRY((spmv_run<double, double, true, false>(A, free_mask, x, B.q, nullptr, nullptr, s)));
    else
        SNP_TRY((spmv_run<double, double, false, false>(A, nullptr, x, B.q, nullptr, nullptr, s)));
    k_init<double><<<gv, kVecBlock, 0, s>>>(A.n, free_mask, b, x, B.r, B.z, B.p, B.q, B.dinv, B.st, B.part, rtol, atol,
                                            (long long)maxit, 0);
    SNP_LAUNCH_CHECK();
    // iterations in chunks; every kernel returns at once after the flag is set, so the
    // overshoot of the last chunk does no work
    PcgState H;
    const int chunk = 32;
    int64_t launched = 0;
    while (true) {
        SNP_CUDA_TRY(cudaMemcpyAsync(&H, B.st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        SNP_CUDA_TRY(cudaStreamSynchronize(s));
        if (H.done || launched > maxit + chunk) break;
        for (int k = 0; k < chunk; ++k) {
            if (free_mask)
                SNP_TRY((spmv_run<double, double, false, true>(A, free_mask, B.p, B.q, B.st, B.part, s)));
            else
                SNP_TRY((spmv_run<double, double, false, true>(A, nullptr, B.p, B.q, B.st, B.part, s)));
            k_update<double><<<gu, kVecBlock, 0, s>>>(A.n, free_mask, x, B.r, B.z, B.p, B.q, B.dinv, B.st, B.part, 0, 0);
            SNP_LAUNCH_CHECK();
            k_pupdate<double><<<gp, kVecBlock, 0, s>>>(A.n, free_mask, B.p, B.z, B.st);
            SNP_LAUNCH_CHECK();
        }
        launched += chunk;
    }
    if (its) *its = H.iter;
    if (res) *res = sqrt(H.rr);
    int stt = SNP_OK;
    if (H.done == 2) stt = SNP_NOT_CONVERGED;
    else if (H.done == 3) stt = SNP_NAN_DETECTED;
    if (status) *status = stt;
    return SNP_OK;
}

}  // namespace snp

extern "C" {

int snp_spmv(int32_t n_rows, const int32_t *row_ptr, const int32_t *col_idx, const double *vals,
             const uint8_t *free_mask, const double *x, double *y, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_rows >= 0, "snp_spmv: negative size");
    if (n_rows == 0) return SNP_OK;
    SNP_REQUIRE(row_ptr && col_idx && vals && x && y, "snp_spmv: NULL argument");
    snp::CsrView<double> A{n_rows, -1, row_ptr, col_idx, vals};
    A.nnz = (int64_t)n_rows * 16;  // thread-per-row choice only
    return snp::spmv_f64(A, free_mask, x, y, snp::as_stream(stream));
}

int snp_pcg(int32_t n_rows, const int32_t *row_ptr, const int32_t *col_idx, const double *vals,
            const uint8_t *free_mask, const double *b, double *x, double rtol, double atol, int64_t maxiter,
            int64_t *iterations, double *res_norm, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_rows > 0, "snp_pcg: n_rows must be positive");
    SNP_REQUIRE(row_ptr && col_idx && vals && b && x, "snp_pcg: NULL argument");
    SNP_REQUIRE(rtol >= 0 && atol >= 0, "snp_pcg: tolerances must be non-negative");
    cudaStream_t s = snp::as_stream(stream);
    // diagonal positions (rows are sorted; found by a search kernel)
    snp::DevBuf<int32_t> diag;
    SNP_TRY(diag.alloc(n_rows));
    SNP_TRY(snp::find_diag(n_rows, row_ptr, col_idx, diag.p, s));
    int32_t nnz_last = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&nnz_last, row_ptr + n_rows, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    snp::CsrView<double> A{n_rows, nnz_last, row_ptr, col_idx, vals};
    snp::Pcg<double, double> pcg;
    SNP_TRY(pcg.reserve(n_rows));
    bool zp = false;
    SNP_TRY(pcg.set_jacobi(A, diag.p, free_mask, s, &zp));
    if (zp) return snp::fail(SNP_ZERO_PIVOT, "snp_pcg: zero or missing diagonal entry on a free row");
    int status = SNP_OK;
    SNP_TRY(pcg.solve(A, free_mask, b, x, rtol, atol, maxiter, false, s, iterations, res_norm, &status));
    if (status == SNP_NOT_CONVERGED) return snp::fail(status, "snp_pcg: maxiter reached");
    if (status == SNP_NAN_DETECTED) return snp::fail(status, "snp_pcg: non-finite residual");
    return SNP_OK;
}

}  // extern "C"
