// Krylov engine types shared by the C-ABI entry points and the Newton solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "snp_internal.cuh"

namespace snp {

template <typename VT>
struct CsrView {
    int32_t n;
    int64_t nnz;
    const int32_t *rp;
    const int32_t *ci;
    const VT *v;
};

// Device-resident CG state, written only by the last block of each reduction.
struct PcgState {
    double rz, pq, alpha, beta, rr, bnorm, atol_eff;
    long long iter, maxit;
    int done;  // 0 running, 1 converged, 2 maxiter, 3 non-finite, 4 zero rhs
    unsigned int counter;
};

// Work space of one CG solve on caller-owned device memory (nothing is allocated).
struct PcgBuffers {
    double *r, *z, *p, *q, *dinv, *part;  // part: 3 * max_blocks doubles
    int32_t *diag;
    PcgState *st;
    int *bad;
    int max_blocks;
};

// Jacobi-PCG (float64) with scipy cg's stopping rule on the given buffers; launches only
// kernels, async copies of scalars and stream synchronisations.
int pcg_on_buffers(const CsrView<double> &A, const uint8_t *free_mask, const double *b, double *x, double rtol,
                   double atol, int64_t maxit, const PcgBuffers &B, cudaStream_t s, int64_t *its, double *res,
                   int *status);

int choose_tpr(int64_t nnz, int32_t n);
int find_diag(int32_t n, const int32_t *rp, const int32_t *ci, int32_t *diag, cudaStream_t s);
int spmv_f64(const CsrView<double> &A, const uint8_t *free_mask, const double *x, double *y, cudaStream_t s);
int spmv_f32(const CsrView<float> &A, const uint8_t *free_mask, const float *x, float *y, cudaStream_t s);
int spmv_f32_f64(const CsrView<float> &A, const uint8_t *free_mask, const double *x, double *y, cudaStream_t s);

// Jacobi-preconditioned CG on the free rows of A (matrix values VT, vectors XT).
template <typename VT, typename XT>
struct Pcg {
    int32_t n = 0, cap = 0;
    DevBuf<XT> r, z, p, q, dinv;
    DevBuf<double> part;
    DevBuf<PcgState> st;
    HostBuf<PcgState> hst;
    DevBuf<int> bad;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const int32_t *key_rp = nullptr;
    const VT *key_v = nullptr;
    const uint8_t *key_fm = nullptr;
    const XT *key_x = nullptr;
    int32_t key_n = 0;
    double last_bnorm = 0.0;
    int64_t launches = 0;  // kernels launched (graph body counted per executed iteration)

    Pcg() = default;
    Pcg(const Pcg &) = delete;
    Pcg &operator=(const Pcg &) = delete;
    ~Pcg();
    int reserve(int32_t n);
    void drop_graph();
    int set_jacobi(const CsrView<VT> &A, const int32_t *diag_pos, const uint8_t *free_mask, cudaStream_t s,
                   bool *zero_pivot);
    // x: in initial guess (ignored when zero_x), out solution; non-free entries set to 0.
    int solve(const CsrView<VT> &A, const uint8_t *free_mask, const XT *b, XT *x, double rtol, double atol,
              int64_t maxit, bool zero_x, cudaStream_t s, int64_t *its, double *res, int *status);

   private:
    int launch_iteration(const CsrView<VT> &A, const uint8_t *free_mask, XT *x, cudaStream_t s, int use_cond,
                         cudaGraphConditionalHandle cond);
    int build_graph(const CsrView<VT> &A, const uint8_t *free_mask, XT *x, cudaStream_t s);
};

}  // namespace snp
