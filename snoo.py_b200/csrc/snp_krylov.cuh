// Krylov engine types shared by the C-ABI entry points and the Newton solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>
#include <functional>

#include "snp_internal.cuh"

namespace snp {

// CG iterations captured per execution of a Krylov graph's conditional WHILE body:
// SNP_PCG_UNROLL (1-16), default 4.  Every execution of the body costs a few microseconds
// beyond its kernels (about 3.5 us per float64 iteration of the 1.16M-tet benchmark with one
// iteration per body); the passes of a solve that finished inside a body return at once, so
// the body's remaining iterations cost only their launches.
inline int pcg_body_unroll() {
    const char *e = getenv("SNP_PCG_UNROLL");
    if (!e || !e[0]) return 4;
    const int u = atoi(e);
    return u < 1 ? 1 : (u > 16 ? 16 : u);
}

// A square sparse matrix: CSR (rp, ci, v), or, when sell_off is set, the SELL-C-sigma layout
// of the same pattern with the values v stored in SELL order (rp/ci still describe the CSR).
template <typename VT>
struct CsrView {
    int32_t n;
    int64_t nnz;
    const int32_t *rp;
    const int32_t *ci;
    const VT *v;
    int64_t n_slices = 0;
    const int64_t *sell_off = nullptr;
    const int32_t *sell_row = nullptr;
    const int32_t *sell_col = nullptr;
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

// ------------------------------------------------------------------ matrix-free Jacobian
//
// The Newton Jacobian of first-order Nedelec curl-curl on affine tetrahedra is stored per
// element as the 3x3 symmetric tensor S_e (six numbers): J_e,jk = s_j s_k chat_j . S_e chat_k,
// chat_j the reference curls of orientation 0 and s_j = +-1 the element's edge signs.  A
// product y = J x is two passes without atomics:
//   element pass  u_e = sum_j s_j x_j chat_j,  v_e = S_e u_e, and the six edge terms
//                 y_e,k = s_k chat_k . v_e stored at their slots of the DoF-ordered incidence
//   DoF pass      y_i = sum of the DoF's slots, a contiguous range

// Element topology of the operator: DoFs with edge signs and the DoF -> (element, local
// edge) incidence, built once per mesh.
struct ElemTopology {
    int64_t n_elems = 0;
    int32_t n = 0;
    DevBuf<int32_t> edof;     // eslot(e, k): DoF, bit 31 set when the edge function is negated
    DevBuf<int32_t> inc_ptr;  // [n + 1]
    DevBuf<int32_t> inc;      // [6 n_elems]   (e << 3 | k), bit 31 = sign, grouped by DoF
    DevBuf<int32_t> pos;      // eslot(e, k): slot of (e, k) in that DoF-ordered list
    DevBuf<double> chat64;    // [18] reference curls of orientation 0
    DevBuf<float> chat32;
};

// One material's elements: gids [count][6], orientation index [count], placed at `offset`.
struct ElemBlock {
    const int32_t *gids;
    const int32_t *orient;
    int64_t count;
    int64_t offset;
};

// Build the topology.  ctab_host: curls at quadrature point 0, [n_orient][6][3].  Sets
// *usable = false (and builds nothing) when the orientation tables are not sign flips of
// orientation 0 or the mesh exceeds the 32-bit incidence encoding.
int build_elem_topology(ElemTopology &top, int32_t n, const ElemBlock *blocks, int n_blocks, const double *ctab_host,
                        int32_t n_orient, cudaStream_t s, bool *usable);

// Per-DoF CG state, split by who reads it: the element pass gathers {z, p} (16 bytes in
// float64, two DoFs per 32-byte sector); {r, x} and 1/diag are read only by the DoF's own
// thread in the DoF pass.
// Per-DoF sums of element-edge terms (indexed by eslot) in incidence order (deterministic):
// F_i = sum Fe - rhs_extra_i (rhs_extra may be NULL), diag_i = sum De.
int elem_sum_to_dofs(const ElemTopology &top, const double *Fe, const double *De, const double *rhs_extra,
                     double *F, double *diag, cudaStream_t s);

// Reduced (Galerkin) system of the matrix-free Jacobian T for a float32 basis V [n][ldv]
// (m <= 128 columns): Jr = V^T J V (m x m, row-major) and, when F is given, g = V^T F, both
// over the free DoFs and summed in float64 in a fixed order.  scratch grows as needed.
template <typename TT>
int elem_reduced_system(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const float *V, int m,
                        int64_t ldv, const double *F, double *Jr, double *g, DevBuf<double> &scratch, cudaStream_t s);

// Block Jacobi of the matrix-free Jacobian T: meta[n] = offset in block | size << 8 (blocks of
// at most 8 consecutive DoFs, never across a multiple of 256; constrained DoFs alone); bmat
// [n][8] float64 work, binv [n][8] float32 rows of the block inverses; *fallback_count (device
// int, accumulated) counts blocks inverted as point Jacobi.
constexpr int kBlockJacobiMax = 8;
template <typename TT>
int block_jacobi_build(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const uint16_t *meta,
                       double *bmat, float *binv, int *fallback_count, cudaStream_t s);
// z = M r on the free DoFs (0 elsewhere), float64 vectors.
int block_jacobi_apply(int32_t n, const uint8_t *free_mask, const uint16_t *meta, const float *binv, const double *r,
                       double *z, cudaStream_t s);

// z = r / diag on the free DoFs (0 elsewhere), float64 vectors.
int point_jacobi_apply(int32_t n, const uint8_t *free_mask, const double *diag, const double *r, double *z,
                       cudaStream_t s);

// x += V coef on the free DoFs (V float32 [n][ldv], m columns; coef float64 [m], device).
int basis_axpy(int32_t n, const uint8_t *free_mask, const float *V, int m, int64_t ldv, const double *coef,
               double *x, cudaStream_t s);

// Read-only view of a finalized Newton solver's device data, for the batched solver.
struct SolverMaterialView {
    int64_t offset, count;
    const int32_t *cells, *gids, *orient;
    const double *Bs;  // [count][nq][3] or NULL
    int32_t n_int;
    const double *relc, *relx;
    const double *phi;  // nodal basis at the quadrature points when diluted, else NULL
    double dil[4];
};
struct SolverView {
    int32_t n;
    int64_t n_free, n_nodes, n_elems;
    int32_t nq, n_orient;
    const double *nodes, *curls, *dphi, *w, *rhs_extra;
    const uint8_t *free_mask;
    const ElemTopology *etop;  // NULL unless the Newton Jacobian is matrix-free
    const uint16_t *bj_meta;   // NULL unless block Jacobi is set
    int n_mats;
    const SolverMaterialView *mats;
};

template <typename TT>
struct alignas(2 * sizeof(TT)) DofPair {
    TT a, b;
};


// Jacobi-PCG on the matrix-free Jacobian (values TT = double or float; sums in double),
// scipy cg's stopping rule, iteration loop in a CUDA-graph conditional WHILE node.
template <typename TT>
struct ElemPcg {
    int32_t n = 0;
    int64_t ne = 0;
    DevBuf<DofPair<TT>> G;  // {z, p}
    DevBuf<DofPair<TT>> R;  // {r, x}
    DevBuf<TT> D;           // 1 / diag(J)
    DevBuf<TT> Y;           // [6 n_elems] element-edge terms in DoF-ordered slots
    DevBuf<double> part;
    DevBuf<PcgState> st;
    HostBuf<PcgState> hst;
    DevBuf<int> bad;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void *key_top = nullptr;
    const TT *key_T = nullptr;
    const uint8_t *key_fm = nullptr;
    const uint16_t *key_bm = nullptr;
    const float *key_bi = nullptr;
    bool l2_window = false;  // the graph's kernels carry the L2 window over Y
    size_t l2_bytes = 0;     // its size, the set-aside raised while a solve runs
    // raise and release the context's persisting-L2 set-aside around each solve (a device-wide
    // setting: off while several solvers run at once, snp_solver_solve_many)
    bool l2_hold = true;
    int64_t launches = 0;

    ElemPcg() = default;
    ElemPcg(const ElemPcg &) = delete;
    ElemPcg &operator=(const ElemPcg &) = delete;
    ~ElemPcg();
    int reserve(int32_t n, int64_t ne);
    void drop_graph();
    // Solve J h = b_scale * b on the free DoFs from h = 0 with Jacobi from diag, or block
    // Jacobi when bj_meta / bj_inv are given (block_jacobi_build); h (float64) gets the
    // iterate, 0 on constrained DoFs.  SNP_ZERO_PIVOT for a zero/non-finite diagonal entry on
    // a free DoF.
    int solve(const ElemTopology &top, const TT *T, const double *diag, const uint8_t *free_mask, const double *b,
              double b_scale, double *h, double rtol, double atol, int64_t maxit, cudaStream_t s, int64_t *its,
              double *res, int *status, const uint16_t *bj_meta = nullptr, const float *bj_inv = nullptr);
    // y = J x on the free rows and columns (0 on constrained rows).
    int apply(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const TT *x, TT *y, cudaStream_t s);

   private:
    int launch_iteration(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const uint16_t *bj_meta,
                         const float *bj_inv, cudaStream_t s, int use_cond, cudaGraphConditionalHandle cond);
    int build_graph(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const uint16_t *bj_meta,
                    const float *bj_inv);
    bool solve_coop(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const uint16_t *bj_meta,
                    const float *bj_inv, cudaStream_t s, int *rc);
    DevBuf<unsigned long long> coop_bar;
    DevBuf<int> coop_err;
};

// Restarted GMRES(m), right-preconditioned, float64 (gmres.cu).  apply_J(x, y): y = J x on the
// free DoFs; apply_M(r, z): z = M r (0 on constrained DoFs).  Solves J h = b_scale b from h = 0
// to ||b_scale b - J h|| <= max(rtol ||b_scale b||, atol) or maxit Arnoldi steps; *status is
// SNP_OK, SNP_NOT_CONVERGED or SNP_NAN_DETECTED.
struct Gmres {
    using Op = std::function<int(const double *, double *)>;
    int64_t n = -1;
    int m = 0;
    int blocks = 0;
    int64_t launches = 0;
    DevBuf<double> V, w, z, part, hdev;
    DevBuf<unsigned int> counter;
    HostBuf<double> hhost;
    int reserve(int64_t n, int m);
    int solve(const Op &apply_J, const Op &apply_M, const uint8_t *free_mask, const double *b, double b_scale,
              double *x, double rtol, double atol, int64_t maxit, cudaStream_t s, int64_t *its, double *res,
              int *status);
};

// The view of a finalized solver (SNP_BAD_ARG when it is not finalized).  Valid while the
// solver lives and no material is added.
int solver_view(const snp_solver *s, SolverView *v);

}  // namespace snp
