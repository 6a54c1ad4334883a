// Internal types shared between the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "snp_common.cuh"

namespace snp {

// Arrays of six values per element (one per element edge, or the six components of a
// symmetric 3x3 tensor) are stored in blocks of 32 elements: value k of element e sits at
// ((e / 32) * 6 + k) * 32 + e % 32.  A warp's 32 consecutive elements read each k as one
// coalesced row, and the six rows lie at fixed offsets from one base address.
__host__ __device__ __forceinline__ int64_t eslot(int64_t e, int k) { return ((e >> 5) * 6 + k) * 32 + (e & 31); }
__host__ __device__ __forceinline__ int64_t eslots_size(int64_t n_elems) { return ((n_elems + 31) >> 5) * 192; }

// Owning device allocation (cudaMalloc'd; freed on destruction).
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        release();
        p = o.p;
        n = o.n;
        o.p = nullptr;
        o.n = 0;
        return *this;
    }
    ~DevBuf() { release(); }
    int alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return fail(SNP_NO_MEMORY, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        n = count;
        return SNP_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// Pinned host allocation.
template <typename T>
struct HostBuf {
    T *p = nullptr;
    HostBuf() = default;
    HostBuf(const HostBuf &) = delete;
    HostBuf &operator=(const HostBuf &) = delete;
    ~HostBuf() {
        if (p) cudaFreeHost(p);
    }
    int alloc(size_t count) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cudaError_t e = cudaMallocHost(reinterpret_cast<void **>(&p), (count ? count : 1) * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return fail(SNP_NO_MEMORY, "cudaMallocHost failed: %s", cudaGetErrorString(e));
        }
        return SNP_OK;
    }
};

int pattern_create(const int32_t *elem_dofs, int64_t n_elems, int32_t dpe, int32_t n_rows, cudaStream_t st,
                   snp_pattern **out);

// Arguments of one curl-curl assembly launch (one material).
struct CurlArgs {
    int64_t n_elems;
    const double *nodes;
    const int32_t *cells;
    const int32_t *gids;
    const int32_t *orient;
    const double *ctab;   // curls at quadrature point 0: [n_orient][6][3]
    int32_t n_orient;
    const double *dphi0;  // d_phi at point 0: [4][3]
    const double *w;      // [Q]
    int32_t nq;
    const double *x;
    const double *Bs;     // [n_elems][Q][3] or null
    int32_t n_int;
    const double *rel_c;
    const double *rel_x;
    const int32_t *slots;  // [n_elems][36] (already offset to this material)
    double *K;
    double *dK;
    double *J;
    float *J32;
    double *rhs;
    double *F;
    // element-tensor outputs (launch_curlcurl_tensor), element-edge arrays indexed by
    // eslot(t_offset + e, k): S_e in float64 or float32 (components xx xy xz yy yz zz), and
    // per element edge k its residual term Fe and Jacobian diagonal term De (summed per DoF
    // afterwards, in a fixed order)
    double *T64;
    float *T32;
    int64_t t_offset;
    double *Fe;
    double *De;
    // element matrices of the two-phase assembly (instead of the atomics into the CSR): block b
    // of ET holds value b of every element, ET[b * et_stride + t_offset + e]; the blocks are
    // K (21, upper triangle row by row: (j, k), j <= k), dK (21), J = K + dK (21), the six
    // residual terms F_e,j and the six reduced-rhs terms, at the block offsets et_k .. et_r
    // (-1: not written)
    double *ET;
    int64_t et_stride;
    int et_k, et_d, et_j, et_f, et_r;
    // diluted steel (reduced formulation only): phi[Q][4] nodal basis at the quadrature
    // points or null; dil = {c_num, m_num, c_den, m_den}, s(z) = (c_num + z m_num) / (c_den + z m_den)
    const double *phi;
    double dil[4];
};

// Give every kernel node of `body` an L2 access policy window over [base, base + bytes) with
// persisting hits (the slot values the element pass writes and the DoF pass reads), raising the
// context's persisting set-aside to cover it; only when the whole range fits the device's
// persisting maximum (returns whether the window was set).  SNP_L2_PERSIST=0 skips.
bool l2_window_on_kernels(cudaGraph_t body, const void *base, size_t bytes);

// Validate the inputs of a curl-curl launch over elements [elem_offset, +n_elems) of `pat` (may
// be NULL) and fill `a` (slots offset to the range; outputs unset).
int fill_args(CurlArgs &a, const snp_pattern *pat, int64_t elem_offset, int64_t n_elems, const double *nodes,
              const int32_t *cells, const int32_t *glob_ids, const int32_t *orientations, const double *curls,
              int32_t n_orient, const double *d_phi, const double *w, int32_t n_quad, const double *x,
              const double *B_s, int32_t n_int, const double *rel_c, const double *rel_x);

// Launch the fused assembly for one material.  Tables must be affine (checked by the caller).
int launch_curlcurl(const CurlArgs &a, cudaStream_t st);

// Batched element-tensor assembly (several problems in one launch).  A segment is one
// material of one problem: its CurlArgs (mesh arrays, source field, reluctance tables,
// dilution; t_offset = the segment's first element in the concatenated element numbering;
// x, T, Fe and De are given per launch), the problem's index and its first DoF in the
// concatenated vectors.  Work items are runs of at most kBatchAsmItem elements of one segment.
struct BatchSeg {
    CurlArgs a;
    int32_t inst;
    int32_t dof_off;
};
struct BatchAsmItem {
    int32_t seg, inst;
    int64_t e0, e1;  // elements [e0, e1) of the segment
};
constexpr int64_t kBatchAsmItem = 2048;
constexpr int kBatchAsmBlock = 128;
// Tables (ctab [n_orient][nq][6][3] read at q = 0, dphi at q = 0, w) are the same for every
// segment.  Items whose problem has run[inst * run_stride] == 0 are skipped.  x: concatenated
// DoF vector; T: float64 (f32 false) or float32 element tensors of the concatenated elements.
int launch_curlcurl_tensor_batch(const BatchSeg *segs, const BatchAsmItem *items, int n_items, int max_n_int,
                                 const double *ctab, int n_orient, int quad_stride_ctab, const double *dphi0,
                                 const double *w, int nq, const double *x, const int32_t *run, int run_stride, void *T,
                                 bool f32, double *Fe, double *De, int grid, cudaStream_t st);

// Element tensors of the Newton Jacobian for one material: S_e = Jm^T (kfac I + M) Jm with
// J_e,jk = chat_j . S_e chat_k (chat_j: reference curls of the element's orientation), plus
// the element terms of diag(J) and of F = K(x) x - rhs(x).  Tables must be affine.
int launch_curlcurl_tensor(const CurlArgs &a, cudaStream_t st);

// Element matrices of the two-phase (deterministic) assembly into a CSR pattern, structure of
// arrays over the pattern's elements: `stride` blocks of n_elems values each, at these block
// offsets (-1: absent): K 21 values (upper triangle, row by row), dK 21, J = K + dK 21, residual
// terms F_e,j 6, reduced-rhs terms 6.  The values are the single-launch kernel's element values
// (the reference kernels' arithmetic), stored instead of added into the CSR.
struct TermLayout {
    int stride = 0;
    int k = -1, d = -1, j = -1, f = -1, r = -1;
};
TermLayout term_layout(int parts);

// Phase 1: the element matrices of one material's elements (a.t_offset = the material's first
// element in the pattern), into terms with n_elems values per block.
int launch_curlcurl_terms(const CurlArgs &a, const TermLayout &L, double *terms, int64_t n_elems, cudaStream_t st);

// Phase 2: every CSR entry of `pat` summed from its element contributions in element order, and
// every entry of F / rhs from the DoF's incidences in element order (no atomics; bitwise
// repeatable); each requested output is overwritten.  J = K + dK per entry when both K and dK
// blocks are present, else from the J block.
int launch_curlcurl_rows(const snp_pattern *pat, const double *terms, const TermLayout &L, double *K, double *dK,
                         double *J, float *J32, double *rhs, double *F, cudaStream_t st);

// Whether launch_curlcurl_rows can serve the pattern (contribution and incidence lists built).
bool rows_supported(const snp_pattern *pat);

// Validate that d_phi and curls do not vary across quadrature points; sets *affine.
int check_affine_tables(const double *curls, int32_t n_orient, const double *d_phi, int32_t nq, cudaStream_t st,
                        bool *affine);

// SELL-C-sigma copy of a CSR pattern (C = 32 rows per slice, rows sorted by length within
// windows of sigma rows, each slice stored column-major and padded to its longest row).
struct SellLayout {
    int64_t n_slices = 0;
    int64_t total = 0;                   // stored entries including padding
    DevBuf<int64_t> slice_off;           // [n_slices + 1] element offset of each slice
    DevBuf<int32_t> slice_row;           // [n_slices * 32] original row of each slot (-1: padding row)
    DevBuf<int32_t> col;                 // [total] column index (padding: the slot's own row, value 0)
    DevBuf<int32_t> csr2sell;            // [nnz] SELL position of each CSR position
    DevBuf<int32_t> diag;                // [n_rows] SELL position of each row's diagonal (-1: none)
    DevBuf<int32_t> slots;               // [n_elems * dpe * dpe] slot map into the SELL values
};

}  // namespace snp

struct snp_pattern {
    int32_t n_rows = 0;
    int64_t nnz = 0;
    int64_t n_elems = 0;
    int32_t dpe = 0;
    snp::DevBuf<int32_t> row_ptr, col_idx, slots, diag_pos;
    // contributions of every CSR entry p: the coupling ids t = e * dpe^2 + a * dpe + b of the
    // element pairs that add into it, in element order, cid[cptr[p] .. cptr[p + 1])
    snp::DevBuf<int32_t> cid, cptr;
    bool has_contrib = false;
    // incidence lists of the rows (6 DoFs per element, fewer than 2^28 elements): row r's
    // (element, local DoF) pairs as e * 8 + k in element order, inc[inc_ptr[r] .. inc_ptr[r + 1])
    snp::DevBuf<int32_t> inc_ptr, inc;
    int32_t max_row = 0;  // entries of the longest row
    bool has_incidence = false;
    // work space of the deterministic grad-grad assembly (element values of one call); calls on
    // one pattern are serialised by its users (one stream)
    mutable snp::DevBuf<double> gg_terms;
};

namespace snp {
// Build the SELL layout of a pattern (and its slot map) on the device.
int build_sell(const snp_pattern *pat, SellLayout &S, cudaStream_t st);
}  // namespace snp
