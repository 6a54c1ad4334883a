// Internal types shared between the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "snp_common.cuh"

namespace snp {

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
};

// Launch the fused assembly for one material.  Tables must be affine (checked by the caller).
int launch_curlcurl(const CurlArgs &a, cudaStream_t st);

// Validate that d_phi and curls do not vary across quadrature points; sets *affine.
int check_affine_tables(const double *curls, int32_t n_orient, const double *d_phi, int32_t nq, cudaStream_t st,
                        bool *affine);

}  // namespace snp

struct snp_pattern {
    int32_t n_rows = 0;
    int64_t nnz = 0;
    int64_t n_elems = 0;
    int32_t dpe = 0;
    snp::DevBuf<int32_t> row_ptr, col_idx, slots, diag_pos;
};
