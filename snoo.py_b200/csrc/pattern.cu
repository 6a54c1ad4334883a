// CSR pattern and element slot map (one-time setup per mesh).
//
// The reference converts every assembly's triplets with scipy (fem_c/interface_c.pyx:367-368:
// csr_array((v,(i,j))) -> sort, sum duplicates).  Here the sort happens once: the
// (row, col) keys of all element couplings are radix-sorted on the device, duplicates
// collapse to one CSR position, and the slot map records for every element coupling
// where its value goes.  Assembly then adds element values straight into CSR values.
#include <cub/cub.cuh>

#include <cstdio>

#include "snp_common.cuh"
#include "snp_internal.cuh"

namespace snp {

namespace {

__global__ void k_make_keys(const int32_t *__restrict__ dofs, int64_t n_elems, int dpe,
                            unsigned long long *__restrict__ keys, uint32_t *__restrict__ ids) {
    const int64_t per = (int64_t)dpe * dpe;
    const int64_t total = n_elems * per;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t e = t / per;
        int ab = (int)(t - e * per);
        int a = ab / dpe, b = ab - a * dpe;
        uint32_t r = (uint32_t)dofs[e * dpe + a];
        uint32_t c = (uint32_t)dofs[e * dpe + b];
        keys[t] = ((unsigned long long)r << 32) | c;
        ids[t] = (uint32_t)t;
    }
}

__global__ void k_check_dofs(const int32_t *__restrict__ dofs, int64_t n, int32_t n_rows, int *bad) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        int32_t d = dofs[t];
        if (d < 0 || d >= n_rows) atomicExch(bad, 1);
    }
}

__global__ void k_heads(const unsigned long long *__restrict__ keys, int64_t n, uint32_t *__restrict__ head) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        head[t] = (t == 0 || keys[t] != keys[t - 1]) ? 1u : 0u;
}

// pos = inclusive scan of heads (1-based position of each sorted key's unique entry)
__global__ void k_scatter(const unsigned long long *__restrict__ keys, const uint32_t *__restrict__ ids,
                          const uint32_t *__restrict__ head, const uint32_t *__restrict__ pos, int64_t n,
                          int32_t *__restrict__ slots, int32_t *__restrict__ col_idx, int32_t *__restrict__ row_cnt,
                          int32_t *__restrict__ diag_pos) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = (int32_t)pos[t] - 1;
        slots[ids[t]] = p;
        if (head[t]) {
            unsigned long long k = keys[t];
            int32_t r = (int32_t)(k >> 32), c = (int32_t)(k & 0xffffffffu);
            col_idx[p] = c;
            atomicAdd(row_cnt + r, 1);
            if (r == c) diag_pos[r] = p;
        }
    }
}

__global__ void k_fill_i32(int32_t *p, int64_t n, int32_t v) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) p[t] = v;
}

// (DoF, e * 8 + k) pairs of every element's DoFs, counted per row
__global__ void k_inc_pairs(const int32_t *__restrict__ dofs, int64_t n_elems, uint32_t *__restrict__ key,
                            int32_t *__restrict__ val, int32_t *__restrict__ cnt) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_elems * 6; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / 6;
        const int k = (int)(t - e * 6);
        const int32_t r = dofs[t];
        key[t] = (uint32_t)r;
        val[t] = (int32_t)((e << 3) | k);
        atomicAdd(cnt + r, 1);
    }
}

// cptr[p] = first sorted coupling of CSR position p (heads of the sorted keys)
__global__ void k_cptr(const uint32_t *__restrict__ head, const uint32_t *__restrict__ pos, int64_t n,
                       int32_t *__restrict__ cptr) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        if (head[t]) cptr[pos[t] - 1] = (int32_t)t;
}

__global__ void k_max_row(int32_t n, const int32_t *__restrict__ rp, int *__restrict__ mx) {
    int m = 0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int len = rp[r + 1] - rp[r];
        m = len > m ? len : m;
    }
    atomicMax(mx, m);
}

int bits_for(uint32_t v) {
    int b = 0;
    while (b < 32 && (1ull << b) <= v) ++b;
    return b;
}

// Row incidence lists (the two-phase assembly's gather order) and the longest row.  Built for
// 6 DoFs per element and fewer than 2^28 elements (the e * 8 + k word); otherwise left empty.
int build_incidence(snp_pattern *P, const int32_t *elem_dofs, cudaStream_t st) {
    const int32_t n = P->n_rows;
    {
        DevBuf<int> mx;
        SNP_TRY(mx.alloc(1));
        SNP_CUDA_TRY(cudaMemsetAsync(mx.p, 0, sizeof(int), st));
        k_max_row<<<stride_grid(n, 256, 4), 256, 0, st>>>(n, P->row_ptr.p, mx.p);
        SNP_LAUNCH_CHECK();
        int h = 0;
        SNP_CUDA_TRY(cudaMemcpyAsync(&h, mx.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        SNP_CUDA_TRY(cudaStreamSynchronize(st));
        P->max_row = h;
    }
    if (P->dpe != 6 || P->n_elems >= ((int64_t)1 << 28)) return SNP_OK;
    const int64_t m = P->n_elems * 6;
    SNP_TRY(P->inc_ptr.alloc((size_t)n + 1));
    SNP_TRY(P->inc.alloc(m > 0 ? m : 1));
    SNP_CUDA_TRY(cudaMemsetAsync(P->inc_ptr.p, 0, sizeof(int32_t) * ((size_t)n + 1), st));
    if (m > 0) {
        DevBuf<uint32_t> key, key2;
        DevBuf<int32_t> val2;
        DevBuf<unsigned char> temp;
        SNP_TRY(key.alloc(m));
        SNP_TRY(key2.alloc(m));
        SNP_TRY(val2.alloc(m));
        k_inc_pairs<<<stride_grid(m, 256, 16), 256, 0, st>>>(elem_dofs, P->n_elems, key.p, P->inc.p, P->inc_ptr.p);
        SNP_LAUNCH_CHECK();
        const int end_bit = bits_for((uint32_t)n);
        cub::DoubleBuffer<uint32_t> dk(key.p, key2.p);
        cub::DoubleBuffer<int32_t> dv(P->inc.p, val2.p);
        size_t tb_sort = 0, tb_scan = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, dk, dv, m, 0, end_bit > 0 ? end_bit : 1, st);
        cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, P->inc_ptr.p, P->inc_ptr.p, n + 1, st);
        SNP_TRY(temp.alloc(tb_sort > tb_scan ? tb_sort : tb_scan));
        // LSD radix sort is stable: within a row the pairs keep their element order
        SNP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tb_sort, dk, dv, m, 0, end_bit > 0 ? end_bit : 1, st));
        if (dv.Current() != P->inc.p)
            SNP_CUDA_TRY(cudaMemcpyAsync(P->inc.p, dv.Current(), sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, st));
        SNP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp.p, tb_scan, P->inc_ptr.p, P->inc_ptr.p, n + 1, st));
        SNP_CUDA_TRY(cudaStreamSynchronize(st));
    }
    P->has_incidence = true;
    return SNP_OK;
}

}  // namespace

int pattern_create(const int32_t *elem_dofs, int64_t n_elems, int32_t dpe, int32_t n_rows, cudaStream_t st,
                   snp_pattern **out) {
    SNP_REQUIRE(out != nullptr, "snp_pattern_create: out is NULL");
    *out = nullptr;
    SNP_REQUIRE(dpe == 4 || dpe == 6, "snp_pattern_create: dofs_per_elem must be 4 or 6 (got %d)", dpe);
    SNP_REQUIRE(n_rows > 0, "snp_pattern_create: n_rows must be positive");
    SNP_REQUIRE(n_elems >= 0, "snp_pattern_create: negative element count");
    const int64_t n = n_elems * dpe * dpe;
    SNP_REQUIRE(n < (int64_t)0xffffffffll, "snp_pattern_create: %lld couplings exceed the 32-bit slot range", (long long)n);
    SNP_REQUIRE(n_elems == 0 || elem_dofs != nullptr, "snp_pattern_create: elem_dofs is NULL");

    snp_pattern *P = new snp_pattern();
    P->n_rows = n_rows;
    P->n_elems = n_elems;
    P->dpe = dpe;
    DevBuf<unsigned long long> keys, keys2;
    DevBuf<uint32_t> ids, ids2, head, pos;
    DevBuf<int> bad;
    DevBuf<unsigned char> temp;
    auto cleanup_fail = [&](int code) {
        delete P;
        return code;
    };
    int rc;
    if ((rc = P->row_ptr.alloc(n_rows + 1)) || (rc = P->diag_pos.alloc(n_rows)) || (rc = P->slots.alloc(n > 0 ? n : 1)) ||
        (rc = bad.alloc(1)))
        return cleanup_fail(rc);
    if (cudaMemsetAsync(bad.p, 0, sizeof(int), st) != cudaSuccess) return cleanup_fail(fail(SNP_CUDA_ERROR, "memset"));
    if (n > 0) {
        k_check_dofs<<<stride_grid(n_elems * dpe, 256, 8), 256, 0, st>>>(elem_dofs, n_elems * dpe, n_rows, bad.p);
        int hbad = 0;
        if (cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: %s", cudaGetErrorString(cudaGetLastError())));
        if (hbad) return cleanup_fail(fail(SNP_BAD_ARG, "snp_pattern_create: a DoF index lies outside [0, %d)", n_rows));
        if ((rc = keys.alloc(n)) || (rc = keys2.alloc(n)) || (rc = ids.alloc(n)) || (rc = ids2.alloc(n)) ||
            (rc = head.alloc(n)) || (rc = pos.alloc(n)))
            return cleanup_fail(rc);
        k_make_keys<<<stride_grid(n, 256, 16), 256, 0, st>>>(elem_dofs, n_elems, dpe, keys.p, ids.p);
        int end_bit = 32 + bits_for((uint32_t)n_rows);
        if (end_bit > 64) end_bit = 64;
        size_t tb_sort = 0, tb_scan = 0;
        cub::DoubleBuffer<unsigned long long> dk(keys.p, keys2.p);
        cub::DoubleBuffer<uint32_t> dv(ids.p, ids2.p);
        cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, dk, dv, n, 0, end_bit, st);
        cub::DeviceScan::InclusiveSum(nullptr, tb_scan, head.p, pos.p, n, st);
        size_t tb_scan2 = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb_scan2, P->row_ptr.p, P->row_ptr.p, n_rows + 1, st);
        size_t tb = tb_sort > tb_scan ? tb_sort : tb_scan;
        if (tb_scan2 > tb) tb = tb_scan2;
        if ((rc = temp.alloc(tb > 0 ? tb : 1))) return cleanup_fail(rc);
        if (cub::DeviceRadixSort::SortPairs(temp.p, tb, dk, dv, n, 0, end_bit, st) != cudaSuccess)
            return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: radix sort failed"));
        k_heads<<<stride_grid(n, 256, 16), 256, 0, st>>>(dk.Current(), n, head.p);
        if (cub::DeviceScan::InclusiveSum(temp.p, tb, head.p, pos.p, n, st) != cudaSuccess)
            return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: scan failed"));
        uint32_t h_nnz = 0;
        if (cudaMemcpyAsync(&h_nnz, pos.p + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: nnz readback failed"));
        P->nnz = h_nnz;
        if ((rc = P->col_idx.alloc(P->nnz))) return cleanup_fail(rc);
        if (cudaMemsetAsync(P->row_ptr.p, 0, sizeof(int32_t) * (n_rows + 1), st) != cudaSuccess)
            return cleanup_fail(fail(SNP_CUDA_ERROR, "memset"));
        k_fill_i32<<<stride_grid(n_rows, 256, 8), 256, 0, st>>>(P->diag_pos.p, n_rows, -1);
        k_scatter<<<stride_grid(n, 256, 16), 256, 0, st>>>(dk.Current(), dv.Current(), head.p, pos.p, n, P->slots.p,
                                                           P->col_idx.p, P->row_ptr.p, P->diag_pos.p);
        if (cub::DeviceScan::ExclusiveSum(temp.p, tb, P->row_ptr.p, P->row_ptr.p, n_rows + 1, st) != cudaSuccess)
            return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: row scan failed"));
        // the sorted couplings (stable radix sort: element order within a position) and the
        // first of each position: every CSR entry's contributions, for the deterministic gather
        if (n < ((int64_t)1 << 31)) {
            if ((rc = P->cid.alloc(n)) || (rc = P->cptr.alloc(P->nnz + 1))) return cleanup_fail(rc);
            if (cudaMemcpyAsync(P->cid.p, dv.Current(), sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st) !=
                cudaSuccess)
                return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: copy of the sorted couplings failed"));
            k_cptr<<<stride_grid(n, 256, 16), 256, 0, st>>>(head.p, pos.p, n, P->cptr.p);
            const int32_t nn = (int32_t)n;
            if (cudaMemcpyAsync(P->cptr.p + P->nnz, &nn, sizeof(int32_t), cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: contribution pointers failed"));
            P->has_contrib = true;
        }
    } else {
        P->nnz = 0;
        if ((rc = P->col_idx.alloc(1))) return cleanup_fail(rc);
        if (cudaMemsetAsync(P->row_ptr.p, 0, sizeof(int32_t) * (n_rows + 1), st) != cudaSuccess)
            return cleanup_fail(fail(SNP_CUDA_ERROR, "memset"));
        k_fill_i32<<<stride_grid(n_rows, 256, 8), 256, 0, st>>>(P->diag_pos.p, n_rows, -1);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cleanup_fail(fail(SNP_CUDA_ERROR, "snp_pattern_create: %s", cudaGetErrorString(e)));
    if ((rc = build_incidence(P, elem_dofs, st))) return cleanup_fail(rc);
    *out = P;
    return SNP_OK;
}

// ------------------------------------------------------------------ SELL-C-sigma layout

namespace {

constexpr int kSellC = 32;
constexpr int kSellSigma = 256;

// key = window * 256 + (255 - min(length, 255)): ascending sort = windows in order, longest first
__global__ void k_sell_keys(int32_t n, const int32_t *__restrict__ rp, uint32_t *__restrict__ key,
                            int32_t *__restrict__ row) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int len = rp[r + 1] - rp[r];
        if (len > 255) len = 255;
        key[r] = (uint32_t)(r / kSellSigma) * 256u + (uint32_t)(255 - len);
        row[r] = (int32_t)r;
    }
}

// slot rows and slice widths (entries of the longest row of each slice)
__global__ void k_sell_slices(int32_t n, int64_t n_slices, const int32_t *__restrict__ rp,
                              const int32_t *__restrict__ sorted_row, int32_t *__restrict__ slice_row,
                              int64_t *__restrict__ width) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n_slices; s += (int64_t)gridDim.x * blockDim.x) {
        int w = 0;
        for (int l = 0; l < kSellC; ++l) {
            const int64_t i = s * kSellC + l;
            const int32_t r = i < n ? sorted_row[i] : -1;
            slice_row[s * kSellC + l] = r;
            if (r >= 0) {
                const int len = rp[r + 1] - rp[r];
                w = len > w ? len : w;
            }
        }
        width[s] = (int64_t)w * kSellC;
    }
}

// one thread per slot: column indices (padding: the slot's own row) and CSR -> SELL positions
__global__ void k_sell_fill(int64_t n_slices, const int64_t *__restrict__ off, const int32_t *__restrict__ slice_row,
                            const int32_t *__restrict__ rp, const int32_t *__restrict__ ci, int32_t *__restrict__ col,
                            int32_t *__restrict__ csr2sell) {
    const int64_t total = n_slices * kSellC;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = t / kSellC;
        const int lane = (int)(t - s * kSellC);
        const int64_t o = off[s];
        const int L = (int)((off[s + 1] - o) / kSellC);
        const int32_t r = slice_row[t];
        const int b = r >= 0 ? rp[r] : 0;
        const int len = r >= 0 ? rp[r + 1] - b : 0;
        for (int k = 0; k < L; ++k) {
            const int64_t pos = o + (int64_t)k * kSellC + lane;
            if (k < len) {
                col[pos] = ci[b + k];
                csr2sell[b + k] = (int32_t)pos;
            } else {
                col[pos] = r >= 0 ? r : 0;
            }
        }
    }
}

__global__ void k_gather_i32(int64_t n, const int32_t *__restrict__ map, const int32_t *__restrict__ idx,
                             int32_t *__restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t i = idx[t];
        out[t] = i >= 0 ? map[i] : -1;
    }
}

}  // namespace

int build_sell(const snp_pattern *pat, SellLayout &S, cudaStream_t st) {
    SNP_REQUIRE(pat != nullptr, "build_sell: pattern is NULL");
    const int32_t n = pat->n_rows;
    const int64_t n_slices = (n + kSellC - 1) / kSellC;
    S.n_slices = n_slices;
    DevBuf<uint32_t> key, key2;
    DevBuf<int32_t> row, row2;
    DevBuf<int64_t> width;
    DevBuf<unsigned char> temp;
    SNP_TRY(key.alloc(n));
    SNP_TRY(key2.alloc(n));
    SNP_TRY(row.alloc(n));
    SNP_TRY(row2.alloc(n));
    SNP_TRY(width.alloc(n_slices + 1));
    SNP_TRY(S.slice_off.alloc(n_slices + 1));
    SNP_TRY(S.slice_row.alloc(n_slices * kSellC));
    k_sell_keys<<<stride_grid(n, 256, 8), 256, 0, st>>>(n, pat->row_ptr.p, key.p, row.p);
    SNP_LAUNCH_CHECK();
    size_t tb_sort = 0, tb_scan = 0;
    cub::DoubleBuffer<uint32_t> dk(key.p, key2.p);
    cub::DoubleBuffer<int32_t> dv(row.p, row2.p);
    cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, dk, dv, n, 0, 32, st);
    cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, width.p, S.slice_off.p, n_slices + 1, st);
    SNP_TRY(temp.alloc(tb_sort > tb_scan ? tb_sort : tb_scan));
    SNP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tb_sort, dk, dv, n, 0, 32, st));
    SNP_CUDA_TRY(cudaMemsetAsync(width.p + n_slices, 0, sizeof(int64_t), st));
    k_sell_slices<<<stride_grid(n_slices, 256, 8), 256, 0, st>>>(n, n_slices, pat->row_ptr.p, dv.Current(),
                                                                 S.slice_row.p, width.p);
    SNP_LAUNCH_CHECK();
    SNP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp.p, tb_scan, width.p, S.slice_off.p, n_slices + 1, st));
    int64_t total = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&total, S.slice_off.p + n_slices, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SNP_CUDA_TRY(cudaStreamSynchronize(st));
    SNP_REQUIRE(total < (int64_t)0x7fffffff, "build_sell: %lld stored entries exceed the 32-bit slot range",
                (long long)total);
    S.total = total;
    SNP_TRY(S.col.alloc(total));
    SNP_TRY(S.csr2sell.alloc(pat->nnz > 0 ? pat->nnz : 1));
    SNP_TRY(S.diag.alloc(n));
    const int64_t n_slot = pat->n_elems * pat->dpe * pat->dpe;
    SNP_TRY(S.slots.alloc(n_slot > 0 ? n_slot : 1));
    k_sell_fill<<<stride_grid(n_slices * kSellC, 256, 16), 256, 0, st>>>(n_slices, S.slice_off.p, S.slice_row.p,
                                                                        pat->row_ptr.p, pat->col_idx.p, S.col.p,
                                                                        S.csr2sell.p);
    SNP_LAUNCH_CHECK();
    k_gather_i32<<<stride_grid(n, 256, 8), 256, 0, st>>>(n, S.csr2sell.p, pat->diag_pos.p, S.diag.p);
    SNP_LAUNCH_CHECK();
    if (n_slot > 0) {
        k_gather_i32<<<stride_grid(n_slot, 256, 16), 256, 0, st>>>(n_slot, S.csr2sell.p, pat->slots.p, S.slots.p);
        SNP_LAUNCH_CHECK();
    }
    SNP_CUDA_TRY(cudaStreamSynchronize(st));
    return SNP_OK;
}

}  // namespace snp

extern "C" {

int snp_pattern_create(const int32_t *elem_dofs, int64_t n_elems, int32_t dofs_per_elem, int32_t n_rows,
                       void *stream, snp_pattern **out) {
    snp::clear_error();
    return snp::pattern_create(elem_dofs, n_elems, dofs_per_elem, n_rows, snp::as_stream(stream), out);
}

int snp_pattern_info(const snp_pattern *pat, int32_t *n_rows, int64_t *nnz, int64_t *n_elems, int32_t *dpe) {
    SNP_REQUIRE(pat != nullptr, "snp_pattern_info: pattern is NULL");
    if (n_rows) *n_rows = pat->n_rows;
    if (nnz) *nnz = pat->nnz;
    if (n_elems) *n_elems = pat->n_elems;
    if (dpe) *dpe = pat->dpe;
    return SNP_OK;
}

int snp_pattern_arrays(const snp_pattern *pat, const int32_t **row_ptr, const int32_t **col_idx, const int32_t **slots) {
    SNP_REQUIRE(pat != nullptr, "snp_pattern_arrays: pattern is NULL");
    if (row_ptr) *row_ptr = pat->row_ptr.p;
    if (col_idx) *col_idx = pat->col_idx.p;
    if (slots) *slots = pat->slots.p;
    return SNP_OK;
}

int snp_pattern_diag(const snp_pattern *pat, const int32_t **diag_pos) {
    SNP_REQUIRE(pat != nullptr, "snp_pattern_diag: pattern is NULL");
    if (diag_pos) *diag_pos = pat->diag_pos.p;
    return SNP_OK;
}

int snp_pattern_destroy(snp_pattern *pat) {
    delete pat;
    return SNP_OK;
}

}  // extern "C"
