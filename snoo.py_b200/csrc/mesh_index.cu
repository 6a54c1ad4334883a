// Point location and nodal output for field maps.
//
// The reference finds the element holding an evaluation point with gmsh
// (get_element_by_coordinates in evaluate_curl_curl_solution / evaluate_interpolation,
// snoopy/evaluators.py:155-295, 297-410) and averages element fields at the mesh nodes in a
// Python loop (compute_nodal_fields, snoopy/curl_curl_assembler.py:2089-2196).  Here a mesh
// index built once on the device serves both:
//
//  * a uniform bucket grid over the nodes' bounding box whose cell edge h is at least the
//    largest extent of any element along any axis.  Elements are bucketed by centroid (a
//    stable radix sort), so the element holding a point has its centroid in one of the 27
//    buckets around the point's own bucket;
//  * one thread per point tests every candidate's barycentric coordinates and keeps the one
//    whose smallest coordinate is largest (ties: the lower element index).  A point whose best
//    smallest coordinate is below -tol lies outside the mesh (element -1);
//  * node -> element incidence (stable radix sort of the 4E (node, element) pairs): a node
//    sums its elements' values in element order, so averages are deterministic.
#include <cub/cub.cuh>

#include <algorithm>
#include <memory>
#include <cfloat>
#include <cmath>
#include <vector>

#include "snp_common.cuh"
#include "snp_internal.cuh"

struct snp_mesh_index {
    int64_t n_nodes = 0, n_elems = 0;
    snp::DevBuf<double> nodes;
    snp::DevBuf<int32_t> cells;
    double bmin[3] = {0, 0, 0}, h[3] = {1, 1, 1};
    int32_t nb[3] = {1, 1, 1};
    int64_t n_buckets = 1;
    int32_t max_bucket = 0;
    snp::DevBuf<int32_t> bucket_ptr, bucket_elems;
    snp::DevBuf<int32_t> node_ptr, node_elems;
};

namespace snp {
namespace {

constexpr int kIdxBlock = 256;

struct Grid {
    double bmin[3], h[3];
    int32_t nb[3];
};

// Per block: min and max of the node coordinates and the largest element extent along any
// axis, written to part[7 * block] = {min x, min y, min z, -max x, -max y, -max z, -extent}
// (all as minima, so one reduction serves every entry).
__global__ void __launch_bounds__(kIdxBlock)
    k_bounds(const double *__restrict__ nodes, int64_t n_nodes, const int32_t *__restrict__ cells, int64_t n_elems,
             double *__restrict__ part, int *__restrict__ bad) {
    double v[7];
    for (int k = 0; k < 7; ++k) v[k] = DBL_MAX;
    const int64_t total = n_nodes > n_elems ? n_nodes : n_elems;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        if (t < n_nodes) {
            for (int k = 0; k < 3; ++k) {
                const double c = nodes[3 * t + k];
                v[k] = fmin(v[k], c);
                v[3 + k] = fmin(v[3 + k], -c);
            }
        }
        if (t < n_elems) {
            double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
            bool ok = true;
            for (int i = 0; i < 4; ++i) {
                const int32_t n = cells[4 * t + i];
                if (n < 0 || n >= n_nodes) {
                    ok = false;
                    break;
                }
                for (int k = 0; k < 3; ++k) {
                    const double c = nodes[3 * (int64_t)n + k];
                    lo[k] = fmin(lo[k], c);
                    hi[k] = fmax(hi[k], c);
                }
            }
            if (!ok) {
                atomicExch(bad, 1);
            } else {
                const double ext = fmax(hi[0] - lo[0], fmax(hi[1] - lo[1], hi[2] - lo[2]));
                v[6] = fmin(v[6], -ext);
            }
        }
    }
    __shared__ double sh[7][kIdxBlock / 32];
    for (int k = 0; k < 7; ++k) {
        double a = v[k];
        for (int o = 16; o > 0; o >>= 1) a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = a;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double a = DBL_MAX;
        for (int w = 0; w < kIdxBlock / 32; ++w) a = fmin(a, sh[threadIdx.x][w]);
        part[7 * blockIdx.x + threadIdx.x] = a;
    }
}

__device__ __forceinline__ int64_t bucket_key(const Grid &g, int32_t b0, int32_t b1, int32_t b2) {
    return (int64_t)b0 + (int64_t)g.nb[0] * ((int64_t)b1 + (int64_t)g.nb[1] * (int64_t)b2);
}

// Bucket of each element's centroid (clamped to the grid).
__global__ void k_elem_buckets(const double *__restrict__ nodes, const int32_t *__restrict__ cells, int64_t n_elems,
                               Grid g, int32_t *__restrict__ key, int32_t *__restrict__ val) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_elems; e += (int64_t)gridDim.x * blockDim.x) {
        int32_t b[3];
        for (int k = 0; k < 3; ++k) {
            double c = 0.0;
            for (int i = 0; i < 4; ++i) c += nodes[3 * (int64_t)cells[4 * e + i] + k];
            c *= 0.25;
            double f = floor((c - g.bmin[k]) / g.h[k]);
            f = fmin(fmax(f, 0.0), (double)(g.nb[k] - 1));
            b[k] = (int32_t)f;
        }
        key[e] = (int32_t)bucket_key(g, b[0], b[1], b[2]);
        val[e] = (int32_t)e;
    }
}

__global__ void k_count(const int32_t *__restrict__ key, int64_t m, int32_t *__restrict__ cnt) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + key[t], 1);
}

// (node, element) pairs of the incidence sort.
__global__ void k_node_pairs(const int32_t *__restrict__ cells, int64_t n_elems, int32_t *__restrict__ key,
                             int32_t *__restrict__ val) {
    const int64_t m = 4 * n_elems;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
        key[t] = cells[t];
        val[t] = (int32_t)(t >> 2);
    }
}

__global__ void k_max_bucket(const int32_t *__restrict__ ptr, int64_t nbk, int *__restrict__ out) {
    int mx = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nbk; t += (int64_t)gridDim.x * blockDim.x)
        mx = max(mx, ptr[t + 1] - ptr[t]);
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

__device__ __forceinline__ double det3(const double *a, const double *b, const double *c) {
    return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
}

// One thread per point: the 27 buckets around it, every candidate's barycentric coordinates
// (Cramer's rule on the edge vectors from node 0), the best smallest coordinate kept.
__global__ void k_locate(const double *__restrict__ nodes, const int32_t *__restrict__ cells,
                         const int32_t *__restrict__ bptr, const int32_t *__restrict__ belem, Grid g,
                         const double *__restrict__ pts, int64_t n_pts, double tol, int32_t *__restrict__ elem,
                         double *__restrict__ bary) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n_pts; p += (int64_t)gridDim.x * blockDim.x) {
        const double x[3] = {pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]};
        double best = -DBL_MAX, bl[4] = {0.0, 0.0, 0.0, 0.0};
        int32_t be = -1;
        if (isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2])) {
            int32_t ip[3];
            for (int k = 0; k < 3; ++k) {
                double f = floor((x[k] - g.bmin[k]) / g.h[k]);
                f = fmin(fmax(f, -2.0), (double)g.nb[k] + 1.0);
                ip[k] = (int32_t)f;
            }
            for (int d2 = -1; d2 <= 1; ++d2) {
                const int32_t b2 = ip[2] + d2;
                if (b2 < 0 || b2 >= g.nb[2]) continue;
                for (int d1 = -1; d1 <= 1; ++d1) {
                    const int32_t b1 = ip[1] + d1;
                    if (b1 < 0 || b1 >= g.nb[1]) continue;
                    for (int d0 = -1; d0 <= 1; ++d0) {
                        const int32_t b0 = ip[0] + d0;
                        if (b0 < 0 || b0 >= g.nb[0]) continue;
                        const int64_t key = bucket_key(g, b0, b1, b2);
                        const int32_t t1 = bptr[key + 1];
                        for (int32_t t = bptr[key]; t < t1; ++t) {
                            const int32_t e = belem[t];
                            double P[4][3];
                            for (int i = 0; i < 4; ++i) {
                                const int64_t n = cells[4 * (int64_t)e + i];
                                for (int k = 0; k < 3; ++k) P[i][k] = nodes[3 * n + k];
                            }
                            double c1[3], c2[3], c3[3], r[3];
                            for (int k = 0; k < 3; ++k) {
                                c1[k] = P[1][k] - P[0][k];
                                c2[k] = P[2][k] - P[0][k];
                                c3[k] = P[3][k] - P[0][k];
                                r[k] = x[k] - P[0][k];
                            }
                            // columns c1, c2, c3: det([c1 c2 c3]) = c1 . (c2 x c3)
                            const double D = det3(c1, c2, c3);
                            const double l1 = det3(r, c2, c3) / D;
                            const double l2 = det3(c1, r, c3) / D;
                            const double l3 = det3(c1, c2, r) / D;
                            const double l0 = 1.0 - l1 - l2 - l3;
                            const double s = fmin(fmin(l0, l1), fmin(l2, l3));
                            if (s > best || (s == best && e < be)) {
                                best = s;
                                be = e;
                                bl[0] = l0;
                                bl[1] = l1;
                                bl[2] = l2;
                                bl[3] = l3;
                            }
                        }
                    }
                }
            }
        }
        const bool inside = be >= 0 && best >= -tol;
        elem[p] = inside ? be : -1;
        if (bary)
            for (int i = 0; i < 4; ++i) bary[4 * p + i] = inside ? bl[i] : 0.0;
    }
}

// out[node][c] = mean over the node's (selected) elements of ev[e][c]; 0 where none.
__global__ void k_nodal_average(int64_t n_nodes, const int32_t *__restrict__ nptr, const int32_t *__restrict__ nelem,
                                const double *__restrict__ ev, int n_comp, const uint8_t *__restrict__ mask,
                                double *__restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n_nodes; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a = nptr[v], b = nptr[v + 1];
        for (int c = 0; c < n_comp; ++c) {
            double s = 0.0;
            int m = 0;
            for (int32_t t = a; t < b; ++t) {
                const int32_t e = nelem[t];
                if (mask && !mask[e]) continue;
                s += ev[(int64_t)e * n_comp + c];
                ++m;
            }
            out[v * n_comp + c] = m ? s / (double)m : 0.0;
        }
    }
}

// out[p][c] = sum_i bary[p][i] nodal[set][cells[e][i]][c] for a located point (else 0).
__global__ void k_interpolate(int64_t n_pts, const int32_t *__restrict__ elem, const double *__restrict__ bary,
                              const int32_t *__restrict__ cells, int64_t n_elems, int64_t n_nodes,
                              const double *__restrict__ nodal, int n_comp, int n_sets,
                              const int32_t *__restrict__ pset, double *__restrict__ out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n_pts; p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t e = elem[p];
        const int32_t s = pset ? pset[p] : 0;
        const bool ok = e >= 0 && e < n_elems && s >= 0 && s < n_sets;
        for (int c = 0; c < n_comp; ++c) {
            double f = 0.0;
            if (ok) {
                const double *base = nodal + (int64_t)s * n_nodes * n_comp;
                for (int i = 0; i < 4; ++i) f += bary[4 * p + i] * base[(int64_t)cells[4 * (int64_t)e + i] * n_comp + c];
            }
            out[p * n_comp + c] = f;
        }
    }
}

Grid grid_of(const snp_mesh_index *mi) {
    Grid g;
    for (int k = 0; k < 3; ++k) {
        g.bmin[k] = mi->bmin[k];
        g.h[k] = mi->h[k];
        g.nb[k] = mi->nb[k];
    }
    return g;
}

// Stable sort of (key, val) pairs by key; writes the sorted values to sorted_val and the
// bucket offsets (exclusive scan of the key counts) to ptr[n_keys + 1].
int sort_into(DevBuf<int32_t> &key, DevBuf<int32_t> &val, int64_t m, int64_t n_keys, int32_t *sorted_val,
              int32_t *ptr, cudaStream_t st) {
    DevBuf<int32_t> key2, cnt;
    SNP_TRY(key2.alloc(m));
    SNP_TRY(cnt.alloc(n_keys + 1));
    DevBuf<int32_t> val_tmp;
    SNP_TRY(val_tmp.alloc(m));
    int end_bit = 1;
    while (end_bit < 31 && (int64_t(1) << end_bit) < n_keys) ++end_bit;
    cub::DoubleBuffer<int32_t> dk(key.p, key2.p);
    cub::DoubleBuffer<int32_t> dv(val.p, val_tmp.p);
    size_t tb_sort = 0, tb_scan = 0;
    SNP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, dk, dv, (int)m, 0, end_bit, st));
    SNP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, cnt.p, ptr, (int)(n_keys + 1), st));
    DevBuf<unsigned char> temp;
    SNP_TRY(temp.alloc(std::max(tb_sort, tb_scan)));
    SNP_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (n_keys + 1), st));
    if (m) {
        k_count<<<stride_grid(m, kIdxBlock, 8), kIdxBlock, 0, st>>>(key.p, m, cnt.p);
        SNP_LAUNCH_CHECK();
        SNP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tb_sort, dk, dv, (int)m, 0, end_bit, st));
        SNP_CUDA_TRY(cudaMemcpyAsync(sorted_val, dv.Current(), sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, st));
    }
    SNP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp.p, tb_scan, cnt.p, ptr, (int)(n_keys + 1), st));
    // the buffers above are freed when this returns: finish their use first
    SNP_CUDA_TRY(cudaStreamSynchronize(st));
    return SNP_OK;
}

}  // namespace
}  // namespace snp

extern "C" {

int snp_mesh_index_create(const double *nodes, int64_t n_nodes, const int32_t *cells, int64_t n_elems, void *stream,
                          snp_mesh_index **out) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(out != nullptr, "snp_mesh_index_create: out is NULL");
    *out = nullptr;
    SNP_REQUIRE(n_nodes > 0 && n_elems > 0, "snp_mesh_index_create: the mesh needs nodes and elements");
    SNP_REQUIRE(n_nodes < INT32_MAX && 4 * n_elems < INT32_MAX, "snp_mesh_index_create: mesh too large for int32 ids");
    SNP_REQUIRE(nodes && cells, "snp_mesh_index_create: NULL argument");
    cudaStream_t st = as_stream(stream);
    auto mi = new snp_mesh_index();
    std::unique_ptr<snp_mesh_index> guard(mi);
    mi->n_nodes = n_nodes;
    mi->n_elems = n_elems;
    SNP_TRY(mi->nodes.alloc(3 * n_nodes));
    SNP_TRY(mi->cells.alloc(4 * n_elems));
    SNP_CUDA_TRY(cudaMemcpyAsync(mi->nodes.p, nodes, sizeof(double) * 3 * n_nodes, cudaMemcpyDeviceToDevice, st));
    SNP_CUDA_TRY(cudaMemcpyAsync(mi->cells.p, cells, sizeof(int32_t) * 4 * n_elems, cudaMemcpyDeviceToDevice, st));

    // bounds, largest element extent and the cell check
    const int nblk = stride_grid(std::max(n_nodes, n_elems), kIdxBlock, 4);
    DevBuf<double> part;
    DevBuf<int> bad;
    SNP_TRY(part.alloc((size_t)7 * nblk));
    SNP_TRY(bad.alloc(1));
    SNP_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    k_bounds<<<nblk, kIdxBlock, 0, st>>>(mi->nodes.p, n_nodes, mi->cells.p, n_elems, part.p, bad.p);
    SNP_LAUNCH_CHECK();
    std::vector<double> hp((size_t)7 * nblk);
    int hbad = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st));
    SNP_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SNP_CUDA_TRY(cudaStreamSynchronize(st));
    SNP_REQUIRE(hbad == 0, "snp_mesh_index_create: cells hold node ids outside [0, %lld)", (long long)n_nodes);
    double v[7];
    for (int k = 0; k < 7; ++k) {
        v[k] = DBL_MAX;
        for (int b = 0; b < nblk; ++b) v[k] = std::min(v[k], hp[(size_t)7 * b + k]);
    }
    const double ext = -v[6];
    SNP_REQUIRE(std::isfinite(ext) && ext > 0.0 && std::isfinite(v[0]) && std::isfinite(v[3]),
                "snp_mesh_index_create: degenerate or non-finite mesh");
    // grid: cells at least the largest element extent, at most max(64, 2E) buckets in all
    double L[3];
    int64_t nbk = 1;
    for (int k = 0; k < 3; ++k) {
        mi->bmin[k] = v[k];
        L[k] = -v[3 + k] - v[k];
        mi->nb[k] = (int32_t)std::max(1.0, std::min(floor(L[k] / ext), 1.0e6));
    }
    const double cap = std::min(double(1 << 28), std::max(64.0, 2.0 * (double)n_elems));
    nbk = (int64_t)mi->nb[0] * mi->nb[1] * mi->nb[2];
    if ((double)nbk > cap) {
        const double f = std::cbrt((double)nbk / cap);
        for (int k = 0; k < 3; ++k) mi->nb[k] = (int32_t)std::max(1.0, floor(mi->nb[k] / f));
    }
    for (int k = 0; k < 3; ++k) mi->h[k] = L[k] > 0.0 ? L[k] / mi->nb[k] : ext;
    mi->n_buckets = (int64_t)mi->nb[0] * mi->nb[1] * mi->nb[2];

    // elements by bucket
    {
        DevBuf<int32_t> key, val;
        SNP_TRY(key.alloc(n_elems));
        SNP_TRY(val.alloc(n_elems));
        SNP_TRY(mi->bucket_ptr.alloc(mi->n_buckets + 1));
        SNP_TRY(mi->bucket_elems.alloc(n_elems));
        k_elem_buckets<<<stride_grid(n_elems, kIdxBlock, 8), kIdxBlock, 0, st>>>(mi->nodes.p, mi->cells.p, n_elems,
                                                                               grid_of(mi), key.p, val.p);
        SNP_LAUNCH_CHECK();
        SNP_TRY(sort_into(key, val, n_elems, mi->n_buckets, mi->bucket_elems.p, mi->bucket_ptr.p, st));
        DevBuf<int> mx;
        SNP_TRY(mx.alloc(1));
        SNP_CUDA_TRY(cudaMemsetAsync(mx.p, 0, sizeof(int), st));
        k_max_bucket<<<stride_grid(mi->n_buckets, kIdxBlock, 4), kIdxBlock, 0, st>>>(mi->bucket_ptr.p, mi->n_buckets,
                                                                                   mx.p);
        SNP_LAUNCH_CHECK();
        int hmx = 0;
        SNP_CUDA_TRY(cudaMemcpyAsync(&hmx, mx.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        SNP_CUDA_TRY(cudaStreamSynchronize(st));
        mi->max_bucket = hmx;
    }
    // node -> element incidence
    {
        const int64_t m = 4 * n_elems;
        DevBuf<int32_t> key, val;
        SNP_TRY(key.alloc(m));
        SNP_TRY(val.alloc(m));
        SNP_TRY(mi->node_ptr.alloc(n_nodes + 1));
        SNP_TRY(mi->node_elems.alloc(m));
        k_node_pairs<<<stride_grid(m, kIdxBlock, 8), kIdxBlock, 0, st>>>(mi->cells.p, n_elems, key.p, val.p);
        SNP_LAUNCH_CHECK();
        SNP_TRY(sort_into(key, val, m, n_nodes, mi->node_elems.p, mi->node_ptr.p, st));
    }
    *out = guard.release();
    return SNP_OK;
}

int snp_mesh_index_info(const snp_mesh_index *mi, int32_t *nb, double *bmin, double *h, int32_t *max_bucket) {
    snp::clear_error();
    SNP_REQUIRE(mi != nullptr, "snp_mesh_index_info: index is NULL");
    for (int k = 0; k < 3; ++k) {
        if (nb) nb[k] = mi->nb[k];
        if (bmin) bmin[k] = mi->bmin[k];
        if (h) h[k] = mi->h[k];
    }
    if (max_bucket) *max_bucket = mi->max_bucket;
    return SNP_OK;
}

int snp_mesh_index_locate(const snp_mesh_index *mi, const double *points, int64_t n_points, double tol, int32_t *elem,
                          double *bary, void *stream) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(mi != nullptr, "snp_mesh_index_locate: index is NULL");
    SNP_REQUIRE(n_points >= 0, "snp_mesh_index_locate: negative point count");
    if (n_points == 0) return SNP_OK;
    SNP_REQUIRE(points && elem, "snp_mesh_index_locate: NULL argument");
    SNP_REQUIRE(std::isfinite(tol) && tol >= 0.0, "snp_mesh_index_locate: tol must be finite and >= 0");
    k_locate<<<stride_grid(n_points, 128, 8), 128, 0, as_stream(stream)>>>(
        mi->nodes.p, mi->cells.p, mi->bucket_ptr.p, mi->bucket_elems.p, grid_of(mi), points, n_points, tol, elem, bary);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_mesh_index_nodal_average(const snp_mesh_index *mi, const double *elem_values, int32_t n_comp,
                                 const uint8_t *elem_mask, double *nodal, void *stream) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(mi != nullptr, "snp_mesh_index_nodal_average: index is NULL");
    SNP_REQUIRE(n_comp >= 1, "snp_mesh_index_nodal_average: n_comp must be >= 1");
    SNP_REQUIRE(elem_values && nodal, "snp_mesh_index_nodal_average: NULL argument");
    k_nodal_average<<<stride_grid(mi->n_nodes, 128, 8), 128, 0, as_stream(stream)>>>(
        mi->n_nodes, mi->node_ptr.p, mi->node_elems.p, elem_values, n_comp, elem_mask, nodal);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_mesh_index_interpolate(const snp_mesh_index *mi, int64_t n_points, const int32_t *elem, const double *bary,
                               const double *nodal, int32_t n_comp, int32_t n_sets, const int32_t *point_set,
                               double *out, void *stream) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(mi != nullptr, "snp_mesh_index_interpolate: index is NULL");
    SNP_REQUIRE(n_points >= 0 && n_comp >= 1 && n_sets >= 1, "snp_mesh_index_interpolate: bad sizes");
    if (n_points == 0) return SNP_OK;
    SNP_REQUIRE(elem && bary && nodal && out, "snp_mesh_index_interpolate: NULL argument");
    k_interpolate<<<stride_grid(n_points, 128, 8), 128, 0, as_stream(stream)>>>(
        n_points, elem, bary, mi->cells.p, mi->n_elems, mi->n_nodes, nodal, n_comp, n_sets, point_set, out);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_mesh_index_destroy(snp_mesh_index *mi) {
    snp::clear_error();
    delete mi;
    return SNP_OK;
}

}  // extern "C"
