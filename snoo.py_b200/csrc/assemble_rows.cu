// Deterministic two-phase assembly of the curl-curl Newton system into a fixed CSR pattern.
//
// The reference sums its element matrices into the global matrix in scipy's COO->CSR
// conversion (fem_c/interface_c.pyx:365-368, csr_array((v, (i, j))) sums duplicates) and adds
// the materials' matrices with K += this_K (curl_curl_assembler.py:900-932).  Here phase 1
// (k_curlcurl_terms in assemble_curlcurl.cu) writes one record per element: the element map
// Jm and kfac = sum_q nu_q w_q / det (with c_a = Jm chat_a the element's curls, as the reference
// kernels form them), the tensor M = sum_q a_q B_q B_q^T of dK, or the reference-frame Jacobian
// tensor SJ, and element vectors such as G (residual) and R (reduced rhs).  Phase 2 (this file)
// forms every CSR row from the records of the elements incident to the row's DoF:
//
//   K_ik = sum over incident (e, a) of kfac_e (c_a . c_b)      (b: e's DoF at column k)
//   F_i  = sum over incident (e, a) of chat_a(e) . G_e
//
// chat_a(e): reference curl of local edge a in the element's orientation table (first-order
// Nedelec on affine tetrahedra, so it does not depend on the quadrature point).
//
// A group of 8 lanes owns one row.  Lane j takes the row's incidences j, j + 8, ...; for its
// incidence (e, a) it forms the six entries of element row a and its F / rhs terms.  The row's
// entries live in the group's registers (lane lg holds positions lg, lg + 8, ...); the lanes'
// entries are broadcast lane by lane and added by their owners, so each entry sums its
// contributions in incidence order.  The row is then written once, coalesced.  Every entry is the sum of its element contributions in
// element order whatever the launch shape: bitwise repeatable, no atomics, no zeroing pass, and
// each output value written exactly once.
#include "snp_common.cuh"
#include "snp_internal.cuh"

namespace snp {

namespace {

constexpr int kRowLanes = 8;
constexpr int kRowBlock = 256;
constexpr int kRowGroups = kRowBlock / kRowLanes;  // rows in flight per block
constexpr int kRowCap = SNP_ROWS_MAX_ENTRIES;

struct RowArgs {
    int32_t n_rows;
    const int32_t *row_ptr, *inc_ptr, *inc;
    const uint2 *loc;
    const double *terms;
    TermLayout L;
    const double *ctab;
    int n_orient, qstride;
    double *K, *dK, *J;
    float *J32;
    double *rhs, *F;
};

// What the row buffers hold, from which record parts.
enum RowMode {
    kRowsNone = 0,  // F / rhs only
    kRowsJ = 1,     // J from SJ (reference frame)
    kRowsK = 2,     // K from Jm, kfac
    kRowsKD = 3,    // K and dK from Jm, kfac, M (J = K + dK)
};

// Row metadata of one row (or of none: i >= n).
struct RowMeta {
    int rs, len, ta, tb;
};

__device__ __forceinline__ RowMeta row_meta(const RowArgs &r, int64_t i) {
    RowMeta m{0, 0, 0, 0};
    if (i < r.n_rows) {
        m.rs = __ldg(r.row_ptr + i);
        m.len = __ldg(r.row_ptr + i + 1) - m.rs;
        m.ta = __ldg(r.inc_ptr + i);
        m.tb = __ldg(r.inc_ptr + i + 1);
    }
    return m;
}

// MODE: RowMode.  Element row a of element e, column l:
//   K_al  = kfac (c_a . c_l),  c = Jm chat (the reference kernels' arithmetic, so entries that
//           are exact zeros there are exact zeros here)
//   dK_al = c_l . (M c_a)
//   J_al  = chat_l . (SJ chat_a)
// NS: row entries per lane (rows of at most 8 NS entries); lane lg of a group owns the row's
// positions lg, lg + 8, ..., held in registers.  Each lane forms the six entries of its own
// incidence, then the group walks its lanes in order: lane j's six (position, value) pairs are
// broadcast by shuffles and the owner of each position adds the value.  A position thus
// receives its contributions in incidence order (one per incidence at most).
// Software pipeline across a group's rows: while row i is formed, the incidence words of the
// group's next row and the metadata of the row after it are already in flight, so each row
// waits on one dependent load (its elements' records) instead of three.
template <int MODE, int NS>
__global__ void __launch_bounds__(kRowBlock, MODE == kRowsKD || MODE == kRowsK ? 2 : (MODE == kRowsJ && NS > 4 ? 3 : 4))
    k_curlcurl_rows(RowArgs r) {
    extern __shared__ double sm[];
    double *s_ctab = sm;
    for (int t = threadIdx.x; t < r.n_orient * 18; t += blockDim.x) {
        const int o = t / 18, q = t - o * 18;
        s_ctab[t] = r.ctab[(int64_t)o * r.qstride + q];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int lg = lane & (kRowLanes - 1);
    const int gbase = lane & ~(kRowLanes - 1);
    const int group = threadIdx.x / kRowLanes;
    const TermLayout L = r.L;
    const int64_t step = (int64_t)gridDim.x * kRowGroups;
    // every lane of a warp runs the same number of row rounds (the shuffles are warp-wide)
    const int64_t first = (int64_t)blockIdx.x * kRowGroups + group;
    const int64_t warp_first = (int64_t)blockIdx.x * kRowGroups + (threadIdx.x / 32) * (32 / kRowLanes);
    const int64_t rounds = warp_first < r.n_rows ? (r.n_rows - 1 - warp_first) / step + 1 : 0;

    RowMeta cur = row_meta(r, first);
    RowMeta nxt = row_meta(r, first + step);
    uint32_t u = 0;
    uint2 lc = make_uint2(0u, 0u);
    if (cur.ta + lg < cur.tb) {
        u = (uint32_t)__ldg(r.inc + cur.ta + lg);
        lc = __ldg(r.loc + cur.ta + lg);
    }
    for (int64_t round = 0; round < rounds; ++round) {
        const int64_t i = first + round * step;
        const bool live = i < r.n_rows;
        // prefetch: the next row's first incidence words, the metadata of the row after it
        uint32_t u_n = 0;
        uint2 lc_n = make_uint2(0u, 0u);
        if (nxt.ta + lg < nxt.tb) {
            u_n = (uint32_t)__ldg(r.inc + nxt.ta + lg);
            lc_n = __ldg(r.loc + nxt.ta + lg);
        }
        const RowMeta nn = row_meta(r, i + 2 * step);

        const int rs = cur.rs, len = cur.len, ta = cur.ta, tb = cur.tb;
        double acc0[NS], acc1[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            acc0[q] = 0.0;
            acc1[q] = 0.0;
        }
        const int my_n = tb - ta;
        const int warp_n = (int)__reduce_max_sync(0xffffffffu, (unsigned)my_n);
        double f_acc = 0.0, r_acc = 0.0;
        for (int c = 0; c * kRowLanes < warp_n; ++c) {
            const int t = ta + c * kRowLanes + lg;
            const bool act = t < tb;
            if (c > 0 && act) {
                u = (uint32_t)__ldg(r.inc + t);
                lc = __ldg(r.loc + t);
            }
            if (!act) lc = make_uint2(0xffffffffu, 0xffffffffu);  // positions 255: owned by nobody
            double v0[6], v1[6], f = 0.0, rr = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                v0[k] = 0.0;
                v1[k] = 0.0;
            }
            if (act) {
                const int64_t e = (int64_t)(u >> 3);
                const int a = (int)(u & 7u);
                const double *rec = r.terms + e * (int64_t)L.stride;
                const double *ct = s_ctab + (int)__ldg(rec + L.o) * 18;
                const double h0 = ct[3 * a], h1 = ct[3 * a + 1], h2 = ct[3 * a + 2];
                if (L.f >= 0) f = h0 * __ldg(rec + L.f) + h1 * __ldg(rec + L.f + 1) + h2 * __ldg(rec + L.f + 2);
                if (L.r >= 0) rr = h0 * __ldg(rec + L.r) + h1 * __ldg(rec + L.r + 1) + h2 * __ldg(rec + L.r + 2);
                if constexpr (MODE == kRowsJ) {
                    double S[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) S[q] = __ldg(rec + L.j + q);
                    const double w0 = S[0] * h0 + S[1] * h1 + S[2] * h2;
                    const double w1 = S[1] * h0 + S[3] * h1 + S[4] * h2;
                    const double w2 = S[2] * h0 + S[4] * h1 + S[5] * h2;
#pragma unroll
                    for (int k = 0; k < 6; ++k) v0[k] = ct[3 * k] * w0 + ct[3 * k + 1] * w1 + ct[3 * k + 2] * w2;
                }
                if constexpr (MODE == kRowsK || MODE == kRowsKD) {
                    double Jm[9];
#pragma unroll
                    for (int q = 0; q < 9; ++q) Jm[q] = __ldg(rec + L.k + q);
                    const double kfac = __ldg(rec + L.k + 9);
                    double ca[3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) ca[q] = Jm[3 * q] * h0 + Jm[3 * q + 1] * h1 + Jm[3 * q + 2] * h2;
                    double ma[3] = {0.0, 0.0, 0.0};
                    if constexpr (MODE == kRowsKD) {
                        double M[6];
#pragma unroll
                        for (int q = 0; q < 6; ++q) M[q] = __ldg(rec + L.d + q);
                        ma[0] = M[0] * ca[0] + M[1] * ca[1] + M[2] * ca[2];
                        ma[1] = M[1] * ca[0] + M[3] * ca[1] + M[4] * ca[2];
                        ma[2] = M[2] * ca[0] + M[4] * ca[1] + M[5] * ca[2];
                    }
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const double g0 = ct[3 * k], g1 = ct[3 * k + 1], g2 = ct[3 * k + 2];
                        double cl[3];
#pragma unroll
                        for (int q = 0; q < 3; ++q) cl[q] = Jm[3 * q] * g0 + Jm[3 * q + 1] * g1 + Jm[3 * q + 2] * g2;
                        v0[k] = kfac * (ca[0] * cl[0] + ca[1] * cl[1] + ca[2] * cl[2]);
                        if constexpr (MODE == kRowsKD) v1[k] = cl[0] * ma[0] + cl[1] * ma[1] + cl[2] * ma[2];
                    }
                }
            }
            // the group's lanes in order: broadcast lane j's entries, owners add them
            const int nj = min(kRowLanes, warp_n - c * kRowLanes);
            for (int j = 0; j < nj; ++j) {
                const int src = gbase + j;
                if constexpr (MODE != kRowsNone) {
                    const uint32_t px = __shfl_sync(0xffffffffu, lc.x, src);
                    const uint32_t py = __shfl_sync(0xffffffffu, lc.y, src);
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const int p = k < 4 ? (int)((px >> (8 * k)) & 0xffu) : (int)((py >> (8 * (k - 4))) & 0xffu);
                        const double a0 = __shfl_sync(0xffffffffu, v0[k], src);
                        double a1 = 0.0;
                        if constexpr (MODE == kRowsKD) a1 = __shfl_sync(0xffffffffu, v1[k], src);
                        const bool mine = (p & (kRowLanes - 1)) == lg;
                        const int slot = p >> 3;
#pragma unroll
                        for (int q = 0; q < NS; ++q) {
                            if (mine && slot == q) {
                                acc0[q] += a0;
                                if constexpr (MODE == kRowsKD) acc1[q] += a1;
                            }
                        }
                    }
                }
                // F and rhs in incidence order (inactive lanes add an exact 0)
                f_acc += __shfl_sync(0xffffffffu, f, src);
                r_acc += __shfl_sync(0xffffffffu, rr, src);
            }
        }
        if (live) {
            if constexpr (MODE != kRowsNone) {
#pragma unroll
                for (int q = 0; q < NS; ++q) {
                    const int l = q * kRowLanes + lg;
                    if (l < len) {
                        if constexpr (MODE == kRowsJ) {
                            if (r.J) r.J[rs + l] = acc0[q];
                            if (r.J32) r.J32[rs + l] = (float)acc0[q];
                        } else {
                            if (r.K) r.K[rs + l] = acc0[q];
                            if constexpr (MODE == kRowsKD) {
                                if (r.dK) r.dK[rs + l] = acc1[q];
                                if (r.J) r.J[rs + l] = acc0[q] + acc1[q];
                                if (r.J32) r.J32[rs + l] = (float)(acc0[q] + acc1[q]);
                            }
                        }
                    }
                }
            }
            if (lg == 0) {
                if (r.F) r.F[i] = f_acc;
                if (r.rhs) r.rhs[i] = r_acc;
            }
        }
        cur = nxt;
        nxt = nn;
        u = u_n;
        lc = lc_n;
    }
}

template <int MODE, int NS>
int launch_rows_ns(const RowArgs &r, cudaStream_t st) {
    const size_t smem = sizeof(double) * (size_t)r.n_orient * 18;
    auto kern = k_curlcurl_rows<MODE, NS>;
    if (smem > 48 * 1024) SNP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t blocks_needed = ((int64_t)r.n_rows + kRowGroups - 1) / kRowGroups;
    kern<<<wave_grid(kern, blocks_needed * kRowBlock, kRowBlock, smem), kRowBlock, smem, st>>>(r);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

// rows of at most 32 entries (the usual first-order tetrahedral meshes) or at most 64
template <int MODE>
int launch_rows_t(const RowArgs &r, int max_row, cudaStream_t st) {
    if (max_row <= 4 * kRowLanes) return launch_rows_ns<MODE, 4>(r, st);
    return launch_rows_ns<MODE, kRowCap / kRowLanes>(r, st);
}

}  // namespace

bool rows_supported(const snp_pattern *pat) {
    return pat != nullptr && pat->dpe == 6 && pat->has_incidence && pat->max_row <= kRowCap;
}

int launch_curlcurl_rows(const snp_pattern *pat, const double *terms, const TermLayout &L, const double *ctab,
                         int n_orient, int quad_stride_ctab, double *K, double *dK, double *J, float *J32, double *rhs,
                         double *F, cudaStream_t st) {
    SNP_REQUIRE(rows_supported(pat), "row assembly: the pattern has no incidence lists or a row longer than %d entries",
                kRowCap);
    SNP_REQUIRE(ctab != nullptr && n_orient >= 1, "row assembly: curls table missing");
    SNP_REQUIRE(pat->n_elems == 0 || terms != nullptr, "row assembly: terms is NULL");
    SNP_REQUIRE(F == nullptr || L.f >= 0, "row assembly: F needs SNP_TERMS_F records");
    SNP_REQUIRE(rhs == nullptr || L.r >= 0, "row assembly: rhs needs SNP_TERMS_RHS records");
    RowArgs r{};
    r.n_rows = pat->n_rows;
    r.row_ptr = pat->row_ptr.p;
    r.loc = pat->inc_loc.p;
    r.inc_ptr = pat->inc_ptr.p;
    r.inc = pat->inc.p;
    r.terms = terms;
    r.L = L;
    r.ctab = ctab;
    r.n_orient = n_orient;
    r.qstride = quad_stride_ctab;
    r.K = K;
    r.dK = dK;
    r.J = J;
    r.J32 = J32;
    r.rhs = rhs;
    r.F = F;
    const bool wj = J != nullptr || J32 != nullptr;
    if (r.n_rows == 0) return SNP_OK;
    if (K == nullptr && dK == nullptr && !wj) return launch_rows_t<kRowsNone>(r, pat->max_row, st);
    if (K == nullptr && dK == nullptr && L.j >= 0) return launch_rows_t<kRowsJ>(r, pat->max_row, st);
    SNP_REQUIRE(L.k >= 0, "row assembly: K, dK and J need SNP_TERMS_K or SNP_TERMS_DK records (J alone: SNP_TERMS_J)");
    if (dK == nullptr && !wj) return launch_rows_t<kRowsK>(r, pat->max_row, st);
    SNP_REQUIRE(L.d >= 0, "row assembly: dK and J = K + dK need SNP_TERMS_DK records");
    return launch_rows_t<kRowsKD>(r, pat->max_row, st);
}

}  // namespace snp

extern "C" {

int snp_curlcurl_terms_stride(int32_t parts, int32_t *stride) {
    snp::clear_error();
    SNP_REQUIRE(stride != nullptr, "snp_curlcurl_terms_stride: stride is NULL");
    SNP_REQUIRE((parts & ~31) == 0, "snp_curlcurl_terms_stride: unknown bits in parts (0x%x)", (unsigned)parts);
    *stride = snp::term_layout(parts).stride;
    return SNP_OK;
}

int snp_curlcurl_rows_supported(const snp_pattern *pat, int32_t *supported) {
    snp::clear_error();
    SNP_REQUIRE(pat != nullptr && supported != nullptr, "snp_curlcurl_rows_supported: NULL argument");
    *supported = snp::rows_supported(pat) ? 1 : 0;
    return SNP_OK;
}

int snp_curlcurl_terms(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems, const double *nodes,
                       const int32_t *cells, const int32_t *glob_ids, const int32_t *orientations, const double *curls,
                       int32_t n_orient, const double *phi, const double *d_phi, const double *w, int32_t n_quad,
                       const double *x, const double *B_s, int32_t n_int, const double *rel_c, const double *rel_x,
                       const double *dilution, int32_t parts, double *terms, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(pat != nullptr, "snp_curlcurl_terms: pattern is NULL");
    SNP_REQUIRE((parts & ~31) == 0, "snp_curlcurl_terms: unknown bits in parts (0x%x)", (unsigned)parts);
    SNP_REQUIRE((phi == nullptr) == (dilution == nullptr), "snp_curlcurl_terms: give both phi and dilution, or neither");
    snp::CurlArgs a;
    SNP_TRY(snp::fill_args(a, pat, elem_offset, n_elems, nodes, cells, glob_ids, orientations, curls, n_orient, d_phi,
                           w, n_quad, x, B_s, n_int, rel_c, rel_x));
    if (B_s != nullptr && phi != nullptr) {
        a.phi = phi;
        for (int i = 0; i < 4; ++i) a.dil[i] = dilution[i];
    }
    const snp::TermLayout L = snp::term_layout(parts);
    return snp::launch_curlcurl_terms(a, L, terms + elem_offset * (int64_t)L.stride, snp::as_stream(stream));
}

int snp_curlcurl_rows(const snp_pattern *pat, const double *terms, int32_t parts, const double *curls,
                      int32_t n_orient, int32_t n_quad, double *K_vals, double *dK_vals, double *J_vals,
                      float *J32_vals, double *rhs, double *F, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(pat != nullptr, "snp_curlcurl_rows: pattern is NULL");
    SNP_REQUIRE((parts & ~31) == 0, "snp_curlcurl_rows: unknown bits in parts (0x%x)", (unsigned)parts);
    SNP_REQUIRE(n_quad >= 1, "snp_curlcurl_rows: n_quad must be >= 1");
    return snp::launch_curlcurl_rows(pat, terms, snp::term_layout(parts), curls, n_orient, n_quad * 18, K_vals,
                                     dK_vals, J_vals, J32_vals, rhs, F, snp::as_stream(stream));
}

}  // extern "C"
