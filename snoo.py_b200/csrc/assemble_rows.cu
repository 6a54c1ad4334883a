// Deterministic two-phase assembly of the curl-curl Newton system into a fixed CSR pattern.
//
// The reference sums its element matrices into the global matrix in scipy's COO->CSR
// conversion (fem_c/interface_c.pyx:365-368, csr_array((v, (i, j))) sums duplicates) and adds
// the materials' matrices with K += this_K (curl_curl_assembler.py:900-932).  Here phase 1
// (k_curlcurl_terms in assemble_curlcurl.cu) writes one record per element: reference-frame
// tensors such as SK = kfac Jm^T Jm and element vectors such as G (residual) and R (reduced
// rhs).  Phase 2 (this file) forms every CSR row from the records of the elements incident to
// the row's DoF:
//
//   K_ik = sum over incident (e, a) of chat_a(e) . SK_e chat_b(e)    (b: e's DoF at column k)
//   F_i  = sum over incident (e, a) of chat_a(e) . G_e
//
// chat_a(e): reference curl of local edge a in the element's orientation table (first-order
// Nedelec on affine tetrahedra, so it does not depend on the quadrature point).
//
// A group of 8 lanes owns one row.  Lane j takes the row's incidences j, j + 8, ...; for its
// incidence (e, a) it forms the six entries of element row a and its F / rhs terms.  Entries go
// into a shared-memory copy of the row in incidence order, one warp-synchronous step per lane
// (an element row's six columns are distinct, so one step never adds twice to an entry); the row
// is then written once, coalesced.  Every entry is the sum of its element contributions in
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
    const int32_t *row_ptr, *slots, *inc_ptr, *inc;
    const double *terms;
    TermLayout L;
    const double *ctab;
    int n_orient, qstride;
    int t0, t1;      // record offsets of the tensors summed into row buffers 0 and 1
    int jsrc;        // J from buffer 0, buffer 1, or their sum (2)
    double *p0, *p1, *pj;
    float *pj32;
    double *rhs, *F;
};

// NB: number of row buffers (tensors gathered per incidence), 0..2
template <int NB>
__global__ void __launch_bounds__(kRowBlock, 4) k_curlcurl_rows(RowArgs r) {
    extern __shared__ double sm[];
    double *s_ctab = sm;
    double *s_buf = sm + r.n_orient * 18;
    for (int t = threadIdx.x; t < r.n_orient * 18; t += blockDim.x) {
        const int o = t / 18, q = t - o * 18;
        s_ctab[t] = r.ctab[(int64_t)o * r.qstride + q];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int lg = lane & (kRowLanes - 1);
    const int gbase = lane & ~(kRowLanes - 1);
    const int group = threadIdx.x / kRowLanes;
    double *buf0 = s_buf + (size_t)group * (NB > 0 ? NB : 1) * kRowCap;
    double *buf1 = buf0 + kRowCap;
    const TermLayout L = r.L;
    const int64_t n_slots_rows = (int64_t)gridDim.x * kRowGroups;
    // every lane of a warp runs the same number of row rounds (the warp-synchronous steps)
    const int64_t first = (int64_t)blockIdx.x * kRowGroups + group;
    const int64_t warp_first = (int64_t)blockIdx.x * kRowGroups + (threadIdx.x / 32) * (32 / kRowLanes);
    const int64_t rounds = warp_first < r.n_rows ? (r.n_rows - 1 - warp_first) / n_slots_rows + 1 : 0;
    for (int64_t round = 0; round < rounds; ++round) {
        const int64_t i = first + round * n_slots_rows;
        const bool live = i < r.n_rows;
        int rs = 0, len = 0, ta = 0, tb = 0;
        if (live) {
            rs = r.row_ptr[i];
            len = r.row_ptr[i + 1] - rs;
            ta = r.inc_ptr[i];
            tb = r.inc_ptr[i + 1];
        }
        if constexpr (NB > 0) {
            for (int l = lg; l < len; l += kRowLanes) {
                buf0[l] = 0.0;
                if constexpr (NB > 1) buf1[l] = 0.0;
            }
        }
        const int my_chunks = (tb - ta + kRowLanes - 1) / kRowLanes;
        const int chunks = __reduce_max_sync(0xffffffffu, (unsigned)my_chunks);
        __syncwarp();
        double f_acc = 0.0, r_acc = 0.0;
        for (int c = 0; c < chunks; ++c) {
            const int t = ta + c * kRowLanes + lg;
            const bool act = t < tb;
            double v0[6], v1[6], f = 0.0, rr = 0.0;
            int pos[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                v0[k] = 0.0;
                v1[k] = 0.0;
                pos[k] = -1;
            }
            if (act) {
                const uint32_t u = (uint32_t)r.inc[t];
                const int64_t e = (int64_t)(u >> 3);
                const int a = (int)(u & 7u);
                const double *rec = r.terms + e * (int64_t)L.stride;
                const double *ct = s_ctab + (int)rec[L.o] * 18;
                const double h0 = ct[3 * a], h1 = ct[3 * a + 1], h2 = ct[3 * a + 2];
                if (L.f >= 0) f = h0 * rec[L.f] + h1 * rec[L.f + 1] + h2 * rec[L.f + 2];
                if (L.r >= 0) rr = h0 * rec[L.r] + h1 * rec[L.r + 1] + h2 * rec[L.r + 2];
                if constexpr (NB > 0) {
                    const int2 *sp = reinterpret_cast<const int2 *>(r.slots + e * 36 + a * 6);
                    const int2 s01 = __ldg(sp), s23 = __ldg(sp + 1), s45 = __ldg(sp + 2);
                    const int sl[6] = {s01.x, s01.y, s23.x, s23.y, s45.x, s45.y};
#pragma unroll
                    for (int k = 0; k < 6; ++k) pos[k] = ((unsigned)(sl[k] - rs) < (unsigned)len) ? sl[k] - rs : -1;
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        const double *S = rec + (b == 0 ? r.t0 : r.t1);
                        const double w0 = S[0] * h0 + S[1] * h1 + S[2] * h2;
                        const double w1 = S[1] * h0 + S[3] * h1 + S[4] * h2;
                        const double w2 = S[2] * h0 + S[4] * h1 + S[5] * h2;
                        double *v = b == 0 ? v0 : v1;
#pragma unroll
                        for (int k = 0; k < 6; ++k) v[k] = ct[3 * k] * w0 + ct[3 * k + 1] * w1 + ct[3 * k + 2] * w2;
                    }
                }
            }
            if constexpr (NB > 0) {
                for (int j = 0; j < kRowLanes; ++j) {
                    if (act && lg == j) {
#pragma unroll
                        for (int k = 0; k < 6; ++k) {
                            if (pos[k] >= 0) {
                                buf0[pos[k]] += v0[k];
                                if constexpr (NB > 1) buf1[pos[k]] += v1[k];
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            // F and rhs in incidence order (inactive lanes add an exact 0)
#pragma unroll
            for (int j = 0; j < kRowLanes; ++j) {
                f_acc += __shfl_sync(0xffffffffu, f, gbase + j);
                r_acc += __shfl_sync(0xffffffffu, rr, gbase + j);
            }
        }
        if (live) {
            if constexpr (NB > 0) {
                for (int l = lg; l < len; l += kRowLanes) {
                    const double b0 = buf0[l];
                    const double b1 = NB > 1 ? buf1[l] : 0.0;
                    if (r.p0) r.p0[rs + l] = b0;
                    if (NB > 1 && r.p1) r.p1[rs + l] = b1;
                    const double jv = r.jsrc == 0 ? b0 : (r.jsrc == 1 ? b1 : b0 + b1);
                    if (r.pj) r.pj[rs + l] = jv;
                    if (r.pj32) r.pj32[rs + l] = (float)jv;
                }
            }
            if (lg == 0) {
                if (r.F) r.F[i] = f_acc;
                if (r.rhs) r.rhs[i] = r_acc;
            }
        }
        __syncwarp();
    }
}

template <int NB>
int launch_rows_t(const RowArgs &r, cudaStream_t st) {
    const size_t smem = sizeof(double) * ((size_t)r.n_orient * 18 + (size_t)kRowGroups * (NB > 0 ? NB : 1) * kRowCap);
    auto kern = k_curlcurl_rows<NB>;
    if (smem > 48 * 1024) SNP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t blocks_needed = ((int64_t)r.n_rows + kRowGroups - 1) / kRowGroups;
    kern<<<wave_grid(kern, blocks_needed * kRowBlock, kRowBlock, smem), kRowBlock, smem, st>>>(r);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
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
    r.slots = pat->slots.p;
    r.inc_ptr = pat->inc_ptr.p;
    r.inc = pat->inc.p;
    r.terms = terms;
    r.L = L;
    r.ctab = ctab;
    r.n_orient = n_orient;
    r.qstride = quad_stride_ctab;
    r.rhs = rhs;
    r.F = F;
    r.t0 = r.t1 = 0;
    r.jsrc = 0;
    const bool wj = J != nullptr || J32 != nullptr;
    int nb = 0;
    if (K == nullptr && dK == nullptr && !wj) {
        nb = 0;
    } else if (wj && dK == nullptr && L.j >= 0) {
        if (K) {
            SNP_REQUIRE(L.k >= 0, "row assembly: K needs SNP_TERMS_K records");
            nb = 2;
            r.t0 = L.k;
            r.t1 = L.j;
            r.p0 = K;
            r.jsrc = 1;
        } else {
            nb = 1;
            r.t0 = L.j;
            r.jsrc = 0;
        }
        r.pj = J;
        r.pj32 = J32;
    } else if (wj) {
        SNP_REQUIRE(L.k >= 0 && L.d >= 0, "row assembly: J needs SNP_TERMS_J or SNP_TERMS_K | SNP_TERMS_DK records");
        nb = 2;
        r.t0 = L.k;
        r.t1 = L.d;
        r.p0 = K;
        r.p1 = dK;
        r.pj = J;
        r.pj32 = J32;
        r.jsrc = 2;
    } else if (K && dK) {
        SNP_REQUIRE(L.k >= 0 && L.d >= 0, "row assembly: K and dK need SNP_TERMS_K | SNP_TERMS_DK records");
        nb = 2;
        r.t0 = L.k;
        r.t1 = L.d;
        r.p0 = K;
        r.p1 = dK;
    } else if (K) {
        SNP_REQUIRE(L.k >= 0, "row assembly: K needs SNP_TERMS_K records");
        nb = 1;
        r.t0 = L.k;
        r.p0 = K;
    } else {
        SNP_REQUIRE(L.d >= 0, "row assembly: dK needs SNP_TERMS_DK records");
        nb = 1;
        r.t0 = L.d;
        r.p0 = dK;
    }
    if (r.n_rows == 0) return SNP_OK;
    if (nb == 0) return launch_rows_t<0>(r, st);
    if (nb == 1) return launch_rows_t<1>(r, st);
    return launch_rows_t<2>(r, st);
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
