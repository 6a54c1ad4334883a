// Deterministic two-phase assembly of the curl-curl Newton system into a fixed CSR pattern.
//
// The reference sums its element matrices into the global matrix in scipy's COO->CSR
// conversion (fem_c/interface_c.pyx:365-368, csr_array((v, (i, j))) sums duplicates) and adds
// the materials' matrices with K += this_K (curl_curl_assembler.py:900-932).  Here phase 1 is
// the single-launch element kernel (k_curlcurl, assemble_curlcurl.cu) storing each element's
// values instead of adding them into the CSR: the 21 values of the upper triangle of K, dK or
// J = K + dK (the reference kernels' arithmetic) and the six residual and reduced-rhs terms, as
// structure-of-arrays blocks over the pattern's elements.  Phase 2 (this file) forms
//
//   A_p = sum over the couplings (e, a, b) of CSR position p, in element order, of A_e,ab
//   F_i = sum over the incidences (e, a) of DoF i, in element order, of F_e,a
//
// from the pattern's sorted coupling list (cid / cptr) and incidence lists (inc / inc_ptr): one
// thread per CSR entry and one per DoF, no atomics, every output written exactly once.  Each
// entry is the same sum whatever the launch shape, so the results are bitwise repeatable.
#include "snp_common.cuh"
#include "snp_internal.cuh"

namespace snp {

namespace {

constexpr int kEntryBlock = 256;

// upper-triangle index of the element pair (a, b): rows j = min, columns k = max, row by row
__device__ __forceinline__ int tri_index(int a, int b) {
    const int j = a < b ? a : b, k = a < b ? b : a;
    return j * 6 - (j * (j - 1)) / 2 + (k - j);
}

// What the entry kernel writes, from which blocks.
enum EntryMode {
    kEntJ = 1,   // J from the J block
    kEntK = 2,   // K from the K block
    kEntKD = 3,  // K and dK from their blocks, J = K + dK
    kEntD = 4,   // dK alone
};

struct EntryArgs {
    int64_t nnz, n_elems;
    const int32_t *cptr, *cid;
    const double *terms;
    int b0, b1;  // block offsets of the first (and second) matrix read
    double *K, *dK, *J;
    float *J32;
};

// value index of coupling id t = e * 36 + a * 6 + b in its block: q * n_elems + e
__device__ __forceinline__ int64_t coupling_index(uint32_t t, int64_t S) {
    const int64_t e = (int64_t)(t / 36u);
    const int ab = (int)(t - (uint32_t)e * 36u);
    return (int64_t)tri_index(ab / 6, ab % 6) * S + e;
}

// Each thread sums kEntU consecutive entries.  The entries' first two contributions are
// requested together before any is added (a CSR entry has 1.9 on average), so a thread keeps
// up to 2 kEntU independent gathers in flight; longer entries finish in a loop.  Every entry's
// sum runs over its contributions in order.
constexpr int kEntU = 4;

template <int MODE>
__global__ void __launch_bounds__(kEntryBlock) k_cc_entries(EntryArgs r) {
    const int64_t S = r.n_elems;
    const double *m0 = r.terms + (int64_t)r.b0 * S;
    const double *m1 = r.terms + (int64_t)r.b1 * S;
    const int64_t n_groups = (r.nnz + kEntU - 1) / kEntU;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_groups; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p0 = g * kEntU;
        int c[kEntU + 1];
#pragma unroll
        for (int u = 0; u <= kEntU; ++u) c[u] = __ldg(r.cptr + (p0 + u < r.nnz ? p0 + u : r.nnz));
        uint32_t t0[kEntU], t1[kEntU];
#pragma unroll
        for (int u = 0; u < kEntU; ++u) {
            t0[u] = c[u + 1] > c[u] ? (uint32_t)__ldg(r.cid + c[u]) : 0u;
            t1[u] = c[u + 1] > c[u] + 1 ? (uint32_t)__ldg(r.cid + c[u] + 1) : 0u;
        }
        double a0[kEntU], a1[kEntU], d0[kEntU], d1[kEntU];
#pragma unroll
        for (int u = 0; u < kEntU; ++u) {
            const int64_t i0 = coupling_index(t0[u], S), i1 = coupling_index(t1[u], S);
            a0[u] = c[u + 1] > c[u] ? __ldg(m0 + i0) : 0.0;
            a1[u] = c[u + 1] > c[u] + 1 ? __ldg(m0 + i1) : 0.0;
            d0[u] = 0.0;
            d1[u] = 0.0;
            if constexpr (MODE == kEntKD) {
                d0[u] = c[u + 1] > c[u] ? __ldg(m1 + i0) : 0.0;
                d1[u] = c[u + 1] > c[u] + 1 ? __ldg(m1 + i1) : 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < kEntU; ++u) {
            const int64_t p = p0 + u;
            if (p >= r.nnz) break;
            double s0 = a0[u], s1 = d0[u];
            if (c[u + 1] > c[u] + 1) {
                s0 += a1[u];
                s1 += d1[u];
            }
            for (int k = c[u] + 2; k < c[u + 1]; ++k) {
                const int64_t ik = coupling_index((uint32_t)__ldg(r.cid + k), S);
                s0 += __ldg(m0 + ik);
                if constexpr (MODE == kEntKD) s1 += __ldg(m1 + ik);
            }
            if constexpr (MODE == kEntJ) {
                if (r.J) r.J[p] = s0;
                if (r.J32) r.J32[p] = (float)s0;
            } else if constexpr (MODE == kEntK) {
                r.K[p] = s0;
            } else if constexpr (MODE == kEntD) {
                r.dK[p] = s0;
            } else {
                if (r.K) r.K[p] = s0;
                if (r.dK) r.dK[p] = s1;
                if (r.J) r.J[p] = s0 + s1;
                if (r.J32) r.J32[p] = (float)(s0 + s1);
            }
        }
    }
}

// F_i and rhs_i from the six-term blocks over DoF i's incidences (e * 8 + a, element order)
__global__ void __launch_bounds__(kEntryBlock)
    k_cc_dofvec(int32_t n, int64_t n_elems, const int32_t *__restrict__ inc_ptr, const int32_t *__restrict__ inc,
                const double *__restrict__ Fe, const double *__restrict__ Re, double *__restrict__ F,
                double *__restrict__ rhs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double f = 0.0, rr = 0.0;
        for (int t = __ldg(inc_ptr + i); t < __ldg(inc_ptr + i + 1); ++t) {
            const uint32_t u = (uint32_t)__ldg(inc + t);
            const int64_t idx = (int64_t)(u & 7u) * n_elems + (int64_t)(u >> 3);
            if (F) f += __ldg(Fe + idx);
            if (rhs) rr += __ldg(Re + idx);
        }
        if (F) F[i] = f;
        if (rhs) rhs[i] = rr;
    }
}

template <int MODE>
int launch_entries(const EntryArgs &r, cudaStream_t st) {
    auto kern = k_cc_entries<MODE>;
    kern<<<wave_grid(kern, (r.nnz + kEntU - 1) / kEntU, kEntryBlock), kEntryBlock, 0, st>>>(r);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

}  // namespace

bool rows_supported(const snp_pattern *pat) {
    return pat != nullptr && pat->dpe == 6 && pat->has_incidence && pat->has_contrib;
}

int launch_curlcurl_rows(const snp_pattern *pat, const double *terms, const TermLayout &L, double *K, double *dK,
                         double *J, float *J32, double *rhs, double *F, cudaStream_t st) {
    SNP_REQUIRE(rows_supported(pat), "row assembly: the pattern has no contribution or incidence lists");
    SNP_REQUIRE(pat->n_elems == 0 || terms != nullptr, "row assembly: terms is NULL");
    SNP_REQUIRE(F == nullptr || L.f >= 0, "row assembly: F needs SNP_TERMS_F blocks");
    SNP_REQUIRE(rhs == nullptr || L.r >= 0, "row assembly: rhs needs SNP_TERMS_RHS blocks");
    const bool wj = J != nullptr || J32 != nullptr;
    EntryArgs r{};
    r.nnz = pat->nnz;
    r.n_elems = pat->n_elems;
    r.cptr = pat->cptr.p;
    r.cid = pat->cid.p;
    r.terms = terms;
    r.K = K;
    r.dK = dK;
    r.J = J;
    r.J32 = J32;
    if (r.nnz > 0 && (K || dK || wj)) {
        if (wj && L.k >= 0 && L.d >= 0) {
            r.b0 = L.k;
            r.b1 = L.d;
            SNP_TRY(launch_entries<kEntKD>(r, st));
        } else if (wj) {
            SNP_REQUIRE(L.j >= 0, "row assembly: J needs SNP_TERMS_J or SNP_TERMS_K | SNP_TERMS_DK blocks");
            SNP_REQUIRE(K == nullptr || L.k >= 0, "row assembly: K needs SNP_TERMS_K blocks");
            SNP_REQUIRE(dK == nullptr, "row assembly: dK needs SNP_TERMS_DK blocks");
            r.b0 = L.j;
            SNP_TRY(launch_entries<kEntJ>(r, st));
            if (K) {
                EntryArgs rk = r;
                rk.J = nullptr;
                rk.J32 = nullptr;
                rk.b0 = L.k;
                SNP_TRY(launch_entries<kEntK>(rk, st));
            }
        } else if (K && dK) {
            SNP_REQUIRE(L.k >= 0 && L.d >= 0, "row assembly: K and dK need SNP_TERMS_K | SNP_TERMS_DK blocks");
            r.b0 = L.k;
            r.b1 = L.d;
            SNP_TRY(launch_entries<kEntKD>(r, st));
        } else if (K) {
            SNP_REQUIRE(L.k >= 0, "row assembly: K needs SNP_TERMS_K blocks");
            r.b0 = L.k;
            SNP_TRY(launch_entries<kEntK>(r, st));
        } else {
            SNP_REQUIRE(L.d >= 0, "row assembly: dK needs SNP_TERMS_DK blocks");
            r.b0 = L.d;
            SNP_TRY(launch_entries<kEntD>(r, st));
        }
    }
    if ((F || rhs) && pat->n_rows > 0) {
        const double *Fe = L.f >= 0 ? terms + (int64_t)L.f * pat->n_elems : nullptr;
        const double *Re = L.r >= 0 ? terms + (int64_t)L.r * pat->n_elems : nullptr;
        k_cc_dofvec<<<wave_grid(k_cc_dofvec, pat->n_rows, kEntryBlock), kEntryBlock, 0, st>>>(
            pat->n_rows, pat->n_elems, pat->inc_ptr.p, pat->inc.p, Fe, Re, F, rhs);
        SNP_LAUNCH_CHECK();
    }
    return SNP_OK;
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
    a.t_offset = elem_offset;
    return snp::launch_curlcurl_terms(a, snp::term_layout(parts), terms, pat->n_elems, snp::as_stream(stream));
}

int snp_curlcurl_rows(const snp_pattern *pat, const double *terms, int32_t parts, double *K_vals, double *dK_vals,
                      double *J_vals, float *J32_vals, double *rhs, double *F, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(pat != nullptr, "snp_curlcurl_rows: pattern is NULL");
    SNP_REQUIRE((parts & ~31) == 0, "snp_curlcurl_rows: unknown bits in parts (0x%x)", (unsigned)parts);
    return snp::launch_curlcurl_rows(pat, terms, snp::term_layout(parts), K_vals, dK_vals, J_vals, J32_vals, rhs, F,
                                     snp::as_stream(stream));
}

}  // extern "C"
