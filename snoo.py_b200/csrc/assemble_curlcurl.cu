// Newton assembly of the curl-curl operator on first-order Nedelec tetrahedra.
//
// Element arithmetic of the reference kernels compute_K_dK_Hcurl (fem_c/ctools.c:960-1193)
// and compute_K_dK_Hcurl_red (fem_c/ctools.c:1195-1388), one thread per element, fused
// with the scatter into a fixed CSR pattern and with the residual F = K(x) x - rhs(x):
//
//   Jm        = sum_i X_i (x) dphi_i                     (ctools.c:373-413)
//   c_j       = Jm curl_hat_j(orientation)               (physical curl = c_j / det)
//   B_q       = B_s,q + sum_j c_j x_j / det              (ctools.c:922-958)
//   nu_q, nu'_q = PCHIP(|B_q|)                           (ctools.c:130-204)
//   K_jk      = sum_q nu_q w_q (c_j . c_k) / det
//   dK_jk     = sum_q [|B_q| >= 1e-14] nu'_q w_q (c_j . B_q)(c_k . B_q) / (det |B_q|)
//   rhs_j     = sum_q (nu0 - nu_q) (c_j . B_s,q) w_q     (reduced kernel, ctools.c:1332-1335)
//
// Diluted steel (compute_K_dK_Hcurl_red_dil, fem_c/ctools.c:1565-1759), reduced kernel only:
//   z_q = sum_i phi_i(q) Z_i,  s_q = (c_num + z_q m_num) / (c_den + z_q m_den)
//   nu_q = s_q PCHIP(s_q |B_q|),  nu'_q = s_q^2 PCHIP'(s_q |B_q|)
//
// For first-order tetrahedra d_phi and the curls do not depend on the quadrature point,
// so Jm, det and c_j are computed once per element and the sums over q factor:
// K_jk = (c_j . c_k) * sum_q nu_q w_q / det.  Without a source field B is constant over
// the element and nu, nu' are evaluated once.  Values agree with the reference's
// per-point sums to rounding.
//
// Data per element: cells 16 B, glob_ids 24 B, orientation 4 B, slot map 144 B, plus
// gathered coordinates and x (mostly cache hits for a locality-ordered mesh).
#include "snp_common.cuh"
#include "snp_internal.cuh"

namespace snp {

namespace {

constexpr int kBlock = 128;

struct SmemLayout {
    int off_ctab, off_dphi, off_w, off_phi, off_relc, off_relx, total;
};

__host__ __device__ inline SmemLayout smem_layout(int n_orient, int nq, int n_int) {
    SmemLayout L;
    int o = 0;
    L.off_ctab = o;
    o += n_orient * 18;
    L.off_dphi = o;
    o += 12;
    L.off_w = o;
    o += nq;
    L.off_phi = o;
    o += 4 * nq;
    int nc = n_int < 0 ? 1 : 4 * n_int;
    int nx = n_int < 0 ? 1 : n_int + 1;
    L.off_relc = o;
    o += nc;
    L.off_relx = o;
    o += nx;
    L.total = o;
    return L;
}

template <typename T>
__device__ __forceinline__ void red_add(T *p, T v) {
    atomicAdd(p, v);
}

// Element values of the two-phase assembly (CurlArgs::ET): the (j, k) pair's K, dK and J, and
// the residual and reduced-rhs terms, each into its block at element eo.
__device__ __forceinline__ void store_pair(const CurlArgs &a, int tri, int64_t eo, double kv, double dv) {
    const int64_t S = a.et_stride;
    if (a.et_k >= 0) a.ET[(a.et_k + tri) * S + eo] = kv;
    if (a.et_d >= 0) a.ET[(a.et_d + tri) * S + eo] = dv;
    if (a.et_j >= 0) a.ET[(a.et_j + tri) * S + eo] = kv + dv;
}

__device__ __forceinline__ void store_vectors(const CurlArgs &a, int64_t eo, const double *Fj, const double *rj) {
    const int64_t S = a.et_stride;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        if (a.et_f >= 0) a.ET[(a.et_f + j) * S + eo] = Fj[j];
        if (a.et_r >= 0) a.ET[(a.et_r + j) * S + eo] = rj ? rj[j] : 0.0;
    }
}

// nu and nu' at one quadrature point; DIL: diluted steel with the point's nodal basis ph[4]
// and the element's node z coordinates Zn[4]
template <bool DIL>
__device__ __forceinline__ double nu_at(const CurlArgs &a, const double *relc, const double *relx, const double *ph,
                                        const double (&Zn)[4], double bm, double &dnu) {
    if constexpr (!DIL) {
        return pchip_eval<double>(a.n_int, relc, relx, bm, dnu);
    } else {
        double z = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) z += ph[i] * Zn[i];
        const double sf = (a.dil[0] + z * a.dil[1]) / (a.dil[2] + z * a.dil[3]);
        const double nu = sf * pchip_eval<double>(a.n_int, relc, relx, sf * bm, dnu);
        dnu *= sf * sf;
        return nu;
    }
}

// HAS_BS: reduced formulation with a source field at each quadrature point.
// NQ: compile-time number of quadrature points (0 = runtime count).
// DIL: diluted steel (with HAS_BS only).
template <bool HAS_BS, int NQ, typename VT, bool DIL>
__global__ void __launch_bounds__(kBlock)
    k_curlcurl(CurlArgs a, int quad_stride_ctab) {
    extern __shared__ double sm[];
    const SmemLayout L = smem_layout(a.n_orient, a.nq, a.n_int);
    double *s_ctab = sm + L.off_ctab;
    double *s_dphi = sm + L.off_dphi;
    double *s_w = sm + L.off_w;
    double *s_phi = sm + L.off_phi;
    double *s_relc = sm + L.off_relc;
    double *s_relx = sm + L.off_relx;
    // stage tables: curls at q = 0 for every orientation, d_phi at q = 0, weights, PCHIP
    for (int t = threadIdx.x; t < a.n_orient * 18; t += blockDim.x) {
        int o = t / 18, r = t - o * 18;
        s_ctab[t] = a.ctab[(int64_t)o * quad_stride_ctab + r];
    }
    for (int t = threadIdx.x; t < 12; t += blockDim.x) s_dphi[t] = a.dphi0[t];
    for (int t = threadIdx.x; t < a.nq; t += blockDim.x) s_w[t] = a.w[t];
    if (a.phi)
        for (int t = threadIdx.x; t < 4 * a.nq; t += blockDim.x) s_phi[t] = a.phi[t];
    const int nc = a.n_int < 0 ? 1 : 4 * a.n_int;
    const int nx = a.n_int < 0 ? 1 : a.n_int + 1;
    for (int t = threadIdx.x; t < nc; t += blockDim.x) s_relc[t] = a.rel_c[t];
    for (int t = threadIdx.x; t < nx; t += blockDim.x) s_relx[t] = (a.n_int < 0) ? 0.0 : a.rel_x[t];
    __syncthreads();

    const int nq = NQ > 0 ? NQ : a.nq;
    double wsum = 0.0;
    for (int q = 0; q < nq; ++q) wsum += s_w[q];

    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.n_elems; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t eo = a.t_offset + e;
        const int4 cv = __ldg(reinterpret_cast<const int4 *>(a.cells) + e);
        const int cidx[4] = {cv.x, cv.y, cv.z, cv.w};
        // Jacobian J[k][l] = sum_i X[i][k] dphi[i][l]
        double Jm[9], Zn[4];
#pragma unroll
        for (int r = 0; r < 9; ++r) Jm[r] = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double X0 = __ldg(a.nodes + 3 * (int64_t)cidx[i]);
            const double X1 = __ldg(a.nodes + 3 * (int64_t)cidx[i] + 1);
            const double X2 = __ldg(a.nodes + 3 * (int64_t)cidx[i] + 2);
            Zn[i] = X2;
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                const double d = s_dphi[3 * i + l];
                Jm[0 + l] += X0 * d;
                Jm[3 + l] += X1 * d;
                Jm[6 + l] += X2 * d;
            }
        }
        const double det = Jm[0] * (Jm[4] * Jm[8] - Jm[7] * Jm[5]) - Jm[1] * (Jm[3] * Jm[8] - Jm[5] * Jm[6]) +
                           Jm[2] * (Jm[3] * Jm[7] - Jm[4] * Jm[6]);
        const double idet = 1.0 / det;
        const int o = __ldg(a.orient + e);
        const double *ct = s_ctab + o * 18;
        int g[6];
        {
            const int2 *gp = reinterpret_cast<const int2 *>(a.gids + 6 * e);
            int2 g01 = __ldg(gp), g23 = __ldg(gp + 1), g45 = __ldg(gp + 2);
            g[0] = g01.x; g[1] = g01.y; g[2] = g23.x; g[3] = g23.y; g[4] = g45.x; g[5] = g45.y;
        }
        double c[6][3], xv[6];
        double Bc[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const double h0 = ct[3 * j], h1 = ct[3 * j + 1], h2 = ct[3 * j + 2];
            c[j][0] = Jm[0] * h0 + Jm[1] * h1 + Jm[2] * h2;
            c[j][1] = Jm[3] * h0 + Jm[4] * h1 + Jm[5] * h2;
            c[j][2] = Jm[6] * h0 + Jm[7] * h1 + Jm[8] * h2;
            xv[j] = __ldg(a.x + g[j]);
            Bc[0] += c[j][0] * xv[j];
            Bc[1] += c[j][1] * xv[j];
            Bc[2] += c[j][2] * xv[j];
        }
        Bc[0] *= idet;
        Bc[1] *= idet;
        Bc[2] *= idet;

        double kfac;                 // sum_q nu_q w_q / det
        double Fj[6];
        const bool want_mat = (a.K != nullptr) | (a.dK != nullptr) | (a.J != nullptr) | (a.J32 != nullptr);
        const int32_t *sl = want_mat ? a.slots + 36 * e : nullptr;
        if constexpr (!HAS_BS) {
            const double bm = sqrt(Bc[0] * Bc[0] + Bc[1] * Bc[1] + Bc[2] * Bc[2]);
            double dnu;
            const double nu = pchip_eval<double>(a.n_int, s_relc, s_relx, bm, dnu);
            kfac = nu * wsum * idet;
            const double af = (bm >= 1e-14) ? dnu * wsum * idet / bm : 0.0;
            double p[6];
#pragma unroll
            for (int j = 0; j < 6; ++j) p[j] = c[j][0] * Bc[0] + c[j][1] * Bc[1] + c[j][2] * Bc[2];
#pragma unroll
            for (int j = 0; j < 6; ++j) Fj[j] = 0.0;
            int tri = 0;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
#pragma unroll
                for (int k = j; k < 6; ++k, ++tri) {
                    const double kv = kfac * (c[j][0] * c[k][0] + c[j][1] * c[k][1] + c[j][2] * c[k][2]);
                    const double dv = af * p[j] * p[k];
                    if (a.ET) store_pair(a, tri, eo, kv, dv);
                    const int s1 = want_mat ? __ldg(sl + j * 6 + k) : 0;
                    if (a.K) red_add(a.K + s1, kv);
                    if (a.dK) red_add(a.dK + s1, dv);
                    if (a.J) red_add(a.J + s1, kv + dv);
                    if (a.J32) red_add(a.J32 + s1, (float)(kv + dv));
                    Fj[j] += kv * xv[k];
                    if (k != j) {
                        const int s2 = want_mat ? __ldg(sl + k * 6 + j) : 0;
                        if (a.K) red_add(a.K + s2, kv);
                        if (a.dK) red_add(a.dK + s2, dv);
                        if (a.J) red_add(a.J + s2, kv + dv);
                        if (a.J32) red_add(a.J32 + s2, (float)(kv + dv));
                        Fj[k] += kv * xv[j];
                    }
                }
            }
            if (a.F) {
#pragma unroll
                for (int j = 0; j < 6; ++j) red_add(a.F + g[j], Fj[j]);
            }
            if (a.ET) store_vectors(a, eo, Fj, nullptr);
        } else {
            // one pass over the quadrature points: accumulate sum_q nu w, the reduced rhs
            // and the 21 dK pair sums (any number of points, fixed register footprint)
            double dk[21], r[6];
#pragma unroll
            for (int t = 0; t < 21; ++t) dk[t] = 0.0;
#pragma unroll
            for (int j = 0; j < 6; ++j) r[j] = 0.0;
            kfac = 0.0;
            const double *bs = a.Bs + (int64_t)e * nq * 3;
#pragma unroll(NQ > 0 ? NQ : 1)
            for (int q = 0; q < nq; ++q) {
                const double s0 = __ldg(bs + 3 * q), s1 = __ldg(bs + 3 * q + 1), s2 = __ldg(bs + 3 * q + 2);
                const double B0 = s0 + Bc[0], B1 = s1 + Bc[1], B2 = s2 + Bc[2];
                const double bm = sqrt(B0 * B0 + B1 * B1 + B2 * B2);
                double dnu;
                const double nu = nu_at<DIL>(a, s_relc, s_relx, s_phi + 4 * q, Zn, bm, dnu);
                const double wq = s_w[q];
                kfac += nu * wq;
                const double aq = (bm >= 1e-14) ? dnu * wq * idet / bm : 0.0;
                const double rq = (kNu0 - nu) * wq;
                double p[6];
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    p[j] = c[j][0] * B0 + c[j][1] * B1 + c[j][2] * B2;
                    r[j] += rq * (c[j][0] * s0 + c[j][1] * s1 + c[j][2] * s2);
                }
                int t = 0;
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    const double apj = aq * p[j];
#pragma unroll
                    for (int k = j; k < 6; ++k) dk[t++] += apj * p[k];
                }
            }
            kfac *= idet;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                if (a.rhs) red_add(a.rhs + g[j], r[j]);
                Fj[j] = -r[j];
            }
            int t = 0;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
#pragma unroll
                for (int k = j; k < 6; ++k) {
                    const double kv = kfac * (c[j][0] * c[k][0] + c[j][1] * c[k][1] + c[j][2] * c[k][2]);
                    if (a.ET) store_pair(a, t, eo, kv, dk[t]);
                    const double dv = dk[t++];
                    const int s1 = want_mat ? __ldg(sl + j * 6 + k) : 0;
                    if (a.K) red_add(a.K + s1, kv);
                    if (a.dK) red_add(a.dK + s1, dv);
                    if (a.J) red_add(a.J + s1, kv + dv);
                    if (a.J32) red_add(a.J32 + s1, (float)(kv + dv));
                    Fj[j] += kv * xv[k];
                    if (k != j) {
                        const int s2 = want_mat ? __ldg(sl + k * 6 + j) : 0;
                        if (a.K) red_add(a.K + s2, kv);
                        if (a.dK) red_add(a.dK + s2, dv);
                        if (a.J) red_add(a.J + s2, kv + dv);
                        if (a.J32) red_add(a.J32 + s2, (float)(kv + dv));
                        Fj[k] += kv * xv[j];
                    }
                }
            }
            if (a.F) {
#pragma unroll
                for (int j = 0; j < 6; ++j) red_add(a.F + g[j], Fj[j]);
            }
            if (a.ET) store_vectors(a, eo, Fj, r);
        }
    }
}

// Reduced rhs only (compute_rhs_Hcurl_red, fem_c/ctools.c:1390-1497).
__global__ void __launch_bounds__(kBlock)
    k_rhs_red(CurlArgs a, int quad_stride_ctab) {
    extern __shared__ double sm[];
    const SmemLayout L = smem_layout(a.n_orient, a.nq, a.n_int);
    double *s_ctab = sm + L.off_ctab;
    double *s_dphi = sm + L.off_dphi;
    double *s_w = sm + L.off_w;
    double *s_phi = sm + L.off_phi;
    double *s_relc = sm + L.off_relc;
    double *s_relx = sm + L.off_relx;
    for (int t = threadIdx.x; t < a.n_orient * 18; t += blockDim.x) {
        int o = t / 18, r = t - o * 18;
        s_ctab[t] = a.ctab[(int64_t)o * quad_stride_ctab + r];
    }
    for (int t = threadIdx.x; t < 12; t += blockDim.x) s_dphi[t] = a.dphi0[t];
    for (int t = threadIdx.x; t < a.nq; t += blockDim.x) s_w[t] = a.w[t];
    if (a.phi)
        for (int t = threadIdx.x; t < 4 * a.nq; t += blockDim.x) s_phi[t] = a.phi[t];
    const int nc = a.n_int < 0 ? 1 : 4 * a.n_int;
    const int nx = a.n_int < 0 ? 1 : a.n_int + 1;
    for (int t = threadIdx.x; t < nc; t += blockDim.x) s_relc[t] = a.rel_c[t];
    for (int t = threadIdx.x; t < nx; t += blockDim.x) s_relx[t] = (a.n_int < 0) ? 0.0 : a.rel_x[t];
    __syncthreads();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.n_elems; e += (int64_t)gridDim.x * blockDim.x) {
        const int4 cv = __ldg(reinterpret_cast<const int4 *>(a.cells) + e);
        const int cidx[4] = {cv.x, cv.y, cv.z, cv.w};
        double Jm[9];
        for (int r = 0; r < 9; ++r) Jm[r] = 0.0;
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 3; ++k) {
                const double X = __ldg(a.nodes + 3 * (int64_t)cidx[i] + k);
                for (int l = 0; l < 3; ++l) Jm[3 * k + l] += X * s_dphi[3 * i + l];
            }
        const double det = Jm[0] * (Jm[4] * Jm[8] - Jm[7] * Jm[5]) - Jm[1] * (Jm[3] * Jm[8] - Jm[5] * Jm[6]) +
                           Jm[2] * (Jm[3] * Jm[7] - Jm[4] * Jm[6]);
        const double idet = 1.0 / det;
        const double *ct = s_ctab + __ldg(a.orient + e) * 18;
        const int32_t *gp = a.gids + 6 * e;
        double c[6][3];
        double Bc[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 6; ++j) {
            for (int k = 0; k < 3; ++k) c[j][k] = Jm[3 * k] * ct[3 * j] + Jm[3 * k + 1] * ct[3 * j + 1] + Jm[3 * k + 2] * ct[3 * j + 2];
            const double xj = __ldg(a.x + __ldg(gp + j));
            for (int k = 0; k < 3; ++k) Bc[k] += c[j][k] * xj;
        }
        for (int k = 0; k < 3; ++k) Bc[k] *= idet;
        double r[6] = {0, 0, 0, 0, 0, 0};
        const double *bs = a.Bs + (int64_t)e * a.nq * 3;
        for (int q = 0; q < a.nq; ++q) {
            const double s0 = __ldg(bs + 3 * q), s1 = __ldg(bs + 3 * q + 1), s2 = __ldg(bs + 3 * q + 2);
            const double B0 = s0 + Bc[0], B1 = s1 + Bc[1], B2 = s2 + Bc[2];
            double dnu;
            const double nu = pchip_eval<double>(a.n_int, s_relc, s_relx, sqrt(B0 * B0 + B1 * B1 + B2 * B2), dnu);
            const double f = (kNu0 - nu) * s_w[q];
            for (int j = 0; j < 6; ++j) r[j] += f * (c[j][0] * s0 + c[j][1] * s1 + c[j][2] * s2);
        }
        for (int j = 0; j < 6; ++j) atomicAdd(a.rhs + __ldg(gp + j), r[j]);
    }
}

__global__ void k_check_affine(const double *curls, int n_orient, const double *dphi, int nq, int *bad) {
    const int64_t per_o = (int64_t)nq * 18;
    const int64_t total = (int64_t)n_orient * per_o + (int64_t)nq * 12;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        if (t < (int64_t)n_orient * per_o) {
            int64_t o = t / per_o, r = t - o * per_o;
            if (curls[o * per_o + r] != curls[o * per_o + (r % 18)]) atomicExch(bad, 1);
        } else {
            int64_t r = t - (int64_t)n_orient * per_o;
            if (dphi[r] != dphi[r % 12]) atomicExch(bad, 1);
        }
    }
}

// Element tensors for the matrix-free Newton Jacobian.  With affine elements every curl is
// c_j = Jm chat_j, so
//   J_e,jk = kfac (c_j . c_k) + sum_q a_q (c_j . B_q)(c_k . B_q) = chat_j . S_e chat_k,
//   S_e    = Jm^T (kfac I + sum_q a_q B_q B_q^T) Jm          (3x3 symmetric, 6 numbers)
// and the residual needs only the reference-frame curl bh = sum_j chat_j x_j:
//   (K x)_j = chat_j . (kfac Jm^T Jm bh),   rhs_j = chat_j . (Jm^T sum_q rq B_s,q).
// One pass over the quadrature points; S_e and the six element terms of F and of diag(J)
// are written once per element (no atomics; the DoF sums follow in a fixed order).
// What the element kernels of the Newton system share about one element e of a material:
// the map Jm, the reference-frame curl of the discrete field bh (Jm bh = det B_element) as
// cb = Jm bh, kfac = sum_q nu_q w_q / det, M = sum_q a_q B_q B_q^T with
// a_q = [|B_q| >= 1e-14] nu'_q w_q / (det |B_q|), Rs = sum_q (nu0 - nu_q) w_q B_s,q, and the
// element's reference curls ct (its orientation's table in shared memory).
struct ElemCore {
    double Jm[9], cb[3], kfac, M[6], Rs[3];
    const double *ct;
    int orient;
};

template <bool HAS_BS, int NQ, bool DIL>
__device__ __forceinline__ void elem_core(const CurlArgs &a, int64_t e, const double *s_ctab, const double *s_dphi,
                                          const double *s_w, const double *s_phi, const double *s_relc,
                                          const double *s_relx, double wsum, ElemCore &c) {
    const int nq = NQ > 0 ? NQ : a.nq;
    const int4 cv = __ldg(reinterpret_cast<const int4 *>(a.cells) + e);
    const int cidx[4] = {cv.x, cv.y, cv.z, cv.w};
    double *Jm = c.Jm;
    double Zn[4];
#pragma unroll
    for (int r = 0; r < 9; ++r) Jm[r] = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const double X0 = __ldg(a.nodes + 3 * (int64_t)cidx[i]);
        const double X1 = __ldg(a.nodes + 3 * (int64_t)cidx[i] + 1);
        const double X2 = __ldg(a.nodes + 3 * (int64_t)cidx[i] + 2);
        Zn[i] = X2;
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const double d = s_dphi[3 * i + l];
            Jm[0 + l] += X0 * d;
            Jm[3 + l] += X1 * d;
            Jm[6 + l] += X2 * d;
        }
    }
    const double det = Jm[0] * (Jm[4] * Jm[8] - Jm[7] * Jm[5]) - Jm[1] * (Jm[3] * Jm[8] - Jm[5] * Jm[6]) +
                       Jm[2] * (Jm[3] * Jm[7] - Jm[4] * Jm[6]);
    const double idet = 1.0 / det;
    c.orient = __ldg(a.orient + e);
    const double *ct = s_ctab + c.orient * 18;
    c.ct = ct;
    int g[6];
    {
        const int2 *gp = reinterpret_cast<const int2 *>(a.gids + 6 * e);
        int2 g01 = __ldg(gp), g23 = __ldg(gp + 1), g45 = __ldg(gp + 2);
        g[0] = g01.x; g[1] = g01.y; g[2] = g23.x; g[3] = g23.y; g[4] = g45.x; g[5] = g45.y;
    }
    // reference-frame curl of the discrete field and the element's own B
    double bh[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const double xj = __ldg(a.x + g[j]);
        bh[0] += ct[3 * j] * xj;
        bh[1] += ct[3 * j + 1] * xj;
        bh[2] += ct[3 * j + 2] * xj;
    }
    double *cb = c.cb;  // Jm bh = det * B_element
#pragma unroll
    for (int r = 0; r < 3; ++r) cb[r] = Jm[3 * r] * bh[0] + Jm[3 * r + 1] * bh[1] + Jm[3 * r + 2] * bh[2];
    const double Bc[3] = {cb[0] * idet, cb[1] * idet, cb[2] * idet};

    double *M = c.M, *Rs = c.Rs;
    Rs[0] = Rs[1] = Rs[2] = 0.0;
    if constexpr (!HAS_BS) {
        const double bm = sqrt(Bc[0] * Bc[0] + Bc[1] * Bc[1] + Bc[2] * Bc[2]);
        double dnu;
        const double nu = pchip_eval<double>(a.n_int, s_relc, s_relx, bm, dnu);
        c.kfac = nu * wsum * idet;
        const double af = (bm >= 1e-14) ? dnu * wsum * idet / bm : 0.0;
        M[0] = af * Bc[0] * Bc[0];
        M[1] = af * Bc[0] * Bc[1];
        M[2] = af * Bc[0] * Bc[2];
        M[3] = af * Bc[1] * Bc[1];
        M[4] = af * Bc[1] * Bc[2];
        M[5] = af * Bc[2] * Bc[2];
    } else {
        double kfac = 0.0;
#pragma unroll
        for (int t = 0; t < 6; ++t) M[t] = 0.0;
        const double *bs = a.Bs + (int64_t)e * nq * 3;
#pragma unroll(NQ > 0 ? NQ : 1)
        for (int q = 0; q < nq; ++q) {
            const double s0 = __ldg(bs + 3 * q), s1 = __ldg(bs + 3 * q + 1), s2 = __ldg(bs + 3 * q + 2);
            const double B0 = s0 + Bc[0], B1 = s1 + Bc[1], B2 = s2 + Bc[2];
            const double bm = sqrt(B0 * B0 + B1 * B1 + B2 * B2);
            double dnu;
            const double nu = nu_at<DIL>(a, s_relc, s_relx, s_phi + 4 * q, Zn, bm, dnu);
            const double wq = s_w[q];
            kfac += nu * wq;
            const double aq = (bm >= 1e-14) ? dnu * wq * idet / bm : 0.0;
            const double rq = (kNu0 - nu) * wq;
            M[0] += aq * B0 * B0;
            M[1] += aq * B0 * B1;
            M[2] += aq * B0 * B2;
            M[3] += aq * B1 * B1;
            M[4] += aq * B1 * B2;
            M[5] += aq * B2 * B2;
            Rs[0] += rq * s0;
            Rs[1] += rq * s1;
            Rs[2] += rq * s2;
        }
        c.kfac = kfac * idet;
    }
}

// Jm^T A Jm of a symmetric A (a: xx xy xz yy yz zz) into S (same order)
__device__ __forceinline__ void congruence(const double *Jm, const double (&A)[9], double (&S)[6]) {
    double P[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) P[3 * r + c] = A[3 * r] * Jm[c] + A[3 * r + 1] * Jm[3 + c] + A[3 * r + 2] * Jm[6 + c];
    int t = 0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = r; c < 3; ++c) S[t++] = Jm[r] * P[c] + Jm[3 + r] * P[3 + c] + Jm[6 + r] * P[6 + c];
}

// Element tensors of one element e of a material (the loop body of k_curlcurl_tensor): S_e into
// T and the six F and diag(J) terms into a.Fe / a.De, all at eslot(a.t_offset + e, .).  The
// tables sit in shared memory (s_*), wsum = sum of the weights.
template <bool HAS_BS, int NQ, typename TT, bool DIL>
__device__ __forceinline__ void tensor_element(const CurlArgs &a, int64_t e, const double *s_ctab,
                                               const double *s_dphi, const double *s_w, const double *s_phi,
                                               const double *s_relc, const double *s_relx, double wsum,
                                               TT *__restrict__ T) {
    ElemCore c;
    elem_core<HAS_BS, NQ, DIL>(a, e, s_ctab, s_dphi, s_w, s_phi, s_relc, s_relx, wsum, c);
    const double *Jm = c.Jm, *M = c.M, *cb = c.cb, *Rs = c.Rs, *ct = c.ct;
    const double kfac = c.kfac;
    // A = kfac I + M;  S = Jm^T A Jm
    const double A[9] = {kfac + M[0], M[1], M[2], M[1], kfac + M[3], M[4], M[2], M[4], kfac + M[5]};
    double S[6];
    congruence(Jm, A, S);
    const int64_t eb = eslot(a.t_offset + e, 0);
#pragma unroll
    for (int t = 0; t < 6; ++t) T[eb + 32 * t] = (TT)S[t];
    // G = kfac Jm^T (Jm bh) - Jm^T Rs;  F_j = chat_j . G
    double G[3];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
        G[cc] = kfac * (Jm[cc] * cb[0] + Jm[3 + cc] * cb[1] + Jm[6 + cc] * cb[2]) -
                (Jm[cc] * Rs[0] + Jm[3 + cc] * Rs[1] + Jm[6 + cc] * Rs[2]);
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const double h0 = ct[3 * j], h1 = ct[3 * j + 1], h2 = ct[3 * j + 2];
        const double sh0 = S[0] * h0 + S[1] * h1 + S[2] * h2;
        const double sh1 = S[1] * h0 + S[3] * h1 + S[4] * h2;
        const double sh2 = S[2] * h0 + S[4] * h1 + S[5] * h2;
        a.Fe[eb + 32 * j] = h0 * G[0] + h1 * G[1] + h2 * G[2];
        a.De[eb + 32 * j] = h0 * sh0 + h1 * sh1 + h2 * sh2;
    }
}

template <bool HAS_BS, int NQ, typename TT, bool DIL>
__global__ void __launch_bounds__(kBlock)
    k_curlcurl_tensor(CurlArgs a, int quad_stride_ctab, TT *__restrict__ T) {
    extern __shared__ double sm[];
    const SmemLayout L = smem_layout(a.n_orient, a.nq, a.n_int);
    double *s_ctab = sm + L.off_ctab;
    double *s_dphi = sm + L.off_dphi;
    double *s_w = sm + L.off_w;
    double *s_phi = sm + L.off_phi;
    double *s_relc = sm + L.off_relc;
    double *s_relx = sm + L.off_relx;
    for (int t = threadIdx.x; t < a.n_orient * 18; t += blockDim.x) {
        int o = t / 18, r = t - o * 18;
        s_ctab[t] = a.ctab[(int64_t)o * quad_stride_ctab + r];
    }
    for (int t = threadIdx.x; t < 12; t += blockDim.x) s_dphi[t] = a.dphi0[t];
    for (int t = threadIdx.x; t < a.nq; t += blockDim.x) s_w[t] = a.w[t];
    if (a.phi)
        for (int t = threadIdx.x; t < 4 * a.nq; t += blockDim.x) s_phi[t] = a.phi[t];
    const int nc = a.n_int < 0 ? 1 : 4 * a.n_int;
    const int nx = a.n_int < 0 ? 1 : a.n_int + 1;
    for (int t = threadIdx.x; t < nc; t += blockDim.x) s_relc[t] = a.rel_c[t];
    for (int t = threadIdx.x; t < nx; t += blockDim.x) s_relx[t] = (a.n_int < 0) ? 0.0 : a.rel_x[t];
    __syncthreads();

    const int nq = NQ > 0 ? NQ : a.nq;
    double wsum = 0.0;
    for (int q = 0; q < nq; ++q) wsum += s_w[q];

    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.n_elems; e += (int64_t)gridDim.x * blockDim.x)
        tensor_element<HAS_BS, NQ, TT, DIL>(a, e, s_ctab, s_dphi, s_w, s_phi, s_relc, s_relx, wsum, T);
}

// Batched element tensors: a grid of resident blocks walks the work items (runs of one
// segment's elements) of all problems; a block stages a segment's reluctance tables (and its
// nodal basis, diluted steel) in shared memory when its item changes segment.  Element e of an
// item is computed exactly as k_curlcurl_tensor computes it for the segment alone.
template <int NQ, typename TT>
__global__ void __launch_bounds__(kBlock)
    k_curlcurl_tensor_batch(const BatchSeg *__restrict__ segs, const BatchAsmItem *__restrict__ items, int n_items,
                            int max_n_int, const double *__restrict__ ctab, int n_orient, int quad_stride_ctab,
                            const double *__restrict__ dphi0, const double *__restrict__ w, int nq_rt,
                            const double *__restrict__ x, const int32_t *__restrict__ run, int run_stride,
                            TT *__restrict__ T, double *__restrict__ Fe, double *__restrict__ De) {
    extern __shared__ double sm[];
    const SmemLayout L = smem_layout(n_orient, nq_rt, max_n_int);
    double *s_ctab = sm + L.off_ctab;
    double *s_dphi = sm + L.off_dphi;
    double *s_w = sm + L.off_w;
    double *s_phi = sm + L.off_phi;
    double *s_relc = sm + L.off_relc;
    double *s_relx = sm + L.off_relx;
    for (int t = threadIdx.x; t < n_orient * 18; t += blockDim.x) {
        int o = t / 18, r = t - o * 18;
        s_ctab[t] = ctab[(int64_t)o * quad_stride_ctab + r];
    }
    for (int t = threadIdx.x; t < 12; t += blockDim.x) s_dphi[t] = dphi0[t];
    for (int t = threadIdx.x; t < nq_rt; t += blockDim.x) s_w[t] = w[t];
    __syncthreads();
    const int nq = NQ > 0 ? NQ : nq_rt;
    double wsum = 0.0;
    for (int q = 0; q < nq; ++q) wsum += s_w[q];
    int cur = -1;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const BatchAsmItem item = items[it];
        if (!run[(int64_t)item.inst * run_stride]) continue;  // uniform across the block
        CurlArgs a = segs[item.seg].a;
        if (item.seg != cur) {
            __syncthreads();
            const int nc = a.n_int < 0 ? 1 : 4 * a.n_int;
            const int nx = a.n_int < 0 ? 1 : a.n_int + 1;
            for (int t = threadIdx.x; t < nc; t += blockDim.x) s_relc[t] = a.rel_c[t];
            for (int t = threadIdx.x; t < nx; t += blockDim.x) s_relx[t] = (a.n_int < 0) ? 0.0 : a.rel_x[t];
            if (a.phi)
                for (int t = threadIdx.x; t < 4 * nq; t += blockDim.x) s_phi[t] = a.phi[t];
            __syncthreads();
            cur = item.seg;
        }
        a.x = x + segs[item.seg].dof_off;
        a.Fe = Fe;
        a.De = De;
        for (int64_t e = item.e0 + threadIdx.x; e < item.e1; e += blockDim.x) {
            if (a.Bs == nullptr)
                tensor_element<false, NQ, TT, false>(a, e, s_ctab, s_dphi, s_w, s_phi, s_relc, s_relx, wsum, T);
            else if (a.phi)
                tensor_element<true, NQ, TT, true>(a, e, s_ctab, s_dphi, s_w, s_phi, s_relc, s_relx, wsum, T);
            else
                tensor_element<true, NQ, TT, false>(a, e, s_ctab, s_dphi, s_w, s_phi, s_relc, s_relx, wsum, T);
        }
    }
}

template <bool HAS_BS, int NQ, typename TT, bool DIL = false>
int launch_tensor_t(const CurlArgs &a, TT *T, cudaStream_t st, size_t smem, int qstride) {
    if (a.n_elems == 0) return SNP_OK;
    auto kern = k_curlcurl_tensor<HAS_BS, NQ, TT, DIL>;
    if (smem > 48 * 1024) SNP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<wave_grid(kern, a.n_elems, kBlock, smem), kBlock, smem, st>>>(a, qstride, T);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

template <typename TT>
int launch_tensor(const CurlArgs &a, TT *T, cudaStream_t st, size_t smem, int qstride) {
    if (a.Bs == nullptr) {
        if (a.nq == 1) return launch_tensor_t<false, 1, TT>(a, T, st, smem, qstride);
        if (a.nq == 4) return launch_tensor_t<false, 4, TT>(a, T, st, smem, qstride);
        return launch_tensor_t<false, 0, TT>(a, T, st, smem, qstride);
    }
    if (a.phi) {
        if (a.nq == 4) return launch_tensor_t<true, 4, TT, true>(a, T, st, smem, qstride);
        return launch_tensor_t<true, 0, TT, true>(a, T, st, smem, qstride);
    }
    if (a.nq == 1) return launch_tensor_t<true, 1, TT>(a, T, st, smem, qstride);
    if (a.nq == 4) return launch_tensor_t<true, 4, TT>(a, T, st, smem, qstride);
    if (a.nq == 5) return launch_tensor_t<true, 5, TT>(a, T, st, smem, qstride);
    return launch_tensor_t<true, 0, TT>(a, T, st, smem, qstride);
}

template <bool HAS_BS, int NQ, bool DIL = false>
int launch_t(const CurlArgs &a, cudaStream_t st, size_t smem, int qstride) {
    if (a.n_elems == 0) return SNP_OK;
    auto kern = k_curlcurl<HAS_BS, NQ, double, DIL>;
    if (smem > 48 * 1024) SNP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = stride_grid(a.n_elems, kBlock, 16);
    kern<<<grid, kBlock, smem, st>>>(a, qstride);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

}  // namespace

int check_affine_tables(const double *curls, int32_t n_orient, const double *d_phi, int32_t nq, cudaStream_t st,
                        bool *affine) {
    DevBuf<int> bad;
    SNP_TRY(bad.alloc(1));
    SNP_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    k_check_affine<<<64, 256, 0, st>>>(curls, n_orient, d_phi, nq, bad.p);
    SNP_LAUNCH_CHECK();
    int h = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SNP_CUDA_TRY(cudaStreamSynchronize(st));
    *affine = (h == 0);
    return SNP_OK;
}

int launch_curlcurl(const CurlArgs &a, cudaStream_t st) {
    const SmemLayout L = smem_layout(a.n_orient, a.nq, a.n_int);
    const size_t smem = sizeof(double) * (size_t)L.total;
    SNP_REQUIRE(smem <= 200 * 1024, "curl-curl assembly: tables need %zu bytes of shared memory (max 200 KiB)", smem);
    const int qstride = a.nq * 18;
    if (a.Bs == nullptr) {
        if (a.nq == 1) return launch_t<false, 1>(a, st, smem, qstride);
        if (a.nq == 4) return launch_t<false, 4>(a, st, smem, qstride);
        return launch_t<false, 0>(a, st, smem, qstride);
    }
    if (a.phi) {
        if (a.nq == 4) return launch_t<true, 4, true>(a, st, smem, qstride);
        return launch_t<true, 0, true>(a, st, smem, qstride);
    }
    if (a.nq == 1) return launch_t<true, 1>(a, st, smem, qstride);
    if (a.nq == 4) return launch_t<true, 4>(a, st, smem, qstride);
    if (a.nq == 5) return launch_t<true, 5>(a, st, smem, qstride);
    return launch_t<true, 0>(a, st, smem, qstride);
}

int launch_curlcurl_tensor(const CurlArgs &a, cudaStream_t st) {
    SNP_REQUIRE((a.T64 == nullptr) != (a.T32 == nullptr), "element tensors: exactly one of T64/T32 must be set");
    SNP_REQUIRE(a.Fe != nullptr && a.De != nullptr, "element tensors: Fe and De are required");
    const SmemLayout L = smem_layout(a.n_orient, a.nq, a.n_int);
    const size_t smem = sizeof(double) * (size_t)L.total;
    SNP_REQUIRE(smem <= 200 * 1024, "curl-curl assembly: tables need %zu bytes of shared memory (max 200 KiB)", smem);
    const int qstride = a.nq * 18;
    if (a.T64) return launch_tensor<double>(a, a.T64, st, smem, qstride);
    return launch_tensor<float>(a, a.T32, st, smem, qstride);
}

TermLayout term_layout(int parts) {
    TermLayout L;
    int o = 0;
    if (parts & SNP_TERMS_K) { L.k = o; o += 21; }
    if (parts & SNP_TERMS_DK) { L.d = o; o += 21; }
    if (parts & SNP_TERMS_J) { L.j = o; o += 21; }
    if (parts & SNP_TERMS_F) { L.f = o; o += 6; }
    if (parts & SNP_TERMS_RHS) { L.r = o; o += 6; }
    L.stride = o;
    return L;
}

int launch_curlcurl_terms(const CurlArgs &a0, const TermLayout &L, double *terms, int64_t n_elems, cudaStream_t st) {
    SNP_REQUIRE(terms != nullptr || a0.n_elems == 0 || L.stride == 0, "element matrices: terms is NULL");
    CurlArgs a = a0;
    a.K = a.dK = a.J = nullptr;
    a.J32 = nullptr;
    a.rhs = a.F = nullptr;
    a.slots = nullptr;
    a.ET = terms;
    a.et_stride = n_elems;
    a.et_k = L.k;
    a.et_d = L.d;
    a.et_j = L.j;
    a.et_f = L.f;
    a.et_r = L.r;
    if (L.stride == 0) return SNP_OK;
    return launch_curlcurl(a, st);
}

template <int NQ, typename TT>
static int launch_batch_t(const BatchSeg *segs, const BatchAsmItem *items, int n_items, int max_n_int,
                          const double *ctab, int n_orient, int qstride, const double *dphi0, const double *w, int nq,
                          const double *x, const int32_t *run, int run_stride, TT *T, double *Fe, double *De, int grid,
                          size_t smem, cudaStream_t st) {
    auto kern = k_curlcurl_tensor_batch<NQ, TT>;
    if (smem > 48 * 1024) SNP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (grid <= 0) grid = wave_grid(kern, (int64_t)n_items * kBlock, kBlock, smem);
    kern<<<grid, kBlock, smem, st>>>(segs, items, n_items, max_n_int, ctab, n_orient, qstride, dphi0, w, nq, x, run,
                                     run_stride, T, Fe, De);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int launch_curlcurl_tensor_batch(const BatchSeg *segs, const BatchAsmItem *items, int n_items, int max_n_int,
                                 const double *ctab, int n_orient, int quad_stride_ctab, const double *dphi0,
                                 const double *w, int nq, const double *x, const int32_t *run, int run_stride, void *T,
                                 bool f32, double *Fe, double *De, int grid, cudaStream_t st) {
    static_assert(kBatchAsmBlock == kBlock, "batched assembly block size");
    if (n_items == 0) return SNP_OK;
    const SmemLayout L = smem_layout(n_orient, nq, max_n_int);
    const size_t smem = sizeof(double) * (size_t)L.total;
    SNP_REQUIRE(smem <= 200 * 1024, "batched assembly: tables need %zu bytes of shared memory", smem);
    if (f32) {
        if (nq == 4)
            return launch_batch_t<4, float>(segs, items, n_items, max_n_int, ctab, n_orient, quad_stride_ctab, dphi0,
                                            w, nq, x, run, run_stride, static_cast<float *>(T), Fe, De, grid, smem, st);
        return launch_batch_t<0, float>(segs, items, n_items, max_n_int, ctab, n_orient, quad_stride_ctab, dphi0, w,
                                        nq, x, run, run_stride, static_cast<float *>(T), Fe, De, grid, smem, st);
    }
    if (nq == 4)
        return launch_batch_t<4, double>(segs, items, n_items, max_n_int, ctab, n_orient, quad_stride_ctab, dphi0, w,
                                         nq, x, run, run_stride, static_cast<double *>(T), Fe, De, grid, smem, st);
    return launch_batch_t<0, double>(segs, items, n_items, max_n_int, ctab, n_orient, quad_stride_ctab, dphi0, w, nq,
                                     x, run, run_stride, static_cast<double *>(T), Fe, De, grid, smem, st);
}

int fill_args(CurlArgs &a, const snp_pattern *pat, int64_t elem_offset, int64_t n_elems, const double *nodes,
                     const int32_t *cells, const int32_t *glob_ids, const int32_t *orientations, const double *curls,
                     int32_t n_orient, const double *d_phi, const double *w, int32_t n_quad, const double *x,
                     const double *B_s, int32_t n_int, const double *rel_c, const double *rel_x) {
    SNP_REQUIRE(n_elems >= 0, "negative element count");
    SNP_REQUIRE(n_quad >= 1, "n_quad must be >= 1");
    SNP_REQUIRE(n_orient >= 1, "n_orient must be >= 1");
    SNP_REQUIRE(n_int == -1 || n_int >= 1, "n_int must be -1 (constant) or >= 1");
    SNP_REQUIRE(rel_c != nullptr && (n_int < 0 || rel_x != nullptr), "reluctance tables are NULL");
    SNP_REQUIRE(n_elems == 0 || (nodes && cells && glob_ids && orientations && curls && d_phi && w && x),
                "a required input pointer is NULL");
    SNP_REQUIRE(((uintptr_t)cells & 15) == 0, "cells must be 16-byte aligned");
    SNP_REQUIRE(((uintptr_t)glob_ids & 7) == 0, "glob_ids must be 8-byte aligned");
    if (pat) {
        SNP_REQUIRE(pat->dpe == 6, "pattern was not built for 6 DoFs per element");
        SNP_REQUIRE(elem_offset >= 0 && elem_offset + n_elems <= pat->n_elems,
                    "element range [%lld, %lld) outside the pattern's %lld elements", (long long)elem_offset,
                    (long long)(elem_offset + n_elems), (long long)pat->n_elems);
    }
    a = CurlArgs{};
    a.n_elems = n_elems;
    a.nodes = nodes;
    a.cells = cells;
    a.gids = glob_ids;
    a.orient = orientations;
    a.ctab = curls;
    a.n_orient = n_orient;
    a.dphi0 = d_phi;
    a.w = w;
    a.nq = n_quad;
    a.x = x;
    a.Bs = B_s;
    a.n_int = n_int;
    a.rel_c = rel_c;
    a.rel_x = rel_x;
    a.slots = pat ? pat->slots.p + 36 * elem_offset : nullptr;
    return SNP_OK;
}

}  // namespace snp

extern "C" {

int snp_curlcurl_assemble(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems, const double *nodes,
                          const int32_t *cells, const int32_t *glob_ids, const int32_t *orientations,
                          const double *curls, int32_t n_orient, const double *d_phi, const double *w,
                          int32_t n_quad, const double *x, const double *B_s, int32_t n_int, const double *rel_c,
                          const double *rel_x, double *K_vals, double *dK_vals, double *J_vals, double *rhs,
                          double *F, void *stream) {
    snp::clear_error();
    const bool want_mat = K_vals || dK_vals || J_vals;
    SNP_REQUIRE(!want_mat || pat != nullptr, "snp_curlcurl_assemble: matrix outputs need a pattern");
    snp::CurlArgs a;
    SNP_TRY(snp::fill_args(a, pat, elem_offset, n_elems, nodes, cells, glob_ids, orientations, curls, n_orient, d_phi,
                           w, n_quad, x, B_s, n_int, rel_c, rel_x));
    a.K = K_vals;
    a.dK = dK_vals;
    a.J = J_vals;
    a.rhs = rhs;
    a.F = F;
    return snp::launch_curlcurl(a, snp::as_stream(stream));
}

int snp_curlcurl_assemble_diluted(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems, const double *nodes,
                                  const int32_t *cells, const int32_t *glob_ids, const int32_t *orientations,
                                  const double *curls, int32_t n_orient, const double *phi, const double *d_phi,
                                  const double *w, int32_t n_quad, const double *x, const double *B_s, int32_t n_int,
                                  const double *rel_c, const double *rel_x, const double *dilution, double *K_vals,
                                  double *dK_vals, double *J_vals, double *rhs, double *F, void *stream) {
    snp::clear_error();
    const bool want_mat = K_vals || dK_vals || J_vals;
    SNP_REQUIRE(!want_mat || pat != nullptr, "snp_curlcurl_assemble_diluted: matrix outputs need a pattern");
    snp::CurlArgs a;
    SNP_TRY(snp::fill_args(a, pat, elem_offset, n_elems, nodes, cells, glob_ids, orientations, curls, n_orient, d_phi,
                           w, n_quad, x, B_s, n_int, rel_c, rel_x));
    if (B_s != nullptr) {
        SNP_REQUIRE(phi != nullptr && dilution != nullptr, "snp_curlcurl_assemble_diluted: phi and dilution are required");
        a.phi = phi;
        for (int i = 0; i < 4; ++i) a.dil[i] = dilution[i];
    }
    a.K = K_vals;
    a.dK = dK_vals;
    a.J = J_vals;
    a.rhs = rhs;
    a.F = F;
    return snp::launch_curlcurl(a, snp::as_stream(stream));
}

int snp_curlcurl_assemble_f32(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems, const double *nodes,
                              const int32_t *cells, const int32_t *glob_ids, const int32_t *orientations,
                              const double *curls, int32_t n_orient, const double *d_phi, const double *w,
                              int32_t n_quad, const double *x, const double *B_s, int32_t n_int, const double *rel_c,
                              const double *rel_x, float *J_vals, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(pat != nullptr, "snp_curlcurl_assemble_f32: pattern is NULL");
    snp::CurlArgs a;
    SNP_TRY(snp::fill_args(a, pat, elem_offset, n_elems, nodes, cells, glob_ids, orientations, curls, n_orient, d_phi,
                           w, n_quad, x, B_s, n_int, rel_c, rel_x));
    a.J32 = J_vals;
    return snp::launch_curlcurl(a, snp::as_stream(stream));
}

int snp_curlcurl_rhs_red(int64_t n_elems, const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                         const int32_t *orientations, const double *curls, int32_t n_orient, const double *d_phi,
                         const double *w, int32_t n_quad, const double *x, const double *B_s, int32_t n_int,
                         const double *rel_c, const double *rel_x, double *rhs, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(rhs != nullptr && (n_elems == 0 || B_s != nullptr), "snp_curlcurl_rhs_red: rhs and B_s are required");
    snp::CurlArgs a;
    SNP_TRY(snp::fill_args(a, nullptr, 0, n_elems, nodes, cells, glob_ids, orientations, curls, n_orient, d_phi, w,
                           n_quad, x, B_s, n_int, rel_c, rel_x));
    a.rhs = rhs;
    if (n_elems == 0) return SNP_OK;
    const snp::SmemLayout L = snp::smem_layout(a.n_orient, a.nq, a.n_int);
    const size_t smem = sizeof(double) * (size_t)L.total;
    SNP_REQUIRE(smem <= 200 * 1024, "tables too large for shared memory");
    if (smem > 48 * 1024)
        SNP_CUDA_TRY(cudaFuncSetAttribute(snp::k_rhs_red, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    snp::k_rhs_red<<<snp::stride_grid(n_elems, snp::kBlock, 16), snp::kBlock, smem, snp::as_stream(stream)>>>(
        a, a.nq * 18);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

}  // extern "C"
