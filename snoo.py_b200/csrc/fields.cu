// Field evaluation: B at quadrature points (compute_B_Hcurl, fem_c/ctools.c:1500-1563),
// physical quadrature points (curl_curl_assembler.py:1521-1593), B at located probe
// points, and Biot-Savart of filament segments (compute_B_line_segs, ctools.c:1761-1923).
#include "snp_common.cuh"
#include "snp_internal.cuh"

namespace snp {
namespace {

// One thread per (element, quadrature point); general tables (per-point d_phi and curls).
__global__ void k_b_hcurl(int64_t n_elems, int nq, const double *__restrict__ nodes, const int32_t *__restrict__ cells,
                          const int32_t *__restrict__ gids, const int32_t *__restrict__ orient,
                          const double *__restrict__ curls, const double *__restrict__ phi,
                          const double *__restrict__ dphi, const double *__restrict__ x, double *__restrict__ points,
                          double *__restrict__ B) {
    const int64_t total = n_elems * nq;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / nq;
        const int q = (int)(t - e * nq);
        double X[4][3];
        for (int i = 0; i < 4; ++i) {
            const int n = cells[4 * e + i];
            for (int k = 0; k < 3; ++k) X[i][k] = nodes[3 * (int64_t)n + k];
        }
        double Jm[9];
        for (int r = 0; r < 9; ++r) Jm[r] = 0.0;
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) Jm[3 * k + l] += X[i][k] * dphi[12 * q + 3 * i + l];
        const double det = Jm[0] * (Jm[4] * Jm[8] - Jm[7] * Jm[5]) - Jm[1] * (Jm[3] * Jm[8] - Jm[5] * Jm[6]) +
                           Jm[2] * (Jm[3] * Jm[7] - Jm[4] * Jm[6]);
        double p[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 3; ++k) p[k] += phi[4 * q + i] * X[i][k];
        const double *ct = curls + ((int64_t)orient[e] * nq + q) * 18;
        double b[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 6; ++j) {
            const double xj = x[gids[6 * e + j]];
            for (int k = 0; k < 3; ++k)
                b[k] += (Jm[3 * k] * ct[3 * j] + Jm[3 * k + 1] * ct[3 * j + 1] + Jm[3 * k + 2] * ct[3 * j + 2]) * xj / det;
        }
        for (int k = 0; k < 3; ++k) {
            if (points) points[3 * t + k] = p[k];
            if (B) B[3 * t + k] = b[k];
        }
    }
}

__global__ void k_quad_points(int64_t n_elems, int nq, const double *__restrict__ nodes,
                              const int32_t *__restrict__ cells, const double *__restrict__ phi,
                              double *__restrict__ points) {
    const int64_t total = n_elems * nq;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / nq;
        const int q = (int)(t - e * nq);
        double p[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 4; ++i) {
            const int n = cells[4 * e + i];
            const double f = phi[4 * q + i];
            for (int k = 0; k < 3; ++k) p[k] += f * nodes[3 * (int64_t)n + k];
        }
        for (int k = 0; k < 3; ++k) points[3 * t + k] = p[k];
    }
}

__global__ void k_b_at_elements(int64_t n_pts, const int32_t *__restrict__ elem, const double *__restrict__ nodes,
                                const int32_t *__restrict__ cells, const int32_t *__restrict__ gids,
                                const int32_t *__restrict__ orient, const double *__restrict__ curls, int nq,
                                const double *__restrict__ dphi, const double *__restrict__ x, double *__restrict__ B) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_pts; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = elem[t];
        double b[3] = {0.0, 0.0, 0.0};
        if (e >= 0) {
            double Jm[9];
            for (int r = 0; r < 9; ++r) Jm[r] = 0.0;
            for (int i = 0; i < 4; ++i) {
                const int n = cells[4 * e + i];
                for (int k = 0; k < 3; ++k)
                    for (int l = 0; l < 3; ++l) Jm[3 * k + l] += nodes[3 * (int64_t)n + k] * dphi[3 * i + l];
            }
            const double det = Jm[0] * (Jm[4] * Jm[8] - Jm[7] * Jm[5]) - Jm[1] * (Jm[3] * Jm[8] - Jm[5] * Jm[6]) +
                               Jm[2] * (Jm[3] * Jm[7] - Jm[4] * Jm[6]);
            const double *ct = curls + (int64_t)orient[e] * nq * 18;
            for (int j = 0; j < 6; ++j) {
                const double xj = x[gids[6 * e + j]];
                for (int k = 0; k < 3; ++k)
                    b[k] += (Jm[3 * k] * ct[3 * j] + Jm[3 * k + 1] * ct[3 * j + 1] + Jm[3 * k + 2] * ct[3 * j + 2]) * xj / det;
            }
        }
        for (int k = 0; k < 3; ++k) B[3 * t + k] = b[k];
    }
}


// rhs of the total-potential formulation from a nodal electric potential:
// rhs[g_k] += sum_q (Jm^-T w_hat_k(q)) . (Jm^-T sum_i dphi_i(q) phi_i) w_q det
// (CurlCurlAssembler.compute_rhs_electric_potential, snoopy/curl_curl_assembler.py:1154-1284).
__global__ void k_rhs_grad_potential(int64_t n_elems, int nq, const double *__restrict__ nodes,
                                     const int32_t *__restrict__ cells, const int32_t *__restrict__ gids,
                                     const int32_t *__restrict__ orient, const double *__restrict__ basis,
                                     const double *__restrict__ dphi, const double *__restrict__ w,
                                     const double *__restrict__ xp, double *__restrict__ rhs) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_elems; e += (int64_t)gridDim.x * blockDim.x) {
        double X[4][3], xv[4];
        for (int i = 0; i < 4; ++i) {
            const int n = cells[4 * e + i];
            for (int k = 0; k < 3; ++k) X[i][k] = nodes[3 * (int64_t)n + k];
            xv[i] = xp[n];
        }
        const double *bt = basis + (int64_t)orient[e] * nq * 18;
        double r[6] = {0, 0, 0, 0, 0, 0};
        for (int q = 0; q < nq; ++q) {
            double Jm[9];
            for (int t = 0; t < 9; ++t) Jm[t] = 0.0;
            double gr[3] = {0.0, 0.0, 0.0};
            for (int i = 0; i < 4; ++i)
                for (int l = 0; l < 3; ++l) {
                    const double d = dphi[12 * q + 3 * i + l];
                    for (int k = 0; k < 3; ++k) Jm[3 * k + l] += X[i][k] * d;
                    gr[l] += d * xv[i];
                }
            const double det = Jm[0] * (Jm[4] * Jm[8] - Jm[7] * Jm[5]) - Jm[1] * (Jm[3] * Jm[8] - Jm[5] * Jm[6]) +
                               Jm[2] * (Jm[3] * Jm[7] - Jm[4] * Jm[6]);
            const double id = 1.0 / det;
            double Ji[9];
            Ji[0] = (Jm[4] * Jm[8] - Jm[7] * Jm[5]) * id;
            Ji[1] = (Jm[2] * Jm[7] - Jm[1] * Jm[8]) * id;
            Ji[2] = (Jm[1] * Jm[5] - Jm[2] * Jm[4]) * id;
            Ji[3] = (Jm[5] * Jm[6] - Jm[3] * Jm[8]) * id;
            Ji[4] = (Jm[0] * Jm[8] - Jm[2] * Jm[6]) * id;
            Ji[5] = (Jm[3] * Jm[2] - Jm[0] * Jm[5]) * id;
            Ji[6] = (Jm[3] * Jm[7] - Jm[6] * Jm[4]) * id;
            Ji[7] = (Jm[6] * Jm[1] - Jm[0] * Jm[7]) * id;
            Ji[8] = (Jm[0] * Jm[4] - Jm[3] * Jm[1]) * id;
            double G[3];
            for (int k = 0; k < 3; ++k) G[k] = Ji[k] * gr[0] + Ji[3 + k] * gr[1] + Ji[6 + k] * gr[2];
            const double f = w[q] * det;
            for (int j = 0; j < 6; ++j) {
                const double *wh = bt + 18 * q + 3 * j;
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += (Ji[k] * wh[0] + Ji[3 + k] * wh[1] + Ji[6 + k] * wh[2]) * G[k];
                r[j] += s * f;
            }
        }
        for (int j = 0; j < 6; ++j) atomicAdd(rhs + gids[6 * e + j], r[j]);
    }
}

constexpr int kBsBlock = 128;

// One thread per target; source segments staged through shared memory in tiles.
// Sources are summed in their input order, as the reference does per target.
__global__ void __launch_bounds__(kBsBlock)
    k_biot_savart(const double *__restrict__ src, int64_t n_src, const double *__restrict__ tar, int64_t n_tar,
                  double current, double rad, double *__restrict__ B) {
    __shared__ double s[kBsBlock * 7];  // per segment: start, end, 1 / |end - start|^2
    const double rad2 = rad * rad;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n_tar; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const bool active = i < n_tar;
        double px = 0.0, py = 0.0, pz = 0.0;
        if (active) {
            px = tar[3 * i];
            py = tar[3 * i + 1];
            pz = tar[3 * i + 2];
        }
        double bx = 0.0, by = 0.0, bz = 0.0;
        for (int64_t j0 = 0; j0 < n_src; j0 += kBsBlock) {
            const int m = (int)((n_src - j0) < kBsBlock ? (n_src - j0) : kBsBlock);
            __syncthreads();
            for (int t = threadIdx.x; t < m * 6; t += blockDim.x) s[(t / 6) * 7 + t % 6] = src[6 * j0 + t];
            __syncthreads();
            for (int t = threadIdx.x; t < m; t += blockDim.x) {
                const double *sg = s + 7 * t;
                const double n0 = sg[3] - sg[0], n1 = sg[4] - sg[1], n2 = sg[5] - sg[2];
                s[7 * t + 6] = 1.0 / (n0 * n0 + n1 * n1 + n2 * n2);
            }
            __syncthreads();
            if (active) {
                for (int jj = 0; jj < m; ++jj) {
                    const double *sg = s + 7 * jj;
                    const double n0 = sg[3] - sg[0], n1 = sg[4] - sg[1], n2 = sg[5] - sg[2];
                    const double d10 = sg[0] - px, d11 = sg[1] - py, d12 = sg[2] - pz;
                    const double d20 = sg[3] - px, d21 = sg[4] - py, d22 = sg[5] - pz;
                    const double nd1 = sqrt(d10 * d10 + d11 * d11 + d12 * d12);
                    const double nd2 = sqrt(d20 * d20 + d21 * d21 + d22 * d22);
                    const double tp = -1.0 * (d10 * n0 + d11 * n1 + d12 * n2) * sg[6];
                    const double p0 = px - (sg[0] + tp * n0), p1 = py - (sg[1] + tp * n1), p2 = pz - (sg[2] + tp * n2);
                    const double dmin2 = p0 * p0 + p1 * p1 + p2 * p2;
                    if ((dmin2 < rad2 && tp <= 1.0 && tp >= 0.0) || nd1 < rad || nd2 < rad) {
                        const double b0 = n1 * p2 - n2 * p1, b1 = n2 * p0 - n0 * p2, b2 = n0 * p1 - n1 * p0;
                        const double nb = sqrt(b0 * b0 + b1 * b1 + b2 * b2);
                        const double f = 2.0 * sqrt(dmin2) / rad / rad / nb;
                        bx += b0 * f;
                        by += b1 * f;
                        bz += b2 * f;
                    } else {
                        // (|d1| + |d2|) / (|d1| |d2| + d1.d2) / |d1| / |d2|, with one division
                        const double dd = d10 * d20 + d11 * d21 + d12 * d22;
                        const double pr = nd1 * nd2;
                        const double f = (nd1 + nd2) / ((pr + dd) * pr);
                        bx += (d11 * d22 - d12 * d21) * f;
                        by += (d12 * d20 - d10 * d22) * f;
                        bz += (d10 * d21 - d11 * d20) * f;
                    }
                }
            }
        }
        if (active) {
            B[3 * i] = bx * current * 1e-7;
            B[3 * i + 1] = by * current * 1e-7;
            B[3 * i + 2] = bz * current * 1e-7;
        }
    }
}

}  // namespace
}  // namespace snp

extern "C" {

int snp_b_hcurl(int64_t n_elems, const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                const int32_t *orientations, const double *curls, int32_t n_orient, const double *phi,
                const double *d_phi, int32_t n_quad, const double *x, double *points, double *B, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_elems >= 0 && n_quad >= 1 && n_orient >= 1, "snp_b_hcurl: bad sizes");
    if (n_elems == 0) return SNP_OK;
    SNP_REQUIRE(nodes && cells && glob_ids && orientations && curls && phi && d_phi && x && (points || B),
                "snp_b_hcurl: NULL argument");
    snp::k_b_hcurl<<<snp::stride_grid(n_elems * n_quad, 128, 16), 128, 0, snp::as_stream(stream)>>>(
        n_elems, n_quad, nodes, cells, glob_ids, orientations, curls, phi, d_phi, x, points, B);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_quad_points(int64_t n_elems, const double *nodes, const int32_t *cells, const double *phi, int32_t n_quad,
                    double *points, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_elems >= 0 && n_quad >= 1, "snp_quad_points: bad sizes");
    if (n_elems == 0) return SNP_OK;
    SNP_REQUIRE(nodes && cells && phi && points, "snp_quad_points: NULL argument");
    snp::k_quad_points<<<snp::stride_grid(n_elems * n_quad, 256, 16), 256, 0, snp::as_stream(stream)>>>(
        n_elems, n_quad, nodes, cells, phi, points);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_b_at_elements(int64_t n_points, const int32_t *elem, const double *nodes, const int32_t *cells,
                      const int32_t *glob_ids, const int32_t *orientations, const double *curls, int32_t n_orient,
                      const double *d_phi, int32_t n_quad, const double *x, double *B, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_points >= 0 && n_quad >= 1 && n_orient >= 1, "snp_b_at_elements: bad sizes");
    if (n_points == 0) return SNP_OK;
    SNP_REQUIRE(elem && nodes && cells && glob_ids && orientations && curls && d_phi && x && B,
                "snp_b_at_elements: NULL argument");
    snp::k_b_at_elements<<<snp::stride_grid(n_points, 128, 8), 128, 0, snp::as_stream(stream)>>>(
        n_points, elem, nodes, cells, glob_ids, orientations, curls, n_quad, d_phi, x, B);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_rhs_grad_potential(int64_t n_elems, const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                           const int32_t *orientations, const double *basis, int32_t n_orient, const double *d_phi,
                           const double *w, int32_t n_quad, const double *x_p, double *rhs, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_elems >= 0 && n_quad >= 1 && n_orient >= 1, "snp_rhs_grad_potential: bad sizes");
    if (n_elems == 0) return SNP_OK;
    SNP_REQUIRE(nodes && cells && glob_ids && orientations && basis && d_phi && w && x_p && rhs,
                "snp_rhs_grad_potential: NULL argument");
    snp::k_rhs_grad_potential<<<snp::stride_grid(n_elems, 128, 16), 128, 0, snp::as_stream(stream)>>>(
        n_elems, n_quad, nodes, cells, glob_ids, orientations, basis, d_phi, w, x_p, rhs);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int snp_biot_savart(const double *src, int64_t n_src, const double *tar, int64_t n_tar, double current, double radius,
                    double *B, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_src >= 0 && n_tar >= 0, "snp_biot_savart: negative sizes");
    if (n_tar == 0) return SNP_OK;
    SNP_REQUIRE(tar && B && (n_src == 0 || src), "snp_biot_savart: NULL argument");
    snp::k_biot_savart<<<snp::stride_grid(n_tar, snp::kBsBlock, 8), snp::kBsBlock, 0, snp::as_stream(stream)>>>(
        src, n_src, tar, n_tar, current, radius, B);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

}  // extern "C"
