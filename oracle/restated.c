/*
 * CPU oracle: a plain-C restatement of snoo.py's element kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load this file's library, and only as the checker.  The
 * product path (snoo.py_b200/csrc) never links or calls it.
 *
 * Every function restates one routine of the reference's fem_c/ctools.c (paths
 * relative to the snoo.py project) and keeps its data layouts, triplet order and
 * branch conditions:
 *   or_pchip              ctools.c:130-204   eval_pchip_interpolator[_derivative]
 *   or_mu                 ctools.c:206-346   Cox-de Boor B-spline mu(log10 H) and dmu/dH
 *   or_curlcurl           ctools.c:960-1193  compute_K_dK_Hcurl
 *                         ctools.c:1195-1388 compute_K_dK_Hcurl_red (B_s != NULL)
 *   or_rhs_red            ctools.c:1390-1497 compute_rhs_Hcurl_red
 *   or_B_hcurl            ctools.c:1500-1563 compute_B_Hcurl
 *   or_gradgrad           ctools.c:730-919   compute_K_dK
 *   or_biot_savart        ctools.c:1761-1923 compute_B_line_segs
 * Tables: d_phi[Q][4][3], curls[n_orient][Q][6][3], w[Q], phi[Q][4]; nodes[N][3];
 * cells[E][4] and glob_ids[E][6] 0-based.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define OR_MAXQ 256
#define OR_MAXT 512

/* ---------------------------------------------------------------- materials */

/* PCHIP in piecewise-polynomial form, c[4][n_int] row-major, knots x[n_int+1].
 * n_int == -1 is the constant law c[0] with zero derivative.  Below x[0] (or NaN)
 * the value and derivative are 0; at or beyond x[n_int] the last cubic is
 * extrapolated.  (ctools.c:130-204) */
double or_pchip(int n_int, const double *c, const double *xk, double x, double *dval)
{
    if (n_int == -1) {
        *dval = 0.0;
        return c[0];
    }
    if (!(x >= xk[0])) {
        *dval = 0.0;
        return 0.0;
    }
    int i;
    if (x >= xk[n_int]) {
        i = n_int - 1;
    } else {
        int lo = 0, hi = n_int - 1; /* largest i with xk[i] <= x */
        while (lo < hi) {
            int mid = (lo + hi + 1) / 2;
            if (xk[mid] <= x) lo = mid; else hi = mid - 1;
        }
        i = lo;
    }
    double d = x - xk[i];
    double c0 = c[i], c1 = c[n_int + i], c2 = c[2 * n_int + i], c3 = c[3 * n_int + i];
    *dval = 3.0 * c0 * d * d + 2.0 * c1 * d + c2;
    return c0 * d * d * d + c1 * d * d + c2 * d + c3;
}

/* Values N[i] of all degree-k basis functions at x (Cox-de Boor, bottom-up, the
 * same expressions as the reference's recursion, ctools.c:206-240), and the
 * derivatives dN[i] (ctools.c:242-268).  n_t = number of knots. */
static void or_bspline_basis(const double *t, int n_t, int k, double x, double *N, double *dN)
{
    double tab[OR_MAXT];
    int m = n_t - 1;
    for (int i = 0; i < m; ++i) tab[i] = (t[i] <= x && x < t[i + 1]) ? 1.0 : 0.0;
    for (int d = 1; d <= k; ++d) {
        int md = n_t - 1 - d;
        if (d == k) {
            for (int i = 0; i < md; ++i) {
                double t1 = 0.0, t2 = 0.0;
                if (t[i + d] != t[i]) t1 = d / (t[i + d] - t[i]) * tab[i];
                if (t[i + d + 1] != t[i + 1]) t2 = d / (t[i + d + 1] - t[i + 1]) * tab[i + 1];
                dN[i] = t1 - t2;
            }
        }
        for (int i = 0; i < md; ++i) {
            double a = 0.0, b = 0.0;
            if (t[i + d] != t[i]) a = (x - t[i]) / (t[i + d] - t[i]) * tab[i];
            if (t[i + d + 1] != t[i + 1]) b = (t[i + d + 1] - x) / (t[i + d + 1] - t[i + 1]) * tab[i + 1];
            tab[i] = a + b;
        }
    }
    if (k == 0)
        for (int i = 0; i < m; ++i) dN[i] = 0.0;
    for (int i = 0; i < n_t - 1 - k; ++i) N[i] = tab[i];
}

/* mu(|H|) and dmu/d|H| (ctools.c:317-346).  type 0 or H < H_min: mu_H_min and 0. */
double or_mu(int type, int k, int n_ctrl, const double *t, const double *c, double H_min,
             double mu_H_min, double H, double *dmu)
{
    if (type == 0 || H < H_min) {
        *dmu = 0.0;
        return mu_H_min;
    }
    double x = log10(H);
    double N[OR_MAXT], dN[OR_MAXT];
    int n_t = n_ctrl + k + 1;
    or_bspline_basis(t, n_t, k, x, N, dN);
    double v = 0.0, dv = 0.0;
    for (int i = 0; i < n_ctrl; ++i) {
        v += c[i] * N[i];
        dv += c[i] * dN[i];
    }
    *dmu = dv / (H * log(10.0));
    return v;
}

/* ---------------------------------------------------------------- geometry */

/* J[q][3][3] = sum_i X_i (x) dphi[q][i] (rows: x,y,z; cols: u,v,w), ctools.c:373-413 */
static void or_jacobian(const double *nodes, const int *cell, const double *dphi_q, double *J)
{
    for (int r = 0; r < 9; ++r) J[r] = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) J[k * 3 + l] += nodes[3 * cell[i] + k] * dphi_q[3 * i + l];
}

/* det and inverse by cofactors, ctools.c:440-460 */
static double or_det_inv(const double *m, double *inv)
{
    double det = m[0] * (m[4] * m[8] - m[7] * m[5]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                 m[2] * (m[3] * m[7] - m[4] * m[6]);
    double id = 1.0 / det;
    inv[0] = (m[4] * m[8] - m[7] * m[5]) * id;
    inv[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    inv[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    inv[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    inv[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    inv[5] = (m[3] * m[2] - m[0] * m[5]) * id;
    inv[6] = (m[3] * m[7] - m[6] * m[4]) * id;
    inv[7] = (m[6] * m[1] - m[0] * m[7]) * id;
    inv[8] = (m[0] * m[4] - m[3] * m[1]) * id;
    return det;
}

static void or_mv(const double *M, const double *v, double *r)
{
    r[0] = M[0] * v[0] + M[1] * v[1] + M[2] * v[2];
    r[1] = M[3] * v[0] + M[4] * v[1] + M[5] * v[2];
    r[2] = M[6] * v[0] + M[7] * v[1] + M[8] * v[2];
}

static void or_mtv(const double *M, const double *v, double *r)
{
    r[0] = M[0] * v[0] + M[3] * v[1] + M[6] * v[2];
    r[1] = M[1] * v[0] + M[4] * v[1] + M[7] * v[2];
    r[2] = M[2] * v[0] + M[5] * v[1] + M[8] * v[2];
}

static double or_dot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* ---------------------------------------------------------------- curl-curl */

/* Element loop of the Newton curl-curl assembly.  Writes 36 triplets per element
 * (j <= k, mirrored when j != k) into ti/tj/vK/vdK in the reference's order.
 * B_s == NULL: plain kernel (ctools.c:960-1193); otherwise reduced kernel with the
 * source field B_s[E][Q][3] and rhs accumulation (ctools.c:1195-1388).
 * sK/sdK (optional) receive, per triplet, the sum of the magnitudes of the terms that make
 * it up (|nu| |cu| |cv| |w| / |det| and |nu'| |cu| |cv| |B| |w| / |det|): the scale of the
 * rounding error any evaluation order makes, used as the comparison scale in the tests.
 * phi/dil (optional, reduced kernel only): diluted steel (compute_K_dK_Hcurl_red_dil,
 * ctools.c:1565-1759).  phi[Q][4] holds the nodal basis at the quadrature points, the point's
 * z is sum_i phi_i Z_i (evaluate_finite_element, ctools.c:480-504), the dilution factor
 * s = (c_num + z m_num) / (c_den + z m_den) (eval_dilution, ctools.c:124-128) with
 * dil = {c_num, m_num, c_den, m_den}, and nu = s PCHIP(s |B|), nu' = s^2 PCHIP'(s |B|).
 * Returns the number of triplets written, or -1 on a bad argument. */
int64_t or_curlcurl(int64_t E, int Q, const double *nodes, const int *cells, const int *glob_ids,
                    const int *orient, const double *curls, const double *dphi, const double *w,
                    const double *x, const double *B_s, int n_int, const double *rel_c,
                    const double *rel_x, int *ti, int *tj, double *vK, double *vdK, double *rhs,
                    double *sK, double *sdK, const double *phi, const double *dil)
{
    if (dil && (!phi || !B_s)) return -1;
    if (Q <= 0 || Q > OR_MAXQ) return -1;
    const double nu0 = 1.0 / 4.0 / M_PI * 1e7;
    double J[OR_MAXQ][9], Jinv[9], det[OR_MAXQ], B[OR_MAXQ][3], Bm[OR_MAXQ], nu[OR_MAXQ], dnu[OR_MAXQ];
    int64_t cnt = 0;
    for (int64_t e = 0; e < E; ++e) {
        const int *cell = cells + 4 * e;
        const int *g = glob_ids + 6 * e;
        const double *ct = curls + (int64_t)3 * Q * 6 * orient[e];
        for (int q = 0; q < Q; ++q) {
            or_jacobian(nodes, cell, dphi + 12 * q, J[q]);
            det[q] = or_det_inv(J[q], Jinv);
        }
        for (int q = 0; q < Q; ++q) {
            for (int d = 0; d < 3; ++d) B[q][d] = B_s ? B_s[(e * Q + q) * 3 + d] : 0.0;
            for (int j = 0; j < 6; ++j) {
                double c[3];
                or_mv(J[q], ct + 3 * (q * 6 + j), c);
                for (int d = 0; d < 3; ++d) B[q][d] += c[d] * x[g[j]] / det[q];
            }
            Bm[q] = sqrt(or_dot(B[q], B[q]));
            if (dil) {
                double z = 0.0;
                for (int i = 0; i < 4; ++i) z += phi[4 * q + i] * nodes[3 * cell[i] + 2];
                const double sf = (dil[0] + z * dil[1]) / (dil[2] + z * dil[3]);
                nu[q] = sf * or_pchip(n_int, rel_c, rel_x, sf * Bm[q], &dnu[q]);
                dnu[q] *= sf * sf;
            } else {
                nu[q] = or_pchip(n_int, rel_c, rel_x, Bm[q], &dnu[q]);
            }
        }
        for (int j = 0; j < 6; ++j) {
            for (int k = j; k < 6; ++k) {
                double aK = 0.0, adK = 0.0, mK = 0.0, mdK = 0.0;
                for (int q = 0; q < Q; ++q) {
                    double cu[3], cv[3];
                    or_mv(J[q], ct + 3 * (q * 6 + j), cu);
                    or_mv(J[q], ct + 3 * (q * 6 + k), cv);
                    aK += nu[q] * or_dot(cu, cv) * w[q] / det[q];
                    double nn = sqrt(or_dot(cu, cu) * or_dot(cv, cv)) * fabs(w[q] / det[q]);
                    mK += fabs(nu[q]) * nn;
                    if (Bm[q] >= 1e-14) {
                        double pu = or_dot(cu, B[q]), pv = or_dot(cv, B[q]);
                        adK += dnu[q] * pu * pv * w[q] / det[q] / Bm[q];
                        mdK += fabs(dnu[q]) * nn * Bm[q];
                    }
                    if (B_s && j == k) rhs[g[j]] += (nu0 - nu[q]) * or_dot(cu, B_s + (e * Q + q) * 3) * w[q];
                }
                ti[cnt] = g[j]; tj[cnt] = g[k]; vK[cnt] = aK; vdK[cnt] = adK;
                if (sK) { sK[cnt] = mK; sdK[cnt] = mdK; }
                ++cnt;
                if (j != k) {
                    ti[cnt] = g[k]; tj[cnt] = g[j]; vK[cnt] = aK; vdK[cnt] = adK;
                    if (sK) { sK[cnt] = mK; sdK[cnt] = mdK; }
                    ++cnt;
                }
            }
        }
    }
    return cnt;
}

/* rhs only, reduced formulation (ctools.c:1390-1497) */
int or_rhs_red(int64_t E, int Q, const double *nodes, const int *cells, const int *glob_ids,
               const int *orient, const double *curls, const double *dphi, const double *w,
               const double *x, const double *B_s, int n_int, const double *rel_c,
               const double *rel_x, double *rhs)
{
    if (Q <= 0 || Q > OR_MAXQ) return -1;
    const double nu0 = 1.0 / 4.0 / M_PI * 1e7;
    double J[OR_MAXQ][9], Jinv[9], det[OR_MAXQ], nu[OR_MAXQ], dnu;
    for (int64_t e = 0; e < E; ++e) {
        const int *cell = cells + 4 * e;
        const int *g = glob_ids + 6 * e;
        const double *ct = curls + (int64_t)3 * Q * 6 * orient[e];
        for (int q = 0; q < Q; ++q) {
            or_jacobian(nodes, cell, dphi + 12 * q, J[q]);
            det[q] = or_det_inv(J[q], Jinv);
            double B[3];
            for (int d = 0; d < 3; ++d) B[d] = B_s[(e * Q + q) * 3 + d];
            for (int j = 0; j < 6; ++j) {
                double c[3];
                or_mv(J[q], ct + 3 * (q * 6 + j), c);
                for (int d = 0; d < 3; ++d) B[d] += c[d] * x[g[j]] / det[q];
            }
            nu[q] = or_pchip(n_int, rel_c, rel_x, sqrt(or_dot(B, B)), &dnu);
        }
        for (int j = 0; j < 6; ++j)
            for (int q = 0; q < Q; ++q) {
                double cu[3];
                or_mv(J[q], ct + 3 * (q * 6 + j), cu);
                rhs[g[j]] += (nu0 - nu[q]) * or_dot(cu, B_s + (e * Q + q) * 3) * w[q];
            }
    }
    return 0;
}

/* Quadrature-point positions and B = J curl_hat x / det (ctools.c:1500-1563) */
int or_B_hcurl(int64_t E, int Q, const double *nodes, const int *cells, const int *glob_ids,
               const int *orient, const double *curls, const double *phi, const double *dphi,
               const double *x, double *points, double *Bout)
{
    if (Q <= 0 || Q > OR_MAXQ) return -1;
    double J[9], Jinv[9];
    for (int64_t e = 0; e < E; ++e) {
        const int *cell = cells + 4 * e;
        const int *g = glob_ids + 6 * e;
        const double *ct = curls + (int64_t)3 * Q * 6 * orient[e];
        for (int q = 0; q < Q; ++q) {
            or_jacobian(nodes, cell, dphi + 12 * q, J);
            double det = or_det_inv(J, Jinv);
            double *p = points + (e * Q + q) * 3;
            double *B = Bout + (e * Q + q) * 3;
            for (int d = 0; d < 3; ++d) {
                p[d] = 0.0;
                B[d] = 0.0;
            }
            for (int i = 0; i < 4; ++i)
                for (int d = 0; d < 3; ++d) p[d] += phi[4 * q + i] * nodes[3 * cell[i] + d];
            for (int j = 0; j < 6; ++j) {
                double c[3];
                or_mv(J, ct + 3 * (q * 6 + j), c);
                for (int d = 0; d < 3; ++d) B[d] += c[d] * x[g[j]] / det;
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- grad-grad */

/* P1 nodal Newton assembly of div(mu grad phi) (ctools.c:730-919).  16 triplets per
 * element: (k, l >= k), mirrored when k != l. */
int64_t or_gradgrad(int64_t E, int Q, const double *nodes, const int *cells, const double *dphi,
                    const double *w, const double *x, int type, int k_deg, int n_ctrl,
                    const double *t, const double *c, double H_min, double mu_H_min, int *ti,
                    int *tj, double *vK, double *vdK, double *sK, double *sdK)
{
    if (Q <= 0 || Q > OR_MAXQ) return -1;
    double J[9], Ji[OR_MAXQ][9], det[OR_MAXQ], H[OR_MAXQ][3], Hm[OR_MAXQ], mu[OR_MAXQ], dmu[OR_MAXQ];
    int64_t cnt = 0;
    for (int64_t e = 0; e < E; ++e) {
        const int *cell = cells + 4 * e;
        for (int q = 0; q < Q; ++q) {
            or_jacobian(nodes, cell, dphi + 12 * q, J);
            det[q] = or_det_inv(J, Ji[q]);
            double gr[3] = {0.0, 0.0, 0.0};
            for (int i = 0; i < 4; ++i)
                for (int d = 0; d < 3; ++d) gr[d] += dphi[12 * q + 3 * i + d] * x[cell[i]];
            or_mtv(Ji[q], gr, H[q]);
            Hm[q] = sqrt(or_dot(H[q], H[q]));
            mu[q] = or_mu(type, k_deg, n_ctrl, t, c, H_min, mu_H_min, Hm[q], &dmu[q]);
        }
        for (int a = 0; a < 4; ++a) {
            for (int b = a; b < 4; ++b) {
                double aK = 0.0, adK = 0.0, mK = 0.0, mdK = 0.0;
                for (int q = 0; q < Q; ++q) {
                    double gu[3], gv[3];
                    or_mtv(Ji[q], dphi + 12 * q + 3 * a, gu);
                    or_mtv(Ji[q], dphi + 12 * q + 3 * b, gv);
                    aK += mu[q] * det[q] * w[q] * or_dot(gu, gv);
                    double nn = sqrt(or_dot(gu, gu) * or_dot(gv, gv)) * fabs(det[q] * w[q]);
                    mK += fabs(mu[q]) * nn;
                    if (Hm[q] >= 1e-14) {
                        adK += dmu[q] * det[q] * w[q] * or_dot(gu, H[q]) * or_dot(gv, H[q]) / Hm[q];
                        mdK += fabs(dmu[q]) * nn * Hm[q];
                    }
                }
                ti[cnt] = cell[a]; tj[cnt] = cell[b]; vK[cnt] = aK; vdK[cnt] = adK;
                if (sK) { sK[cnt] = mK; sdK[cnt] = mdK; }
                ++cnt;
                if (a != b) {
                    ti[cnt] = cell[b]; tj[cnt] = cell[a]; vK[cnt] = aK; vdK[cnt] = adK;
                    if (sK) { sK[cnt] = mK; sdK[cnt] = mdK; }
                    ++cnt;
                }
            }
        }
    }
    return cnt;
}

/* ---------------------------------------------------------------- Biot-Savart */

/* B of straight line segments src[S][6] at targets tar[T][3], times current*1e-7.
 * Inside a radius-rad "sausage" around a segment the field is that of a uniform
 * cylindrical conductor (ctools.c:1761-1923). */
void or_biot_savart(const double *src, int64_t S, const double *tar, int64_t T, double current,
                    double rad, double *Bout)
{
    for (int64_t i = 0; i < T; ++i) {
        double bx = 0.0, by = 0.0, bz = 0.0;
        const double *p = tar + 3 * i;
        for (int64_t j = 0; j < S; ++j) {
            const double *s = src + 6 * j;
            double n[3] = {s[3] - s[0], s[4] - s[1], s[5] - s[2]};
            double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
            double d1[3] = {s[0] - p[0], s[1] - p[1], s[2] - p[2]};
            double d2[3] = {s[3] - p[0], s[4] - p[1], s[5] - p[2]};
            double n1 = sqrt(or_dot(d1, d1)), n2 = sqrt(or_dot(d2, d2));
            double tp = -1.0 * or_dot(d1, n) / nn;
            double pm[3] = {p[0] - (s[0] + tp * n[0]), p[1] - (s[1] + tp * n[1]), p[2] - (s[2] + tp * n[2])};
            double dmin2 = or_dot(pm, pm);
            if ((dmin2 < rad * rad && tp <= 1.0 && tp >= 0.0) || n1 < rad || n2 < rad) {
                double bd[3] = {n[1] * pm[2] - n[2] * pm[1], n[2] * pm[0] - n[0] * pm[2], n[0] * pm[1] - n[1] * pm[0]};
                double nb = sqrt(or_dot(bd, bd));
                double f = 2.0 * sqrt(dmin2) / rad / rad / nb;
                bx += bd[0] * f;
                by += bd[1] * f;
                bz += bd[2] * f;
            } else {
                double dd = or_dot(d1, d2);
                double f = (n1 + n2) / (n1 * n2 + dd) / n1 / n2;
                bx += (d1[1] * d2[2] - d1[2] * d2[1]) * f;
                by += (d1[2] * d2[0] - d1[0] * d2[2]) * f;
                bz += (d1[0] * d2[1] - d1[1] * d2[0]) * f;
            }
        }
        Bout[3 * i] = bx * current * 1e-7;
        Bout[3 * i + 1] = by * current * 1e-7;
        Bout[3 * i + 2] = bz * current * 1e-7;
    }
}
