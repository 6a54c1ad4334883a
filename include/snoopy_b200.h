/*
 * snoopy_b200: sm_100a kernels for snoo.py's nonlinear magnetostatic path, behind a
 * plain C ABI (load with ctypes / cffi / dlopen).
 *
 * Conventions
 *   - Every pointer argument is a DEVICE pointer unless its comment says "host".
 *   - Indices are 0-based int32 (the reference subtracts gmsh's 1 before calling C,
 *     snoopy/curl_curl_assembler.py:916-917).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).  Calls
 *     are asynchronous on it unless their comment says they synchronise.
 *   - Every function returns an snp_status; snp_last_error() gives the message of the
 *     calling thread's last failure.  The reference's C returns void and prints
 *     (fem_c/ctools.c:428, fem_c/interface_c.pyx:71,234,952-959).
 *   - The single-launch assembly entry points ACCUMULATE (+=) into their outputs, like the
 *     reference's `K += this_K` per material (snoopy/curl_curl_assembler.py:928-930): zero
 *     first.  The two-phase curl-curl assembly (snp_curlcurl_terms + snp_curlcurl_rows)
 *     overwrites its outputs.
 *
 * Table layouts are the reference C kernels' (fem_c/ctools.c):
 *   nodes[N][3]; cells[E][4]; glob_ids[E][6]; orientations[E];
 *   d_phi[Q][4][3]; curls[n_orient][Q][6][3]; w[Q]; phi[Q][4].
 * Materials:
 *   reluctance  (fem_c/ctools.h:56-63, interface_c.pyx:226-234):
 *       n_int == -1 -> constant nu = rel_c[0]; else PCHIP in PP form,
 *       rel_c[4][n_int] row-major, rel_x[n_int+1].
 *   permeability (fem_c/ctools.h:44-54, interface_c.pyx:56-68):
 *       type 0 -> mu = mu_H_min; type 1 -> cubic (degree k) B-spline in log10|H| with
 *       knots t[n_ctrl+k+1], coefficients c[n_ctrl], constant mu_H_min below H_min.
 */
#ifndef SNOOPY_B200_H
#define SNOOPY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SNP_OK = 0,
    SNP_BAD_ARG = 1,
    SNP_CUDA_ERROR = 2,
    SNP_NOT_CONVERGED = 3,
    SNP_NAN_DETECTED = 4,
    SNP_ZERO_PIVOT = 5,
    SNP_NO_MEMORY = 6
} snp_status;

/* Message of the calling thread's last failure ("" if none). */
const char *snp_last_error(void);

/* ABI version of this library. */
int snp_version(void);

/* ------------------------------------------------------------------ CSR pattern
 * Replaces the COO->CSR conversion of fem_c/interface_c.pyx:154-155,367-368
 * (csr_array((vals,(i,j))): duplicates summed, sorted column indices).  The pattern of
 * an element -> DoF connectivity holds row_ptr/col_idx and the slot map
 * slot[e][a][b] = position of (elem_dofs[e][a], elem_dofs[e][b]) in the CSR arrays, so
 * assembly scatters element values straight into CSR values. */
typedef struct snp_pattern snp_pattern;

/* elem_dofs[n_elems][dofs_per_elem] (device).  dofs_per_elem is 6 (edge elements) or 4
 * (nodal P1).  Synchronises `stream` (the nnz is read back). */
int snp_pattern_create(const int32_t *elem_dofs, int64_t n_elems, int32_t dofs_per_elem, int32_t n_rows,
                       void *stream, snp_pattern **out);
/* Host outputs: rows, nnz, elements, dofs per element. */
int snp_pattern_info(const snp_pattern *pat, int32_t *n_rows, int64_t *nnz, int64_t *n_elems, int32_t *dofs_per_elem);
/* Device arrays owned by the pattern: row_ptr[n_rows+1], col_idx[nnz], slots[n_elems*dpe*dpe]. */
int snp_pattern_arrays(const snp_pattern *pat, const int32_t **row_ptr, const int32_t **col_idx, const int32_t **slots);
/* Position of each row's diagonal entry, diag_pos[n_rows] (-1 if absent). */
int snp_pattern_diag(const snp_pattern *pat, const int32_t **diag_pos);
int snp_pattern_destroy(snp_pattern *pat);

/* ------------------------------------------------------------------ curl-curl assembly
 * Replaces fem_c.compute_stiffness_and_jacobi_matrix_curl_curl (fem_c/interface_c.pyx:162-374)
 * -> compute_K_dK_Hcurl (fem_c/ctools.c:960-1193) when B_s == NULL and
 * compute_K_dK_Hcurl_red (fem_c/ctools.c:1195-1388) otherwise.
 *
 * One material's elements, which are elements [elem_offset, elem_offset + n_elems) of
 * `pat`.  First-order tetrahedra with quadrature-independent tables (affine elements).
 * Outputs (each may be NULL), accumulated:
 *   K_vals[nnz]   stiffness values K(x)             (reference K)
 *   dK_vals[nnz]  Newton correction dK(x)           (reference dK)
 *   J_vals[nnz]   Jacobian K + dK                   (reference dK + K)
 *   rhs[n]        reduced rhs sum (nu0 - nu) curl w.B_s w (reduced kernel only)
 *   F[n]          residual K(x) x - rhs(x)
 * B_s[n_elems][Q][3] or NULL.  x[n] the DoF vector. */
int snp_curlcurl_assemble(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems,
                          const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                          const int32_t *orientations, const double *curls, int32_t n_orient,
                          const double *d_phi, const double *w, int32_t n_quad,
                          const double *x, const double *B_s,
                          int32_t n_int, const double *rel_c, const double *rel_x,
                          double *K_vals, double *dK_vals, double *J_vals, double *rhs, double *F,
                          void *stream);

/* Same element arithmetic (float64) accumulating float32 Jacobian values K + dK
 * (mixed-precision Newton: the Krylov solve runs on these, the residual F stays float64
 * through snp_curlcurl_assemble with only F requested).  Same source as
 * snp_curlcurl_assemble (fem_c/ctools.c:960-1388). */
int snp_curlcurl_assemble_f32(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems,
                              const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                              const int32_t *orientations, const double *curls, int32_t n_orient,
                              const double *d_phi, const double *w, int32_t n_quad,
                              const double *x, const double *B_s,
                              int32_t n_int, const double *rel_c, const double *rel_x,
                              float *J_vals, void *stream);

/* Diluted steel.  Replaces fem_c.compute_stiffness_and_jacobi_matrix_curl_curl_diluted
 * (fem_c/interface_c.pyx:698-926) -> compute_K_dK_Hcurl_red_dil (fem_c/ctools.c:1565-1759).
 * As snp_curlcurl_assemble, and with B_s the reluctance at each quadrature point is
 * nu = s PCHIP(s |B|), nu' = s^2 PCHIP'(s |B|) with s = (c_num + z m_num) / (c_den + z m_den),
 * z = sum_i phi[q][i] Z_i the point's z coordinate; phi is device f64[n_quad][4] (the nodal
 * basis at the points) and dilution host f64[4] = {c_num, m_num, c_den, m_den}.  Without
 * B_s the plain kernel runs and phi/dilution are not read (the reference's air branch,
 * interface_c.pyx:874-886). */
int snp_curlcurl_assemble_diluted(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems,
                                  const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                                  const int32_t *orientations, const double *curls, int32_t n_orient,
                                  const double *phi, const double *d_phi, const double *w, int32_t n_quad,
                                  const double *x, const double *B_s,
                                  int32_t n_int, const double *rel_c, const double *rel_x,
                                  const double *dilution,
                                  double *K_vals, double *dK_vals, double *J_vals, double *rhs, double *F,
                                  void *stream);

/* Reduced rhs only.  Replaces fem_c.compute_rhs_Hcurl_red_c (fem_c/interface_c.pyx:377-552)
 * -> compute_rhs_Hcurl_red (fem_c/ctools.c:1390-1497).  Accumulates into rhs[n]. */
int snp_curlcurl_rhs_red(int64_t n_elems, const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                         const int32_t *orientations, const double *curls, int32_t n_orient,
                         const double *d_phi, const double *w, int32_t n_quad, const double *x,
                         const double *B_s, int32_t n_int, const double *rel_c, const double *rel_x,
                         double *rhs, void *stream);

/* Deterministic two-phase form of snp_curlcurl_assemble[_diluted] over a whole pattern (same
 * element arithmetic, fem_c/ctools.c:960-1388 and 1565-1759; the reference's sum over
 * elements happens in scipy's COO->CSR conversion, fem_c/interface_c.pyx:365-368).
 *
 * Phase 1, once per material: snp_curlcurl_terms stores the element values of elements
 * [elem_offset, elem_offset + n_elems) in `terms`: stride blocks (snp_curlcurl_terms_stride) of
 * the pattern's n_elems doubles each, value b of element e at terms[b * n_elems + e].  `parts`
 * (SNP_TERMS_* bits) selects the blocks: the 21 upper-triangle values of the element's K, dK
 * or J = K + dK, its six residual terms (F = K(x) x - rhs(x)), its six reduced-rhs terms.  phi
 * and dilution as for snp_curlcurl_assemble_diluted (both NULL: plain steel).
 *
 * Phase 2, once: snp_curlcurl_rows forms every CSR entry as the sum of its element
 * contributions in element order (one thread per entry, over the pattern's sorted coupling
 * list) and every entry of F / rhs over the DoF's incidences, with no atomics, and OVERWRITES
 * each requested output (no zeroing needed): K_vals needs SNP_TERMS_K, dK_vals SNP_TERMS_DK,
 * J_vals / J32_vals SNP_TERMS_K | SNP_TERMS_DK (J = K + dK per entry, as the reference's dK + K)
 * or SNP_TERMS_J, F SNP_TERMS_F, rhs SNP_TERMS_RHS (elements without a source field give 0).
 * Results are bitwise repeatable.  Needs a pattern built with 6 DoFs per element and fewer than
 * 2^31 couplings (snp_curlcurl_rows_supported). */
#define SNP_TERMS_K 1
#define SNP_TERMS_DK 2
#define SNP_TERMS_J 4
#define SNP_TERMS_F 8
#define SNP_TERMS_RHS 16
int snp_curlcurl_terms_stride(int32_t parts, int32_t *stride);
int snp_curlcurl_rows_supported(const snp_pattern *pat, int32_t *supported);
int snp_curlcurl_terms(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems,
                       const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                       const int32_t *orientations, const double *curls, int32_t n_orient,
                       const double *phi, const double *d_phi, const double *w, int32_t n_quad,
                       const double *x, const double *B_s,
                       int32_t n_int, const double *rel_c, const double *rel_x, const double *dilution,
                       int32_t parts, double *terms, void *stream);
int snp_curlcurl_rows(const snp_pattern *pat, const double *terms, int32_t parts,
                      double *K_vals, double *dK_vals, double *J_vals, float *J32_vals,
                      double *rhs, double *F, void *stream);

/* ------------------------------------------------------------------ grad-grad assembly
 * Replaces fem_c.compute_stiffness_and_jacobi_matrix (fem_c/interface_c.pyx:11-160)
 * -> compute_K_dK (fem_c/ctools.c:730-919).  P1 nodal elements [elem_offset, +n_elems)
 * of a pattern built with dofs_per_elem = 4 over `cells`.  Outputs may be NULL, accumulated:
 * K_vals, dK_vals, J_vals = K + dK (all [nnz]).  Each CSR entry gets one addition per call, the
 * sum of its contributions from these elements in element order, so repeated calls give bitwise
 * the same values (SNP_ASSEMBLY=atomic: float64 atomics per contribution instead).  The call
 * keeps its element values in a work array of the pattern: calls on one pattern must not
 * overlap on the GPU. */
int snp_gradgrad_assemble(const snp_pattern *pat, int64_t elem_offset, int64_t n_elems,
                          const double *nodes, const int32_t *cells, const double *d_phi,
                          const double *w, int32_t n_quad, const double *x,
                          int32_t perm_type, int32_t degree, int32_t n_ctrl, const double *knots,
                          const double *ctrl, double H_min, double mu_H_min,
                          double *K_vals, double *dK_vals, double *J_vals, void *stream);

/* ------------------------------------------------------------------ fields
 * B at quadrature points.  Replaces fem_c.compute_B_Hcurl (fem_c/interface_c.pyx:555-696)
 * -> compute_B_Hcurl (fem_c/ctools.c:1500-1563).  points[E][Q][3], B[E][Q][3]. */
int snp_b_hcurl(int64_t n_elems, const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                const int32_t *orientations, const double *curls, int32_t n_orient, const double *phi,
                const double *d_phi, int32_t n_quad, const double *x, double *points, double *B,
                void *stream);

/* Physical quadrature points only, points[E][Q][3] (snoopy/curl_curl_assembler.py:1521-1593). */
int snp_quad_points(int64_t n_elems, const double *nodes, const int32_t *cells, const double *phi,
                    int32_t n_quad, double *points, void *stream);

/* B of one element-constant curl at arbitrary points: B[i] = curl of x in element elem[i]
 * (first-order elements; elem[i] < 0 gives 0).  Probe evaluation
 * (snoopy/evaluators.py:155-295 locates points with gmsh; here the caller passes elem). */
int snp_b_at_elements(int64_t n_points, const int32_t *elem, const double *nodes, const int32_t *cells,
                      const int32_t *glob_ids, const int32_t *orientations, const double *curls,
                      int32_t n_orient, const double *d_phi, int32_t n_quad, const double *x, double *B,
                      void *stream);

/* ---------------------------------------------------------------- field maps
 * Mesh index for point location and nodal output.  Replaces gmsh's point location
 * (get_element_by_coordinates in snoopy/evaluators.py:155-295, 297-410) and the Python loop of
 * CurlCurlAssembler.compute_nodal_fields (snoopy/curl_curl_assembler.py:2089-2196).  Built once
 * per mesh (device copies of nodes[N][3] and cells[E][4]; cells are checked): a uniform bucket
 * grid with cell edge >= the largest element extent, elements bucketed by centroid, and the
 * node -> element incidence. */
typedef struct snp_mesh_index snp_mesh_index;

int snp_mesh_index_create(const double *nodes, int64_t n_nodes, const int32_t *cells, int64_t n_elems,
                          void *stream, snp_mesh_index **out);

/* Grid shape (nb[3] buckets, origin bmin[3], cell edges h[3]) and the fullest bucket's size;
 * any output may be NULL. */
int snp_mesh_index_info(const snp_mesh_index *mi, int32_t *nb, double *bmin, double *h, int32_t *max_bucket);

/* For each point (device f64[n_points][3]): the element holding it, elem[i] (-1 when the best
 * candidate's smallest barycentric coordinate is below -tol, or the point is not finite), and,
 * when bary is not NULL, its barycentric coordinates bary[i][4] in the element's node order
 * (0 outside).  Among elements holding a point (faces, edges) the one with the largest smallest
 * coordinate wins, ties to the lower element index. */
int snp_mesh_index_locate(const snp_mesh_index *mi, const double *points, int64_t n_points, double tol,
                          int32_t *elem, double *bary, void *stream);

/* nodal[v][c] = mean of elem_values[e][c] over the elements e of node v with elem_mask[e] != 0
 * (all elements when elem_mask is NULL), summed in element order; 0 for a node with none
 * (compute_nodal_fields, curl_curl_assembler.py:2185-2196). */
int snp_mesh_index_nodal_average(const snp_mesh_index *mi, const double *elem_values, int32_t n_comp,
                                 const uint8_t *elem_mask, double *nodal, void *stream);

/* out[i][c] = sum_k bary[i][k] nodal[s][cells[elem[i]][k]][c] with s = point_set[i] (0 when
 * point_set is NULL); 0 for elem[i] outside [0, E) or s outside [0, n_sets).  nodal holds
 * n_sets arrays of N x n_comp values (evaluate_interpolation, snoopy/evaluators.py:297-410). */
int snp_mesh_index_interpolate(const snp_mesh_index *mi, int64_t n_points, const int32_t *elem,
                               const double *bary, const double *nodal, int32_t n_comp, int32_t n_sets,
                               const int32_t *point_set, double *out, void *stream);

int snp_mesh_index_destroy(snp_mesh_index *mi);

/* Source rhs of the total-potential formulation from a nodal electric potential x_p[N]:
 * rhs[g_k] += sum_q (J^-T w_hat_k) . (J^-T grad_hat phi) w_q det, with the edge basis
 * functions basis[n_orient][Q][6][3] (not their curls).  Replaces the pure-Python
 * CurlCurlAssembler.compute_rhs_electric_potential (snoopy/curl_curl_assembler.py:1154-1284).
 * Accumulates into rhs[n]. */
int snp_rhs_grad_potential(int64_t n_elems, const double *nodes, const int32_t *cells, const int32_t *glob_ids,
                           const int32_t *orientations, const double *basis, int32_t n_orient, const double *d_phi,
                           const double *w, int32_t n_quad, const double *x_p, double *rhs, void *stream);

/* Biot-Savart of straight filament segments.  Replaces fem_c.compute_B_line_segs_cpp
 * (fem_c/interface_c.pyx:928-991) -> compute_B_line_segs (fem_c/ctools.c:1761-1923).
 * src[S][6], tar[T][3], B[T][3] (overwritten). */
int snp_biot_savart(const double *src, int64_t n_src, const double *tar, int64_t n_tar, double current,
                    double radius, double *B, void *stream);

/* ------------------------------------------------------------------ sparse linear algebra
 * y = A x on the rows/cols with free[i] != 0 (free == NULL: all).  Rows with free[i] == 0
 * give y[i] = 0, and their columns are skipped.  (scipy `J @ x`, `J[mask,:][:,mask]`,
 * snoopy/red_mvp_solver.py:186,195-196.) */
int snp_spmv(int32_t n_rows, const int32_t *row_ptr, const int32_t *col_idx, const double *vals,
             const uint8_t *free_mask, const double *x, double *y, void *stream);

/* Jacobi-preconditioned CG on A restricted to the free DoFs, with scipy.sparse.linalg.cg's
 * stopping rule ||r|| < max(atol, rtol ||b_free||) (snoopy/red_mvp_solver.py:199-203).
 * x: in = initial guess (free entries), out = solution (non-free entries set to 0).
 * maxiter < 0: 10 * n_free like scipy.  Host outputs: iterations, final ||r||.
 * Synchronises `stream`.  Returns SNP_NOT_CONVERGED when maxiter is reached (x is the
 * last iterate) and SNP_NAN_DETECTED on a non-finite residual. */
int snp_pcg(int32_t n_rows, const int32_t *row_ptr, const int32_t *col_idx, const double *vals,
            const uint8_t *free_mask, const double *b, double *x, double rtol, double atol,
            int64_t maxiter, int64_t *iterations, double *res_norm, void *stream);

/* snp_pcg for callers that cannot allocate device memory while they solve (a service whose
 * device memory is all handed to its own pool at start-up, or a loop where cudaFree's implicit
 * device synchronisation would stall other streams).  No counterpart in the reference.
 * Same arguments, results and statuses as snp_pcg, but the work vectors live in one static
 * device array of SNP_PCG_NOALLOC_MAX_ROWS rows (about 11 MB, held by every GPU that loads
 * this library until the process exits); larger systems are rejected with SNP_BAD_ARG.
 * Nothing is allocated: no cudaMalloc, cudaFree or allocating library call.  Every call looks
 * the array's device address up for the calling thread's current device and context, and
 * synchronises `stream`.  All calls share the array, which keeps the last call's contents:
 * calls whose work overlaps on the GPU race and must be serialised by the caller. */
#define SNP_PCG_NOALLOC_MAX_ROWS 262144
int snp_pcg_noalloc(int32_t n_rows, const int32_t *row_ptr, const int32_t *col_idx, const double *vals,
                    const uint8_t *free_mask, const double *b, double *x, double rtol, double atol,
                    int64_t maxiter, int64_t *iterations, double *res_norm, void *stream);

/* ------------------------------------------------------------------ Newton solver
 * Persistent device problem for the Newton loops of RedMVPSolver.solve
 * (snoopy/red_mvp_solver.py:121-224) and MVPSolver.solve_nonlin (snoopy/mvp_solver.py:222-334):
 * owns the concatenated element lists, the CSR pattern and slot map, the Dirichlet mask,
 * the source fields and all work vectors. */
typedef struct snp_solver snp_solver;

/* Tables are shared by all materials; free_mask[n_dofs] (device) marks non-Dirichlet DoFs.
 * Everything is copied into the solver. */
int snp_solver_create(int32_t n_dofs, const double *nodes, int64_t n_nodes, const double *curls,
                      int32_t n_orient, const double *d_phi, const double *w, int32_t n_quad,
                      const uint8_t *free_mask, void *stream, snp_solver **out);

/* Append one material (the reference's per-volume-tag loop).  B_s[n_elems][Q][3] or NULL. */
int snp_solver_add_material(snp_solver *s, const int32_t *cells, const int32_t *glob_ids,
                            const int32_t *orientations, int64_t n_elems, int32_t n_int,
                            const double *rel_c, const double *rel_x, const double *B_s);

/* Extra constant rhs added to every residual (MVPSolver's coil source rhs_mvp), or NULL. */
int snp_solver_set_rhs(snp_solver *s, const double *rhs);

/* Build the CSR pattern over all materials.  Synchronises. */
int snp_solver_finalize(snp_solver *s);

/* Solve options (host struct). */
typedef struct {
    int32_t mode;            /* 0: the reference's increment test and CG(atol=tol, rtol=1e-5);
                                1: relative Newton residual ||F_free|| <= tol ||F_free(x0)|| */
    double tol;              /* mode 0: increment tolerance (reference default 1e-4); mode 1: residual rtol */
    int64_t cg_maxiter;      /* < 0: 10 * n_free (scipy default) */
    int32_t max_newton;      /* reference default 25 */
    double cg_rtol;          /* mode 0: scipy default 1e-5; mode 1: cap of the adaptive forcing term */
    int32_t precision;       /* 0: float64 throughout; 1: float32 Jacobian + Krylov inside float64 Newton */
    int32_t verbose;         /* print one line per Newton step to stdout */
    int32_t line_search;     /* mode 1: step length where the energy slope F(x + a h).h has halved (safeguarded secant) */
    double res_ref;          /* mode 1: > 0 replaces ||F_free(x0)|| in the criterion (pass ||F_free(0)|| to hold a
                                warm start to the zero-start target); a start with ||F_free(x0)|| > res_ref is
                                replaced by x0 = 0 (stats.start_dropped) */
} snp_solve_opts;

/* Solve statistics (host struct). */
typedef struct {
    int32_t newton_iterations;
    int64_t cg_iterations;       /* total */
    double res0;                 /* ||F_free(x0)|| */
    double res;                  /* ||F_free(x_final)|| (mode 1; mode 0: at the last assembly) */
    double t_assemble_ms, t_krylov_ms, t_total_ms;
    int32_t status;
    int64_t kernel_launches;     /* this library's kernels launched by the solve (graph nodes counted per execution) */
    int32_t residual_evals;      /* extra residual-only assemblies of the line search */
    int32_t start_dropped;       /* 1 when the initial guess was replaced by 0 (see res_ref) */
    int32_t galerkin_steps;      /* Galerkin corrections applied to the start (snp_solver_set_galerkin_basis) */
} snp_solve_stats;

/* x[n_dofs] (device): in = initial guess, out = solution.  Synchronises. */
int snp_solver_solve(snp_solver *s, double *x, const snp_solve_opts *opts, snp_solve_stats *stats);

/* Assemble at x into the solver's pattern and copy out (each may be NULL):
 * K_vals/J_vals [nnz], rhs/F [n].  Uses the solver's materials and source fields. */
int snp_solver_assemble(snp_solver *s, const double *x, double *K_vals, double *J_vals, double *rhs,
                        double *F, void *stream);

/* Storage of the Jacobian inside the residual-mode Newton loop, chosen at finalize from the
 * environment variable SNP_JACOBIAN ("elem" default, "csr", "sell"):
 *   SNP_LAYOUT_ELEM  matrix-free: per element the 3x3 symmetric tensor S_e with
 *                    J_e,jk = s_j s_k chat_j . S_e chat_k (first-order Nedelec, affine tets);
 *                    falls back to CSR when the orientation tables are not sign flips
 *   SNP_LAYOUT_CSR   assembled CSR on the solver's pattern
 *   SNP_LAYOUT_SELL  assembled SELL-C-sigma (C = 32, sigma = 256) copy of that pattern
 * Reference-semantics solves (mode 0) and snp_solver_assemble always use the CSR. */
#define SNP_LAYOUT_CSR 0
#define SNP_LAYOUT_SELL 1
#define SNP_LAYOUT_ELEM 2
int snp_solver_jacobian_layout(const snp_solver *s, int *layout);

/* Solve `count` independent problems concurrently: instance i runs snp_solver_solve(solvers[i],
 * x[i], &opts[i], &stats[i]) on its own host thread (at most n_threads at a time; <= 0: one
 * per instance), each on the stream its solver was created with, so the GPU overlaps the
 * instances' kernels.  status[i] (may be NULL) receives each instance's status; the return
 * value is the first failure's, with its message.  Solvers must be distinct and should have
 * distinct streams (a shared stream serialises them).  The reference solves one design per
 * process (red_mvp_solver.py:121-224); this is the batched form. */
int snp_solver_solve_many(snp_solver *const *solvers, int32_t count, double *const *x, const snp_solve_opts *opts,
                          snp_solve_stats *stats, int32_t n_threads, int32_t *status);

/* ------------------------------------------------------------------ batched Newton solver
 * Many problems of uneven size solved by one set of launches: the problems' elements and
 * DoFs are concatenated (each problem at its own element and DoF offset, padded to the
 * reduction units), every pass of the residual-mode Newton loop (element-tensor assembly,
 * block-Jacobi build, the PCG's element and DoF passes, the line search's trial points and
 * the Newton update) is one launch over all problems, each problem keeps its own Newton, CG
 * and line-search state on the device, and the whole Newton loop of all problems is one CUDA
 * graph (conditional WHILE nodes for the Newton, CG and line-search loops) launched once per
 * solve.  Every sum runs in a fixed order that depends only on the problem itself, so a
 * problem's answer is bitwise the same whatever else is in the batch.  The reference solves
 * one design per call (red_mvp_solver.py:121-224) and a design study loops over designs
 * (examples/plot_example_baseline.py:61-91); this is the batched form of that loop. */
typedef struct snp_batch snp_batch;

/* Build a batch over `count` finalized solvers with the matrix-free Jacobian layout
 * (SNP_LAYOUT_ELEM) and block Jacobi set (snp_solver_set_block_jacobi), all with the same
 * quadrature and orientation tables.  The batch reads each solver's mesh coordinates, source
 * fields, materials and extra rhs when it solves (later snp_solver_set_nodes / _set_source
 * calls are seen); the solvers must outlive the batch.  Allocates the concatenated arrays and
 * a CUDA stream of its own; synchronises. */
int snp_batch_create(snp_solver *const *solvers, int32_t count, snp_batch **out);

/* Residual-mode Newton (opts[i].mode must be 1; precision the same for all) of every problem at
 * once: x[i] (device, [n_dofs of problem i]) in = initial guess, out = solution; per-problem
 * stats and status (SNP_OK, SNP_NOT_CONVERGED, SNP_NAN_DETECTED, SNP_ZERO_PIVOT) as
 * snp_solver_solve reports them; Galerkin warm-start bases are not used.  Returns the first
 * failing problem's status.  Synchronises the device before it starts and its stream at the end. */
int snp_batch_solve(snp_batch *b, double *const *x, const snp_solve_opts *opts, snp_solve_stats *stats,
                    int32_t *status);

/* Autotuner: times the candidate launch shapes of the element pass (block size 128, 256 or
 * 512 threads) and of the batched assembly (grid of one or two waves of resident blocks) on
 * this batch and keeps the fastest for later solves.  The shapes change no arithmetic (every
 * reduction order is fixed by the data), only the time.  Synchronises. */
int snp_batch_tune(snp_batch *b, int32_t precision);

typedef struct {
    int32_t problems;
    int64_t dofs, elements;        /* concatenated, padding included */
    int32_t pass1_block;           /* element-pass block size in use */
    int32_t asm_waves;             /* assembly grid: waves of resident blocks */
    int32_t graph;                 /* 1 when the Newton loop runs as one CUDA graph */
    double tuned_pass1_us[3];      /* autotuner's timings of the element pass at 128/256/512 (0: not tuned) */
    double tuned_asm_us[2];        /* ... and of the assembly at one/two waves */
} snp_batch_info;
int snp_batch_get_info(const snp_batch *b, snp_batch_info *info);

int snp_batch_destroy(snp_batch *b);

/* Matrix-free Newton assembly at x (device, [n_dofs]): the element tensors of the Jacobian
 * (float64 for precision 0, float32 for 1; afterwards snp_solver_jacobian_apply with that
 * precision applies J(x)) and, when F is not NULL, the residual F = K(x) x - rhs(x) - rhs_extra
 * ([n_dofs], device).  Needs the SNP_LAYOUT_ELEM layout.  Replaces, for the Newton loop, the
 * K/dK/rhs assembly of compute_K_dK_Hcurl[_red] (fem_c/ctools.c:960-1388). */
int snp_solver_assemble_tensors(snp_solver *s, const double *x, int precision, double *F, void *stream);

/* y = J x on the free rows and columns (y = 0 on constrained rows) with the Newton Jacobian
 * the solver holds from its last solve, in the layout the solver's Krylov loop uses.
 * precision 0: the float64 Jacobian, x/y double[n]; precision 1: the float32 Jacobian of a
 * mixed-precision solve, x/y float[n].  SNP_BAD_ARGUMENT when no solve of that precision ran.
 * No counterpart in the reference (Jacobian-vector product of the Newton step). */
int snp_solver_jacobian_apply(snp_solver *s, int precision, const void *x, void *y, void *stream);

/* Galerkin (reduced) Newton system in the span of a basis V (device float32, row-major
 * [n_dofs][ldv], the first m <= 128 columns used) with the Jacobian of the last
 * snp_solver_assemble_tensors of that precision: Jr = V^T J V (device float64 [m][m],
 * row-major) and, when F is not NULL, g = V^T F (device float64 [m]), both over the free DoFs,
 * summed in float64 in a fixed order (deterministic).  Needs the SNP_LAYOUT_ELEM layout.  The
 * correction x + V c with Jr c = -g moves a warm start to the Newton point of the reduced
 * space.  No counterpart in the reference (it has no warm start). */
int snp_solver_reduced_system(snp_solver *s, int precision, const float *V, int32_t m, int64_t ldv, const double *F,
                              double *Jr, double *g, void *stream);

/* Block-Jacobi preconditioner for the residual-mode (mode 1) Krylov solves of the
 * SNP_LAYOUT_ELEM layout, in place of point Jacobi.  meta (HOST uint16[n_dofs]) partitions the
 * DoFs into blocks of 1..8 consecutive DoFs that never cross a multiple of 256:
 * meta[i] = (offset of DoF i in its block) | (block size << 8); a constrained DoF must be a
 * block of its own.  Before every Krylov solve the block-diagonal entries of the Newton
 * Jacobian are summed from the element tensors (per DoF row, fixed order), each block is
 * inverted by Cholesky in float64 (point Jacobi for a block with a pivot below 1e-12 of its
 * diagonal) and stored in float32; the DoF pass forms z = M r per block.  Deterministic.  For
 * edge DoFs numbered by their lower node, blocks of the edges that share that node halve the CG
 * iterations of the window-frame yoke.  meta = NULL goes back to point Jacobi.  The
 * reference-semantics mode keeps point Jacobi (red_mvp_solver.py:199 builds
 * M = diags(1 / diag(J))).  Synchronises (meta is checked and uploaded). */
int snp_solver_set_block_jacobi(snp_solver *s, const uint16_t *meta);

/* Krylov method of the residual-mode Newton steps (the reference's scipy cg in each Newton step,
 * red_mvp_solver.py:199-203): SNP_KRYLOV_CG (default) or SNP_KRYLOV_GMRES, restarted GMRES(restart)
 * with right preconditioning by the same block or point Jacobi, float64 only (a mixed-precision
 * solve with GMRES returns SNP_BAD_ARG), matrix-free Jacobian layout.  Each Arnoldi step counts as
 * one iteration in snp_solve_stats.cg_iterations. */
#define SNP_KRYLOV_CG 0
#define SNP_KRYLOV_GMRES 1
int snp_solver_set_krylov(snp_solver *s, int32_t method, int32_t restart);

/* z = M r (device float64 [n_dofs]) with the block Jacobi built from the element tensors of
 * the last snp_solver_assemble_tensors of that precision; *fallback_blocks (host, may be NULL)
 * receives the number of blocks inverted as point Jacobi.  Synchronises when fallback_blocks
 * is given.  No counterpart in the reference. */
int snp_solver_precond_apply(snp_solver *s, int precision, const double *r, double *z, int32_t *fallback_blocks,
                             void *stream);

/* The block-Jacobi rows built from the element tensors of the last snp_solver_assemble_tensors
 * of that precision: bmat (device f64 [n_dofs][8], row i = J_(i, b0 + c) over DoF i's block
 * starting at b0) and binv (device f32 [n_dofs][8], the rows of the block inverses); either
 * may be NULL.  Inspection and test entry. */
int snp_solver_block_jacobi_export(snp_solver *s, int precision, double *bmat, float *binv, void *stream);

/* HOST: c = -A^-1 g for the symmetric positive semi-definite m x m Galerkin system A (host
 * row-major) and g (host [m]); the solve snp_solver_solve applies to the reduced system of an
 * attached basis.  Cholesky of the Jacobi-scaled A; a direction whose pivot falls below 1e-10
 * of its diagonal (a dependent basis column) is left out (c = 0 there).  SNP_BAD_ARG for a
 * non-positive or non-finite diagonal entry. */
int snp_spd_solve(int32_t m, const double *A, const double *g, double *c);

/* Attach a basis (device float32, row-major [n_dofs][ldv], first m <= 128 columns) to the
 * solver's mode-1 solves: the start first takes up to `steps` Galerkin Newton steps
 * x += V c, (V^T J V) c = -V^T F (snp_solver_reduced_system; the m x m system by Cholesky on
 * the host), each undone and ending the corrections when it does not lower ||F_free||; the
 * res_ref drop rule then applies to the corrected start.  Without res_ref the convergence target
 * stays relative to the uncorrected start's ||F_free|| (stats.res0).  V
 * must stay valid while attached; V = NULL, m = 0 or steps = 0 detaches.  Needs the
 * SNP_LAYOUT_ELEM layout.  No counterpart in the reference. */
int snp_solver_set_galerkin_basis(snp_solver *s, const float *V, int32_t m, int64_t ldv, int32_t steps);

/* Replace the node coordinates (device f64[n_nodes][3]) of a solver's mesh: same topology,
 * moved nodes (a morphed geometry).  The CSR pattern, element topology and materials stay.
 * No counterpart in the reference (it rebuilds everything per geometry). */
int snp_solver_set_nodes(snp_solver *s, const double *nodes, void *stream);

/* Replace the source field of material `material` (device f64[n_elems][n_quad][3], the
 * material must have been added with one), e.g. after moving the coils or nodes. */
int snp_solver_set_source(snp_solver *s, int32_t material, const double *B_s, void *stream);

/* Diluted steel for material `material` (RedMVPSolverDiluted, snoopy/red_mvp_solver_diluted.py):
 * phi device f64[n_quad][4] (nodal basis at the quadrature points, copied) and dilution host
 * f64[4] = {c_num, m_num, c_den, m_den}; dilution NULL switches it off again.  Applies to a
 * material with a source field only, as in the reference.  Not while a solve is running. */
int snp_solver_set_dilution(snp_solver *s, int32_t material, const double *phi, const double *dilution);

/* The solver's CSR pattern (owned by the solver). */
int snp_solver_pattern(const snp_solver *s, const snp_pattern **pat);

int snp_solver_destroy(snp_solver *s);

/* ---------------------------------------------------------------- warm-start surrogate
 * Dense kernels of the learned warm start: an MLP that maps design parameters to POD
 * coefficients of the converged edge-DoF vector.  None has a counterpart in the reference
 * (snoo.py has no surrogate); BF16 arrays are passed as raw 16-bit words. */

/* POD reconstruction of the warm start (the surrogate's x = mean + U c, the projection GEMM of
 * the learned warm start; the reference has no surrogate): out[p][i] = mean[i] + sum_c V[i][c] coef[p][c] for
 * p < P (<= 32) vectors, V float32 [n][ldv] with m <= 128 columns, coef float64 [P][m] (device),
 * mean float64 [n] or NULL, out float64 [P][ldo].  float64 products and sums in a fixed order.
 * Asynchronous on the stream. */
int snp_basis_combine(int32_t n, const float *V, int32_t m, int64_t ldv, const double *coef, int32_t P,
                      const double *mean, double *out, int64_t ldo, void *stream);

/* C[M,N] = A[M,K] . B[N,K]^T (+ bias[N]) on the tcgen05 tensor cores: A, B row-major BF16
 * with K contiguous (K and lda, ldb multiples of 8, A and B 16-byte aligned), FP32
 * accumulation.  Outputs (either may be NULL): C FP32 [M, ldc]; H BF16 [M, ldh] = act(C)
 * with act 0 = identity, 1 = GELU (0.5 z (1 + erf(z / sqrt 2))).  *err (device int, caller
 * zeroes it) is set to 1 if a tensor-core wait timed out.  Asynchronous on the stream. */
int snp_gemm_bf16(int32_t M, int32_t N, int32_t K, const void *A, int32_t lda, const void *B, int32_t ldb,
                  const float *bias, int32_t act, float *C, int32_t ldc, void *H, int32_t ldh, int32_t *err,
                  void *stream);

/* dZ = dH * GELU'(Z), element-wise over count values; BF16 and/or FP32 output. */
int snp_gelu_backward(int64_t count, const float *dH, const float *Z, void *dZ_bf16, float *dZ_f32, void *stream);

/* out[c][r] = in[r][c] for a rows x cols BF16 matrix (row strides ldi, ldo). */
int snp_transpose_bf16(int32_t rows, int32_t cols, const void *in, int32_t ldi, void *out, int32_t ldo, void *stream);

/* out[c] = sum_r in[r][c] (FP32; bias gradients). */
int snp_col_sum(int32_t rows, int32_t cols, const float *in, int32_t ld, float *out, void *stream);

/* One Adam step (bias-corrected, step >= 1) on FP32 weights w with gradient g and moments m,
 * v; refreshes the BF16 copy w_bf16 when not NULL. */
int snp_adam_step(int64_t count, float *w, const float *g, float *m, float *v, void *w_bf16, float lr, float beta1,
                  float beta2, float eps, int32_t step, void *stream);

/* dY = scale * (Y - T) over count values (gradient of a mean-squared error), with an
 * optional BF16 copy. */
int snp_mse_grad(int64_t count, const float *Y, const float *T, float scale, float *dY, void *dY_bf16, void *stream);

/* BF16 (round to nearest even) copy of count FP32 values. */
int snp_f32_to_bf16(int64_t count, const float *in, void *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SNOOPY_B200_H */
