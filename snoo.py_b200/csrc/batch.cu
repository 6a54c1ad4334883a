// Batched residual-mode Newton solver (snp_batch_*): many problems of uneven size, one launch
// per pass over all of them, each problem's Newton, CG and line-search state on the device,
// and the whole Newton loop as one CUDA graph.
//
// The reference solves one magnet design per call (snoopy/red_mvp_solver.py:121-224) and a
// design study loops over designs (examples/plot_example_baseline.py:61-91).  Here the designs'
// element and DoF arrays are concatenated:
//
//   DoFs      problem p owns [dof_off_p, dof_off_p + n_p), padded to a multiple of kUnit (2048):
//             DoF-indexed kernels take one unit (8 tiles of 256 DoFs) per block iteration and
//             write one partial sum per unit.  Padding DoFs are constrained (free mask 0) and
//             have empty incidence ranges.
//   elements  problem p owns [elem_off_p, elem_off_p + ne_p), elem_off_p a multiple of kChunk
//             (1024): the element pass takes one chunk per block iteration and writes one
//             partial sum per chunk.  Per-element arrays keep the single-problem solver's
//             32-element blocks (eslot), copied at offset 6 elem_off_p.
//   incidence the problems' DoF-ordered incidence lists one after another, (e << 3 | k) with
//             the concatenated element index.
//
// Sums: the unit / chunk partials are summed per problem by the last block of the launch, one
// warp per problem, in the partials' order (lane-strided sequential sums, then a fixed shuffle
// tree).  None of a problem's sums depends on the other problems or on the launch shape, so a
// problem's iterates are bitwise those it has when solved alone in a batch of one.
//
// Newton loop (the single-problem solver's residual mode, csrc/solver.cu): Eisenstat-Walker
// inner tolerances, block-Jacobi PCG, the energy line search, the relative residual test, the
// drop rule for starts worse than res_ref.  Every decision is taken per problem on the device
// by the last block of the launch that produced its inputs; a WHILE node repeats the Newton,
// CG and line-search bodies while any problem needs them, and kernels skip the units and
// chunks of problems that do not.  Every loop is bounded: CG by its iteration cap, the line
// search by 12 trials, Newton by max_newton, and the Newton controller counts its passes.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "snp_common.cuh"
#include "snp_elem.cuh"
#include "snp_internal.cuh"
#include "snp_krylov.cuh"
#include "snp_reduce.cuh"

namespace snp {
namespace {

constexpr int kBB = kBjTile;             // threads of the DoF-indexed kernels (one block-Jacobi tile)
constexpr int kUnitTiles = 8;            // tiles per DoF partial-sum unit
constexpr int kUnit = kBB * kUnitTiles;  // DoFs per unit
constexpr int kChunk = 256;              // elements per element-pass partial-sum chunk (one warp's work)
constexpr int kGroup = 16;               // elements per warp step of the element pass (two lanes each)
constexpr int kGroups = kChunk / kGroup;

// CG outcome per problem (as the single-problem PcgState.done, plus idle and zero pivot)
enum : int { CG_RUN = 0, CG_CONV = 1, CG_MAXIT = 2, CG_NAN = 3, CG_ZERO_RHS = 4, CG_IDLE = 5, CG_PIVOT = 6 };

// Where each problem stands in its Newton loop.  Every pass of the solver's loop advances each
// problem by its own next step, so problems do not wait for one another:
//   HEAD     start of a Newton step: inner tolerance, block-Jacobi build, PCG start
//   CG       one PCG iteration per pass
//   EXTRACT  CG finished: the direction, the line search opened
//   LS       one trial point of the line search per pass
//   ACCEPT   the accepted trial point becomes x; converged, out of steps, or the next HEAD
enum : int { PH_DONE = 0, PH_HEAD = 1, PH_CG = 2, PH_EXTRACT = 3, PH_LS = 4, PH_ACCEPT = 5, PH_LIVE = 6 };

struct BInst {
    int32_t dof_off, n;
    int32_t unit0, n_units;
    int64_t elem_off, ne;
    int32_t chunk0, n_chunks;
    const double *rhs_extra;  // [n] or NULL
};

// Device state of one problem.  `run` (int32, first member so the assembly can stride over it)
// marks the problems that take part in the next assembly and residual sums.
struct BState {
    int32_t run;
    int32_t active, status, it, ls_it, res_evals, dropped, bad, line_search, max_newton, cg_done, ph;
    long long cg_iter, cg_maxit, cg_total;
    double rz, pq, alpha, beta, rr, bnorm, atol_eff;
    double fn, res0, F0, fprev, eta_prev, eta, tol, res_ref, eta_max;
    double g0, g, f2, alpha_ls, a_lo, g_lo, a_hi, g_hi;
};
static_assert(sizeof(BState) % 4 == 0, "BState is strided in int32 units");

struct BCtl {
    unsigned int counter;
    int any_active, any_cg, any_ls;
    unsigned long long launches;
    int passes;
    int fallback_blocks;
    int any_phase[8];  // per phase (PH_LIVE: any problem not done), for the host-driven loop
};

constexpr int kMaxPasses = 4000000;  // passes of the solver's loop before every problem is stopped

struct BOpts {
    double tol, res_ref, eta_max;
    long long cg_maxit;
    int max_newton, line_search;
};

// one count per launch (the kernels of this library executed by the solve)
__device__ __forceinline__ void count_launch(BCtl *ctl) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&ctl->launches, 1ull);
}

// Sum of part[(first + j) * width + comp], j < count, lane-strided sequential sums then a
// fixed shuffle tree: the same bits whichever warp computes it; every lane gets the result.
__device__ __forceinline__ double warp_ordered_sum(const double *part, int64_t first, int count, int width, int comp) {
    const int lane = threadIdx.x & 31;
    double v = 0.0;
    int j = lane;
    for (; j + 96 < count; j += 128) {
        const double a0 = __ldcg(part + (first + j) * width + comp);
        const double a1 = __ldcg(part + (first + j + 32) * width + comp);
        const double a2 = __ldcg(part + (first + j + 64) * width + comp);
        const double a3 = __ldcg(part + (first + j + 96) * width + comp);
        v += a0;
        v += a1;
        v += a2;
        v += a3;
    }
    for (; j < count; j += 32) v += __ldcg(part + (first + j) * width + comp);
    return warp_sum(v);
}

// ---------------------------------------------------------------- start of a solve

// x: zero on constrained and padding DoFs; per-problem state from the options
__global__ void k_b_init(int n_inst, const BOpts *__restrict__ opts, BState *__restrict__ st, int64_t n_tot,
                         const uint8_t *__restrict__ free_mask, double *__restrict__ x, BCtl *ctl) {
    count_launch(ctl);
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid < n_inst) {
        BState s;
        memset(&s, 0, sizeof(s));
        const BOpts o = opts[tid];
        s.run = 1;
        s.tol = o.tol;
        s.res_ref = o.res_ref;
        s.eta_max = o.eta_max;
        s.cg_maxit = o.cg_maxit;
        s.max_newton = o.max_newton;
        s.line_search = o.line_search;
        s.cg_done = CG_IDLE;
        s.status = SNP_OK;
        st[tid] = s;
    }
    if (tid == 0) {
        ctl->passes = 0;
        ctl->fallback_blocks = 0;
    }
    for (int64_t i = tid; i < n_tot; i += (int64_t)gridDim.x * blockDim.x)
        if (!free_mask[i]) x[i] = 0.0;
}

// x = 0 on the problems whose start was dropped (run set by the start controller)
__global__ void k_b_zero_run(const int32_t *__restrict__ unit_inst, int64_t n_units, const BState *__restrict__ st,
                             double *__restrict__ x, BCtl *ctl) {
    count_launch(ctl);
    for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
        if (!st[unit_inst[u]].run) continue;
        for (int k = threadIdx.x; k < kUnit; k += blockDim.x) x[u * kUnit + k] = 0.0;
    }
}

// ---------------------------------------------------------------- residual sums + controllers

enum : int { SUM_START = 0, SUM_DROP = 1, SUM_LS = 2 };

// Per DoF of the problems with run set: F = sum of the element terms - rhs_extra, diag(J) = sum
// of the diagonal terms (incidence order); per unit the free sums of F^2 and (line search) F.h.
// The last block finishes the controller step of MODE for every problem.
template <int MODE>
__global__ void __launch_bounds__(kBB)
    k_b_sum(int n_inst, const BInst *__restrict__ inst, const int32_t *__restrict__ unit_inst, int64_t n_units,
            const uint8_t *__restrict__ free_mask, const int32_t *__restrict__ inc_ptr,
            const int32_t *__restrict__ inc, const double *__restrict__ Fe, const double *__restrict__ De,
            const double *__restrict__ h, double *__restrict__ F, double *__restrict__ diag, BState *st,
            double *part, BCtl *ctl, int use_cond, cudaGraphConditionalHandle cond) {
    __shared__ double sh2[2][32];
    __shared__ int s_any;
    count_launch(ctl);
    for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
        const int p = unit_inst[u];
        if (!st[p].run) continue;  // uniform across the block
        const int32_t dof_off = inst[p].dof_off, n_p = inst[p].n;
        const double *rhs_extra = inst[p].rhs_extra;
        double f2 = 0.0, fh = 0.0;
        for (int t = 0; t < kUnitTiles; ++t) {
            const int64_t i = u * kUnit + t * kBB + threadIdx.x;
            double f = 0.0, d = 0.0;
            for (int k = inc_ptr[i]; k < inc_ptr[i + 1]; ++k) {
                const uint32_t w = (uint32_t)inc[k] & ~kSignBit;
                const int64_t idx = eslot((int64_t)(w >> 3), (int)(w & 7u));
                f += Fe[idx];
                d += De[idx];
            }
            const int64_t loc = i - dof_off;
            if (rhs_extra && loc < n_p) f -= rhs_extra[loc];
            F[i] = f;
            diag[i] = d;
            if (free_mask[i]) {
                f2 += f * f;
                if (MODE == SUM_LS) fh += f * h[i];
            }
        }
        block_sum2(f2, fh, sh2);
        if (threadIdx.x == 0) {
            part[2 * u] = f2;
            part[2 * u + 1] = fh;
        }
        __syncthreads();
    }
    if (!last_block(&ctl->counter)) return;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int p = warp; p < n_inst; p += nw) {
        BState &s = st[p];
        const bool ran = s.run != 0;
        double f2 = 0.0, fh = 0.0;
        if (ran) {
            f2 = warp_ordered_sum(part, inst[p].unit0, inst[p].n_units, 2, 0);
            fh = warp_ordered_sum(part, inst[p].unit0, inst[p].n_units, 2, 1);
        }
        if (lane != 0) continue;
        if (MODE == SUM_START) {
            s.f2 = f2;
            s.res0 = sqrt(f2);
            s.fn = s.res0;
            // a start worse than x = 0 (by the zero-start residual, up to rounding of the two
            // evaluations) is dropped for x = 0
            s.dropped = (s.res_ref > 0.0 && !(s.fn <= s.res_ref * (1.0 + 1e-9))) ? 1 : 0;
            s.run = s.dropped;
        } else if (MODE == SUM_DROP) {
            if (ran) {
                s.f2 = f2;
                s.fn = sqrt(f2);
            }
            s.run = 0;
            s.F0 = s.res_ref > 0.0 ? s.res_ref : s.res0;
            if (!(s.fn == s.fn)) {
                s.status = SNP_NAN_DETECTED;
                s.active = 0;
            } else {
                s.active = (s.F0 == 0.0 || s.fn <= s.tol * s.F0) ? 0 : 1;
            }
            s.ph = s.active ? PH_HEAD : PH_DONE;
            if (s.active) atomicOr(&s_any, 1);
        } else {  // SUM_LS: one trial point of the line search
            if (!ran) continue;
            s.f2 = f2;
            s.g = fh;
            if (s.ls_it > 0) s.res_evals += 1;
            bool accept = !s.line_search;
            if (!accept) {
                // the full step is kept unless it overshoots (slope above +0.5 |phi'(0)|); inside
                // the bracket a trial must have |phi'| <= 0.5 |phi'(0)|, an undershoot raising the
                // lower end and an overshoot lowering the upper end
                const double g = fh, c = 0.5 * fabs(s.g0);
                if (!(g == g) || s.ls_it >= 11) accept = true;
                else if (s.ls_it == 0 ? !(g > c) : fabs(g) <= c) accept = true;
                if (!accept) {
                    if (g < -c) {
                        s.a_lo = s.alpha_ls;
                        s.g_lo = g;
                    } else {
                        s.a_hi = s.alpha_ls;
                        s.g_hi = g;
                    }
                    const double a_new = s.a_lo - s.g_lo * (s.a_hi - s.a_lo) / (s.g_hi - s.g_lo);
                    const double width = s.a_hi - s.a_lo;
                    s.alpha_ls = fmin(fmax(a_new, s.a_lo + 0.01 * width), s.a_hi - 0.01 * width);
                }
            }
            s.ls_it += 1;
            s.run = accept ? 0 : 1;
            if (accept) s.ph = PH_ACCEPT;
            if (!accept) atomicOr(&s_any, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int any = s_any;
        if (MODE == SUM_DROP) ctl->any_active = any;
        if (MODE == SUM_LS) ctl->any_ls = any;
        if (MODE != SUM_START && use_cond) cudaGraphSetConditional(cond, any ? 1u : 0u);
    }
}

// ---------------------------------------------------------------- Newton step

// Inner tolerance of every active problem (Eisenstat-Walker choice 2 with the safeguards of the
// single-problem solver); idle CG for the others.
__global__ void k_b_step_begin(int n_inst, BState *st, int f32, BCtl *ctl) {
    count_launch(ctl);
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_inst) return;
    BState &s = st[p];
    if (s.ph != PH_HEAD) return;
    double eta = s.eta_max;
    if (s.it > 0) {
        const double ratio = s.fn / s.fprev;
        eta = 0.9 * ratio * ratio;
        const double sg = 0.9 * s.eta_prev * s.eta_prev;
        if (sg > 0.1 && sg > eta) eta = sg;
        if (eta > s.eta_max) eta = s.eta_max;
    }
    const double floor_eta = 0.5 * s.tol * s.F0 / s.fn;
    if (eta < floor_eta) eta = floor_eta;
    if (f32 && eta < 1e-6) eta = 1e-6;
    if (eta > 0.5) eta = 0.5;
    s.fprev = s.fn;
    s.eta_prev = eta;
    s.eta = eta;
    s.bad = 0;
    s.cg_done = CG_RUN;
}

// block-Jacobi rows of the active problems' DoFs
template <typename TT>
__global__ void __launch_bounds__(kBB)
    k_b_bj_entries(int64_t n_tot, const int32_t *__restrict__ unit_inst, const BState *__restrict__ st,
                   const uint8_t *__restrict__ free_mask, const int32_t *__restrict__ inc_ptr,
                   const int32_t *__restrict__ inc, const int32_t *__restrict__ edof, const TT *__restrict__ T,
                   const TT *__restrict__ chat, const uint16_t *__restrict__ meta, double *__restrict__ bmat,
                   BCtl *ctl) {
    __shared__ double sc[18];
    count_launch(ctl);
    if (threadIdx.x < 18) sc[threadIdx.x] = (double)chat[threadIdx.x];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_tot; i += (int64_t)gridDim.x * blockDim.x) {
        if (st[unit_inst[i / kUnit]].ph != PH_HEAD) continue;
        double row[kBjMax];
#pragma unroll
        for (int c = 0; c < kBjMax; ++c) row[c] = 0.0;
        if (free_mask[i]) bj_entries_row(i, inc_ptr, inc, edof, T, sc, (unsigned)meta[i], row);
#pragma unroll
        for (int c = 0; c < kBjMax; ++c) bmat[i * kBjMax + c] = row[c];
    }
}

__global__ void __launch_bounds__(128)
    k_b_bj_invert(int64_t n_tot, const int32_t *__restrict__ unit_inst, const BState *__restrict__ st,
                  const uint8_t *__restrict__ free_mask, const uint16_t *__restrict__ meta,
                  const double *__restrict__ bmat, float *__restrict__ binv, BCtl *ctl) {
    count_launch(ctl);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_tot; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned mt = meta[i];
        if (mt & 0xffu) continue;
        if (st[unit_inst[i / kUnit]].ph != PH_HEAD) continue;
        bj_invert_block(i, (int)(mt >> 8), free_mask[i] != 0, free_mask, bmat, binv, &ctl->fallback_blocks);
    }
}

// PCG start of every active problem: r = -F, z = M r (block Jacobi), x = 0 (R.b), p = 0 (G.b);
// the last block sets each problem's tolerance (rtol = eta) and its CG status.
template <typename TT>
__global__ void __launch_bounds__(kBB)
    k_b_pcg_init(int n_inst, const BInst *__restrict__ inst, const int32_t *__restrict__ unit_inst, int64_t n_units,
                 const uint8_t *__restrict__ free_mask, const double *__restrict__ F, const double *__restrict__ diag,
                 const uint16_t *__restrict__ meta, const float *__restrict__ binv, DofPair<TT> *__restrict__ G,
                 DofPair<TT> *__restrict__ R, BState *st, double *part, BCtl *ctl, int use_cond,
                 cudaGraphConditionalHandle cond) {
    __shared__ double sh2[2][32];
    __shared__ TT s_r[kBB];
    __shared__ int s_any;
    count_launch(ctl);
    for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
        const int p = unit_inst[u];
        if (st[p].ph != PH_HEAD) continue;  // uniform across the block
        double rz = 0.0, rr = 0.0;
        int bad = 0;
        for (int t = 0; t < kUnitTiles; ++t) {
            const int64_t i = u * kUnit + t * kBB + threadIdx.x;
            const bool fr = free_mask[i] != 0;
            TT r = TT(0);
            unsigned mt = 0;
            float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
            if (fr) {
                const double dg = diag[i];
                if (dg == 0.0 || !isfinite(dg)) bad = 1;
                r = (TT)(-F[i]);
                mt = meta[i];
                bj_load(binv, i, ma, mb);
            }
            s_r[threadIdx.x] = r;
            __syncthreads();
            const TT z = fr ? bj_row(mt, ma, mb, s_r, threadIdx.x) : TT(0);
            G[i] = DofPair<TT>{z, TT(0)};
            R[i] = DofPair<TT>{r, TT(0)};
            rz += (double)r * (double)z;
            rr += (double)r * (double)r;
            __syncthreads();
        }
        if (bad) atomicExch(&st[p].bad, 1);
        block_sum2(rz, rr, sh2);
        if (threadIdx.x == 0) {
            part[2 * u] = rz;
            part[2 * u + 1] = rr;
        }
        __syncthreads();
    }
    if (!last_block(&ctl->counter)) return;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int p = warp; p < n_inst; p += nw) {
        BState &s = st[p];
        if (s.ph != PH_HEAD) continue;
        const double rz = warp_ordered_sum(part, inst[p].unit0, inst[p].n_units, 2, 0);
        const double rr = warp_ordered_sum(part, inst[p].unit0, inst[p].n_units, 2, 1);
        if (lane != 0) continue;
        s.rz = rz;
        s.rr = rr;
        s.bnorm = sqrt(rr);
        s.atol_eff = s.eta * s.bnorm;
        s.cg_iter = 0;
        s.alpha = 0.0;
        s.beta = 0.0;
        int done = CG_RUN;
        if (s.bad) done = CG_PIVOT;
        else if (rr == 0.0) done = CG_ZERO_RHS;
        else if (!(rr == rr) || isinf(rr)) done = CG_NAN;
        else if (sqrt(rr) < s.atol_eff) done = CG_CONV;
        else if (s.cg_maxit <= 0) done = CG_MAXIT;
        s.cg_done = done;
        s.ph = done == CG_RUN ? PH_CG : PH_EXTRACT;
        if (done == CG_RUN) atomicOr(&s_any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->any_cg = s_any;
        if (use_cond) cudaGraphSetConditional(cond, s_any ? 1u : 0u);
    }
}

// The problems in their CG phase, compacted for the CG passes (k_b_cg_list, once per CG phase
// node): act[0] = m, act[1 + j] = the j-th such problem (problem order), act[1 + n_inst + j] and
// act[2 + 2 n_inst + j] the prefix sums of their units and chunks (m + 1 entries each).  The
// passes walk only those units and chunks, so a pass with one problem left costs that problem's
// work and not a sweep over every problem's.  A problem that leaves CG during the unrolled CG
// iterations of the node stays listed and is skipped by its phase test.
inline int act_size(int n_inst) { return 3 + 3 * n_inst; }

__global__ void k_b_cg_list(int n_inst, const BInst *__restrict__ inst, const BState *__restrict__ st,
                            int32_t *__restrict__ act, BCtl *ctl) {
    count_launch(ctl);
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int32_t *ids = act + 1, *up = act + 1 + n_inst, *cp = act + 2 + 2 * n_inst;
    int m = 0;
    up[0] = 0;
    cp[0] = 0;
    for (int p = 0; p < n_inst; ++p) {
        if (st[p].ph != PH_CG) continue;
        ids[m] = p;
        up[m + 1] = up[m] + inst[p].n_units;
        cp[m + 1] = cp[m] + inst[p].n_chunks;
        ++m;
    }
    act[0] = m;
}

// the listed problem j (< m) whose prefix range [pre[j], pre[j + 1]) holds k
__device__ __forceinline__ int act_find(const int32_t *__restrict__ pre, int m, int64_t k) {
    int lo = 0, hi = m;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= k) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Element pass of a CG iteration over the chunks of the problems still iterating: as the
// single-problem k_epass1 (two lanes per element, three edges each).  Four warps of a block
// share a chunk, four steps of 16 elements each (so that one problem left alone still has a
// warp per 64 elements); each step's p.Jp partial is summed by a fixed shuffle tree and added to
// the warp's sum in step order, and the chunk's sum is the four warps' sums added in warp order
// (shared memory, one block barrier per chunk step): fixed whatever the batch and launch shape.
constexpr int kSplit = 4;                     // warps per chunk
constexpr int kWarpGroups = kGroups / kSplit;  // steps per warp
template <typename TT, int BS>
__global__ void __launch_bounds__(BS, 1024 / BS)
    k_b_pass1(int n_inst, const BInst *__restrict__ inst, const int32_t *__restrict__ act,
              const int32_t *__restrict__ edof, const int32_t *__restrict__ pos, const TT *__restrict__ T,
              const TT *__restrict__ chat, const DofPair<TT> *__restrict__ G, TT *__restrict__ Y, BState *st,
              double *part, BCtl *ctl) {
    __shared__ TT sc[18];
    count_launch(ctl);
    if (threadIdx.x < 18) sc[threadIdx.x] = chat[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int h = lane & 1;  // edges 3h .. 3h+2
    const int warp = threadIdx.x >> 5;
    constexpr int kWarps = BS / 32;
    // as the single solver's element pass: a group's streamed words are requested before its
    // gathers, the chunk's first group's before its problem's state is read (every padded chunk
    // position is allocated, so the words are read unconditionally and used only for elements of
    // the problem), and in float32 each group's words one group ahead
    constexpr bool kAhead = sizeof(TT) == 4;
    int32_t d[3], ps[3], nd[3], nps[3];
    TT th[3], nth[3];
    auto stream_in = [&](int64_t c, int g, int32_t(&od)[3], int32_t(&ops)[3], TT(&oth)[3]) {
        const int64_t eb = eslot(c * kChunk + g * kGroup + (lane >> 1), 0);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            od[j] = __ldcs(edof + eb + 32 * (3 * h + j));
            ops[j] = __ldcs(pos + eb + 32 * (3 * h + j));
            oth[j] = __ldcs(T + eb + 32 * (3 * h + j));
        }
    };
    __shared__ double s_acc[kWarps];
    const int m = act[0];
    const int32_t *cpre = act + 2 + 2 * n_inst;
    const int64_t total = cpre[m];
    constexpr int kPerStep = kWarps / kSplit;  // chunks per block step
    const int q = warp % kSplit;               // this warp's quarter of its chunk
    for (int64_t kb = (int64_t)blockIdx.x * kPerStep; kb < total; kb += (int64_t)gridDim.x * kPerStep) {
        const int64_t k = kb + warp / kSplit;
        bool active = k < total;
        int p = 0;
        int64_t c = 0;
        if (active) {
            const int j = act_find(cpre, m, k);
            p = act[1 + j];
            c = inst[p].chunk0 + (k - cpre[j]);
            stream_in(c, q * kWarpGroups, d, ps, th);
            active = st[p].ph == PH_CG;  // uniform across the warp
        }
        double acc = 0.0;
        if (active) {
            const TT beta = (TT)st[p].beta;
            const int64_t e_end = inst[p].elem_off + inst[p].ne;
#pragma unroll 1
            for (int g = q * kWarpGroups; g < (q + 1) * kWarpGroups; ++g) {
                const int64_t e = c * kChunk + g * kGroup + (lane >> 1);
                const bool valid = e < e_end;
                if constexpr (kAhead) {
                    if (g > q * kWarpGroups) {
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            d[j] = nd[j];
                            ps[j] = nps[j];
                            th[j] = nth[j];
                        }
                    }
                    if (g + 1 < (q + 1) * kWarpGroups) stream_in(c, g + 1, nd, nps, nth);
                } else {
                    if (g > q * kWarpGroups) stream_in(c, g, d, ps, th);
                }
                DofPair<TT> w[3];
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    w[j] = valid ? G[(uint32_t)d[j] & ~kSignBit] : DofPair<TT>{TT(0), TT(0)};
                TT u0 = TT(0), u1 = TT(0), u2 = TT(0);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    TT pk = pnext(beta, w[j].b, w[j].a);
                    if (d[j] < 0) pk = -pk;
                    const TT *cc = sc + 3 * (3 * h + j);
                    u0 += pk * cc[0];
                    u1 += pk * cc[1];
                    u2 += pk * cc[2];
                }
                if (!valid) u0 = u1 = u2 = TT(0);
                // u_e = (edges 0-2) + (edges 3-5), added in that order on both lanes
                const TT o0 = __shfl_xor_sync(0xffffffffu, u0, 1);
                const TT o1 = __shfl_xor_sync(0xffffffffu, u1, 1);
                const TT o2 = __shfl_xor_sync(0xffffffffu, u2, 1);
                if (h) {
                    u0 = o0 + u0;
                    u1 = o1 + u1;
                    u2 = o2 + u2;
                } else {
                    u0 = u0 + o0;
                    u1 = u1 + o1;
                    u2 = u2 + o2;
                }
                TT t[6];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const TT other = __shfl_xor_sync(0xffffffffu, th[j], 1);
                    t[j] = h ? other : th[j];
                    t[3 + j] = h ? th[j] : other;
                }
                const TT v0 = t[0] * u0 + t[1] * u1 + t[2] * u2;
                const TT v1 = t[1] * u0 + t[3] * u1 + t[4] * u2;
                const TT v2 = t[2] * u0 + t[4] * u1 + t[5] * u2;
                double dot = 0.0;
                if (valid && !h) dot = (double)u0 * (double)v0 + (double)u1 * (double)v1 + (double)u2 * (double)v2;
                if (valid) {
#pragma unroll
                    for (int j = 0; j < 3; ++j) Y[ps[j]] = edge_term(sc, 3 * h + j, d[j] < 0, v0, v1, v2);
                }
                acc += warp_sum(dot);
            }
        }
        if (lane == 0) s_acc[warp] = acc;
        __syncthreads();
        if (active && q == 0 && lane == 0)
            part[c] = ((s_acc[warp] + s_acc[warp + 1]) + s_acc[warp + 2]) + s_acc[warp + 3];
        __syncthreads();
    }
    if (!last_block(&ctl->counter)) return;
    const int nw = blockDim.x >> 5;
    for (int p = warp; p < n_inst; p += nw) {
        BState &s = st[p];
        if (s.ph != PH_CG) continue;
        const double pq = warp_ordered_sum(part, inst[p].chunk0, inst[p].n_chunks, 1, 0);
        if (lane == 0) {
            s.pq = pq;
            s.alpha = s.rz / pq;
        }
    }
}

// DoF pass of a CG iteration over the units of the problems still iterating: q_i = sum of the
// DoF's slots, r -= alpha q, z = M r over the DoF's block (the tile's r in shared memory),
// p = z + beta p, x += alpha p; the last block moves each problem's CG state on.
template <typename TT>
__global__ void __launch_bounds__(kBB)
    k_b_pass2(int n_inst, const BInst *__restrict__ inst, const int32_t *__restrict__ act,
              const uint8_t *__restrict__ free_mask, const int32_t *__restrict__ inc_ptr, const TT *__restrict__ Y,
              const uint16_t *__restrict__ meta, const float *__restrict__ binv, DofPair<TT> *__restrict__ G,
              DofPair<TT> *__restrict__ R, BState *st, double *part, BCtl *ctl, int use_cond,
              cudaGraphConditionalHandle cond) {
    __shared__ double sh2[2][32];
    __shared__ TT s_r[kBB];
    __shared__ int s_any;
    count_launch(ctl);
    const int m = act[0];
    const int32_t *upre = act + 1 + n_inst;
    const int64_t total = upre[m];
    for (int64_t k = blockIdx.x; k < total; k += gridDim.x) {
        const int j = act_find(upre, m, k);
        const int p = act[1 + j];
        const int64_t u = inst[p].unit0 + (k - upre[j]);
        // as the single solver's DoF pass: each tile's slot range one tile ahead (the unit's first
        // before its problem's state is read), in float32 the DoF states too, the DoF's other
        // words before the slot values
        constexpr bool kStateAhead = sizeof(TT) == 4;
        int nb0, nb1;
        DofPair<TT> ng{TT(0), TT(0)}, nrx{TT(0), TT(0)};
        {
            const int64_t i0 = u * kUnit + threadIdx.x;
            nb0 = __ldcs(inc_ptr + i0);
            nb1 = __ldcs(inc_ptr + i0 + 1);
            if constexpr (kStateAhead) {
                ng = G[i0];
                nrx = R[i0];
            }
        }
        if (st[p].ph != PH_CG) continue;  // uniform across the block
        const TT alpha = (TT)st[p].alpha, beta = (TT)st[p].beta;
        double rz = 0.0, rr = 0.0;
        for (int t = 0; t < kUnitTiles; ++t) {
            const int64_t i = u * kUnit + t * kBB + threadIdx.x;
            const bool fr = free_mask[i] != 0;
            const int b0 = nb0, b1 = nb1;
            DofPair<TT> g = ng, rx = nrx;
            if (t + 1 < kUnitTiles) {
                nb0 = __ldcs(inc_ptr + i + kBB);
                nb1 = __ldcs(inc_ptr + i + kBB + 1);
                if constexpr (kStateAhead) {
                    ng = G[i + kBB];
                    nrx = R[i + kBB];
                }
            }
            if constexpr (!kStateAhead) {
                if (fr) {
                    g = G[i];
                    rx = R[i];
                }
            }
            TT r = TT(0);
            unsigned mt = 0;
            float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
            if (fr) {
                mt = meta[i];
                if constexpr (sizeof(TT) == 4) bj_load(binv, i, ma, mb);
                else bj_prefetch(binv, i);
                double q = 0.0;
                for (int k = b0; k < b1; ++k) q += (double)Y[k];
                r = rx.a - alpha * (TT)q;
            }
            s_r[threadIdx.x] = r;
            __syncthreads();
            if (fr) {
                if constexpr (sizeof(TT) == 8) bj_load(binv, i, ma, mb);
                const TT z = bj_row(mt, ma, mb, s_r, threadIdx.x);
                const TT pp = pnext(beta, g.b, g.a);
                G[i] = DofPair<TT>{z, pp};
                R[i] = DofPair<TT>{r, rx.b + alpha * pp};
                rz += (double)r * (double)z;
                rr += (double)r * (double)r;
            }
            __syncthreads();
        }
        block_sum2(rz, rr, sh2);
        if (threadIdx.x == 0) {
            part[2 * u] = rz;
            part[2 * u + 1] = rr;
        }
        __syncthreads();
    }
    if (!last_block(&ctl->counter)) return;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int p = warp; p < n_inst; p += nw) {
        BState &s = st[p];
        if (s.ph != PH_CG) continue;
        const double rz_new = warp_ordered_sum(part, inst[p].unit0, inst[p].n_units, 2, 0);
        const double rr_new = warp_ordered_sum(part, inst[p].unit0, inst[p].n_units, 2, 1);
        if (lane != 0) continue;
        s.beta = rz_new / s.rz;
        s.rz = rz_new;
        s.rr = rr_new;
        s.cg_iter += 1;
        int done = CG_RUN;
        if (!(rr_new == rr_new) || isinf(rr_new)) done = CG_NAN;
        else if (sqrt(rr_new) < s.atol_eff) done = CG_CONV;
        else if (s.cg_iter >= s.cg_maxit) done = CG_MAXIT;
        s.cg_done = done;
        if (done != CG_RUN) s.ph = PH_EXTRACT;
        if (done == CG_RUN) atomicOr(&s_any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->any_cg = s_any;
        if (use_cond && !s_any) cudaGraphSetConditional(cond, 0u);
    }
}

// Newton direction h = the CG iterate (active problems) and g0 = F.h; the last block ends each
// problem's CG (non-finite residual: the problem stops with SNP_NAN_DETECTED, a zero pivot with
// SNP_ZERO_PIVOT) and opens its line search.
template <typename TT>
__global__ void __launch_bounds__(kBB)
    k_b_extract(int n_inst, const BInst *__restrict__ inst, const int32_t *__restrict__ unit_inst, int64_t n_units,
                const uint8_t *__restrict__ free_mask, const DofPair<TT> *__restrict__ R, const double *__restrict__ F,
                double *__restrict__ h, BState *st, double *part, BCtl *ctl, int use_cond,
                cudaGraphConditionalHandle cond) {
    __shared__ double sh[32];
    __shared__ int s_any;
    count_launch(ctl);
    for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
        const int p = unit_inst[u];
        if (st[p].ph != PH_EXTRACT) continue;  // uniform across the block
        double fh = 0.0;
        for (int t = 0; t < kUnitTiles; ++t) {
            const int64_t i = u * kUnit + t * kBB + threadIdx.x;
            const double hv = (double)R[i].b;
            h[i] = hv;
            if (free_mask[i]) fh += F[i] * hv;
        }
        fh = block_sum(fh, sh);
        if (threadIdx.x == 0) part[u] = fh;
        __syncthreads();
    }
    if (!last_block(&ctl->counter)) return;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int p = warp; p < n_inst; p += nw) {
        BState &s = st[p];
        if (s.ph != PH_EXTRACT) continue;
        const double g0 = warp_ordered_sum(part, inst[p].unit0, inst[p].n_units, 1, 0);
        if (lane != 0) continue;
        s.cg_total += s.cg_iter;
        if (s.cg_done == CG_NAN) {
            s.status = SNP_NAN_DETECTED;
            s.active = 0;
            s.ph = PH_DONE;
            s.it += 1;
            continue;
        }
        if (s.cg_done == CG_PIVOT) {
            s.status = SNP_ZERO_PIVOT;
            s.active = 0;
            s.ph = PH_DONE;
            continue;
        }
        s.g0 = s.line_search ? g0 : 0.0;
        s.alpha_ls = 1.0;
        s.a_lo = 0.0;
        s.g_lo = s.g0;
        s.a_hi = 1.0;
        s.g_hi = 0.0;
        s.ls_it = 0;
        s.run = 1;
        s.ph = PH_LS;
        atomicOr(&s_any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->any_ls = s_any;
        if (use_cond) cudaGraphSetConditional(cond, s_any ? 1u : 0u);
    }
}

// trial point xw = x + alpha h on the free DoFs of the problems still searching
__global__ void __launch_bounds__(kBB)
    k_b_axpy(const int32_t *__restrict__ unit_inst, int64_t n_units, const uint8_t *__restrict__ free_mask,
             const double *__restrict__ x, const double *__restrict__ h, double *__restrict__ xw,
             const BState *__restrict__ st, BCtl *ctl) {
    count_launch(ctl);
    for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
        const int p = unit_inst[u];
        if (!st[p].run) continue;
        const double a = st[p].alpha_ls;
        for (int t = 0; t < kUnitTiles; ++t) {
            const int64_t i = u * kUnit + t * kBB + threadIdx.x;
            xw[i] = free_mask[i] ? x[i] + a * h[i] : x[i];
        }
    }
}

// x = the accepted trial point; the last block takes each active problem's Newton decision
__global__ void __launch_bounds__(kBB)
    k_b_accept(int n_inst, const int32_t *__restrict__ unit_inst, int64_t n_units, const double *__restrict__ xw,
               double *__restrict__ x, BState *st, BCtl *ctl, int use_cond, cudaGraphConditionalHandle cond) {
    __shared__ int s_any;
    count_launch(ctl);
    for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
        const int p = unit_inst[u];
        if (st[p].ph != PH_ACCEPT) continue;
        for (int t = 0; t < kUnitTiles; ++t) {
            const int64_t i = u * kUnit + t * kBB + threadIdx.x;
            x[i] = xw[i];
        }
    }
    if (!last_block(&ctl->counter)) return;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    const bool stop_all = ctl->passes >= kMaxPasses;
    for (int p = threadIdx.x; p < n_inst; p += blockDim.x) {
        BState &s = st[p];
        if (s.ph != PH_ACCEPT) continue;
        s.fn = sqrt(s.f2);
        s.it += 1;
        if (!(s.fn == s.fn)) {
            s.status = SNP_NAN_DETECTED;
            s.active = 0;
        } else if (s.F0 == 0.0 || s.fn <= s.tol * s.F0) {
            s.active = 0;
        } else if (s.it >= s.max_newton || stop_all) {
            s.status = SNP_NOT_CONVERGED;
            s.active = 0;
        }
        s.ph = s.active ? PH_HEAD : PH_DONE;
        if (s.active) atomicOr(&s_any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->any_active = s_any;
        if (use_cond) cudaGraphSetConditional(cond, s_any ? 1u : 0u);
    }
}

// Whether any problem stands at `phase` (PH_LIVE: any problem not done): the condition of the
// next IF node (or of the loop's WHILE node), and the host-driven loop's flag.  With PH_LIVE it
// also counts the loop's passes and, past kMaxPasses, stops every problem.
__global__ void k_b_flag(int n_inst, BState *st, int phase, BCtl *ctl, int use_cond, cudaGraphConditionalHandle cond) {
    __shared__ int s_any;
    count_launch(ctl);
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    const bool stop = phase == PH_LIVE && ctl->passes >= kMaxPasses;
    for (int p = threadIdx.x; p < n_inst; p += blockDim.x) {
        BState &s = st[p];
        if (stop && s.ph != PH_DONE) {
            s.status = SNP_NOT_CONVERGED;
            s.active = 0;
            s.run = 0;
            s.ph = PH_DONE;
        }
        const bool hit = phase == PH_LIVE ? s.ph != PH_DONE : s.ph == phase;
        if (hit) atomicOr(&s_any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (phase == PH_LIVE) ctl->passes += 1;
        ctl->any_phase[phase] = s_any;
        if (use_cond) cudaGraphSetConditional(cond, s_any ? 1u : 0u);
    }
}

// every problem takes part in the next assembly (the autotuner's timing of it)
__global__ void k_b_set_run(int n_inst, BState *st) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_inst; p += gridDim.x * blockDim.x) st[p].run = 1;
}

// ---------------------------------------------------------------- batch build

enum : int { CP_EDOF = 0, CP_ADD = 1, CP_INC = 2 };

// out[i] = in[i] shifted: CP_EDOF DoF part + add (sign kept), CP_ADD + add,
// CP_INC (e << 3 | k | sign) with e + eadd
__global__ void k_b_copy_shift(int64_t m, const int32_t *__restrict__ in, int32_t *__restrict__ out, int mode,
                               int64_t add, int64_t eadd) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)in[t];
        uint32_t o;
        if (mode == CP_EDOF) o = (uint32_t)((int64_t)(v & ~kSignBit) + add) | (v & kSignBit);
        else if (mode == CP_ADD) o = (uint32_t)((int64_t)v + add);
        else o = ((((v & ~kSignBit) >> 3) + (uint32_t)eadd) << 3 | (v & 7u)) | (v & kSignBit);
        out[t] = (int32_t)o;
    }
}

__global__ void k_b_fill_i32(int64_t m, int32_t *out, int32_t v) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) out[t] = v;
}

__global__ void k_b_fill_u16(int64_t m, uint16_t *out, uint16_t v) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) out[t] = v;
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

}  // namespace
}  // namespace snp

struct snp_batch {
    int32_t count = 0;
    std::vector<snp::SolverView> views;
    std::vector<snp::BInst> h_inst;
    int64_t n_tot = 0, e_tot = 0, inc_tot = 0, n_units = 0, n_chunks = 0;
    int32_t nq = 0, n_orient = 0, max_n_int = 1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    snp::DevBuf<snp::BInst> inst;
    snp::DevBuf<snp::BState> st;
    snp::HostBuf<snp::BState> hst;
    snp::DevBuf<snp::BOpts> opts;
    snp::DevBuf<snp::BCtl> ctl;
    snp::HostBuf<snp::BCtl> hctl;
    snp::DevBuf<int32_t> unit_inst, chunk_inst, edof, pos, inc, inc_ptr;
    snp::DevBuf<int32_t> act;  // the problems in CG, compacted (k_b_cg_list)
    snp::DevBuf<uint8_t> free_mask;
    snp::DevBuf<uint16_t> meta;
    snp::DevBuf<double> x, xw, h, F, diag, Fe, De, bmat, part;
    snp::DevBuf<float> binv;
    snp::DevBuf<double> T;       // float64 tensors, or float32 in the same bytes
    snp::DevBuf<double> Gv, Rv;  // DofPair<double>, or DofPair<float> in the same bytes
    snp::DevBuf<double> Y;
    snp::DevBuf<double> chat64;
    snp::DevBuf<float> chat32;
    snp::DevBuf<snp::BatchSeg> segs;
    snp::DevBuf<snp::BatchAsmItem> items;
    int32_t n_items = 0;
    const double *ctab = nullptr, *dphi = nullptr, *w = nullptr;
    // launch shapes (autotuner)
    int pass1_block = 256, asm_waves = 1;
    double tuned_pass1_us[3] = {0, 0, 0}, tuned_asm_us[2] = {0, 0};
    // one graph per precision, rebuilt when the launch shapes change
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int graph_shape[2][2] = {{0, 0}, {0, 0}};
    bool use_graph = true;

    ~snp_batch() {
        drop_graphs();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graphs() {
        for (int k = 0; k < 2; ++k) {
            if (exec[k]) cudaGraphExecDestroy(exec[k]);
            if (graph[k]) cudaGraphDestroy(graph[k]);
            exec[k] = nullptr;
            graph[k] = nullptr;
        }
    }

    template <typename TT>
    TT *Tp() { return reinterpret_cast<TT *>(T.p); }
    template <typename TT>
    snp::DofPair<TT> *Gp() { return reinterpret_cast<snp::DofPair<TT> *>(Gv.p); }
    template <typename TT>
    snp::DofPair<TT> *Rp() { return reinterpret_cast<snp::DofPair<TT> *>(Rv.p); }
    template <typename TT>
    TT *Yp() { return reinterpret_cast<TT *>(Y.p); }
    template <typename TT>
    const TT *chat() const;

    int grid_units() const { return (int)std::min<int64_t>(n_units, (int64_t)snp::sm_count() * 8); }
    int grid_chunks(int block) const {
        const int per_sm = std::max(1, 2048 / block);
        const int64_t need = (n_chunks * snp::kSplit + block / 32 - 1) / (block / 32);  // kSplit warps per chunk
        return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)snp::sm_count() * per_sm));
    }
    int run_stride() const { return (int)(sizeof(snp::BState) / sizeof(int32_t)); }

    // ------------------------------------------------------------ phases (launch sequences)
    template <typename TT>
    int assemble(const double *xv, cudaStream_t s) {
        const int grid = (int)std::min<int64_t>(n_items, (int64_t)snp::sm_count() * 4 * asm_waves);
        return snp::launch_curlcurl_tensor_batch(segs.p, items.p, n_items, max_n_int, ctab, n_orient, nq * 18, dphi, w,
                                                 nq, xv, &st.p->run, run_stride(), Tp<TT>(), sizeof(TT) == 4, Fe.p,
                                                 De.p, grid, s);
    }

    template <int MODE>
    int sum(cudaStream_t s, int use_cond, cudaGraphConditionalHandle c) {
        snp::k_b_sum<MODE><<<grid_units(), snp::kBB, 0, s>>>(count, inst.p, unit_inst.p, n_units, free_mask.p,
                                                             inc_ptr.p, inc.p, Fe.p, De.p, h.p, F.p, diag.p, st.p,
                                                             part.p, ctl.p, use_cond, c);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    // start: x masked, assembly + sums at x, the drop rule, F0 and the first convergence test
    template <typename TT>
    int phase_start(cudaStream_t s, int use_cond, cudaGraphConditionalHandle newton) {
        const int g = (int)std::min<int64_t>((n_tot + 255) / 256, (int64_t)snp::sm_count() * 8);
        snp::k_b_init<<<std::max<int>(g, (count + 255) / 256), 256, 0, s>>>(count, opts.p, st.p, n_tot, free_mask.p,
                                                                           x.p, ctl.p);
        SNP_LAUNCH_CHECK();
        SNP_TRY(assemble<TT>(x.p, s));
        SNP_TRY(sum<snp::SUM_START>(s, 0, 0));
        snp::k_b_zero_run<<<grid_units(), snp::kBB, 0, s>>>(unit_inst.p, n_units, st.p, x.p, ctl.p);
        SNP_LAUNCH_CHECK();
        SNP_TRY(assemble<TT>(x.p, s));
        SNP_TRY(sum<snp::SUM_DROP>(s, 0, 0));
        return flag(s, snp::PH_LIVE, use_cond, newton);
    }

    int flag(cudaStream_t s, int phase, int use_cond, cudaGraphConditionalHandle c) {
        snp::k_b_flag<<<1, 256, 0, s>>>(count, st.p, phase, ctl.p, use_cond, c);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    template <typename TT>
    int phase_step_head(cudaStream_t s, int use_cond, cudaGraphConditionalHandle cg) {
        snp::k_b_step_begin<<<(count + 127) / 128, 128, 0, s>>>(count, st.p, sizeof(TT) == 4 ? 1 : 0, ctl.p);
        SNP_LAUNCH_CHECK();
        const int gb = (int)std::min<int64_t>((n_tot + snp::kBB - 1) / snp::kBB, (int64_t)snp::sm_count() * 8);
        snp::k_b_bj_entries<TT><<<gb, snp::kBB, 0, s>>>(n_tot, unit_inst.p, st.p, free_mask.p, inc_ptr.p, inc.p,
                                                         edof.p, Tp<TT>(), chat<TT>(), meta.p, bmat.p, ctl.p);
        SNP_LAUNCH_CHECK();
        const int gi = (int)std::min<int64_t>((n_tot + 127) / 128, (int64_t)snp::sm_count() * 8);
        snp::k_b_bj_invert<<<gi, 128, 0, s>>>(n_tot, unit_inst.p, st.p, free_mask.p, meta.p, bmat.p, binv.p, ctl.p);
        SNP_LAUNCH_CHECK();
        snp::k_b_pcg_init<TT><<<grid_units(), snp::kBB, 0, s>>>(count, inst.p, unit_inst.p, n_units, free_mask.p, F.p,
                                                                diag.p, meta.p, binv.p, Gp<TT>(), Rp<TT>(), st.p,
                                                                part.p, ctl.p, 0, 0);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    template <typename TT>
    int pass1(cudaStream_t s, int block) {
        switch (block) {
            case 128:
                snp::k_b_pass1<TT, 128><<<grid_chunks(128), 128, 0, s>>>(count, inst.p, act.p, edof.p,
                                                                         pos.p, Tp<TT>(), chat<TT>(), Gp<TT>(),
                                                                         Yp<TT>(), st.p, part.p, ctl.p);
                break;
            case 512:
                snp::k_b_pass1<TT, 512><<<grid_chunks(512), 512, 0, s>>>(count, inst.p, act.p, edof.p,
                                                                         pos.p, Tp<TT>(), chat<TT>(), Gp<TT>(),
                                                                         Yp<TT>(), st.p, part.p, ctl.p);
                break;
            default:
                snp::k_b_pass1<TT, 256><<<grid_chunks(256), 256, 0, s>>>(count, inst.p, act.p, edof.p,
                                                                         pos.p, Tp<TT>(), chat<TT>(), Gp<TT>(),
                                                                         Yp<TT>(), st.p, part.p, ctl.p);
                break;
        }
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    // the compacted list of the problems in CG, for the passes of the CG iterations that follow
    int cg_list(cudaStream_t s) {
        snp::k_b_cg_list<<<1, 32, 0, s>>>(count, inst.p, st.p, act.p, ctl.p);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    // the CG phase: the list, then `reps` CG iterations
    template <typename TT>
    int phase_cg(cudaStream_t s, int reps) {
        SNP_TRY(cg_list(s));
        for (int r = 0; r < reps; ++r) SNP_TRY(phase_cg_body<TT>(s, 0, 0));
        return SNP_OK;
    }

    template <typename TT>
    int phase_cg_body(cudaStream_t s, int use_cond, cudaGraphConditionalHandle cg) {
        SNP_TRY(pass1<TT>(s, pass1_block));
        snp::k_b_pass2<TT><<<grid_units(), snp::kBB, 0, s>>>(count, inst.p, act.p, free_mask.p,
                                                             inc_ptr.p, Yp<TT>(), meta.p, binv.p, Gp<TT>(), Rp<TT>(),
                                                             st.p, part.p, ctl.p, use_cond, cg);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    template <typename TT>
    int phase_extract(cudaStream_t s, int use_cond, cudaGraphConditionalHandle ls) {
        snp::k_b_extract<TT><<<grid_units(), snp::kBB, 0, s>>>(count, inst.p, unit_inst.p, n_units, free_mask.p,
                                                               Rp<TT>(), F.p, h.p, st.p, part.p, ctl.p, use_cond, ls);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    template <typename TT>
    int phase_ls_body(cudaStream_t s, int use_cond, cudaGraphConditionalHandle ls) {
        snp::k_b_axpy<<<grid_units(), snp::kBB, 0, s>>>(unit_inst.p, n_units, free_mask.p, x.p, h.p, xw.p, st.p,
                                                        ctl.p);
        SNP_LAUNCH_CHECK();
        SNP_TRY(assemble<TT>(xw.p, s));
        SNP_TRY(sum<snp::SUM_LS>(s, use_cond, ls));
        return SNP_OK;
    }

    int phase_accept(cudaStream_t s, int use_cond, cudaGraphConditionalHandle newton) {
        snp::k_b_accept<<<grid_units(), snp::kBB, 0, s>>>(count, unit_inst.p, n_units, xw.p, x.p, st.p, ctl.p,
                                                          use_cond, newton);
        SNP_LAUNCH_CHECK();
        return SNP_OK;
    }

    // ------------------------------------------------------------ graph
    // The solve as graph nodes: launches captured into the graph after `tail` (the capture's
    // last nodes become the new tail), and WHILE nodes whose bodies are filled the same way.
    struct Seq {
        cudaGraph_t g = nullptr;
        std::vector<cudaGraphNode_t> tail;
    };

    template <typename Fn>
    int capture(Seq &q, cudaStream_t cs, Fn &&launches) {
        SNP_CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, q.g, q.tail.empty() ? nullptr : q.tail.data(), nullptr,
                                                   q.tail.size(), cudaStreamCaptureModeThreadLocal));
        const int rc = launches(cs);
        const cudaGraphNode_t *deps = nullptr;
        size_t nd = 0;
        cudaStreamCaptureStatus cst;
        const cudaError_t e = cudaStreamGetCaptureInfo(cs, &cst, nullptr, nullptr, &deps, &nd);
        std::vector<cudaGraphNode_t> nt;
        if (e == cudaSuccess && deps) nt.assign(deps, deps + nd);
        cudaGraph_t out = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &out);
        SNP_TRY(rc);
        SNP_CUDA_TRY(e);
        SNP_CUDA_TRY(e2);
        q.tail = nt;
        return SNP_OK;
    }

    int add_cond(Seq &q, cudaGraphConditionalHandle hnd, cudaGraphConditionalNodeType type, Seq *body) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hnd;
        cp.conditional.type = type;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        SNP_CUDA_TRY(cudaGraphAddNode(&node, q.g, q.tail.empty() ? nullptr : q.tail.data(), q.tail.size(), &cp));
        q.tail.assign(1, node);
        body->g = cp.conditional.phGraph_out[0];
        body->tail.clear();
        return SNP_OK;
    }

    // One pass of the solver's loop as graph nodes in `nb`: for each phase, a flag kernel and an
    // IF node over that phase's kernels; then the loop's own condition.  The CG phase's node
    // holds pcg_body_unroll() CG iterations (a problem whose CG ends inside it leaves the phase,
    // and the remaining iterations skip its units), so a pass's fixed cost (six flag kernels,
    // five conditional nodes) is shared by several CG iterations.
    template <typename TT>
    int build_pass(Seq &nb, cudaStream_t cs, const cudaGraphConditionalHandle *hp, cudaGraphConditionalHandle hn) {
        const int phases[5] = {snp::PH_HEAD, snp::PH_CG, snp::PH_EXTRACT, snp::PH_LS, snp::PH_ACCEPT};
        const int cg_unroll = snp::pcg_body_unroll();
        for (int k = 0; k < 5; ++k) {
            const int ph = phases[k];
            SNP_TRY(capture(nb, cs, [&](cudaStream_t s) { return flag(s, ph, 1, hp[k]); }));
            Seq body;
            SNP_TRY(add_cond(nb, hp[k], cudaGraphCondTypeIf, &body));
            SNP_TRY(capture(body, cs, [&](cudaStream_t s) -> int {
                return ph == snp::PH_CG ? phase_cg<TT>(s, cg_unroll) : phase_body<TT>(ph, s);
            }));
        }
        return capture(nb, cs, [&](cudaStream_t s) { return flag(s, snp::PH_LIVE, 1, hn); });
    }

    // the kernels of one phase (host loop and graph alike)
    template <typename TT>
    int phase_body(int ph, cudaStream_t s) {
        switch (ph) {
            case snp::PH_HEAD: return phase_step_head<TT>(s, 0, 0);
            case snp::PH_CG: return phase_cg<TT>(s, 1);
            case snp::PH_EXTRACT: return phase_extract<TT>(s, 0, 0);
            case snp::PH_LS: return phase_ls_body<TT>(s, 0, 0);
            default: return phase_accept(s, 0, 0);
        }
    }

    template <typename TT>
    int build_graph_t(cudaGraph_t g, cudaStream_t cs) {
        cudaGraphConditionalHandle hn, hp[5];
        SNP_CUDA_TRY(cudaGraphConditionalHandleCreate(&hn, g, 0, 0));
        for (auto &h : hp) SNP_CUDA_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
        Seq top;
        top.g = g;
        SNP_TRY(capture(top, cs, [&](cudaStream_t s) { return phase_start<TT>(s, 1, hn); }));
        Seq nb;
        SNP_TRY(add_cond(top, hn, cudaGraphCondTypeWhile, &nb));
        return build_pass<TT>(nb, cs, hp, hn);
    }

    template <typename TT>
    int ensure_graph() {
        const int k = sizeof(TT) == 4 ? 1 : 0;
        if (exec[k] && graph_shape[k][0] == pass1_block && graph_shape[k][1] == asm_waves) return SNP_OK;
        if (exec[k]) cudaGraphExecDestroy(exec[k]);
        if (graph[k]) cudaGraphDestroy(graph[k]);
        exec[k] = nullptr;
        graph[k] = nullptr;
        cudaGraph_t g = nullptr;
        SNP_CUDA_TRY(cudaGraphCreate(&g, 0));
        cudaStream_t cs = nullptr;
        int rc = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess ? SNP_OK : SNP_CUDA_ERROR;
        if (rc == SNP_OK) rc = build_graph_t<TT>(g, cs);
        if (rc == SNP_OK && cudaGraphInstantiate(&exec[k], g, 0) != cudaSuccess) {
            exec[k] = nullptr;
            rc = snp::fail(SNP_CUDA_ERROR, "batched solver: the Newton-loop graph did not instantiate");
        }
        if (cs) cudaStreamDestroy(cs);
        if (rc != SNP_OK) {
            cudaGetLastError();
            if (exec[k]) cudaGraphExecDestroy(exec[k]);
            exec[k] = nullptr;
            cudaGraphDestroy(g);
            return rc;
        }
        graph[k] = g;
        graph_shape[k][0] = pass1_block;
        graph_shape[k][1] = asm_waves;
        return SNP_OK;
    }

    // ------------------------------------------------------------ host-driven loop (no graph)
    int read_ctl() {
        SNP_CUDA_TRY(cudaMemcpyAsync(hctl.p, ctl.p, sizeof(snp::BCtl), cudaMemcpyDeviceToHost, stream));
        SNP_CUDA_TRY(cudaStreamSynchronize(stream));
        return SNP_OK;
    }

    template <typename TT>
    int run_host_loop() {
        SNP_TRY(phase_start<TT>(stream, 0, 0));
        SNP_TRY(read_ctl());
        const int phases[5] = {snp::PH_HEAD, snp::PH_CG, snp::PH_EXTRACT, snp::PH_LS, snp::PH_ACCEPT};
        while (hctl.p->any_phase[snp::PH_LIVE]) {
            for (int ph : phases) {
                SNP_TRY(flag(stream, ph, 0, 0));
                SNP_TRY(read_ctl());
                if (hctl.p->any_phase[ph]) SNP_TRY(phase_body<TT>(ph, stream));
            }
            SNP_TRY(flag(stream, snp::PH_LIVE, 0, 0));
            SNP_TRY(read_ctl());
        }
        return SNP_OK;
    }

    template <typename TT>
    int solve_t(snp_solve_stats *stats, int32_t *status) {
        SNP_CUDA_TRY(cudaMemsetAsync(ctl.p, 0, sizeof(snp::BCtl), stream));
        bool graph_ok = false;
        if (use_graph) {
            graph_ok = ensure_graph<TT>() == SNP_OK;
            if (!graph_ok) {
                snp::clear_error();
                use_graph = false;  // the host-driven loop from now on
            }
        }
        SNP_CUDA_TRY(cudaEventRecord(ev0, stream));
        if (graph_ok) SNP_CUDA_TRY(cudaGraphLaunch(exec[sizeof(TT) == 4 ? 1 : 0], stream));
        else SNP_TRY(run_host_loop<TT>());
        SNP_CUDA_TRY(cudaEventRecord(ev1, stream));
        SNP_CUDA_TRY(cudaMemcpyAsync(hst.p, st.p, sizeof(snp::BState) * count, cudaMemcpyDeviceToHost, stream));
        SNP_CUDA_TRY(cudaMemcpyAsync(hctl.p, ctl.p, sizeof(snp::BCtl), cudaMemcpyDeviceToHost, stream));
        SNP_CUDA_TRY(cudaStreamSynchronize(stream));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        for (int p = 0; p < count; ++p) {
            const snp::BState &s = hst.p[p];
            snp_solve_stats S;
            memset(&S, 0, sizeof(S));
            S.newton_iterations = s.it;
            S.cg_iterations = s.cg_total;
            S.res0 = s.res0;
            S.res = s.fn;
            S.t_total_ms = ms;
            S.status = s.status;
            S.kernel_launches = (int64_t)hctl.p->launches;
            S.residual_evals = s.res_evals;
            S.start_dropped = s.dropped;
            if (stats) stats[p] = S;
            if (status) status[p] = s.status;
        }
        return SNP_OK;
    }
};

template <>
const double *snp_batch::chat<double>() const {
    return chat64.p;
}
template <>
const float *snp_batch::chat<float>() const {
    return chat32.p;
}

namespace snp {
namespace {

// Time `reps` launches of fn on the batch's stream (CUDA events), in microseconds per launch.
template <typename Fn>
int time_launches(snp_batch *b, int reps, Fn &&fn, double *us) {
    for (int k = 0; k < 2; ++k) SNP_TRY(fn());
    SNP_CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
    for (int k = 0; k < reps; ++k) SNP_TRY(fn());
    SNP_CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
    SNP_CUDA_TRY(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    SNP_CUDA_TRY(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    *us = 1e3 * ms / reps;
    return SNP_OK;
}

// Autotuner body: the state of a solve's first CG iteration (x = 0 assembled, block Jacobi,
// PCG started), then each candidate shape timed on it.
template <typename TT>
int tune_t(snp_batch *b) {
    cudaStream_t s = b->stream;
    SNP_CUDA_TRY(cudaMemsetAsync(b->ctl.p, 0, sizeof(BCtl), s));
    SNP_CUDA_TRY(cudaMemsetAsync(b->x.p, 0, sizeof(double) * b->n_tot, s));
    SNP_TRY(b->phase_start<TT>(s, 0, 0));
    SNP_TRY(b->phase_step_head<TT>(s, 0, 0));
    SNP_TRY(b->cg_list(s));
    const int blocks[3] = {128, 256, 512};
    double best = 1e300;
    int best_b = b->pass1_block;
    for (int k = 0; k < 3; ++k) {
        double us = 0.0;
        SNP_TRY(time_launches(b, 10, [&]() { return b->pass1<TT>(s, blocks[k]); }, &us));
        b->tuned_pass1_us[k] = us;
        if (us < best) {
            best = us;
            best_b = blocks[k];
        }
    }
    k_b_set_run<<<(b->count + 127) / 128, 128, 0, s>>>(b->count, b->st.p);
    SNP_LAUNCH_CHECK();
    double best_a = 1e300;
    int best_w = b->asm_waves;
    for (int wv = 1; wv <= 2; ++wv) {
        b->asm_waves = wv;
        double us = 0.0;
        SNP_TRY(time_launches(b, 5, [&]() { return b->assemble<TT>(b->x.p, s); }, &us));
        b->tuned_asm_us[wv - 1] = us;
        if (us < best_a) {
            best_a = us;
            best_w = wv;
        }
    }
    b->pass1_block = best_b;
    b->asm_waves = best_w;
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    return SNP_OK;
}

}  // namespace
}  // namespace snp

extern "C" {

int snp_batch_create(snp_solver *const *solvers, int32_t count, snp_batch **out) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(out != nullptr, "snp_batch_create: out is NULL");
    *out = nullptr;
    SNP_REQUIRE(count >= 1 && solvers != nullptr, "snp_batch_create: need at least one solver");
    auto B = std::make_unique<snp_batch>();
    B->count = count;
    B->views.resize(count);
    for (int p = 0; p < count; ++p) {
        SNP_REQUIRE(solvers[p] != nullptr, "snp_batch_create: solver %d is NULL", p);
        for (int q = 0; q < p; ++q)
            SNP_REQUIRE(solvers[q] != solvers[p], "snp_batch_create: solvers %d and %d are the same", q, p);
        SNP_TRY(solver_view(solvers[p], &B->views[p]));
        const SolverView &v = B->views[p];
        SNP_REQUIRE(v.etop != nullptr, "snp_batch_create: solver %d does not use the matrix-free Jacobian layout", p);
        SNP_REQUIRE(v.bj_meta != nullptr, "snp_batch_create: solver %d has no block-Jacobi partition", p);
        SNP_REQUIRE(v.nq == B->views[0].nq && v.n_orient == B->views[0].n_orient,
                    "snp_batch_create: solver %d has other quadrature or orientation tables than solver 0", p);
    }
    // every solver's work so far (its setup on its own stream) precedes the copies below
    SNP_CUDA_TRY(cudaDeviceSynchronize());
    SNP_CUDA_TRY(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    SNP_CUDA_TRY(cudaEventCreate(&B->ev0));
    SNP_CUDA_TRY(cudaEventCreate(&B->ev1));
    cudaStream_t s = B->stream;
    const SolverView &v0 = B->views[0];
    B->nq = v0.nq;
    B->n_orient = v0.n_orient;
    // the tables of every problem must equal problem 0's (they are read once per launch)
    {
        const size_t nc = (size_t)v0.n_orient * v0.nq * 18;
        const size_t nd = (size_t)v0.nq * 13;
        std::vector<double> c0(nc), ci(nc), d0(nd), di(nd);
        auto fetch = [&](const SolverView &v, std::vector<double> &c, std::vector<double> &d) -> int {
            SNP_CUDA_TRY(cudaMemcpy(c.data(), v.curls, nc * sizeof(double), cudaMemcpyDeviceToHost));
            SNP_CUDA_TRY(cudaMemcpy(d.data(), v.dphi, (size_t)v.nq * 12 * sizeof(double), cudaMemcpyDeviceToHost));
            SNP_CUDA_TRY(cudaMemcpy(d.data() + (size_t)v.nq * 12, v.w, (size_t)v.nq * sizeof(double),
                                    cudaMemcpyDeviceToHost));
            return SNP_OK;
        };
        SNP_TRY(fetch(v0, c0, d0));
        for (int p = 1; p < count; ++p) {
            SNP_TRY(fetch(B->views[p], ci, di));
            SNP_REQUIRE(ci == c0 && di == d0, "snp_batch_create: solver %d has other quadrature tables than solver 0", p);
        }
    }
    B->ctab = v0.curls;
    B->dphi = v0.dphi;
    B->w = v0.w;
    // offsets
    int64_t dof = 0, el = 0, incn = 0;
    B->h_inst.resize(count);
    for (int p = 0; p < count; ++p) {
        const SolverView &v = B->views[p];
        BInst I{};
        I.dof_off = (int32_t)dof;
        I.n = v.n;
        I.unit0 = (int32_t)(dof / kUnit);
        I.n_units = (int32_t)(round_up(v.n, kUnit) / kUnit);
        I.elem_off = el;
        I.ne = v.n_elems;
        I.chunk0 = (int32_t)(el / kChunk);
        I.n_chunks = (int32_t)(round_up(std::max<int64_t>(v.n_elems, 1), kChunk) / kChunk);
        I.rhs_extra = v.rhs_extra;
        B->h_inst[p] = I;
        dof += (int64_t)I.n_units * kUnit;
        el += (int64_t)I.n_chunks * kChunk;
        incn += 6 * v.n_elems;
        for (int m = 0; m < v.n_mats; ++m)
            if (v.mats[m].n_int > B->max_n_int) B->max_n_int = v.mats[m].n_int;
        SNP_REQUIRE(dof < ((int64_t)1 << 31) && incn < ((int64_t)1 << 31) && el < ((int64_t)1 << 28),
                    "snp_batch_create: the batch exceeds the 32-bit DoF / incidence encoding at problem %d", p);
    }
    B->n_tot = dof;
    B->e_tot = el;
    B->inc_tot = incn;
    B->n_units = dof / kUnit;
    B->n_chunks = el / kChunk;
    // device arrays
    const int64_t es = eslots_size(el);
    SNP_TRY(B->inst.alloc(count));
    SNP_TRY(B->st.alloc(count));
    SNP_TRY(B->hst.alloc(count));
    SNP_TRY(B->opts.alloc(count));
    SNP_TRY(B->ctl.alloc(1));
    SNP_TRY(B->hctl.alloc(1));
    SNP_TRY(B->unit_inst.alloc(B->n_units));
    SNP_TRY(B->chunk_inst.alloc(B->n_chunks));
    SNP_TRY(B->act.alloc(snp::act_size(count)));
    SNP_TRY(B->edof.alloc(es));
    SNP_TRY(B->pos.alloc(es));
    SNP_TRY(B->inc.alloc(std::max<int64_t>(incn, 1)));
    SNP_TRY(B->inc_ptr.alloc(dof + 1));
    SNP_TRY(B->free_mask.alloc(dof));
    SNP_TRY(B->meta.alloc(dof));
    for (auto *buf : {&B->x, &B->xw, &B->h, &B->F, &B->diag}) SNP_TRY(buf->alloc(dof));
    SNP_TRY(B->Fe.alloc(es));
    SNP_TRY(B->De.alloc(es));
    SNP_TRY(B->T.alloc(es));
    SNP_TRY(B->bmat.alloc((size_t)dof * kBjMax));
    SNP_TRY(B->binv.alloc((size_t)dof * kBjMax));
    SNP_TRY(B->Gv.alloc(2 * dof));
    SNP_TRY(B->Rv.alloc(2 * dof));
    SNP_TRY(B->Y.alloc(std::max<int64_t>(incn, 1)));
    SNP_TRY(B->part.alloc(2 * std::max(B->n_units, B->n_chunks) + 2));
    SNP_CUDA_TRY(cudaMemcpyAsync(B->inst.p, B->h_inst.data(), sizeof(BInst) * count, cudaMemcpyHostToDevice, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->edof.p, 0, sizeof(int32_t) * es, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->pos.p, 0, sizeof(int32_t) * es, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->free_mask.p, 0, dof, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->T.p, 0, sizeof(double) * es, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->Fe.p, 0, sizeof(double) * es, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->De.p, 0, sizeof(double) * es, s));
    for (auto *buf : {&B->x, &B->xw, &B->h, &B->F, &B->diag})
        SNP_CUDA_TRY(cudaMemsetAsync(buf->p, 0, sizeof(double) * dof, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->Gv.p, 0, sizeof(double) * 2 * dof, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->Rv.p, 0, sizeof(double) * 2 * dof, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->bmat.p, 0, sizeof(double) * dof * kBjMax, s));
    SNP_CUDA_TRY(cudaMemsetAsync(B->binv.p, 0, sizeof(float) * dof * kBjMax, s));
    k_b_fill_u16<<<stride_grid(dof, 256, 8), 256, 0, s>>>(dof, B->meta.p, (uint16_t)(1u << 8));
    SNP_LAUNCH_CHECK();
    std::vector<int32_t> ui(B->n_units), ci(B->n_chunks);
    std::vector<BatchSeg> segs;
    std::vector<BatchAsmItem> items;
    int64_t inc_off = 0;
    for (int p = 0; p < count; ++p) {
        const SolverView &v = B->views[p];
        const BInst &I = B->h_inst[p];
        for (int u = 0; u < I.n_units; ++u) ui[I.unit0 + u] = p;
        for (int c = 0; c < I.n_chunks; ++c) ci[I.chunk0 + c] = p;
        const ElemTopology &tp = *v.etop;
        const int64_t esi = eslots_size(v.n_elems);
        const int64_t m6 = 6 * v.n_elems;
        const int g = stride_grid(std::max<int64_t>(esi, m6), 256, 8);
        k_b_copy_shift<<<g, 256, 0, s>>>(esi, tp.edof.p, B->edof.p + 6 * I.elem_off, CP_EDOF, I.dof_off, 0);
        SNP_LAUNCH_CHECK();
        k_b_copy_shift<<<g, 256, 0, s>>>(esi, tp.pos.p, B->pos.p + 6 * I.elem_off, CP_ADD, inc_off, 0);
        SNP_LAUNCH_CHECK();
        k_b_copy_shift<<<g, 256, 0, s>>>(m6, tp.inc.p, B->inc.p + inc_off, CP_INC, 0, I.elem_off);
        SNP_LAUNCH_CHECK();
        k_b_copy_shift<<<stride_grid(v.n + 1, 256, 8), 256, 0, s>>>(v.n + 1, tp.inc_ptr.p, B->inc_ptr.p + I.dof_off,
                                                                   CP_ADD, inc_off, 0);
        SNP_LAUNCH_CHECK();
        const int64_t pad = (int64_t)I.n_units * kUnit - v.n;  // padding DoFs: empty incidence ranges
        if (pad > 0) {
            k_b_fill_i32<<<stride_grid(pad, 256, 8), 256, 0, s>>>(pad, B->inc_ptr.p + I.dof_off + v.n + 1,
                                                                 (int32_t)(inc_off + m6));
            SNP_LAUNCH_CHECK();
        }
        SNP_CUDA_TRY(cudaMemcpyAsync(B->free_mask.p + I.dof_off, v.free_mask, v.n, cudaMemcpyDeviceToDevice, s));
        SNP_CUDA_TRY(
            cudaMemcpyAsync(B->meta.p + I.dof_off, v.bj_meta, sizeof(uint16_t) * v.n, cudaMemcpyDeviceToDevice, s));
        for (int m = 0; m < v.n_mats; ++m) {
            const SolverMaterialView &mv = v.mats[m];
            if (mv.count == 0) continue;
            BatchSeg sg{};
            sg.a.n_elems = mv.count;
            sg.a.nodes = v.nodes;
            sg.a.cells = mv.cells;
            sg.a.gids = mv.gids;
            sg.a.orient = mv.orient;
            sg.a.ctab = v.curls;
            sg.a.n_orient = v.n_orient;
            sg.a.dphi0 = v.dphi;
            sg.a.w = v.w;
            sg.a.nq = v.nq;
            sg.a.Bs = mv.Bs;
            sg.a.n_int = mv.n_int;
            sg.a.rel_c = mv.relc;
            sg.a.rel_x = mv.relx;
            sg.a.phi = mv.phi;
            for (int k = 0; k < 4; ++k) sg.a.dil[k] = mv.dil[k];
            sg.a.t_offset = I.elem_off + mv.offset;
            sg.inst = p;
            sg.dof_off = I.dof_off;
            const int sid = (int)segs.size();
            segs.push_back(sg);
            for (int64_t e0 = 0; e0 < mv.count; e0 += kBatchAsmItem)
                items.push_back(BatchAsmItem{sid, p, e0, std::min<int64_t>(mv.count, e0 + kBatchAsmItem)});
        }
        inc_off += m6;
    }
    SNP_CUDA_TRY(cudaMemcpyAsync(B->unit_inst.p, ui.data(), sizeof(int32_t) * ui.size(), cudaMemcpyHostToDevice, s));
    SNP_CUDA_TRY(cudaMemcpyAsync(B->chunk_inst.p, ci.data(), sizeof(int32_t) * ci.size(), cudaMemcpyHostToDevice, s));
    SNP_TRY(B->segs.alloc(std::max<size_t>(segs.size(), 1)));
    SNP_TRY(B->items.alloc(std::max<size_t>(items.size(), 1)));
    SNP_CUDA_TRY(cudaMemcpyAsync(B->segs.p, segs.data(), sizeof(BatchSeg) * segs.size(), cudaMemcpyHostToDevice, s));
    SNP_CUDA_TRY(
        cudaMemcpyAsync(B->items.p, items.data(), sizeof(BatchAsmItem) * items.size(), cudaMemcpyHostToDevice, s));
    B->n_items = (int32_t)items.size();
    SNP_TRY(B->chat64.alloc(18));
    SNP_TRY(B->chat32.alloc(18));
    SNP_CUDA_TRY(cudaMemcpyAsync(B->chat64.p, v0.etop->chat64.p, 18 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    SNP_CUDA_TRY(cudaMemcpyAsync(B->chat32.p, v0.etop->chat32.p, 18 * sizeof(float), cudaMemcpyDeviceToDevice, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));  // the host vectors above are read by the copies
    const char *env = getenv("SNP_BATCH_GRAPH");
    B->use_graph = !(env && env[0] == '0');
    *out = B.release();
    return SNP_OK;
}

int snp_batch_solve(snp_batch *b, double *const *x, const snp_solve_opts *opts, snp_solve_stats *stats,
                    int32_t *status) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(b != nullptr && x != nullptr && opts != nullptr, "snp_batch_solve: NULL argument");
    const int prec = opts[0].precision;
    SNP_REQUIRE(prec == 0 || prec == 1, "snp_batch_solve: precision must be 0 or 1");
    std::vector<BOpts> ho(b->count);
    for (int p = 0; p < b->count; ++p) {
        const snp_solve_opts &o = opts[p];
        SNP_REQUIRE(x[p] != nullptr, "snp_batch_solve: x[%d] is NULL", p);
        SNP_REQUIRE(o.mode == 1, "snp_batch_solve: problem %d: only the residual mode (1) is batched", p);
        SNP_REQUIRE(o.precision == prec, "snp_batch_solve: problem %d: every problem needs the same precision", p);
        SNP_REQUIRE(o.max_newton >= 1 && o.tol > 0, "snp_batch_solve: problem %d: max_newton >= 1 and tol > 0", p);
        BOpts bo;
        bo.tol = o.tol;
        bo.res_ref = o.res_ref;
        const double em = o.cg_rtol > 0 ? o.cg_rtol : 0.1;
        bo.eta_max = em > 0.5 ? 0.5 : em;
        bo.cg_maxit = o.cg_maxiter < 0 ? 10 * (long long)b->views[p].n_free : (long long)o.cg_maxiter;
        bo.max_newton = o.max_newton;
        bo.line_search = o.line_search ? 1 : 0;
        ho[p] = bo;
    }
    cudaStream_t s = b->stream;
    // the caller's work on any stream (x prepared there, solver inputs changed) precedes the solve
    SNP_CUDA_TRY(cudaDeviceSynchronize());
    SNP_CUDA_TRY(cudaMemcpyAsync(b->opts.p, ho.data(), sizeof(BOpts) * b->count, cudaMemcpyHostToDevice, s));
    for (int p = 0; p < b->count; ++p)
        SNP_CUDA_TRY(cudaMemcpyAsync(b->x.p + b->h_inst[p].dof_off, x[p], sizeof(double) * b->h_inst[p].n,
                                     cudaMemcpyDeviceToDevice, s));
    SNP_TRY(prec == 1 ? b->solve_t<float>(stats, status) : b->solve_t<double>(stats, status));
    for (int p = 0; p < b->count; ++p)
        SNP_CUDA_TRY(cudaMemcpyAsync(x[p], b->x.p + b->h_inst[p].dof_off, sizeof(double) * b->h_inst[p].n,
                                     cudaMemcpyDeviceToDevice, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    for (int p = 0; p < b->count; ++p) {
        const int st = b->hst.p[p].status;
        if (st != SNP_OK)
            return fail(st, "snp_batch_solve: problem %d: %s", p,
                        st == SNP_NOT_CONVERGED  ? "Newton did not reach the tolerance"
                        : st == SNP_NAN_DETECTED ? "non-finite residual"
                                                 : "zero Jacobian diagonal on a free DoF");
    }
    return SNP_OK;
}

int snp_batch_tune(snp_batch *b, int32_t precision) {
    using namespace snp;
    clear_error();
    SNP_REQUIRE(b != nullptr, "snp_batch_tune: batch is NULL");
    SNP_REQUIRE(precision == 0 || precision == 1, "snp_batch_tune: precision must be 0 or 1");
    // options of a plain solve for the state the candidates are timed on
    std::vector<BOpts> ho(b->count);
    for (int p = 0; p < b->count; ++p) ho[p] = BOpts{1e-8, 0.0, 0.1, 10 * (long long)b->views[p].n_free, 60, 1};
    SNP_CUDA_TRY(cudaDeviceSynchronize());
    SNP_CUDA_TRY(cudaMemcpyAsync(b->opts.p, ho.data(), sizeof(BOpts) * b->count, cudaMemcpyHostToDevice, b->stream));
    return precision == 1 ? tune_t<float>(b) : tune_t<double>(b);
}

int snp_batch_get_info(const snp_batch *b, snp_batch_info *info) {
    snp::clear_error();
    SNP_REQUIRE(b != nullptr && info != nullptr, "snp_batch_get_info: NULL argument");
    info->problems = b->count;
    info->dofs = b->n_tot;
    info->elements = b->e_tot;
    info->pass1_block = b->pass1_block;
    info->asm_waves = b->asm_waves;
    info->graph = b->use_graph ? 1 : 0;
    for (int k = 0; k < 3; ++k) info->tuned_pass1_us[k] = b->tuned_pass1_us[k];
    for (int k = 0; k < 2; ++k) info->tuned_asm_us[k] = b->tuned_asm_us[k];
    return SNP_OK;
}

int snp_batch_destroy(snp_batch *b) {
    delete b;
    return SNP_OK;
}

}  // extern "C"
