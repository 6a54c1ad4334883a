// Matrix-free Newton Jacobian and its Jacobi-PCG.
//
// The assembled Jacobian of the reference (a CSR built by scipy from element triplets,
// snoopy/red_mvp_solver.py:160-203) costs 12 bytes per stored entry and ~16 entries per row
// on a tetrahedral mesh.  For first-order Nedelec elements on affine tetrahedra each element
// block is J_e,jk = s_j s_k chat_j . S_e chat_k with a 3x3 symmetric S_e, so the operator is
// kept as six numbers per element plus the fixed topology, and a product is two passes:
//
//   element pass  p_j formed on the fly, u_e = sum_j s_j p_j chat_j, v_e = S_e u_e, p.q
//                 partial sums (p.J p = sum_e u_e . v_e); each edge term s_k chat_k . v_e
//                 is stored in the slot that (e, k) holds in the DoF-ordered incidence list
//   DoF pass      q_i = sum of DoF i's slots (a contiguous range, no gathers), then the CG
//                 update of the DoF: p = z + beta p, x += alpha p, r -= alpha q,
//                 z = dinv r, r.z and r.r partial sums
//
// Every slot has one writer and every sum runs in a fixed order, so the iteration is
// deterministic without atomics.  The per-DoF CG state is split so the element pass gathers only {z, p}
// (16 bytes per DoF in float64).  The direction p_k = z_k + beta p_(k-1) is formed in both
// passes by the same rounded expression, so both see the same p.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cub/cub.cuh>

#include "snp_common.cuh"
#include "snp_elem.cuh"
#include "snp_internal.cuh"
#include "snp_krylov.cuh"
#include "snp_reduce.cuh"

namespace snp {

namespace {

constexpr int kEBlock = 256;
#ifndef SNP_PASS1_MIN_BLOCKS
#define SNP_PASS1_MIN_BLOCKS 4
#endif
constexpr int kPass1MinBlocks = SNP_PASS1_MIN_BLOCKS;  // resident blocks per SM the element pass asks for

// ---------------------------------------------------------------- topology build

__global__ void k_edof(int64_t count, int64_t offset, int64_t ne, const int32_t *__restrict__ gids,
                       const int32_t *__restrict__ orient, const int8_t *__restrict__ sgn, int32_t n_orient,
                       int32_t n, int32_t *__restrict__ edof, int *bad) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x) {
        const int o = orient[e];
        if (o < 0 || o >= n_orient) {
            atomicExch(bad, 1);
            continue;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int32_t g = gids[6 * e + k];
            if (g < 0 || g >= n) {
                atomicExch(bad, 1);
                continue;
            }
            edof[eslot(offset + e, k)] = (int32_t)((uint32_t)g | (sgn[6 * o + k] < 0 ? kSignBit : 0u));
        }
    }
}

// sort keys (DoF) and values (e << 3 | k | sign) of every element edge; counts per DoF
__global__ void k_inc_keys(int64_t ne, const int32_t *__restrict__ edof, int32_t *__restrict__ key,
                           int32_t *__restrict__ val, int32_t *__restrict__ count) {
    const int64_t total = 6 * ne;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / 6;
        const int k = (int)(t - 6 * e);
        const uint32_t d = (uint32_t)edof[eslot(e, k)];
        const int32_t g = (int32_t)(d & ~kSignBit);
        key[t] = g;
        val[t] = (int32_t)(((uint32_t)e << 3) | (uint32_t)k | (d & kSignBit));
        atomicAdd(count + g, 1);
    }
}

// per-DoF sums of element-edge terms, in incidence order
__global__ void k_sum_to_dofs(int32_t n, int64_t ne, const int32_t *__restrict__ inc_ptr,
                              const int32_t *__restrict__ inc, const double *__restrict__ Fe,
                              const double *__restrict__ De, const double *__restrict__ rhs_extra,
                              double *__restrict__ F, double *__restrict__ diag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double f = 0.0, d = 0.0;
        for (int t = inc_ptr[i]; t < inc_ptr[i + 1]; ++t) {
            const uint32_t u = (uint32_t)inc[t] & ~kSignBit;
            const int64_t idx = eslot(u >> 3, (int)(u & 7u));
            f += Fe[idx];
            d += De[idx];
        }
        F[i] = rhs_extra ? f - rhs_extra[i] : f;
        diag[i] = d;
    }
}

// slot of every (e, k) in the DoF-ordered incidence list
__global__ void k_inc_pos(int64_t m, int64_t ne, const int32_t *__restrict__ inc, int32_t *__restrict__ pos) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t u = (uint32_t)inc[t] & ~kSignBit;
        pos[eslot(u >> 3, (int)(u & 7u))] = (int32_t)t;
    }
}

// ---------------------------------------------------------------- PCG kernels

template <typename TT>
__global__ void __launch_bounds__(kEBlock)
    k_einit(int32_t n, const uint8_t *__restrict__ free_mask, const double *__restrict__ b, double b_scale,
            const double *__restrict__ diag, DofPair<TT> *__restrict__ G, DofPair<TT> *__restrict__ R,
            TT *__restrict__ D, PcgState *st, double *part, double rtol, double atol, long long maxit, int *bad) {
    __shared__ double sh[32];
    double rz = 0.0, rr = 0.0, bb = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        TT r = TT(0), d = TT(0), z = TT(0);
        if (is_free(free_mask, i)) {
            const double dg = diag[i];
            if (dg == 0.0 || !isfinite(dg)) {
                atomicExch(bad, 1);
            } else {
                d = (TT)(1.0 / dg);
            }
            r = (TT)(b_scale * b[i]);
            z = d * r;
            rz += (double)r * (double)z;
            rr += (double)r * (double)r;
            bb += (double)r * (double)r;
        }
        G[i] = DofPair<TT>{z, TT(0)};
        R[i] = DofPair<TT>{r, TT(0)};
        D[i] = d;
    }
    const double a0 = block_sum(rz, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x] = a0;
    const double a1 = block_sum(rr, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x + 1] = a1;
    const double a2 = block_sum(bb, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x + 2] = a2;
    if (last_block(&st->counter)) {
        const double s_rz = reduce_parts(part, gridDim.x, 3, 0, sh);
        const double s_rr = reduce_parts(part, gridDim.x, 3, 1, sh);
        const double s_bb = reduce_parts(part, gridDim.x, 3, 2, sh);
        if (threadIdx.x == 0) {
            st->rz = s_rz;
            st->rr = s_rr;
            st->bnorm = sqrt(s_bb);
            st->atol_eff = fmax(atol, rtol * st->bnorm);
            st->iter = 0;
            st->maxit = maxit;
            st->alpha = 0.0;
            st->beta = 0.0;
            int done = 0;
            if (s_bb == 0.0) done = 4;
            else if (!(s_rr == s_rr) || isinf(s_rr)) done = 3;
            else if (sqrt(s_rr) < st->atol_eff) done = 1;
            else if (maxit <= 0) done = 2;
            st->done = done;
        }
    }
}

template <typename TT>
__device__ __forceinline__ void load_chat(TT *sc, const TT *chat) {
    if (threadIdx.x < 18) sc[threadIdx.x] = chat[threadIdx.x];
    __syncthreads();
}

// element pass of a CG iteration: p from the DoF states, v_e = S_e u_e, p.J p -> alpha, and
// the six edge terms into their incidence slots.  Two lanes per element, three edges each:
// each lane gathers three DoF states, the halves of u_e meet through one shuffle, and each
// lane stores its three edge terms (half the registers of one lane per element, so twice
// the resident warps keep the same number of gathers in flight).
template <typename TT>
__global__ void __launch_bounds__(kEBlock, kPass1MinBlocks)
    k_epass1(int64_t ne, const int32_t *__restrict__ edof, const int32_t *__restrict__ pos,
             const TT *__restrict__ T, const TT *__restrict__ chat, const DofPair<TT> *__restrict__ G,
             TT *__restrict__ Y, PcgState *st, double *part) {
    __shared__ TT sc[18];
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31;
    const int h = lane & 1;  // edges 3h .. 3h+2
    // a warp takes 16 consecutive elements per pass; the loop bound is uniform across the warp
    const int64_t wstride = (int64_t)gridDim.x * (blockDim.x >> 5) * 16;
    const int64_t first = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 16;
    // every streamed word of a pass is requested before its gathers: the lane's three DoF words,
    // slots and tensor components (the partner lane holds the other three); the first pass's
    // words before the CG state is read
    // In float32 the words of the warp's next pass are requested while this pass gathers, one
    // pass ahead (in float64 their registers need a lower occupancy target, which cost more:
    // 78.1 -> 79-82 us per iteration at 1.16M tets with three blocks per SM).
    constexpr bool kAhead = sizeof(TT) == 4;
    int32_t d[3], ps[3], nd[3], nps[3];
    TT th[3], nth[3];
    auto stream_in = [&](int64_t e0, int32_t(&od)[3], int32_t(&ops)[3], TT(&oth)[3]) {
        const int64_t e = e0 + (lane >> 1);
        const bool valid = e < ne;
        const int64_t eb = eslot(valid ? e : 0, 0);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            od[j] = valid ? __ldcs(edof + eb + 32 * (3 * h + j)) : 0;
            ops[j] = valid ? __ldcs(pos + eb + 32 * (3 * h + j)) : 0;
            oth[j] = valid ? __ldcs(T + eb + 32 * (3 * h + j)) : TT(0);
        }
    };
    if (first < ne) stream_in(first, d, ps, th);
    if (st->done) return;
    load_chat(sc, chat);
    const TT beta = (TT)st->beta;
    double dot = 0.0;
#pragma unroll 1
    for (int64_t e0 = first; e0 < ne; e0 += wstride) {
        const int64_t e = e0 + (lane >> 1);
        const bool valid = e < ne;
        if constexpr (kAhead) {
            if (e0 != first) {
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    d[j] = nd[j];
                    ps[j] = nps[j];
                    th[j] = nth[j];
                }
            }
            if (e0 + wstride < ne) stream_in(e0 + wstride, nd, nps, nth);
        } else {
            if (e0 != first) stream_in(e0, d, ps, th);
        }
        DofPair<TT> w[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) w[j] = G[(uint32_t)d[j] & ~kSignBit];
        TT u0 = TT(0), u1 = TT(0), u2 = TT(0);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            TT pk = pnext(beta, w[j].b, w[j].a);
            if (d[j] < 0) pk = -pk;
            const TT *c = sc + 3 * (3 * h + j);
            u0 += pk * c[0];
            u1 += pk * c[1];
            u2 += pk * c[2];
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
        if (!valid) continue;
        const TT v0 = t[0] * u0 + t[1] * u1 + t[2] * u2;
        const TT v1 = t[1] * u0 + t[3] * u1 + t[4] * u2;
        const TT v2 = t[2] * u0 + t[4] * u1 + t[5] * u2;
        if (!h) dot += (double)u0 * (double)v0 + (double)u1 * (double)v1 + (double)u2 * (double)v2;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Y[ps[j]] = edge_term(sc, 3 * h + j, d[j] < 0, v0, v1, v2);
    }
    dot = block_sum(dot, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = dot;
    if (last_block(&st->counter)) {
        const double pq = reduce_parts(part, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) {
            st->pq = pq;
            st->alpha = st->rz / pq;
        }
    }
}

// DoF pass of a CG iteration: q_i = sum of the DoF's incidence slots, then the update of DoF i
template <typename TT>
__global__ void __launch_bounds__(kEBlock)
    k_epass2(int32_t n, const uint8_t *__restrict__ free_mask, const int32_t *__restrict__ inc_ptr,
             const TT *__restrict__ Y, DofPair<TT> *__restrict__ G, DofPair<TT> *__restrict__ R,
             const TT *__restrict__ D, PcgState *st, double *part, int use_cond, cudaGraphConditionalHandle cond) {
    __shared__ double sh2[2][32];
    if (st->done) {
        if (use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
        return;
    }
    const TT alpha = (TT)st->alpha, beta = (TT)st->beta;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (!is_free(free_mask, i)) continue;
        const DofPair<TT> g = G[i];
        const DofPair<TT> rx = R[i];
        const TT dv = D[i];
        const int b0 = __ldcs(inc_ptr + i), b1 = __ldcs(inc_ptr + i + 1);
        double q = 0.0;
        for (int t = b0; t < b1; ++t) q += (double)Y[t];
        const TT p = pnext(beta, g.b, g.a);
        const TT r = rx.a - alpha * (TT)q;
        const TT z = dv * r;
        G[i] = DofPair<TT>{z, p};
        R[i] = DofPair<TT>{r, rx.b + alpha * p};
        rz += (double)r * (double)z;
        rr += (double)r * (double)r;
    }
    block_sum2(rz, rr, sh2);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rz;
        part[2 * blockIdx.x + 1] = rr;
    }
    if (last_block(&st->counter)) {
        double a = 0.0, b = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            a += __ldcg(part + 2 * i);
            b += __ldcg(part + 2 * i + 1);
        }
        __syncthreads();
        block_sum2(a, b, sh2);
        if (threadIdx.x == 0) {
            const double rz_new = a, rr_new = b;
            st->beta = rz_new / st->rz;
            st->rz = rz_new;
            st->rr = rr_new;
            st->iter += 1;
            int done = 0;
            if (!(rr_new == rr_new) || isinf(rr_new)) done = 3;
            else if (sqrt(rr_new) < st->atol_eff) done = 1;
            else if (st->iter >= st->maxit) done = 2;
            st->done = done;
            if (use_cond && done) cudaGraphSetConditional(cond, 0);
        }
    }
}

template <typename TT>
__global__ void k_eextract(int32_t n, const DofPair<TT> *__restrict__ R, double *__restrict__ h) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        h[i] = (double)R[i].b;
}

// ---------------------------------------------------------------- plain product y = J x

template <typename TT>
__global__ void __launch_bounds__(kEBlock)
    k_eapply1(int64_t ne, const int32_t *__restrict__ edof, const int32_t *__restrict__ pos,
              const TT *__restrict__ T, const TT *__restrict__ chat, const uint8_t *__restrict__ free_mask,
              const TT *__restrict__ x, TT *__restrict__ Y) {
    __shared__ TT sc[18];
    load_chat(sc, chat);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t eb = eslot(e, 0);
        int32_t d[6];
        TT u0 = TT(0), u1 = TT(0), u2 = TT(0);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            d[k] = edof[eb + 32 * k];
            const uint32_t g = (uint32_t)d[k] & ~kSignBit;
            TT xk = is_free(free_mask, g) ? x[g] : TT(0);
            if (d[k] < 0) xk = -xk;
            u0 += xk * sc[3 * k];
            u1 += xk * sc[3 * k + 1];
            u2 += xk * sc[3 * k + 2];
        }
        TT t[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) t[k] = T[eb + 32 * k];
        const TT v0 = t[0] * u0 + t[1] * u1 + t[2] * u2;
        const TT v1 = t[1] * u0 + t[3] * u1 + t[4] * u2;
        const TT v2 = t[2] * u0 + t[4] * u1 + t[5] * u2;
#pragma unroll
        for (int k = 0; k < 6; ++k) Y[pos[eb + 32 * k]] = edge_term(sc, k, d[k] < 0, v0, v1, v2);
    }
}

template <typename TT>
__global__ void __launch_bounds__(kEBlock)
    k_eapply2(int32_t n, const uint8_t *__restrict__ free_mask, const int32_t *__restrict__ inc_ptr,
              const TT *__restrict__ Y, TT *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double q = 0.0;
        if (is_free(free_mask, i))
            for (int t = inc_ptr[i]; t < inc_ptr[i + 1]; ++t) q += (double)Y[t];
        y[i] = (TT)q;
    }
}

// ---------------------------------------------------------------- reduced (Galerkin) system
//
// Jr = V^T J V for a basis V [n][ldv] (float32, m <= 128 columns) on the free DoFs:
// Jr = sum_e W_e^T S_e W_e with W_e = sum_k s_k chat_k V[dof_k, :] (3 x m, the curls of the
// basis columns on element e).  A block takes one 64 x 64 block (bi, bj), bi <= bj, of Jr and a
// share of the 32-element eslot groups; per group it forms W_e (columns of block bi) and
// S_e W_e (columns of block bj) in shared memory (96 rows each), then every thread adds the
// 96 rank-1 terms of its 4 x 4 piece in float64 registers.  Block partials are summed in a
// fixed order by k_rsys_sum, so the result is deterministic.

constexpr int kRsB = 64;         // output block edge
constexpr int kRsRows = 3 * 32;  // rows of W per eslot group
constexpr size_t kRsSmem = 2 * sizeof(double) * kRsRows * kRsB;

__device__ __forceinline__ void rsys_job(int job, int nb, int &bi, int &bj) {
    bi = 0;
    while (job >= nb - bi) {
        job -= nb - bi;
        ++bi;
    }
    bj = bi + job;
}

template <typename TT>
__global__ void __launch_bounds__(256)
    k_rsys_jac(int64_t ne, const int32_t *__restrict__ edof, const TT *__restrict__ T, const TT *__restrict__ chat,
               const uint8_t *__restrict__ free_mask, const float *__restrict__ V, int m, int64_t ldv, int nb,
               double *__restrict__ part) {
    extern __shared__ double rs_smem[];
    double *Wi = rs_smem;                  // [96][64]  W_e, columns of block bi
    double *Yj = rs_smem + kRsRows * kRsB;  // [96][64]  S_e W_e, columns of block bj
    __shared__ uint32_t s_d[32][6];
    __shared__ double s_t[32][6];
    __shared__ double sc[18];
    int bi, bj;
    rsys_job(blockIdx.y, nb, bi, bj);
    if (threadIdx.x < 18) sc[threadIdx.x] = (double)chat[threadIdx.x];
    const int ti = threadIdx.x >> 4, tj = threadIdx.x & 15;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    const int64_t n_groups = (ne + 31) >> 5;
    for (int64_t grp = blockIdx.x; grp < n_groups; grp += gridDim.x) {
        __syncthreads();  // the previous group's rows are consumed
        if (threadIdx.x < 192) {
            const int k = threadIdx.x >> 5, l = threadIdx.x & 31;
            const bool valid = (grp << 5) + l < ne;
            const int64_t idx = (grp * 6 + k) * 32 + l;
            s_d[l][k] = valid ? (uint32_t)edof[idx] : 0u;
            s_t[l][k] = valid ? (double)T[idx] : 0.0;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < 32 * kRsB; q += blockDim.x) {
            const int c = q & (kRsB - 1), l = q >> 6;
            const int ci = bi * kRsB + c, cj = bj * kRsB + c;
            double wi[3] = {0.0, 0.0, 0.0}, wj[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const uint32_t d = s_d[l][k];
                const uint32_t g = d & ~kSignBit;
                if (!is_free(free_mask, g)) continue;
                double vi = ci < m ? (double)V[(int64_t)g * ldv + ci] : 0.0;
                double vj = cj < m ? (double)V[(int64_t)g * ldv + cj] : 0.0;
                if (d & kSignBit) {
                    vi = -vi;
                    vj = -vj;
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    wi[a] = fma(vi, sc[3 * k + a], wi[a]);
                    wj[a] = fma(vj, sc[3 * k + a], wj[a]);
                }
            }
            const double *t = s_t[l];  // xx xy xz yy yz zz (zero for the padding of the last group)
            Wi[(3 * l + 0) * kRsB + c] = wi[0];
            Wi[(3 * l + 1) * kRsB + c] = wi[1];
            Wi[(3 * l + 2) * kRsB + c] = wi[2];
            Yj[(3 * l + 0) * kRsB + c] = t[0] * wj[0] + t[1] * wj[1] + t[2] * wj[2];
            Yj[(3 * l + 1) * kRsB + c] = t[1] * wj[0] + t[3] * wj[1] + t[4] * wj[2];
            Yj[(3 * l + 2) * kRsB + c] = t[2] * wj[0] + t[4] * wj[1] + t[5] * wj[2];
        }
        __syncthreads();
#pragma unroll 4
        for (int r = 0; r < kRsRows; ++r) {
            const double2 a01 = *reinterpret_cast<const double2 *>(Wi + r * kRsB + 4 * ti);
            const double2 a23 = *reinterpret_cast<const double2 *>(Wi + r * kRsB + 4 * ti + 2);
            const double2 b01 = *reinterpret_cast<const double2 *>(Yj + r * kRsB + 4 * tj);
            const double2 b23 = *reinterpret_cast<const double2 *>(Yj + r * kRsB + 4 * tj + 2);
            const double av[4] = {a01.x, a01.y, a23.x, a23.y};
            const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
    }
    double *out = part + ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * (kRsB * kRsB);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) out[(4 * ti + a) * kRsB + 4 * tj + b] = acc[a][b];
}

// Jr from the block partials: one thread per entry of each (bi, bj) block, partials summed in
// block order; the mirror (bj, bi) is written for off-diagonal blocks.
__global__ void k_rsys_jac_sum(int n_parts, int n_jobs, int nb, int m, const double *__restrict__ part,
                               double *__restrict__ Jr) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_jobs * kRsB * kRsB) return;
    const int job = t / (kRsB * kRsB), ij = t - job * kRsB * kRsB;
    int bi, bj;
    rsys_job(job, nb, bi, bj);
    const int r = bi * kRsB + ij / kRsB, c = bj * kRsB + (ij & (kRsB - 1));
    if (r >= m || c >= m) return;
    double s = 0.0;
    for (int p = 0; p < n_parts; ++p) s += part[((int64_t)job * n_parts + p) * (kRsB * kRsB) + ij];
    Jr[(int64_t)r * m + c] = s;
    if (bi != bj) Jr[(int64_t)c * m + r] = s;
}

// g = V^T F over the free DoFs: 64 columns per block row (grid.y), four DoFs per pass.
__global__ void __launch_bounds__(256)
    k_rsys_rhs(int32_t n, const uint8_t *__restrict__ free_mask, const float *__restrict__ V, int m, int64_t ldv,
               const double *__restrict__ F, double *__restrict__ part) {
    __shared__ double sh[4][kRsB];
    const int c = blockIdx.y * kRsB + (threadIdx.x & (kRsB - 1)), lane4 = threadIdx.x >> 6;
    double acc = 0.0;
    if (c < m)
        for (int64_t i = (int64_t)blockIdx.x * 4 + lane4; i < n; i += (int64_t)gridDim.x * 4)
            if (is_free(free_mask, i)) acc = fma((double)V[i * ldv + c], F[i], acc);
    sh[lane4][threadIdx.x & (kRsB - 1)] = acc;
    __syncthreads();
    if (threadIdx.x < kRsB)
        part[((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * kRsB + threadIdx.x] =
            (sh[0][threadIdx.x] + sh[1][threadIdx.x]) + (sh[2][threadIdx.x] + sh[3][threadIdx.x]);
}

__global__ void k_rsys_rhs_sum(int n_parts, int m, const double *__restrict__ part, double *__restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    const int cb = c / kRsB, cl = c & (kRsB - 1);
    double s = 0.0;
    for (int p = 0; p < n_parts; ++p) s += part[((int64_t)cb * n_parts + p) * kRsB + cl];
    g[c] = s;
}

// ---------------------------------------------------------------- block Jacobi
//
// The DoFs are cut into blocks of at most kBjMax consecutive free DoFs (for edge DoFs numbered
// by their lower node: the edges that share that node) that never cross a multiple of kBjTile;
// meta[i] = offset of DoF i in its block | block size << 8, constrained DoFs are blocks of their
// own.  Per Newton step the block-diagonal entries of J are summed per DoF row over the DoF's
// incidence list (fixed order), each block is inverted by Cholesky (point Jacobi for a block
// whose pivot falls below 1e-12 of its diagonal) and stored as float32 rows of kBjMax, and the
// PCG's DoF pass stages r of a kBjTile-DoF tile in shared memory so that each DoF forms
// z_i = sum_j M_ij r_j over its block.

static_assert(kBjTile == kEBlock, "the DoF pass stages one block-Jacobi tile per block");

template <typename TT>
__global__ void __launch_bounds__(kEBlock)
    k_bj_entries(int32_t n, const uint8_t *__restrict__ free_mask, const int32_t *__restrict__ inc_ptr,
                 const int32_t *__restrict__ inc, const int32_t *__restrict__ edof, const TT *__restrict__ T,
                 const TT *__restrict__ chat, const uint16_t *__restrict__ meta, double *__restrict__ bmat) {
    __shared__ double sc[18];
    if (threadIdx.x < 18) sc[threadIdx.x] = (double)chat[threadIdx.x];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double row[kBjMax];
#pragma unroll
        for (int c = 0; c < kBjMax; ++c) row[c] = 0.0;
        if (is_free(free_mask, i)) bj_entries_row(i, inc_ptr, inc, edof, T, sc, (unsigned)meta[i], row);
#pragma unroll
        for (int c = 0; c < kBjMax; ++c) bmat[i * kBjMax + c] = row[c];
    }
}

// one thread per block: the block's inverse (bj_invert_block)
__global__ void __launch_bounds__(128)
    k_bj_invert(int32_t n, const uint8_t *__restrict__ free_mask, const uint16_t *__restrict__ meta,
                const double *__restrict__ bmat, float *__restrict__ binv, int *n_fallback) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned mt = meta[i];
        if (mt & 0xffu) continue;
        bj_invert_block(i, (int)(mt >> 8), is_free(free_mask, i), free_mask, bmat, binv, n_fallback);
    }
}

template <typename TT>
__global__ void __launch_bounds__(kEBlock)
    k_einit_bj(int32_t n, const uint8_t *__restrict__ free_mask, const double *__restrict__ b, double b_scale,
               const double *__restrict__ diag, const uint16_t *__restrict__ meta, const float *__restrict__ binv,
               DofPair<TT> *__restrict__ G, DofPair<TT> *__restrict__ R, PcgState *st, double *part, double rtol,
               double atol, long long maxit, int *bad) {
    __shared__ double sh[32];
    __shared__ TT s_r[kBjTile];
    double rz = 0.0, rr = 0.0;
    for (int64_t base = (int64_t)blockIdx.x * kBjTile; base < n; base += (int64_t)gridDim.x * kBjTile) {
        const int64_t i = base + threadIdx.x;
        const bool fr = i < n && is_free(free_mask, i);
        TT r = TT(0);
        unsigned mt = 0;
        float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
        if (fr) {
            const double dg = diag[i];
            if (dg == 0.0 || !isfinite(dg)) atomicExch(bad, 1);
            r = (TT)(b_scale * b[i]);
            mt = meta[i];
            bj_load(binv, i, ma, mb);
        }
        s_r[threadIdx.x] = r;
        __syncthreads();
        if (i < n) {
            const TT z = fr ? bj_row(mt, ma, mb, s_r, threadIdx.x) : TT(0);
            G[i] = DofPair<TT>{z, TT(0)};
            R[i] = DofPair<TT>{r, TT(0)};
            rz += (double)r * (double)z;
            rr += (double)r * (double)r;
        }
        __syncthreads();
    }
    const double a0 = block_sum(rz, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x] = a0;
    const double a1 = block_sum(rr, sh);
    if (threadIdx.x == 0) part[3 * blockIdx.x + 1] = a1;
    if (threadIdx.x == 0) part[3 * blockIdx.x + 2] = a1;
    if (last_block(&st->counter)) {
        const double s_rz = reduce_parts(part, gridDim.x, 3, 0, sh);
        const double s_rr = reduce_parts(part, gridDim.x, 3, 1, sh);
        if (threadIdx.x == 0) {
            st->rz = s_rz;
            st->rr = s_rr;
            st->bnorm = sqrt(s_rr);
            st->atol_eff = fmax(atol, rtol * st->bnorm);
            st->iter = 0;
            st->maxit = maxit;
            st->alpha = 0.0;
            st->beta = 0.0;
            int done = 0;
            if (s_rr == 0.0) done = 4;
            else if (!(s_rr == s_rr) || isinf(s_rr)) done = 3;
            else if (sqrt(s_rr) < st->atol_eff) done = 1;
            else if (maxit <= 0) done = 2;
            st->done = done;
        }
    }
}

template <typename TT>
__global__ void __launch_bounds__(kEBlock)
    k_epass2_bj(int32_t n, const uint8_t *__restrict__ free_mask, const int32_t *__restrict__ inc_ptr,
                const TT *__restrict__ Y, const uint16_t *__restrict__ meta, const float *__restrict__ binv,
                DofPair<TT> *__restrict__ G, DofPair<TT> *__restrict__ R, PcgState *st, double *part, int use_cond,
                cudaGraphConditionalHandle cond) {
    __shared__ double sh2[2][32];
    // float64: r of the tile in two alternating buffers, so a tile needs one barrier: it writes
    // the buffer its predecessor's predecessor read, which every thread has finished with once
    // past the barrier in between (77.8 -> 77.0 us per iteration at 1.16M tets; in float32 the
    // second barrier per tile measured slightly faster, 56.3 against 56.8 us, and stays)
    constexpr bool kTwoBuffers = sizeof(TT) == 8;
    __shared__ TT s_r2[2][kBjTile];
    // each tile's slot range is read one tile ahead (the first one before the CG state), so
    // that a tile's slot values are requested together with its DoF words
    // In float32 the tile's DoF states {z, p}, {r, x} are read one tile ahead as well (in float64
    // their registers would cost a resident block per SM).
    constexpr bool kStateAhead = sizeof(TT) == 4;
    const int64_t tstride = (int64_t)gridDim.x * kBjTile;
    int nb0 = 0, nb1 = 0;
    DofPair<TT> ng{TT(0), TT(0)}, nrx{TT(0), TT(0)};
    {
        const int64_t i0 = (int64_t)blockIdx.x * kBjTile + threadIdx.x;
        if (i0 < n) {
            nb0 = __ldcs(inc_ptr + i0);
            nb1 = __ldcs(inc_ptr + i0 + 1);
            if constexpr (kStateAhead) {
                ng = G[i0];
                nrx = R[i0];
            }
        }
    }
    if (st->done) {
        if (use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(cond, 0);
        return;
    }
    const TT alpha = (TT)st->alpha, beta = (TT)st->beta;
    double rz = 0.0, rr = 0.0;
    int par = 0;
    for (int64_t base = (int64_t)blockIdx.x * kBjTile; base < n; base += tstride, par ^= (kTwoBuffers ? 1 : 0)) {
        TT *s_r = s_r2[par];
        const int64_t i = base + threadIdx.x;
        const bool fr = i < n && is_free(free_mask, i);
        const int b0 = nb0, b1 = nb1;
        DofPair<TT> g = ng, rx = nrx;
        if (i + tstride < n) {
            nb0 = __ldcs(inc_ptr + i + tstride);
            nb1 = __ldcs(inc_ptr + i + tstride + 1);
            if constexpr (kStateAhead) {
                ng = G[i + tstride];
                nrx = R[i + tstride];
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
            // the DoF's words are requested before the slot values and the tile barrier; in
            // float64 the block row only as an L1 prefetch (its registers would cost a block per SM)
            mt = meta[i];
            if constexpr (sizeof(TT) == 4) bj_load(binv, i, ma, mb);
            else bj_prefetch(binv, i);
            double q = 0.0;
            for (int t = b0; t < b1; ++t) q += (double)Y[t];
            r = rx.a - alpha * (TT)q;
        }
        s_r[threadIdx.x] = r;
        __syncthreads();
        if (fr) {
            if constexpr (sizeof(TT) == 8) bj_load(binv, i, ma, mb);
            const TT z = bj_row(mt, ma, mb, s_r, threadIdx.x);
            const TT p = pnext(beta, g.b, g.a);
            G[i] = DofPair<TT>{z, p};
            R[i] = DofPair<TT>{r, rx.b + alpha * p};
            rz += (double)r * (double)z;
            rr += (double)r * (double)r;
        }
        if constexpr (!kTwoBuffers) __syncthreads();
    }
    block_sum2(rz, rr, sh2);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rz;
        part[2 * blockIdx.x + 1] = rr;
    }
    if (last_block(&st->counter)) {
        double a = 0.0, b = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            a += __ldcg(part + 2 * i);
            b += __ldcg(part + 2 * i + 1);
        }
        __syncthreads();
        block_sum2(a, b, sh2);
        if (threadIdx.x == 0) {
            const double rz_new = a, rr_new = b;
            st->beta = rz_new / st->rz;
            st->rz = rz_new;
            st->rr = rr_new;
            st->iter += 1;
            int done = 0;
            if (!(rr_new == rr_new) || isinf(rr_new)) done = 3;
            else if (sqrt(rr_new) < st->atol_eff) done = 1;
            else if (st->iter >= st->maxit) done = 2;
            st->done = done;
            if (use_cond && done) cudaGraphSetConditional(cond, 0);
        }
    }
}

// ---------------------------------------------------------------- one-launch PCG (cooperative)
//
// The whole Krylov loop of one Newton step in one cooperative launch (every block resident):
// per iteration the element pass and the DoF pass of k_epass1 / k_epass2_bj (or k_epass2) run
// back to back, separated by grid barriers instead of kernel boundaries; every block sums the
// per-block partials itself, in block order, so all blocks take the same alpha, beta and
// stopping decision without a serial last-block step.  Block 0 mirrors the state into *st for
// the host.  Each barrier wait is bounded: a block that gives up records the failure in *err
// and leaves; the others then give up at their next barrier.

struct GridBarrier {
    unsigned long long count;
};

constexpr long long kCoopSpin = 1ll << 26;

__device__ __forceinline__ bool grid_sync(GridBarrier *bar, unsigned long long &target, int *err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&bar->count, 1ull);
        target += gridDim.x;
        int ok = 0;
        for (long long k = 0; k < kCoopSpin; ++k) {
            unsigned long long c;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(c) : "l"(&bar->count) : "memory");
            if (c >= target) {
                ok = 1;
                break;
            }
        }
        if (!ok) atomicExch(err, 1);
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// sum of part[i * 3 + comp] over i < gridDim.x, the same order in every block; all threads
__device__ __forceinline__ double coop_sum(const double *part, int comp, double *sh) {
    double v = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v += __ldcg(part + 3 * i + comp);
    v = block_sum(v, sh);
    __shared__ double s_v;
    if (threadIdx.x == 0) s_v = v;
    __syncthreads();
    v = s_v;
    __syncthreads();
    return v;
}

template <typename TT, bool BJ>
__global__ void __launch_bounds__(kEBlock, kPass1MinBlocks)
    k_pcg_coop(int64_t ne, int32_t n, const int32_t *__restrict__ edof, const int32_t *__restrict__ pos,
               const TT *__restrict__ T, const TT *__restrict__ chat, const uint8_t *__restrict__ free_mask,
               const int32_t *__restrict__ inc_ptr, const uint16_t *__restrict__ meta, const float *__restrict__ binv,
               const TT *__restrict__ D, DofPair<TT> *__restrict__ G, DofPair<TT> *__restrict__ R, TT *__restrict__ Y,
               PcgState *st, double *part, GridBarrier *bar, int *err) {
    __shared__ TT sc[18];
    __shared__ double sh[32];
    __shared__ double sh2[2][32];
    __shared__ TT s_r[kBjTile];
    if (st->done) return;  // uniform: written by the start kernel before this launch
    if (threadIdx.x < 18) sc[threadIdx.x] = chat[threadIdx.x];
    __syncthreads();
    double rz = st->rz;
    const double atol_eff = st->atol_eff;
    const long long maxit = st->maxit;
    long long iter = 0;
    double beta = 0.0;
    unsigned long long target = 0;
    const int lane = threadIdx.x & 31;
    const int h = lane & 1;
    const int64_t wstride = (int64_t)gridDim.x * (blockDim.x >> 5) * 16;
    for (;;) {
        // ---- element pass (k_epass1)
        const TT tb = (TT)beta;
        double dot = 0.0;
#pragma unroll 1
        for (int64_t e0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 16; e0 < ne; e0 += wstride) {
            const int64_t e = e0 + (lane >> 1);
            const bool valid = e < ne;
            const int64_t eb = eslot(valid ? e : 0, 0);
            int32_t d[3], ps[3];
            TT th[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                d[j] = valid ? __ldcs(edof + eb + 32 * (3 * h + j)) : 0;
                ps[j] = valid ? __ldcs(pos + eb + 32 * (3 * h + j)) : 0;
                th[j] = valid ? __ldcs(T + eb + 32 * (3 * h + j)) : TT(0);
            }
            DofPair<TT> w[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) w[j] = G[(uint32_t)d[j] & ~kSignBit];
            TT u0 = TT(0), u1 = TT(0), u2 = TT(0);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                TT pk = pnext(tb, w[j].b, w[j].a);
                if (d[j] < 0) pk = -pk;
                const TT *c = sc + 3 * (3 * h + j);
                u0 += pk * c[0];
                u1 += pk * c[1];
                u2 += pk * c[2];
            }
            if (!valid) u0 = u1 = u2 = TT(0);
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
            if (!valid) continue;
            const TT v0 = t[0] * u0 + t[1] * u1 + t[2] * u2;
            const TT v1 = t[1] * u0 + t[3] * u1 + t[4] * u2;
            const TT v2 = t[2] * u0 + t[4] * u1 + t[5] * u2;
            if (!h) dot += (double)u0 * (double)v0 + (double)u1 * (double)v1 + (double)u2 * (double)v2;
#pragma unroll
            for (int j = 0; j < 3; ++j) Y[ps[j]] = edge_term(sc, 3 * h + j, d[j] < 0, v0, v1, v2);
        }
        dot = block_sum(dot, sh);
        if (threadIdx.x == 0) part[3 * blockIdx.x] = dot;
        if (!grid_sync(bar, target, err)) return;
        const double pq = coop_sum(part, 0, sh);
        const double alpha = rz / pq;
        // ---- DoF pass (k_epass2_bj / k_epass2)
        const TT ta = (TT)alpha;
        double rz_n = 0.0, rr_n = 0.0;
        if constexpr (BJ) {
            for (int64_t base = (int64_t)blockIdx.x * kBjTile; base < n; base += (int64_t)gridDim.x * kBjTile) {
                const int64_t i = base + threadIdx.x;
                const bool fr = i < n && is_free(free_mask, i);
                DofPair<TT> g{TT(0), TT(0)}, rx{TT(0), TT(0)};
                TT r = TT(0);
                unsigned mt = 0;
                float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
                if (fr) {
                    mt = meta[i];
                    if constexpr (sizeof(TT) == 4) bj_load(binv, i, ma, mb);
                    else bj_prefetch(binv, i);
                    g = G[i];
                    rx = R[i];
                    const int b0 = __ldcs(inc_ptr + i), b1 = __ldcs(inc_ptr + i + 1);
                    double q = 0.0;
                    for (int k = b0; k < b1; ++k) q += (double)Y[k];
                    r = rx.a - ta * (TT)q;
                }
                s_r[threadIdx.x] = r;
                __syncthreads();
                if (fr) {
                    if constexpr (sizeof(TT) == 8) bj_load(binv, i, ma, mb);
                    const TT z = bj_row(mt, ma, mb, s_r, threadIdx.x);
                    const TT p = pnext(tb, g.b, g.a);
                    G[i] = DofPair<TT>{z, p};
                    R[i] = DofPair<TT>{r, rx.b + ta * p};
                    rz_n += (double)r * (double)z;
                    rr_n += (double)r * (double)r;
                }
                __syncthreads();
            }
        } else {
            for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
                 i += (int64_t)gridDim.x * blockDim.x) {
                if (!is_free(free_mask, i)) continue;
                const DofPair<TT> g = G[i];
                const DofPair<TT> rx = R[i];
                const TT dv = D[i];
                const int b0 = __ldcs(inc_ptr + i), b1 = __ldcs(inc_ptr + i + 1);
                double q = 0.0;
                for (int k = b0; k < b1; ++k) q += (double)Y[k];
                const TT p = pnext(tb, g.b, g.a);
                const TT r = rx.a - ta * (TT)q;
                const TT z = dv * r;
                G[i] = DofPair<TT>{z, p};
                R[i] = DofPair<TT>{r, rx.b + ta * p};
                rz_n += (double)r * (double)z;
                rr_n += (double)r * (double)r;
            }
        }
        block_sum2(rz_n, rr_n, sh2);
        if (threadIdx.x == 0) {
            part[3 * blockIdx.x + 1] = rz_n;
            part[3 * blockIdx.x + 2] = rr_n;
        }
        if (!grid_sync(bar, target, err)) return;
        const double rz_new = coop_sum(part, 1, sh);
        const double rr_new = coop_sum(part, 2, sh);
        beta = rz_new / rz;
        rz = rz_new;
        iter += 1;
        int done = 0;
        if (!(rr_new == rr_new) || isinf(rr_new)) done = 3;
        else if (sqrt(rr_new) < atol_eff) done = 1;
        else if (iter >= maxit) done = 2;
        if (done) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                st->pq = pq;
                st->alpha = alpha;
                st->beta = beta;
                st->rz = rz;
                st->rr = rr_new;
                st->iter = iter;
                st->done = done;
            }
            return;
        }
    }
}

__global__ void k_bj_apply(int32_t n, const uint8_t *__restrict__ free_mask, const uint16_t *__restrict__ meta,
                           const float *__restrict__ binv, const double *__restrict__ r_in, double *__restrict__ z_out) {
    __shared__ double s_r[kBjTile];
    for (int64_t base = (int64_t)blockIdx.x * kBjTile; base < n; base += (int64_t)gridDim.x * kBjTile) {
        const int64_t i = base + threadIdx.x;
        const bool fr = i < n && is_free(free_mask, i);
        unsigned mt = 0;
        float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
        if (fr) {
            mt = meta[i];
            bj_load(binv, i, ma, mb);
        }
        s_r[threadIdx.x] = fr ? r_in[i] : 0.0;
        __syncthreads();
        if (i < n) z_out[i] = fr ? bj_row(mt, ma, mb, s_r, threadIdx.x) : 0.0;
        __syncthreads();
    }
}

// x_i += sum_c V[i][c] coef_c on the free DoFs: one warp per DoF, lanes over the columns,
// then a fixed shuffle tree (deterministic).
__global__ void k_basis_axpy(int32_t n, const uint8_t *__restrict__ free_mask, const float *__restrict__ V, int m,
                             int64_t ldv, const double *__restrict__ coef, double *__restrict__ x) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        if (!is_free(free_mask, i)) continue;
        double acc = 0.0;
        for (int c = lane; c < m; c += 32) acc = fma((double)V[i * ldv + c], coef[c], acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) x[i] += acc;
    }
}

template <typename TT>
const TT *chat_ptr(const ElemTopology &top);
template <>
const double *chat_ptr<double>(const ElemTopology &top) {
    return top.chat64.p;
}
template <>
const float *chat_ptr<float>(const ElemTopology &top) {
    return top.chat32.p;
}

}  // namespace

// ---------------------------------------------------------------- topology

int build_elem_topology(ElemTopology &top, int32_t n, const ElemBlock *blocks, int n_blocks, const double *ctab_host,
                        int32_t n_orient, cudaStream_t s, bool *usable) {
    *usable = false;
    SNP_REQUIRE(n > 0 && n_orient >= 1 && ctab_host != nullptr, "element topology: bad arguments");
    int64_t ne = 0;
    for (int b = 0; b < n_blocks; ++b) ne = ne > blocks[b].offset + blocks[b].count ? ne : blocks[b].offset + blocks[b].count;
    if (ne <= 0 || ne >= ((int64_t)1 << 28)) return SNP_OK;  // (e << 3 | k) must fit in 31 bits
    // every orientation's curls must be +-(orientation 0's), edge by edge
    std::vector<int8_t> sgn((size_t)n_orient * 6, 1);
    for (int o = 0; o < n_orient; ++o)
        for (int j = 0; j < 6; ++j) {
            const double *c = ctab_host + ((size_t)o * 6 + j) * 3;
            const double *c0 = ctab_host + (size_t)j * 3;
            bool plus = true, minus = true;
            for (int k = 0; k < 3; ++k) {
                plus = plus && (c[k] == c0[k]);
                minus = minus && (c[k] == -c0[k]);
            }
            if (!plus && !minus) return SNP_OK;
            sgn[(size_t)o * 6 + j] = plus ? 1 : -1;
        }
    DevBuf<int8_t> d_sgn;
    DevBuf<int> bad;
    SNP_TRY(d_sgn.alloc(sgn.size()));
    SNP_TRY(bad.alloc(1));
    SNP_CUDA_TRY(cudaMemcpyAsync(d_sgn.p, sgn.data(), sgn.size(), cudaMemcpyHostToDevice, s));
    SNP_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    SNP_TRY(top.edof.alloc(eslots_size(ne)));
    SNP_CUDA_TRY(cudaMemsetAsync(top.edof.p, 0, sizeof(int32_t) * eslots_size(ne), s));
    for (int b = 0; b < n_blocks; ++b) {
        if (blocks[b].count == 0) continue;
        k_edof<<<stride_grid(blocks[b].count, 256, 8), 256, 0, s>>>(blocks[b].count, blocks[b].offset, ne,
                                                                     blocks[b].gids, blocks[b].orient, d_sgn.p,
                                                                     n_orient, n, top.edof.p, bad.p);
        SNP_LAUNCH_CHECK();
    }
    // incidence: stable radix sort of (DoF, entry) pairs keeps each DoF's entries in (e, k) order
    const int64_t m = 6 * ne;
    DevBuf<int32_t> key, key2, val, cnt;
    SNP_TRY(key.alloc(m));
    SNP_TRY(key2.alloc(m));
    SNP_TRY(val.alloc(m));
    SNP_TRY(top.inc.alloc(m));
    SNP_TRY(cnt.alloc((size_t)n + 1));
    SNP_TRY(top.inc_ptr.alloc((size_t)n + 1));
    SNP_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * ((size_t)n + 1), s));
    k_inc_keys<<<stride_grid(m, 256, 8), 256, 0, s>>>(ne, top.edof.p, key.p, val.p, cnt.p);
    SNP_LAUNCH_CHECK();
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < (int64_t)n) ++end_bit;
    cub::DoubleBuffer<int32_t> dk(key.p, key2.p);
    cub::DoubleBuffer<int32_t> dv(val.p, top.inc.p);
    size_t tb_sort = 0, tb_scan = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, dk, dv, (int)m, 0, end_bit, s);
    cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, cnt.p, top.inc_ptr.p, n + 1, s);
    DevBuf<unsigned char> temp;
    SNP_TRY(temp.alloc(tb_sort > tb_scan ? tb_sort : tb_scan));
    SNP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, tb_sort, dk, dv, (int)m, 0, end_bit, s));
    if (dv.Current() != top.inc.p)
        SNP_CUDA_TRY(cudaMemcpyAsync(top.inc.p, dv.Current(), sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, s));
    SNP_CUDA_TRY(cub::DeviceScan::ExclusiveSum(temp.p, tb_scan, cnt.p, top.inc_ptr.p, n + 1, s));
    SNP_TRY(top.pos.alloc(eslots_size(ne)));
    SNP_CUDA_TRY(cudaMemsetAsync(top.pos.p, 0, sizeof(int32_t) * eslots_size(ne), s));
    k_inc_pos<<<stride_grid(m, 256, 8), 256, 0, s>>>(m, ne, top.inc.p, top.pos.p);
    SNP_LAUNCH_CHECK();
    double c64[18];
    float c32[18];
    for (int t = 0; t < 18; ++t) {
        c64[t] = ctab_host[t];
        c32[t] = (float)ctab_host[t];
    }
    SNP_TRY(top.chat64.alloc(18));
    SNP_TRY(top.chat32.alloc(18));
    SNP_CUDA_TRY(cudaMemcpyAsync(top.chat64.p, c64, sizeof(c64), cudaMemcpyHostToDevice, s));
    SNP_CUDA_TRY(cudaMemcpyAsync(top.chat32.p, c32, sizeof(c32), cudaMemcpyHostToDevice, s));
    int hbad = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    SNP_REQUIRE(hbad == 0, "element topology: a DoF index or orientation is out of range");
    top.n_elems = ne;
    top.n = n;
    *usable = true;
    return SNP_OK;
}

int elem_sum_to_dofs(const ElemTopology &top, const double *Fe, const double *De, const double *rhs_extra,
                     double *F, double *diag, cudaStream_t s) {
    SNP_REQUIRE(top.n > 0 && top.n_elems > 0, "element sums: topology not built");
    k_sum_to_dofs<<<stride_grid(top.n, kEBlock, 8), kEBlock, 0, s>>>(top.n, top.n_elems, top.inc_ptr.p, top.inc.p, Fe,
                                                                    De, rhs_extra, F, diag);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

// ---------------------------------------------------------------- PCG engine

template <typename TT>
ElemPcg<TT>::~ElemPcg() {
    drop_graph();
}

template <typename TT>
void ElemPcg<TT>::drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
}

template <typename TT>
int ElemPcg<TT>::reserve(int32_t n_, int64_t ne_) {
    if (n_ == n && ne_ == ne && G.p) return SNP_OK;
    drop_graph();
    n = n_;
    ne = ne_;
    SNP_TRY(G.alloc(n));
    SNP_TRY(R.alloc(n));
    SNP_TRY(D.alloc(n));
    SNP_TRY(Y.alloc(6 * ne));
    const int gmax = sm_count() * 8 + 1;
    SNP_TRY(part.alloc(3 * (size_t)gmax));
    SNP_TRY(st.alloc(1));
    SNP_TRY(hst.alloc(1));
    SNP_TRY(bad.alloc(1));
    SNP_CUDA_TRY(cudaMemset(st.p, 0, sizeof(PcgState)));
    return SNP_OK;
}

template <typename TT>
int ElemPcg<TT>::launch_iteration(const ElemTopology &top, const TT *T, const uint8_t *free_mask,
                                  const uint16_t *bj_meta, const float *bj_inv, cudaStream_t s, int use_cond,
                                  cudaGraphConditionalHandle cond) {
    const TT *chat = chat_ptr<TT>(top);
    k_epass1<TT><<<wave_grid(k_epass1<TT>, 2 * ne, kEBlock), kEBlock, 0, s>>>(ne, top.edof.p, top.pos.p, T, chat, G.p,
                                                                         Y.p, st.p, part.p);
    SNP_LAUNCH_CHECK();
    if (bj_meta)
        k_epass2_bj<TT><<<wave_grid(k_epass2_bj<TT>, n, kEBlock), kEBlock, 0, s>>>(
            n, free_mask, top.inc_ptr.p, Y.p, bj_meta, bj_inv, G.p, R.p, st.p, part.p, use_cond, cond);
    else
        k_epass2<TT><<<wave_grid(k_epass2<TT>, n, kEBlock), kEBlock, 0, s>>>(n, free_mask, top.inc_ptr.p, Y.p, G.p,
                                                                            R.p, D.p, st.p, part.p, use_cond, cond);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

// L2 residency of the slot values between the element pass (which writes them) and the DoF
// pass (which reads them): the iteration's kernel nodes get an access policy window over Y with
// persisting hits, and this context's persisting L2 set-aside is raised to cover it (up to the
// device's maximum; it lasts as long as the context).  Measured on the 1.16M-tet benchmark: 92.5
// -> 84.1 us per float64 PCG iteration.  SNP_L2_PERSIST=0 leaves the nodes' cache policy alone.
bool l2_window_on_kernels(cudaGraph_t body, const void *base, size_t bytes) {
    const char *env = getenv("SNP_L2_PERSIST");
    if (env && env[0] == '0') return false;
    int dev = 0, max_persist = 0, max_win = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, dev) != cudaSuccess ||
        max_persist <= 0 || max_win <= 0) {
        cudaGetLastError();
        return false;
    }
    // only a window that covers the whole array: a partial one (hit ratio below 1) marks the
    // rest streaming, which evicts it early and made a 187 MB slot array three times slower
    if (bytes > (size_t)max_win || bytes > (size_t)max_persist) return false;
    const size_t win = bytes, keep = bytes;
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, keep) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaKernelNodeAttrValue v = {};
    v.accessPolicyWindow.base_ptr = const_cast<void *>(base);
    v.accessPolicyWindow.num_bytes = win;
    v.accessPolicyWindow.hitRatio = 1.0f;
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    size_t n = 0;
    if (cudaGraphGetNodes(body, nullptr, &n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return false;
    }
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(body, nodes.data(), &n) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
            cudaGraphKernelNodeSetAttribute(nd, cudaKernelNodeAttributeAccessPolicyWindow, &v);
    }
    cudaGetLastError();
    return true;
}

template <typename TT>
int ElemPcg<TT>::build_graph(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const uint16_t *bj_meta,
                             const float *bj_inv) {
    drop_graph();
    l2_window = false;
    const char *env = getenv("SNP_PCG_GRAPH");
    if (env && env[0] == '0') return SNP_OK;
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) {
        cudaGetLastError();
        return SNP_OK;
    }
    cudaGraphConditionalHandle h;
    cudaGraphNode_t node;
    cudaGraphNodeParams cp = {};
    bool ok = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&node, g, nullptr, 0, &cp) == cudaSuccess;
    }
    cudaStream_t cs = nullptr;
    if (ok) ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            const int unroll = pcg_body_unroll();
            int rc = SNP_OK;
            for (int u = 0; u < unroll && rc == SNP_OK; ++u)
                rc = launch_iteration(top, T, free_mask, bj_meta, bj_inv, cs, 1, h);
            cudaGraph_t out = nullptr;
            cudaError_t e = cudaStreamEndCapture(cs, &out);
            ok = (rc == SNP_OK) && e == cudaSuccess;
            if (ok) {
                l2_bytes = sizeof(TT) * 6 * (size_t)ne;
                l2_window = l2_window_on_kernels(body, Y.p, l2_bytes);
            }
        }
    }
    if (ok) ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
    if (cs) cudaStreamDestroy(cs);
    if (!ok) {
        cudaGetLastError();
        clear_error();
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        cudaGraphDestroy(g);
        return SNP_OK;
    }
    graph = g;
    key_top = &top;
    key_T = T;
    key_fm = free_mask;
    key_bm = bj_meta;
    key_bi = bj_inv;
    return SNP_OK;
}

// The iteration loop as one cooperative launch (k_pcg_coop); false when the device cannot
// hold the grid (the caller then uses the graph).  *rc: the launch's status and the barrier's.
template <typename TT>
bool ElemPcg<TT>::solve_coop(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const uint16_t *bj_meta,
                             const float *bj_inv, cudaStream_t s, int *rc) {
    *rc = SNP_OK;
    auto kern = bj_meta ? k_pcg_coop<TT, true> : k_pcg_coop<TT, false>;
    int dev = 0, coop = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        !coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kEBlock, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return false;
    }
    const int grid = sm_count() * per_sm;
    if ((size_t)grid * 3 > part.n) return false;  // part holds 3 x (8 blocks per SM + 1)
    if (!coop_bar.p && (coop_bar.alloc(1) != SNP_OK || coop_err.alloc(1) != SNP_OK)) {
        clear_error();
        return false;
    }
    if (cudaMemsetAsync(coop_bar.p, 0, sizeof(GridBarrier), s) != cudaSuccess ||
        cudaMemsetAsync(coop_err.p, 0, sizeof(int), s) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int64_t ne_ = ne;
    int32_t n_ = n;
    const int32_t *edof = top.edof.p, *pos = top.pos.p, *ip = top.inc_ptr.p;
    const TT *chat = chat_ptr<TT>(top);
    const TT *Dp = D.p;
    DofPair<TT> *Gp = G.p, *Rp = R.p;
    TT *Yp = Y.p;
    PcgState *stp = st.p;
    double *pp = part.p;
    GridBarrier *bp = reinterpret_cast<GridBarrier *>(coop_bar.p);
    int *ep = coop_err.p;
    void *args[] = {&ne_, &n_, &edof, &pos, &T, &chat, &free_mask, &ip, &bj_meta, &bj_inv, &Dp, &Gp, &Rp, &Yp,
                    &stp, &pp, &bp, &ep};
    const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kern), dim3(grid), dim3(kEBlock),
                                                      args, 0, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int herr = 0;
    if (cudaMemcpyAsync(&herr, coop_err.p, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        *rc = fail(SNP_CUDA_ERROR, "element PCG: %s", cudaGetErrorString(cudaGetLastError()));
        return true;
    }
    if (herr) *rc = fail(SNP_CUDA_ERROR, "element PCG: a grid barrier of the one-launch loop timed out");
    return true;
}

template <typename TT>
int ElemPcg<TT>::solve(const ElemTopology &top, const TT *T, const double *diag, const uint8_t *free_mask,
                       const double *b, double b_scale, double *h, double rtol, double atol, int64_t maxit,
                       cudaStream_t s, int64_t *its, double *res, int *status, const uint16_t *bj_meta,
                       const float *bj_inv) {
    bool hold = false;  // this solve raised the L2 set-aside
    SNP_REQUIRE((bj_meta == nullptr) == (bj_inv == nullptr), "element PCG: block Jacobi needs both meta and inverse");
    SNP_REQUIRE(top.n > 0 && top.n_elems > 0, "element PCG: topology not built");
    SNP_TRY(reserve(top.n, top.n_elems));
    if (maxit < 0) maxit = 10 * (int64_t)n;
    SNP_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    if (bj_meta)
        k_einit_bj<TT><<<wave_grid(k_einit_bj<TT>, n, kEBlock), kEBlock, 0, s>>>(
            n, free_mask, b, b_scale, diag, bj_meta, bj_inv, G.p, R.p, st.p, part.p, rtol, atol, (long long)maxit, bad.p);
    else
        k_einit<TT><<<wave_grid(k_einit<TT>, n, kEBlock), kEBlock, 0, s>>>(n, free_mask, b, b_scale, diag, G.p, R.p,
                                                                          D.p, st.p, part.p, rtol, atol,
                                                                          (long long)maxit, bad.p);
    SNP_LAUNCH_CHECK();
    launches += 1;
    int hbad = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    if (hbad) {
        if (status) *status = SNP_ZERO_PIVOT;
        return fail(SNP_ZERO_PIVOT, "element PCG: zero or non-finite Jacobian diagonal on a free DoF");
    }
    int64_t chunk_launches = -1;
    const char *coop_env = getenv("SNP_PCG_COOP");
    if (coop_env && coop_env[0] == '1') {
        int coop_rc = SNP_OK;
        if (solve_coop(top, T, free_mask, bj_meta, bj_inv, s, &coop_rc)) {
            SNP_TRY(coop_rc);
            chunk_launches = 1;
            goto extract;
        }
    }
    {
    const bool same = exec && key_top == &top && key_T == T && key_fm == free_mask && key_bm == bj_meta &&
                      key_bi == bj_inv;
    if (!same) SNP_TRY(build_graph(top, T, free_mask, bj_meta, bj_inv));
    }
    hold = exec && l2_window && l2_hold;
    if (exec) {
        // the L2 set-aside for the slot values' persisting lines, only while this solve runs
        if (hold && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, l2_bytes) != cudaSuccess) cudaGetLastError();
        SNP_CUDA_TRY(cudaGraphLaunch(exec, s));
    } else {
        const int chunk = 32;
        int64_t launched = 0;
        while (true) {
            for (int k = 0; k < chunk; ++k) SNP_TRY(launch_iteration(top, T, free_mask, bj_meta, bj_inv, s, 0, 0));
            launched += chunk;
            SNP_CUDA_TRY(cudaMemcpyAsync(hst.p, st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
            SNP_CUDA_TRY(cudaStreamSynchronize(s));
            if (hst.p->done || launched > maxit + chunk) break;
        }
        chunk_launches = 2 * launched;
    }
extract:
    k_eextract<TT><<<stride_grid(n, kEBlock, 8), kEBlock, 0, s>>>(n, R.p, h);
    SNP_LAUNCH_CHECK();
    SNP_CUDA_TRY(cudaMemcpyAsync(hst.p, st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    // the slot values' persisting lines go back to normal and the set-aside is released once
    // the solve is over, so that they do not hold the L2 against whatever the program runs next
    if (hold) {
        cudaCtxResetPersistingL2Cache();
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
        cudaGetLastError();
    }
    const PcgState &H = *hst.p;
    launches += 1 + (chunk_launches >= 0 ? chunk_launches : 2 * (H.iter > 0 ? H.iter : 1));
    if (its) *its = H.iter;
    if (res) *res = sqrt(H.rr);
    int stt = SNP_OK;
    if (H.done == 2) stt = SNP_NOT_CONVERGED;
    else if (H.done == 3) stt = SNP_NAN_DETECTED;
    if (status) *status = stt;
    return SNP_OK;
}

template <typename TT>
int ElemPcg<TT>::apply(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const TT *x, TT *y,
                       cudaStream_t s) {
    SNP_REQUIRE(top.n > 0 && top.n_elems > 0, "element operator: topology not built");
    SNP_TRY(reserve(top.n, top.n_elems));
    const TT *chat = chat_ptr<TT>(top);
    k_eapply1<TT><<<wave_grid(k_eapply1<TT>, ne, kEBlock), kEBlock, 0, s>>>(ne, top.edof.p, top.pos.p, T, chat,
                                                                           free_mask, x, Y.p);
    SNP_LAUNCH_CHECK();
    k_eapply2<TT><<<wave_grid(k_eapply2<TT>, n, kEBlock), kEBlock, 0, s>>>(n, free_mask, top.inc_ptr.p, Y.p, y);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

template <typename TT>
int elem_reduced_system(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const float *V, int m,
                        int64_t ldv, const double *F, double *Jr, double *g, DevBuf<double> &scratch,
                        cudaStream_t s) {
    SNP_REQUIRE(top.n > 0 && top.n_elems > 0, "reduced system: topology not built");
    SNP_REQUIRE(V != nullptr && Jr != nullptr, "reduced system: V or Jr is NULL");
    SNP_REQUIRE(m >= 1 && m <= 2 * kRsB && ldv >= m, "reduced system: need 1 <= m <= %d and ldv >= m", 2 * kRsB);
    SNP_REQUIRE(F == nullptr || g != nullptr, "reduced system: F given without g");
    const int nb = (m + kRsB - 1) / kRsB, n_jobs = nb * (nb + 1) / 2;
    // set once per process (thread-safe static initialisation)
    static const cudaError_t smem_rc = [] {
        cudaError_t e = cudaFuncSetAttribute(k_rsys_jac<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRsSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_rsys_jac<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRsSmem);
        return e;
    }();
    SNP_CUDA_TRY(smem_rc);
    const int64_t n_groups = (top.n_elems + 31) >> 5;
    int per_sm = resident_blocks(reinterpret_cast<const void *>(k_rsys_jac<TT>), 256, kRsSmem);
    if (per_sm < 1) per_sm = 1;
    int64_t gx = ((int64_t)sm_count() * per_sm + n_jobs - 1) / n_jobs;
    if (gx > n_groups) gx = n_groups;
    const int gr = 4 * sm_count();
    const size_t need = (size_t)n_jobs * gx * kRsB * kRsB + (size_t)nb * gr * kRsB;
    if (scratch.n < need) SNP_TRY(scratch.alloc(need));
    double *pj = scratch.p, *pr = scratch.p + (size_t)n_jobs * gx * kRsB * kRsB;
    k_rsys_jac<TT><<<dim3((unsigned)gx, (unsigned)n_jobs), 256, kRsSmem, s>>>(top.n_elems, top.edof.p, T,
                                                                            chat_ptr<TT>(top), free_mask, V, m, ldv,
                                                                            nb, pj);
    SNP_LAUNCH_CHECK();
    const int tot = n_jobs * kRsB * kRsB;
    k_rsys_jac_sum<<<(tot + 255) / 256, 256, 0, s>>>((int)gx, n_jobs, nb, m, pj, Jr);
    SNP_LAUNCH_CHECK();
    if (F) {
        k_rsys_rhs<<<dim3((unsigned)gr, (unsigned)nb), 256, 0, s>>>(top.n, free_mask, V, m, ldv, F, pr);
        SNP_LAUNCH_CHECK();
        k_rsys_rhs_sum<<<(m + 127) / 128, 128, 0, s>>>(gr, m, pr, g);
        SNP_LAUNCH_CHECK();
    }
    return SNP_OK;
}

template <typename TT>
int block_jacobi_build(const ElemTopology &top, const TT *T, const uint8_t *free_mask, const uint16_t *meta,
                       double *bmat, float *binv, int *fallback_count, cudaStream_t s) {
    SNP_REQUIRE(top.n > 0 && top.n_elems > 0, "block Jacobi: topology not built");
    SNP_REQUIRE(meta && bmat && binv && fallback_count, "block Jacobi: NULL buffer");
    k_bj_entries<TT><<<wave_grid(k_bj_entries<TT>, top.n, kEBlock), kEBlock, 0, s>>>(
        top.n, free_mask, top.inc_ptr.p, top.inc.p, top.edof.p, T, chat_ptr<TT>(top), meta, bmat);
    SNP_LAUNCH_CHECK();
    k_bj_invert<<<stride_grid(top.n, 128, 8), 128, 0, s>>>(top.n, free_mask, meta, bmat, binv, fallback_count);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

template int block_jacobi_build<double>(const ElemTopology &, const double *, const uint8_t *, const uint16_t *,
                                        double *, float *, int *, cudaStream_t);
template int block_jacobi_build<float>(const ElemTopology &, const float *, const uint8_t *, const uint16_t *,
                                       double *, float *, int *, cudaStream_t);

int block_jacobi_apply(int32_t n, const uint8_t *free_mask, const uint16_t *meta, const float *binv, const double *r,
                       double *z, cudaStream_t s) {
    SNP_REQUIRE(meta && binv && r && z && n > 0, "block Jacobi apply: bad arguments");
    k_bj_apply<<<wave_grid(k_bj_apply, n, kEBlock), kEBlock, 0, s>>>(n, free_mask, meta, binv, r, z);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

int basis_axpy(int32_t n, const uint8_t *free_mask, const float *V, int m, int64_t ldv, const double *coef,
               double *x, cudaStream_t s) {
    SNP_REQUIRE(V != nullptr && coef != nullptr && x != nullptr && m >= 1 && ldv >= m, "basis axpy: bad arguments");
    k_basis_axpy<<<wave_grid(k_basis_axpy, 32 * (int64_t)n, kEBlock), kEBlock, 0, s>>>(n, free_mask, V, m, ldv, coef, x);
    SNP_LAUNCH_CHECK();
    return SNP_OK;
}

template int elem_reduced_system<double>(const ElemTopology &, const double *, const uint8_t *, const float *, int,
                                         int64_t, const double *, double *, double *, DevBuf<double> &, cudaStream_t);
template int elem_reduced_system<float>(const ElemTopology &, const float *, const uint8_t *, const float *, int,
                                        int64_t, const double *, double *, double *, DevBuf<double> &, cudaStream_t);

template struct ElemPcg<double>;
template struct ElemPcg<float>;

}  // namespace snp
