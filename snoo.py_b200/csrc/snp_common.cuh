// Shared helpers of the snoopy_b200 CUDA library: error plumbing, launch geometry and
// the device-side material laws.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "snoopy_b200.h"

namespace snp {

// Record a message for snp_last_error() and return `code`.
int fail(int code, const char *fmt, ...);
void clear_error();

#define SNP_CUDA_TRY(expr)                                                                              \
    do {                                                                                                \
        cudaError_t _e = (expr);                                                                        \
        if (_e != cudaSuccess)                                                                          \
            return ::snp::fail(SNP_CUDA_ERROR, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                               __FILE__, __LINE__);                                                     \
    } while (0)

#define SNP_LAUNCH_CHECK() SNP_CUDA_TRY(cudaGetLastError())

#define SNP_REQUIRE(cond, ...)                                          \
    do {                                                                \
        if (!(cond)) return ::snp::fail(SNP_BAD_ARG, __VA_ARGS__);      \
    } while (0)

#define SNP_TRY(expr)                  \
    do {                               \
        int _s = (expr);               \
        if (_s != SNP_OK) return _s;   \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (148 on B200); cached per device.
int sm_count();

// Grid for a grid-stride loop over n items: a multiple of the SM count, at most
// `per_sm` blocks per SM, never more blocks than needed.
inline int stride_grid(int64_t n, int block, int per_sm) {
    int64_t need = (n + block - 1) / block;
    int64_t cap = (int64_t)sm_count() * per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

// Blocks of `block` threads (with `smem` dynamic shared bytes) of `kernel` that one SM holds
// at once (occupancy API, cached per kernel and device; at most 8, at least 1).
int resident_blocks(const void *kernel, int block, size_t smem);

// Grid for a grid-stride kernel: enough blocks for n_threads, capped at one full wave of
// resident blocks, so no block waits for a second wave.
template <typename Kernel>
inline int wave_grid(Kernel kernel, int64_t n_threads, int block, size_t smem = 0) {
    int64_t need = (n_threads + block - 1) / block;
    if (need < 1) need = 1;
    const int64_t cap = (int64_t)sm_count() * resident_blocks(reinterpret_cast<const void *>(kernel), block, smem);
    return (int)(need < cap ? need : cap);
}

constexpr double kNu0 = 1.0 / 4.0 / 3.14159265358979323846 * 1e7;  // vacuum reluctance

// ---------------------------------------------------------------- material laws

// PCHIP reluctance in piecewise-polynomial form (c[4][n_int] row-major, knots x[n_int+1]):
// n_int == -1 is the constant c[0]; below x[0] (or NaN) 0; at/after x[n_int] the last
// cubic extrapolates.  Binary search instead of the reference's linear scan
// (fem_c/ctools.c:130-204); same interval choice.
template <typename T>
__device__ __forceinline__ T pchip_eval(int n_int, const T *__restrict__ c, const T *__restrict__ xk, T x, T &dval) {
    if (n_int < 0) {
        dval = T(0);
        return c[0];
    }
    if (!(x >= xk[0])) {
        dval = T(0);
        return T(0);
    }
    int i;
    if (x >= xk[n_int]) {
        i = n_int - 1;
    } else {
        int lo = 0, hi = n_int - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (xk[mid] <= x) lo = mid; else hi = mid - 1;
        }
        i = lo;
    }
    T d = x - xk[i];
    T c0 = c[i], c1 = c[n_int + i], c2 = c[2 * n_int + i], c3 = c[3 * n_int + i];
    dval = (T(3) * c0 * d + T(2) * c1) * d + c2;
    return ((c0 * d + c1) * d + c2) * d + c3;
}

// mu(|H|) and dmu/d|H| of the B-spline permeability in x = log10|H| (fem_c/ctools.c:206-346).
// Only the k+1 basis functions whose support holds x are evaluated; their values are the
// reference recursion's, term by term.  Beyond the last knot every basis function is 0
// (half-open intervals), as in the reference.
constexpr int kMaxSplineDegree = 7;

__device__ __forceinline__ double bspline_mu(int type, int k, int n_ctrl, const double *__restrict__ t,
                                             const double *__restrict__ c, double H_min, double mu_H_min,
                                             double H, double &dmu) {
    if (type == 0 || H < H_min) {
        dmu = 0.0;
        return mu_H_min;
    }
    double x = log10(H);
    int n_t = n_ctrl + k + 1;
    // span s: t[s] <= x < t[s+1]
    if (!(x >= t[0]) || !(x < t[n_t - 1])) {
        dmu = 0.0;
        return 0.0;
    }
    int lo = 0, hi = n_t - 2;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (t[mid] <= x) lo = mid; else hi = mid - 1;
    }
    int s = lo;
    // N[d][r] = N_{s-d+r, d}(x), r = 0..d
    double N[kMaxSplineDegree + 2];
    double Nprev[kMaxSplineDegree + 2];
    for (int r = 0; r <= k + 1; ++r) N[r] = 0.0;
    N[0] = 1.0;
    double dN[kMaxSplineDegree + 2];
    for (int r = 0; r <= k + 1; ++r) dN[r] = 0.0;
    for (int d = 1; d <= k; ++d) {
        for (int r = 0; r < d; ++r) Nprev[r] = N[r];
        // basis i = s-d+r, r = 0..d; uses N_{i,d-1} (= Nprev[r-1]) and N_{i+1,d-1} (= Nprev[r])
        for (int r = 0; r <= d; ++r) {
            int i = s - d + r;
            if (i > n_t - 2 - d) {  // no degree-d basis function with this index
                N[r] = 0.0;
                dN[r] = 0.0;
                continue;
            }
            double lft = (r >= 1) ? Nprev[r - 1] : 0.0;
            double rgt = (r < d) ? Nprev[r] : 0.0;
            double a = 0.0, b = 0.0;
            if (i >= 0 && t[i + d] != t[i]) a = (x - t[i]) / (t[i + d] - t[i]) * lft;
            if (i + 1 >= 0 && t[i + d + 1] != t[i + 1]) b = (t[i + d + 1] - x) / (t[i + d + 1] - t[i + 1]) * rgt;
            if (d == k) {
                double t1 = 0.0, t2 = 0.0;
                if (i >= 0 && t[i + d] != t[i]) t1 = d / (t[i + d] - t[i]) * lft;
                if (i + 1 >= 0 && t[i + d + 1] != t[i + 1]) t2 = d / (t[i + d + 1] - t[i + 1]) * rgt;
                dN[r] = t1 - t2;
            }
            N[r] = a + b;
        }
    }
    double v = 0.0, dv = 0.0;
    for (int r = 0; r <= k; ++r) {
        int i = s - k + r;
        if (i >= 0 && i < n_ctrl) {
            v += c[i] * N[r];
            dv += c[i] * dN[r];
        }
    }
    if (k == 0) dv = 0.0;
    dmu = dv / (H * log(10.0));
    return v;
}

// ---------------------------------------------------------------- reductions

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; result valid in thread 0.  `sh` holds >= 32 values.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T *sh) {
    v = warp_sum(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : T(0);
    if (wid == 0) v = warp_sum(v);
    return v;
}

}  // namespace snp
