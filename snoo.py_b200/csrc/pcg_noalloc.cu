// snp_pcg_noalloc: the Jacobi-preconditioned CG of snp_pcg for callers that cannot allocate
// device memory.
//
// Some callers may not call cudaMalloc/cudaFree at the point where they solve: a service that
// hands all device memory to its own pool at start-up and forbids allocation afterwards, or a
// latency-critical loop where cudaFree's implicit device synchronisation would stall other
// streams.  snp_pcg allocates its work vectors on every call; this entry point takes them from
// one statically sized array in device memory instead.  The array is part of the module image:
// every GPU that loads this library holds it until the process exits.
//
// Host code cannot use the array's name as a device address (it names a host-side shadow), so
// every call looks the address up with cudaGetSymbolAddress, with the calling thread's current
// device current, and checks the result.  The lookup allocates nothing; doing it per call (not
// once per device) keeps the address right after cudaDeviceReset or when another context of
// the device becomes current, either of which reloads the module at a new address.
// The call synchronises `stream` (it reads the row count and the CG state back).
// All calls share the array: calls whose work overlaps on the GPU (different streams, threads
// or processes sharing a context) race on it and must be serialised by the caller.
#include "snp_common.cuh"
#include "snp_internal.cuh"
#include "snp_krylov.cuh"

namespace snp {
namespace {

constexpr int64_t kMaxRows = SNP_PCG_NOALLOC_MAX_ROWS;
constexpr int kMaxBlocks = 4096;  // partial-sum slots (>= the 8 blocks per SM the kernels launch)

// layout of the scratch array (byte offsets, each 256-byte aligned)
constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kVecBytes = align256(sizeof(double) * kMaxRows);
constexpr size_t kOffR = 0;
constexpr size_t kOffZ = kOffR + kVecBytes;
constexpr size_t kOffP = kOffZ + kVecBytes;
constexpr size_t kOffQ = kOffP + kVecBytes;
constexpr size_t kOffDinv = kOffQ + kVecBytes;
constexpr size_t kOffDiag = kOffDinv + kVecBytes;
constexpr size_t kOffPart = kOffDiag + align256(sizeof(int32_t) * kMaxRows);
constexpr size_t kOffState = kOffPart + align256(sizeof(double) * 3 * kMaxBlocks);
constexpr size_t kOffBad = kOffState + align256(sizeof(PcgState));
constexpr size_t kScratchBytes = kOffBad + 256;

static __device__ __align__(256) unsigned char g_pcg_scratch[kScratchBytes];

// Device address of g_pcg_scratch in the current device's current context.
int scratch_address(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        return fail(SNP_CUDA_ERROR, "snp_pcg_noalloc: cudaGetSymbolAddress of the scratch array failed: %s",
                    cudaGetErrorString(e));
    }
    *out = static_cast<unsigned char *>(p);
    return SNP_OK;
}

}  // namespace
}  // namespace snp

extern "C" int snp_pcg_noalloc(int32_t n_rows, const int32_t *row_ptr, const int32_t *col_idx, const double *vals,
                               const uint8_t *free_mask, const double *b, double *x, double rtol, double atol,
                               int64_t maxiter, int64_t *iterations, double *res_norm, void *stream) {
    snp::clear_error();
    SNP_REQUIRE(n_rows > 0, "snp_pcg_noalloc: n_rows must be positive");
    SNP_REQUIRE(n_rows <= snp::kMaxRows,
                "snp_pcg_noalloc: %d rows exceed the static work space of %lld rows (use snp_pcg)", n_rows,
                (long long)snp::kMaxRows);
    SNP_REQUIRE(row_ptr && col_idx && vals && b && x, "snp_pcg_noalloc: NULL argument");
    SNP_REQUIRE(rtol >= 0 && atol >= 0, "snp_pcg_noalloc: tolerances must be non-negative");
    cudaStream_t s = snp::as_stream(stream);
    unsigned char *base = nullptr;
    SNP_TRY(snp::scratch_address(&base));
    snp::PcgBuffers B;
    B.r = reinterpret_cast<double *>(base + snp::kOffR);
    B.z = reinterpret_cast<double *>(base + snp::kOffZ);
    B.p = reinterpret_cast<double *>(base + snp::kOffP);
    B.q = reinterpret_cast<double *>(base + snp::kOffQ);
    B.dinv = reinterpret_cast<double *>(base + snp::kOffDinv);
    B.diag = reinterpret_cast<int32_t *>(base + snp::kOffDiag);
    B.part = reinterpret_cast<double *>(base + snp::kOffPart);
    B.st = reinterpret_cast<snp::PcgState *>(base + snp::kOffState);
    B.bad = reinterpret_cast<int *>(base + snp::kOffBad);
    B.max_blocks = snp::kMaxBlocks;
    int32_t nnz = 0;
    SNP_CUDA_TRY(cudaMemcpyAsync(&nnz, row_ptr + n_rows, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    SNP_CUDA_TRY(cudaStreamSynchronize(s));
    snp::CsrView<double> A{n_rows, nnz, row_ptr, col_idx, vals};
    int status = SNP_OK;
    SNP_TRY(snp::pcg_on_buffers(A, free_mask, b, x, rtol, atol, maxiter, B, s, iterations, res_norm, &status));
    if (status == SNP_NOT_CONVERGED) return snp::fail(status, "snp_pcg_noalloc: maxiter reached");
    if (status == SNP_NAN_DETECTED) return snp::fail(status, "snp_pcg_noalloc: non-finite residual");
    return SNP_OK;
}
