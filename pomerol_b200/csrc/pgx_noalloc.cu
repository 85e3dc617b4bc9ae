// Allocation-free eigensolve of one symmetric block (pgx_eigh_noalloc).
//
// Some callers cannot let a library call cudaMalloc: their device memory is
// owned by an outer allocator (an application's caching pool or a fixed
// arena with a budget), and an allocation behind its back would break that
// accounting.  For them this entry point diagonalises one real symmetric
// block on buffers the caller passes in, and keeps its own workspace in the
// file-scope array below instead of allocating.
//
// The array holds the Householder workspace (reused for the eigenvectors of
// the tridiagonal), the accumulated factor, the inverse-iteration scratch,
// the tridiagonal with its eigenvalues and index arrays, and the small
// descriptor lists of one block of at most PGX_NOALLOC_MAX_DIM states
// (about 3 MiB).  Every GPU that loads this
// library holds it until the process exits.  All calls on a device share it
// and it keeps the last call's contents: calls whose work overlaps on the GPU
// (different streams, or host threads racing) corrupt each other and must be
// serialised by the caller.  The first call on a device looks up the array's
// device address (cudaGetSymbolAddress) with that device current; that first
// call should come before any stream capture.

#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "pgx_common.cuh"
#include "pgx_internal.h"

namespace {

constexpr long NA_N = PGX_NOALLOC_MAX_DIM;
// layout in doubles:
//   A (n^2) | Zc (n^2) | S (4 n^2) | tri (2n) | lam (n) | sb, rank (3n ints = 2n doubles)
//   | work items (128) | GEMM problem (32) | GEMM tile index (64) | descriptors (8)
constexpr long NA_A = 0;
constexpr long NA_ZC = NA_A + NA_N * NA_N;
constexpr long NA_S = NA_ZC + NA_N * NA_N;
constexpr long NA_TRI = NA_S + 4 * NA_N * NA_N;
constexpr long NA_LAM = NA_TRI + 2 * NA_N;
constexpr long NA_INT = NA_LAM + NA_N;
constexpr long NA_ITEMS = NA_INT + 2 * NA_N;
constexpr long NA_GPROB = NA_ITEMS + 128;
constexpr long NA_GTILE = NA_GPROB + 32;
constexpr long NA_META = NA_GTILE + 64;
constexpr long NA_TOTAL = NA_META + 8;

static __device__ __align__(256) double g_noalloc_scratch[NA_TOTAL];

// Host-side descriptors staged into the array's last 64 bytes.
struct NaMeta {
    int order;   // CTA -> block
    int dims;    // block size
    long moff;   // matrix offset
    long eoff;   // vector offset
    int status;  // cleared before every call
    int pad;
};
static_assert(sizeof(NaMeta) <= 8 * sizeof(double), "descriptor slot too small");

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_mu;
double* g_base[NA_MAX_DEVICES] = {};

// Device address of the scratch array on the current device, looked up once.
int scratch_base(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) {
        cudaGetLastError();
        return PGX_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_base[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return PGX_ERR_CUDA;
        }
        g_base[dev] = static_cast<double*>(p);
    }
    *out = g_base[dev];
    return PGX_OK;
}

}  // namespace

extern "C" int pgx_eigh_noalloc(const double* H, int32_t n, double* E, double* U, void* stream) {
    if (!H || !E || !U) return PGX_ERR_ARG;
    if (n < 1 || n > PGX_NOALLOC_MAX_DIM) return PGX_ERR_ARG;  // size beyond the static workspace
    double* base = nullptr;
    const int rc = scratch_base(&base);
    if (rc != PGX_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        const std::vector<int> dims{n};
        size_t tile_bytes = 0;
        PGX_CHECK(pgx::eigh_item_bytes(dims) <= 128 * sizeof(double), PGX_ERR_ARG, "item list too long");
        PGX_CHECK(pgx::eigh_vec_scratch_doubles(dims) <= (size_t)(NA_TRI - NA_S), PGX_ERR_ARG, "vector scratch too small");
        PGX_CHECK(pgx::eigh_gemm_bytes(dims, &tile_bytes) <= 32 * sizeof(double) && tile_bytes <= 64 * sizeof(double),
                  PGX_ERR_ARG, "GEMM lists too long");
        NaMeta* meta = reinterpret_cast<NaMeta*>(base + NA_META);
        const NaMeta h{0, n, 0, 0, 0, 0};
        PGX_CUDA(cudaMemcpyAsync(meta, &h, sizeof(h), cudaMemcpyHostToDevice, st));
        pgx::EighDev d;
        d.dims = &meta->dims;
        d.moff = &meta->moff;
        d.eoff = &meta->eoff;
        d.H = H;
        d.A = base + NA_A;
        d.Zc = base + NA_ZC;
        d.tri = base + NA_TRI;
        d.lam = base + NA_LAM;
        d.sb = reinterpret_cast<int*>(base + NA_INT);
        d.rank = d.sb + 2 * n;
        d.S = base + NA_S;
        d.items = base + NA_ITEMS;
        d.gemm_probs = base + NA_GPROB;
        d.gemm_tiles = base + NA_GTILE;
        d.U = U;
        d.E = E;
        d.status = &meta->status;
        pgx::launch_eigh_raw(d, dims, {0L}, st);
        int status = 0;
        PGX_CUDA(cudaMemcpyAsync(&status, &meta->status, sizeof(int), cudaMemcpyDeviceToHost, st));
        PGX_CUDA(cudaStreamSynchronize(st));
        return status == 0 ? PGX_OK : PGX_ERR_NUMERIC;
    } catch (const pgx::Error& e) {
        return e.code;
    } catch (...) {
        return PGX_ERR_ARG;
    }
}
