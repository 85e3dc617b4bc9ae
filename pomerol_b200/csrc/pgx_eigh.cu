// K1: batched FP64 symmetric eigensolver.
//
// Replaces Eigen::SelfAdjointEigenSolver as called by HamiltonianPart::computeImpl
// (HamiltonianPart.cpp:90-102).  Stages:
//   1. Householder reduction to tridiagonal form T and explicit accumulation
//      of the orthogonal factor Q (Golub & Van Loan, "Matrix Computations",
//      4th ed., 8.3.1):
//      eigh_cluster_kernel, one thread-block cluster of 1-8 CTAs per block
//      with the matrix in distributed shared memory (blocks up to 464 states);
//      eigh_kernel, one CTA per block with the matrix in global memory
//      (larger blocks).  Q is stored column-major.
//   2. bisect_kernel, one thread per eigenvalue: bisection with Sturm counts
//      on the unreduced pieces of T (8.4.1).
//   3. vector_kernel, one thread per eigenvalue: inverse iteration with a
//      partial-pivoting tridiagonal LU; ortho_kernel: modified Gram-Schmidt
//      inside chains of close eigenvalues; eigenvalues are ranked so that the
//      output is ascending.
//   4. U = Q Z as one batched FP64 GEMM over all blocks.
// A non-finite eigenvector sets a device status word instead of trapping.

#include <cooperative_groups.h>

#include <cmath>
#include <cstring>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

constexpr int EIGH_THREADS = 512;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the CTA; result valid in every thread.  `red` holds >= 32 doubles.
__device__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double r = (lane < nw) ? red[lane] : 0.0;
    r = warp_sum(r);
    return r;
}

struct EighArgs {
    const int* order;          // CTA -> block (largest first)
    const int* dims;
    const long* moff;          // matrix offset of block b (elements)
    const long* eoff;          // vector offset of block b
    const double* H;           // packed input blocks (row-major)
    double* A;                 // workspace copy (destroyed)
    double* Zc;                // workspace, column-major accumulated factor
    double* tri;               // per block: diagonal then sub-diagonal (2 n)
};

// Householder reduction of one block and accumulation of its orthogonal
// factor (column-major), one CTA per block.
__global__ void __launch_bounds__(EIGH_THREADS) eigh_kernel(EighArgs g) {
    extern __shared__ double sh[];
    __shared__ double red[32];

    const int b = g.order[blockIdx.x];
    const int n = g.dims[b];
    const long mo = g.moff[b], eo = g.eoff[b];
    const double* Hb = g.H + mo;
    double* A = g.A + mo;
    double* Z = g.Zc + mo;
    const int tid = threadIdx.x, nt = blockDim.x;

    double* v = sh;            // n   Householder vector
    double* w = sh + n;        // n   p / w vectors
    double* dg = sh + 2 * n;   // n   diagonal
    double* ed = sh + 3 * n;   // n   sub-diagonal

    for (long i = tid; i < (long)n * n; i += nt) A[i] = Hb[i];
    __syncthreads();

    // ---------------- Householder tridiagonalisation (lower) ----------------
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        const long base = (long)(k + 1) * n + (k + 1);  // B(i,j) = A[base + i*n + j]
        double part = 0.0;
        for (int i = tid; i < m; i += nt) {
            double x = A[(long)(k + 1 + i) * n + k];
            v[i] = x;
            if (i > 0) part += x * x;
        }
        double sigma = block_sum(part, red);
        const double x0 = v[0];
        if (tid == 0) dg[k] = A[(long)k * n + k];
        if (sigma == 0.0) {
            if (tid == 0) ed[k] = x0;
            __syncthreads();
            if (tid == 0) A[(long)(k + 1) * n + k] = 0.0;  // marks tau = 0 below
            continue;
        }
        const double mu = sqrt(x0 * x0 + sigma);
        const double alpha = (x0 > 0.0) ? -mu : mu;   // v0 = x0 - alpha, no cancellation
        const double v0 = x0 - alpha;
        const double tau = 2.0 / (sigma + v0 * v0);
        __syncthreads();
        if (tid == 0) { v[0] = v0; ed[k] = alpha; }
        __syncthreads();
        // p = tau * B v  (B symmetric: p_i = sum_j B(j,i) v_j, coalesced over i);
        // four independent accumulators keep several loads in flight
        for (int i = tid; i < m; i += nt) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
            const double* col = A + base + i;
            int j = 0;
            for (; j + 3 < m; j += 4) {
                const double b0 = col[(long)j * n], b1 = col[(long)(j + 1) * n], b2 = col[(long)(j + 2) * n],
                             b3 = col[(long)(j + 3) * n];
                a0 = fma(b0, v[j], a0);
                a1 = fma(b1, v[j + 1], a1);
                a2 = fma(b2, v[j + 2], a2);
                a3 = fma(b3, v[j + 3], a3);
            }
            for (; j < m; ++j) a0 = fma(col[(long)j * n], v[j], a0);
            w[i] = tau * ((a0 + a1) + (a2 + a3));
        }
        __syncthreads();
        part = 0.0;
        for (int i = tid; i < m; i += nt) part += v[i] * w[i];
        const double K = 0.5 * tau * block_sum(part, red);
        __syncthreads();
        for (int i = tid; i < m; i += nt) w[i] -= K * v[i];
        __syncthreads();
        // B -= v w^T + w v^T  (rows in groups of four: loads issued before stores)
        for (int i = tid; i < m; i += nt) {
            const double vi = v[i], wi = w[i];
            double* colp = A + base + i;
            int j = 0;
            for (; j + 3 < m; j += 4) {
                double b0 = colp[(long)j * n], b1 = colp[(long)(j + 1) * n], b2 = colp[(long)(j + 2) * n],
                       b3 = colp[(long)(j + 3) * n];
                b0 -= v[j] * wi + w[j] * vi;
                b1 -= v[j + 1] * wi + w[j + 1] * vi;
                b2 -= v[j + 2] * wi + w[j + 2] * vi;
                b3 -= v[j + 3] * wi + w[j + 3] * vi;
                colp[(long)j * n] = b0;
                colp[(long)(j + 1) * n] = b1;
                colp[(long)(j + 2) * n] = b2;
                colp[(long)(j + 3) * n] = b3;
            }
            for (; j < m; ++j) colp[(long)j * n] -= v[j] * wi + w[j] * vi;
        }
        // keep v (scaled by sqrt(tau)) in column k below the diagonal
        const double st = sqrt(tau);
        for (int i = tid; i < m; i += nt) A[(long)(k + 1 + i) * n + k] = v[i] * st;
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            dg[n - 2] = A[(long)(n - 2) * n + (n - 2)];
            ed[n - 2] = A[(long)(n - 1) * n + (n - 2)];
            if (n == 2) ed[0] = A[(long)1 * n + 0];
        }
        dg[n - 1] = A[(long)(n - 1) * n + (n - 1)];
        ed[n - 1] = 0.0;
    }
    // ---------------- accumulate Q = H_0 ... H_{n-3} (column-major) ----------------
    for (long i = tid; i < (long)n * n; i += nt) Z[i] = ((i / n) == (i % n)) ? 1.0 : 0.0;
    __syncthreads();
    const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    for (int k = n - 3; k >= 0; --k) {
        const int m = n - k - 1;
        for (int i = tid; i < m; i += nt) v[i] = A[(long)(k + 1 + i) * n + k];  // sqrt(tau) v
        __syncthreads();
        // columns j >= k+1: Q(:,j) -= u (u^T Q(:,j)),  u = sqrt(tau) v
        for (int j = k + 1 + wid; j < n; j += nw) {
            double* col = Z + (long)j * n + (k + 1);
            double s = 0.0;
            for (int i = lane; i < m; i += 32) s += v[i] * col[i];
            s = warp_sum(s);
            for (int i = lane; i < m; i += 32) col[i] -= v[i] * s;
        }
        __syncthreads();
    }
    // hand the tridiagonal (diagonal, sub-diagonal) to the bisection stage
    for (int i = tid; i < n; i += nt) {
        g.tri[2 * eo + i] = dg[i];
        g.tri[2 * eo + n + i] = ed[i];
    }
}

// ----------------------------------------------------------------------------
// Householder stage on a thread-block cluster (blocks whose matrix fits in
// the shared memory of up to 8 CTAs: 464 states at 220 KB per CTA).
//
// The C CTAs of a cluster hold the block's symmetric matrix in distributed
// shared memory, row r in CTA r mod C (cyclic, so the shrinking trailing
// matrix stays spread over all CTAs).  Step k of the reduction:
//   (A) cluster barrier; every CTA reads row k (= the column below the
//       diagonal) from its owner and forms the Householder vector v, tau;
//   each CTA computes p = tau B v on its own rows and its share of v.p;
//   (B) cluster barrier; every CTA gathers all of p and the v.p shares,
//       forms w = p - (tau/2)(v.p) v and applies B -= v w^T + w v^T to its
//       own rows.
// CTA 0 stores d_k, e_k and sqrt(tau) v (row k of V in global memory).
// Q = H_0 ... H_{n-3} is then formed from V with the CTAs owning columns
// j = c (mod C) of Q: a column's update needs only that column, so this
// phase has no cross-CTA traffic.  The outputs (tridiagonal, column-major Q)
// are those of eigh_kernel.
constexpr int CL_THREADS = 512;
constexpr int CL_MAX_DIM = CL_THREADS + 1;  // the prefetch of a reflector uses one element per thread

struct ClusterArgs {
    const int* blocks;  // cluster -> block
    const int* dims;
    const long* moff;
    const long* eoff;
    const double* H;
    double* V;          // per block n x n: row k holds sqrt(tau_k) v_k in columns k+1..n-1
    double* Zc;         // per block: Q column-major
    double* tri;
};

__host__ __device__ inline size_t cluster_smem_doubles(int n, int C) {
    const int R = (n + C - 1) / C;
    return (size_t)R * n + 2 * (size_t)n + R + 2;
}

__global__ void __launch_bounds__(CL_THREADS) eigh_cluster_kernel(ClusterArgs g) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ double sh[];
    __shared__ double red[32];
    const int C = (int)cl.num_blocks();
    const int c = (int)cl.block_rank();
    const int b = g.blocks[blockIdx.x / C];
    const int n = g.dims[b];
    const long mo = g.moff[b], eo = g.eoff[b];
    const int R = (n + C - 1) / C;
    const int nrows = (n - c + C - 1) / C;  // rows (and later columns) c, c + C, ...
    double* slab = sh;                      // R x n rows | later R x n columns of Q
    double* v = sh + (size_t)R * n;         // n
    double* w = v + n;                      // n
    double* p = w + n;                      // R
    double* dslot = p + R;                  // 1
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    const double* Hb = g.H + mo;
    double* V = g.V + mo;

    for (long idx = tid; idx < (long)nrows * n; idx += nt) {
        const int lr = (int)(idx / n), j = (int)(idx % n);
        slab[idx] = Hb[(long)(c + C * lr) * n + j];
    }
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        cl.sync();  // (A) row k is final; the p slots of the previous step are free
        const double* rowk = cl.map_shared_rank(slab, k % C) + (size_t)(k / C) * n;
        double part = 0.0;
        for (int i = tid; i < m; i += nt) {
            const double x = rowk[k + 1 + i];
            v[i] = x;
            if (i > 0) part += x * x;
        }
        const double sigma = block_sum(part, red);
        const double x0 = v[0];
        const double dk = rowk[k];
        double tau = 0.0, alpha = x0, v0 = x0;
        if (sigma != 0.0) {
            const double mu = sqrt(x0 * x0 + sigma);
            alpha = (x0 > 0.0) ? -mu : mu;  // v0 = x0 - alpha without cancellation
            v0 = x0 - alpha;
            tau = 2.0 / (sigma + v0 * v0);
        }
        __syncthreads();
        if (tid == 0) v[0] = v0;
        __syncthreads();
        // p = tau B v on own rows r >= k+1 (one warp per row)
        const int lr0 = (k + 1 - c + C - 1) / C;
        double dpart = 0.0;
        for (int lr = lr0 + wid; lr < nrows; lr += nw) {
            const double* row = slab + (size_t)lr * n + (k + 1);
            double s = 0.0;
            for (int j = lane; j < m; j += 32) s = fma(row[j], v[j], s);
            s = warp_sum(s) * tau;
            if (lane == 0) {
                p[lr] = s;
                dpart += v[c + C * lr - (k + 1)] * s;
            }
        }
        const double dsum = block_sum(dpart, red);
        if (tid == 0) dslot[0] = dsum;
        cl.sync();  // (B) p and the v.p shares of every CTA are complete
        double dtot = 0.0;
        for (int q = 0; q < C; ++q) dtot += cl.map_shared_rank(dslot, q)[0];
        const double K = 0.5 * tau * dtot;
        for (int i = tid; i < m; i += nt) {
            const int r = k + 1 + i;
            w[i] = cl.map_shared_rank(p, r % C)[r / C] - K * v[i];
        }
        __syncthreads();
        for (int lr = lr0 + wid; lr < nrows; lr += nw) {
            double* row = slab + (size_t)lr * n + (k + 1);
            const int i = c + C * lr - (k + 1);
            const double vi = v[i], wi = w[i];
            for (int j = lane; j < m; j += 32) row[j] -= vi * w[j] + wi * v[j];
        }
        if (c == 0) {
            if (tid == 0) {
                g.tri[2 * eo + k] = dk;
                g.tri[2 * eo + n + k] = alpha;
            }
            const double st = sqrt(tau);
            for (int i = tid; i < m; i += nt) V[(size_t)k * n + k + 1 + i] = v[i] * st;
        }
    }
    cl.sync();
    if (c == 0 && tid == 0) {
        auto elem = [&](int r, int j) { return cl.map_shared_rank(slab, r % C)[(size_t)(r / C) * n + j]; };
        if (n >= 2) {
            g.tri[2 * eo + n - 2] = elem(n - 2, n - 2);
            g.tri[2 * eo + n + n - 2] = elem(n - 1, n - 2);
        }
        g.tri[2 * eo + n - 1] = elem(n - 1, n - 1);
        g.tri[2 * eo + n + n - 1] = 0.0;
    }
    __threadfence();
    cl.sync();  // V is visible to every CTA; no CTA reads another's shared memory after this point

    // ---- Q = H_0 ... H_{n-3}, columns j = c + C t of Q in shared memory (column-major)
    double* Qs = slab;
    double* u = v;
    for (long idx = tid; idx < (long)nrows * n; idx += nt) {
        const int t = (int)(idx / n), i = (int)(idx % n);
        Qs[idx] = (i == c + C * t) ? 1.0 : 0.0;
    }
    double pre = 0.0;
    if (n >= 3 && tid < 2) pre = V[(size_t)(n - 3) * n + (n - 2) + tid];
    for (int k = n - 3; k >= 0; --k) {
        const int m = n - k - 1;
        __syncthreads();  // the previous reflector is no longer read
        if (tid < m) u[tid] = pre;
        __syncthreads();
        if (k >= 1 && tid < m + 1) pre = V[(size_t)(k - 1) * n + k + tid];
        const int t0 = (k + 1 - c + C - 1) / C;
        for (int t = t0 + wid; t < nrows; t += nw) {
            double* col = Qs + (size_t)t * n + (k + 1);
            double s = 0.0;
            for (int i = lane; i < m; i += 32) s = fma(u[i], col[i], s);
            s = warp_sum(s);
            for (int i = lane; i < m; i += 32) col[i] -= u[i] * s;
        }
    }
    __syncthreads();
    for (long idx = tid; idx < (long)nrows * n; idx += nt) {
        const int t = (int)(idx / n), i = (int)(idx % n);
        g.Zc[mo + (long)(c + C * t) * n + i] = Qs[idx];
    }
}

// ----------------------------------------------------------------------------
// Tridiagonal stage.  T (diagonal d, sub-diagonal e) is split into unreduced
// pieces where |e_i| <= eps (|d_i| + |d_i+1|) or |e_i| <= 8 eps ||T|| (a
// perturbation of T of the size of the Householder stage's own backward
// error).  Exact degeneracies of H show up as such splits, so eigenvectors of
// different pieces are orthogonal by support.
//   * eigenvalues: bisection with Sturm counts, one thread per eigenvalue
//     (Golub & Van Loan, 8.4.1), as 32-point multisection by one warp;
//   * eigenvectors: two steps of inverse iteration, one thread per
//     eigenvalue (Golub & Van Loan, 8.2.2).  Each solve factors T - lambda I
//     by Gaussian elimination with partial pivoting.  In a chain of
//     eigenvalues whose neighbours are closer than 1e-4 ||T|| the shifts are
//     nudged apart, so coincident eigenvalues get distinct vectors, and a
//     second kernel orthogonalises each member (modified Gram-Schmidt, twice)
//     against the earlier members closer than 1e-4 ||T||; mixing only among
//     such close eigenvalues keeps the residuals at the eps ||T|| level.  The
//     start vector is a fixed hash of (index, row).
struct TriItem {
    int block, j0, j1, pad;
    long soff;  // vector_kernel: this CTA's scratch, 4 n TRI_THREADS doubles at S + soff
};

struct TriArgs {
    const TriItem* items;
    const int* dims;
    const long* moff;
    const long* eoff;
    const double* tri;  // per block: d (n), e (n)
    double* lam;        // per block: eigenvalues, ascending inside each piece
    int* sb;            // per block: 2 n ints (first and last row of the piece)
    int* rank;          // per block: n ints (position in the ascending order)
    double* Z;          // per block: n x n column-major eigenvectors of T, sorted
    double* S;          // per vector_kernel CTA: 4 arrays of n x TRI_THREADS, thread-interleaved
    double* E;          // eigenvalues, ascending
    int* status;
};

constexpr int TRI_THREADS = 32;  // vector_kernel: one warp per CTA, so the CTAs spread over all SMs
constexpr double EPS = 2.220446049250313e-16;
constexpr double SAFE_MIN = 2.2250738585072014e-308;
constexpr double SPLIT_ABS = 8.0;   // absolute split threshold, units of eps ||T||
constexpr double CHAIN_TOL = 1e-4;  // chain / orthogonalisation window, units of ||T||
constexpr int INV_ITERS = 2;        // inverse iterations per eigenvector

// Loads d and e of one block into shared memory, zeroes the split points and
// returns ||T|| (max row sum); every thread of the CTA must call it.
__device__ double load_tri(const double* tri, long eo, int n, double* d, double* e) {
    __shared__ double red[32];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        d[i] = tri[2 * eo + i];
        e[i] = (i < n - 1) ? tri[2 * eo + n + i] : 0.0;
    }
    __syncthreads();
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        m = fmax(m, fabs(d[i]) + fabs(e[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    double tn = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tn = fmax(tn, red[w]);
    for (int i = threadIdx.x; i < n - 1; i += blockDim.x)
        if (fabs(e[i]) <= EPS * (fabs(d[i]) + fabs(d[i + 1])) || fabs(e[i]) <= SPLIT_ABS * EPS * tn) e[i] = 0.0;
    __syncthreads();
    return tn;
}

__device__ void piece_of(const double* e, int n, int j, int& a, int& b) {
    a = j;
    b = j;
    while (a > 0 && e[a - 1] != 0.0) --a;
    while (b < n - 1 && e[b] != 0.0) ++b;
}

// Multisection with one warp per eigenvalue: each round the 32 lanes take the
// Sturm counts at 32 equally spaced interior points of the bracketing
// interval, narrowing it 33-fold (about 11 rounds to full precision).
constexpr int BIS_WARPS = 8;  // eigenvalues per CTA
constexpr int BIS_THREADS = 32 * BIS_WARPS;

// number of eigenvalues of T[a..b] below x
__device__ int sturm(const double* d, const double* e, int a, int b, double x, double pivmin) {
    double q = d[a] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    int cnt = q < 0.0;
    for (int i = a + 1; i <= b; ++i) {
        q = (d[i] - x) - e[i - 1] * (e[i - 1] / q);
        if (fabs(q) < pivmin) q = -pivmin;
        cnt += q < 0.0;
    }
    return cnt;
}

__global__ void __launch_bounds__(BIS_THREADS) bisect_kernel(TriArgs g, const TriItem* bitems) {
    extern __shared__ double sh[];
    const TriItem it = bitems[blockIdx.x];
    const int n = g.dims[it.block];
    const long eo = g.eoff[it.block];
    double* d = sh;
    double* e = sh + n;
    load_tri(g.tri, eo, n, d, e);
    const int lane = threadIdx.x & 31;
    const int j = it.j0 + (int)(threadIdx.x >> 5);
    if (j >= it.j1) return;
    int a, b;
    piece_of(e, n, j, a, b);
    double lo = 1e300, hi = -1e300, em = 0.0;
    for (int i = a; i <= b; ++i) {
        const double r = (i > a ? fabs(e[i - 1]) : 0.0) + (i < b ? fabs(e[i]) : 0.0);
        lo = fmin(lo, d[i] - r);
        hi = fmax(hi, d[i] + r);
        if (i < b) em = fmax(em, e[i] * e[i]);
    }
    const double pivmin = SAFE_MIN * fmax(1.0, em);
    const double gn = fmax(fabs(lo), fabs(hi));
    const double w = 2.0 * EPS * gn + pivmin;
    lo -= w;
    hi += w;
    const double atol = 0.25 * EPS * gn + pivmin;
    const int k = j - a;
    // every lane holds the same lo, hi: the loop and its exits are warp-uniform
    for (int round = 0; round < 64; ++round) {
        if (hi - lo <= atol + 2.0 * EPS * fmin(fabs(lo), fabs(hi))) break;
        const double step = (hi - lo) / 33.0;
        if (!(lo + step > lo && lo + step * 32.0 < hi)) break;  // interval at the resolution of doubles
        const int cnt = sturm(d, e, a, b, lo + step * (lane + 1), pivmin);
        // counts grow with x: the eigenvalue lies between point `below` and `below + 1`
        const int below = __popc(__ballot_sync(0xffffffffu, cnt <= k));
        const double nlo = (below > 0) ? lo + step * below : lo;
        const double nhi = (below < 32) ? lo + step * (below + 1) : hi;
        lo = nlo;
        hi = nhi;
    }
    if (lane == 0) {
        g.lam[eo + j] = 0.5 * (lo + hi);
        g.sb[2 * eo + j] = a;
        g.sb[2 * eo + n + j] = b;
    }
}

// pseudo-random start vector entry in [-1, 1) for eigen-index j, row i
__device__ __forceinline__ double start_entry(int j, int i) {
    unsigned x = (unsigned)j * 0x9E3779B1u + (unsigned)i * 0x85EBCA77u + 0x165667B1u;
    x ^= x >> 15;
    x *= 0x2C1B3C6Du;
    x ^= x >> 12;
    x *= 0x297A2D39u;
    x ^= x >> 15;
    return (double)x * (2.0 / 4294967296.0) - 1.0;
}

// z := (T[a..b] - lm I)^-1 z by Gaussian elimination with partial pivoting;
// the factorisation and the forward elimination share one sweep, the upper
// factor's three diagonals are kept in u1, u2, u3 for the back substitution.
// Pivots smaller than pfloor in magnitude are replaced by +-pfloor.
// Both sweeps are a chain of dependent divisions; the values the chain
// passes on stay in registers, and the vector entries each sweep reads are
// loaded LU_BATCH rows ahead, so a batch waits for memory once.  Entry i of
// each vector is at index i * st: the lanes of a warp interleave their
// vectors, so a warp at the same row reads and writes one contiguous segment.
constexpr int LU_BATCH = 8;

__device__ void lu_solve(const double* d, const double* e, int a, int b, double lm, double pfloor,
                         double* __restrict__ z, double* __restrict__ u1, double* __restrict__ u2,
                         double* __restrict__ u3, int st) {
    double p = d[a] - lm, q = (a < b) ? e[a] : 0.0;
    double zk = z[(long)a * st];
    for (int k0 = a; k0 < b; k0 += LU_BATCH) {
        double zn[LU_BATCH];
#pragma unroll
        for (int t = 0; t < LU_BATCH; ++t)
            if (k0 + t < b) zn[t] = z[(long)(k0 + t + 1) * st];
#pragma unroll
        for (int t = 0; t < LU_BATCH; ++t) {
            const int k = k0 + t;
            if (k >= b) break;
            const double sub = e[k], dn = d[k + 1] - lm, en = (k + 1 < b) ? e[k + 1] : 0.0;
            const double zk1 = zn[t];
            // row interchange when the sub-diagonal entry is the larger pivot; both
            // cases share one division and are selected without branching
            const bool sw = fabs(sub) > fabs(p);
            const double num = sw ? p : sub, den = sw ? sub : p;
            const double l = (den != 0.0) ? num / den : 0.0;
            const double w1 = sw ? sub : p, w2 = sw ? dn : q, w3 = sw ? en : 0.0;
            const double np = sw ? q - l * dn : dn - l * q;
            const double nq = sw ? -l * en : en;
            const double zout = sw ? zk1 : zk;
            const double znext = sw ? zk - l * zk1 : zk1 - l * zk;
            const long o = (long)k * st;
            u1[o] = w1;
            u2[o] = w2;
            u3[o] = w3;
            z[o] = zout;
            zk = znext;
            p = np;
            q = nq;
        }
    }
    // back substitution; x1, x2 carry the two solution entries below row k
    double x1 = 0.0, x2 = 0.0;
    for (int k0 = b; k0 >= a; k0 -= LU_BATCH) {
        double v1[LU_BATCH], v2[LU_BATCH], v3[LU_BATCH], vz[LU_BATCH];
#pragma unroll
        for (int t = 0; t < LU_BATCH; ++t) {
            const int k = k0 - t;
            if (k < a) break;
            const long o = (long)k * st;
            v1[t] = (k == b) ? p : u1[o];
            vz[t] = (k == b) ? zk : z[o];
            v2[t] = (k + 1 <= b) ? u2[o] : 0.0;
            v3[t] = (k + 2 <= b) ? u3[o] : 0.0;
        }
#pragma unroll
        for (int t = 0; t < LU_BATCH; ++t) {
            const int k = k0 - t;
            if (k < a) break;
            double piv = v1[t];
            if (fabs(piv) < pfloor) piv = (piv >= 0.0) ? pfloor : -pfloor;
            double r = vz[t];
            if (k + 1 <= b) r -= v2[t] * x1;
            if (k + 2 <= b) r -= v3[t] * x2;
            const double xk = r / piv;
            z[(long)k * st] = xk;
            x2 = x1;
            x1 = xk;
        }
    }
}

// z /= ||z|| over rows a..b (stride st); false when the norm is zero or not finite
__device__ bool normalize(double* z, int a, int b, int st) {
    double nn = 0.0;
    for (int i = a; i <= b; ++i) nn = fma(z[(long)i * st], z[(long)i * st], nn);
    if (!(nn > 0.0) || !isfinite(nn)) return false;
    const double inv = rsqrt(nn);
    for (int i = a; i <= b; ++i) z[(long)i * st] *= inv;
    return true;
}

// One thread per eigenvalue, the same work in every thread: two steps of
// inverse iteration.  Within a chain (neighbours closer than CHAIN_TOL ||T||)
// the shifts are nudged apart so coincident eigenvalues start from distinct
// shifts; ortho_kernel then orthogonalises the members of each chain.
__global__ void __launch_bounds__(TRI_THREADS) vector_kernel(TriArgs g) {
    extern __shared__ double sh[];
    const TriItem it = g.items[blockIdx.x];
    const int n = g.dims[it.block];
    const long eo = g.eoff[it.block], mo = g.moff[it.block];
    double* d = sh;
    double* e = sh + n;
    double* lam = sh + 2 * n;
    const double tn = load_tri(g.tri, eo, n, d, e);
    for (int i = threadIdx.x; i < n; i += blockDim.x) lam[i] = g.lam[eo + i];
    __syncthreads();
    const double ortol = CHAIN_TOL * tn;
    const double pfloor = (tn > 0.0) ? EPS * tn : 1.0;
    const int* sa = g.sb + 2 * eo;
    const int* sbe = sa + n;
    double* Zb = g.Z + mo;
    // this thread's working vector and LU diagonals, interleaved with the CTA's other threads
    const int st = blockDim.x;
    double* zt = g.S + it.soff + threadIdx.x;
    double* u1 = zt + (long)n * st;
    double* u2 = u1 + (long)n * st;
    double* u3 = u2 + (long)n * st;
    for (int j = it.j0 + threadIdx.x; j < it.j1; j += blockDim.x) {
        const int a = sa[j], b = sbe[j];
        // shift: the eigenvalue, raised above its chain predecessor's shift where they coincide
        int h = j;
        while (h > a && lam[h] - lam[h - 1] <= ortol) --h;
        double lm = -1e308;
        for (int t = h; t <= j; ++t) {
            const double lt = lam[t], sep = 10.0 * EPS * fmax(fabs(lt), 1e-3 * tn);
            lm = (t > h && lt < lm + sep) ? lm + sep : lt;
        }
        int rk = 0;
        for (int i = 0; i < n; ++i) rk += (lam[i] < lam[j]) || (lam[i] == lam[j] && i < j);
        g.rank[eo + j] = rk;
        g.E[eo + rk] = lam[j];
        double* z = Zb + (long)rk * n;
        bool ok = true;
        if (a == b) {
            for (int i = 0; i < n; ++i) z[i] = (i == a) ? 1.0 : 0.0;
        } else {
            for (int i = a; i <= b; ++i) zt[(long)i * st] = start_entry(j, i);
            for (int t = 0; t < INV_ITERS && ok; ++t) {
                lu_solve(d, e, a, b, lm, pfloor, zt, u1, u2, u3, st);
                ok = normalize(zt, a, b, st);
            }
            for (int i = 0; i < n; ++i) z[i] = (i >= a && i <= b) ? zt[(long)i * st] : 0.0;
        }
        if (!ok) atomicExch(g.status, PGX_ERR_NUMERIC);
    }
}

// Modified Gram-Schmidt, applied twice, of each chain member against the
// earlier members closer than CHAIN_TOL ||T||; one thread per chain head.
__global__ void __launch_bounds__(TRI_THREADS) ortho_kernel(TriArgs g) {
    extern __shared__ double sh[];
    const TriItem it = g.items[blockIdx.x];
    const int n = g.dims[it.block];
    const long eo = g.eoff[it.block], mo = g.moff[it.block];
    double* d = sh;
    double* e = sh + n;
    double* lam = sh + 2 * n;
    const double tn = load_tri(g.tri, eo, n, d, e);
    for (int i = threadIdx.x; i < n; i += blockDim.x) lam[i] = g.lam[eo + i];
    __syncthreads();
    const double ortol = CHAIN_TOL * tn;
    const int* sa = g.sb + 2 * eo;
    const int* sbe = sa + n;
    const int* rank = g.rank + eo;
    double* Zb = g.Z + mo;
    for (int j = it.j0 + threadIdx.x; j < it.j1; j += blockDim.x) {
        const int a = sa[j], b = sbe[j];
        if (j > a && lam[j] - lam[j - 1] <= ortol) continue;  // not the head of a chain
        bool ok = true;
        for (int jj = j + 1; jj <= b && lam[jj] - lam[jj - 1] <= ortol; ++jj) {
            double* z = Zb + (long)rank[jj] * n;
            for (int pass = 0; pass < 2 && ok; ++pass) {
                for (int pp = jj - 1; pp >= j && lam[jj] - lam[pp] <= ortol; --pp) {
                    const double* qv = Zb + (long)rank[pp] * n;
                    double dot = 0.0;
                    for (int i = a; i <= b; ++i) dot = fma(qv[i], z[i], dot);
                    for (int i = a; i <= b; ++i) z[i] = fma(-dot, qv[i], z[i]);
                }
                ok = normalize(z, a, b, 1);
            }
        }
        if (!ok) atomicExch(g.status, PGX_ERR_NUMERIC);
    }
}

// ----------------------------------------------------------------------------
// Complex Hermitian blocks.  H = R + iI (R symmetric, I antisymmetric) has the
// real symmetric embedding [[R, -I], [I, R]] of twice the size; every
// eigenvalue of H appears twice in it, and for a real eigenvector [a; b] of
// the pair, a + ib is an eigenvector of H (unit norm).  The embedding is
// diagonalised by the real stages above; cx_extract_kernel then forms the
// complex eigenvectors.

// block b of H (complex, row-major n x n) -> block b of the embedding (2n x 2n)
__global__ void cx_embed_kernel(const int* dims, const long* moff, const long* moff2, const double* H, double* H2) {
    const int b = blockIdx.y, n = dims[b];
    const cd* Hb = reinterpret_cast<const cd*>(H) + moff[b];
    double* E = H2 + moff2[b];
    const long nn = (long)n * n, n2 = 2L * n;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nn; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e / n), j = (int)(e % n);
        const cd h = Hb[e];
        E[i * n2 + j] = h.x;
        E[i * n2 + n + j] = -h.y;
        E[(n + i) * n2 + j] = h.y;
        E[(n + i) * n2 + n + j] = h.x;
    }
}

// One thread per cluster of equal eigenvalues of the embedding (2m values):
// the m complex eigenvectors of H are taken from the 2m candidates a + ib by
// modified Gram-Schmidt (twice), keeping those with a residual norm above 1/2.
// A cluster is a run of consecutive eigenvalues closer than tol.
__global__ void cx_extract_kernel(const int* dims, const long* moff, const long* eoff, const long* moff2,
                                  const long* eoff2, const double* E2, const double* U2, double* E, cd* U, double tol,
                                  int* status) {
    const int b = blockIdx.x, n = dims[b];
    const long n2 = 2L * n;
    const double* Eb2 = E2 + eoff2[b];
    const double* Ub2 = U2 + moff2[b];
    double* Eb = E + eoff[b];
    cd* Ub = U + moff[b];
    for (int j = threadIdx.x; j < 2 * n; j += blockDim.x) {
        if (j > 0 && Eb2[j] - Eb2[j - 1] <= tol) continue;  // not the start of a cluster
        int jend = j;
        while (jend + 1 < 2 * n && Eb2[jend + 1] - Eb2[jend] <= tol) ++jend;
        const int sz = jend - j + 1, m = sz / 2, c0 = j / 2;
        if ((sz & 1) || (j & 1)) {
            atomicExch(status, PGX_ERR_NUMERIC);
            continue;
        }
        int acc = 0;
        for (int k = 0; k < sz && acc < m; ++k) {
            cd* v = Ub + (c0 + acc);  // column c0 + acc, stride n
            for (int i = 0; i < n; ++i) v[(long)i * n] = cd{Ub2[i * n2 + j + k], Ub2[(n + i) * n2 + j + k]};
            for (int pass = 0; pass < 2; ++pass)
                for (int q = 0; q < acc; ++q) {
                    const cd* u = Ub + (c0 + q);
                    double px = 0.0, py = 0.0;  // u^H v
                    for (int i = 0; i < n; ++i) {
                        const cd a = u[(long)i * n], c = v[(long)i * n];
                        px += a.x * c.x + a.y * c.y;
                        py += a.x * c.y - a.y * c.x;
                    }
                    for (int i = 0; i < n; ++i) {
                        const cd a = u[(long)i * n];
                        v[(long)i * n].x -= px * a.x - py * a.y;
                        v[(long)i * n].y -= px * a.y + py * a.x;
                    }
                }
            double nn = 0.0;
            for (int i = 0; i < n; ++i) nn += abs2(v[(long)i * n]);
            if (nn > 0.25) {
                const double inv = rsqrt(nn);
                for (int i = 0; i < n; ++i) v[(long)i * n] = v[(long)i * n] * inv;
                Eb[c0 + acc] = Eb2[j + 2 * acc];
                ++acc;
            }
        }
        if (acc < m) atomicExch(status, PGX_ERR_NUMERIC);
    }
}

}  // namespace

// Work items, largest blocks first: vector_kernel takes TRI_THREADS
// eigen-indices per CTA, bisect_kernel BIS_WARPS; both lists go into one
// descriptor upload (vector items, then bisection items).
static void tri_plan(const std::vector<int>& dims, std::vector<TriItem>& items, size_t* n_vec = nullptr) {
    std::vector<int> order(dims.size());
    for (size_t b = 0; b < dims.size(); ++b) order[b] = (int)b;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return dims[x] > dims[y]; });
    long soff = 0;
    for (int b : order)
        for (int j0 = 0; j0 < dims[b]; j0 += TRI_THREADS) {
            items.push_back(TriItem{b, j0, std::min(dims[b], j0 + TRI_THREADS), 0, soff});
            soff += 4L * dims[b] * TRI_THREADS;
        }
    if (n_vec) *n_vec = items.size();
    for (int b : order)
        for (int j0 = 0; j0 < dims[b]; j0 += BIS_WARPS)
            items.push_back(TriItem{b, j0, std::min(dims[b], j0 + BIS_WARPS), 0, 0});
}

// doubles of vector_kernel scratch (EighDev::S)
size_t eigh_vec_scratch_doubles(const std::vector<int>& dims) {
    size_t s = 0;
    for (int n : dims) s += 4 * (size_t)n * TRI_THREADS * ((n + TRI_THREADS - 1) / TRI_THREADS);
    return std::max<size_t>(s, 1);
}

constexpr int CL_SIZES[4] = {1, 2, 4, 8};
constexpr size_t CL_SMEM_MAX = 220 * 1024;

// Householder stage plan: the block list of each cluster size (largest
// blocks first) and the blocks left to the single-CTA global-memory kernel.
struct HhPlan {
    std::vector<int> cls[4];
    std::vector<int> global;
};

static HhPlan hh_plan(const std::vector<int>& dims) {
    std::vector<int> order(dims.size());
    for (size_t b = 0; b < dims.size(); ++b) order[b] = (int)b;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return dims[x] > dims[y]; });
    HhPlan h;
    for (int b : order) {
        const int n = dims[b];
        int q = -1;
        if (n <= CL_MAX_DIM)
            for (int i = 0; i < 4 && q < 0; ++i)
                if (cluster_smem_doubles(n, CL_SIZES[i]) * sizeof(double) <= CL_SMEM_MAX) q = i;
        if (q < 0) h.global.push_back(b);
        else h.cls[q].push_back(b);
    }
    return h;
}

// descriptor bytes: bisection items, then one int per block (Householder lists)
size_t eigh_item_bytes(const std::vector<int>& dims) {
    std::vector<TriItem> items;
    tri_plan(dims, items);
    return items.size() * sizeof(TriItem) + dims.size() * sizeof(int);
}

size_t eigh_gemm_bytes(const std::vector<int>& dims, size_t* tiles_bytes) {
    if (tiles_bytes) *tiles_bytes = gemm_index_bytes(dims.size());
    return std::max<size_t>(dims.size(), 1) * sizeof(GemmProblem<double, double, double>);
}

// All eigensolver stages on caller-provided device buffers (no allocation),
// enqueued on stream st (asynchronous).
void launch_eigh_raw(const EighDev& d, const std::vector<int>& dims, const std::vector<long>& moff,
                     cudaStream_t st) {
    int dmax = 1;
    for (int x : dims) dmax = std::max(dmax, x);
    // descriptors: bisection items and the Householder block lists, one upload
    std::vector<TriItem> items;
    size_t n_vec = 0;
    tri_plan(dims, items, &n_vec);
    const size_t n_bis = items.size() - n_vec;
    HhPlan hp = hh_plan(dims);
    // a cluster size the device cannot schedule falls back to the global-memory kernel
    ClusterArgs ca;
    ca.dims = d.dims;
    ca.moff = d.moff;
    ca.eoff = d.eoff;
    ca.H = d.H;
    ca.V = d.A;
    ca.Zc = d.Zc;
    ca.tri = d.tri;
    size_t cl_smem[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; ++q) {
        if (hp.cls[q].empty()) continue;
        for (int b : hp.cls[q]) cl_smem[q] = std::max(cl_smem[q], cluster_smem_doubles(dims[b], CL_SIZES[q]) * sizeof(double));
        PGX_CUDA(cudaFuncSetAttribute(eigh_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CL_SMEM_MAX));
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL_SIZES[q];
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)CL_SIZES[q]);
        cfg.blockDim = dim3(CL_THREADS);
        cfg.dynamicSmemBytes = cl_smem[q];
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, eigh_cluster_kernel, &cfg) != cudaSuccess || nclusters < 1) {
            cudaGetLastError();
            hp.global.insert(hp.global.end(), hp.cls[q].begin(), hp.cls[q].end());
            hp.cls[q].clear();
        }
    }
    std::vector<int> lists(hp.global);
    size_t cl_off[4];
    for (int q = 0; q < 4; ++q) {
        cl_off[q] = lists.size();
        lists.insert(lists.end(), hp.cls[q].begin(), hp.cls[q].end());
    }
    std::vector<char> host(items.size() * sizeof(TriItem) + lists.size() * sizeof(int));
    std::memcpy(host.data(), items.data(), items.size() * sizeof(TriItem));
    std::memcpy(host.data() + items.size() * sizeof(TriItem), lists.data(), lists.size() * sizeof(int));
    h2d(d.items, host.data(), host.size(), st);
    const int* d_lists = reinterpret_cast<const int*>(static_cast<const char*>(d.items) + items.size() * sizeof(TriItem));

    // LAPACK operation counts: tridiagonalisation 4/3 n^3, forming Q 4/3 n^3;
    // minimum DRAM traffic: read H, write Q and the tridiagonal
    auto hh_work = [&](const std::vector<int>& bl, double& fl, double& by) {
        fl = by = 0.0;
        for (int b : bl) {
            const double n = dims[b];
            fl += 8.0 / 3.0 * n * n * n;
            by += 16.0 * n * n + 16.0 * n;
        }
    };
    // the launches are independent: with side streams, cluster class q > 0 runs
    // on aux[q - 1] while the main stream runs the global-memory kernel and class 0
    const bool fork = d.aux[0] && d.aux[1] && d.aux[2] && d.fork;
    if (fork) {
        PGX_CUDA(cudaEventRecord(d.fork, st));
        for (int i = 0; i < 3; ++i) PGX_CUDA(cudaStreamWaitEvent(d.aux[i], d.fork, 0));
    }
    if (!hp.global.empty()) {
        int gmax = 1;
        for (int b : hp.global) gmax = std::max(gmax, dims[b]);
        const size_t smem = 4 * sizeof(double) * (size_t)gmax;
        PGX_CHECK(smem <= 200 * 1024, PGX_ERR_ARG, "block too large for the single-CTA eigensolver (d > 6400)");
        PGX_CUDA(cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        EighArgs a;
        a.order = d_lists;
        a.dims = d.dims;
        a.moff = d.moff;
        a.eoff = d.eoff;
        a.H = d.H;
        a.A = d.A;
        a.Zc = d.Zc;
        a.tri = d.tri;
        double fl, by;
        hh_work(hp.global, fl, by);
        ProfRange pr("eigh_kernel", st, fl, by);
        eigh_kernel<<<(unsigned)hp.global.size(), EIGH_THREADS, smem, st>>>(a);
        check_launch("eigh_kernel");
    }
    for (int q = 0; q < 4; ++q) {
        if (hp.cls[q].empty()) continue;
        const cudaStream_t sq = (fork && q > 0) ? d.aux[q - 1] : st;
        ca.blocks = d_lists + cl_off[q];
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL_SIZES[q];
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3((unsigned)(hp.cls[q].size() * CL_SIZES[q]));
        cfg.blockDim = dim3(CL_THREADS);
        cfg.dynamicSmemBytes = cl_smem[q];
        cfg.stream = sq;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        double fl, by;
        hh_work(hp.cls[q], fl, by);
        static const char* names[4] = {"eigh_cluster_kernel<1>", "eigh_cluster_kernel<2>", "eigh_cluster_kernel<4>",
                                       "eigh_cluster_kernel<8>"};
        ProfRange pr(names[q], sq, fl, by);
        PGX_CUDA(cudaLaunchKernelEx(&cfg, eigh_cluster_kernel, ca));
        check_launch("eigh_cluster_kernel");
    }
    if (fork) {
        for (int i = 0; i < 3; ++i) {
            PGX_CUDA(cudaEventRecord(d.join[i], d.aux[i]));
            PGX_CUDA(cudaStreamWaitEvent(st, d.join[i], 0));
        }
    }

    TriArgs t;
    t.items = static_cast<const TriItem*>(d.items);
    t.dims = d.dims;
    t.moff = d.moff;
    t.eoff = d.eoff;
    t.tri = d.tri;
    t.lam = d.lam;
    t.sb = d.sb;
    t.rank = d.rank;
    t.Z = d.A;   // the Householder workspace is free again
    t.S = d.S;
    t.E = d.E;
    t.status = d.status;
    const size_t smem_b = 2 * sizeof(double) * (size_t)dmax, smem_v = 3 * sizeof(double) * (size_t)dmax;
    const TriItem* bis_items = static_cast<const TriItem*>(d.items) + n_vec;
    PGX_CUDA(cudaFuncSetAttribute(bisect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
    PGX_CUDA(cudaFuncSetAttribute(vector_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_v));
    PGX_CUDA(cudaFuncSetAttribute(ortho_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_v));
    double esum = 0.0, msum = 0.0;
    for (int n : dims) {
        esum += n;
        msum += (double)n * n;
    }
    {
        ProfRange pr("bisect_kernel", st, 0.0, 16.0 * esum + 8.0 * esum + 8.0 * esum);
        bisect_kernel<<<(unsigned)n_bis, BIS_THREADS, smem_b, st>>>(t, bis_items);
        check_launch("bisect_kernel");
    }
    {
        ProfRange pr("vector_kernel", st, 0.0, 8.0 * msum + 48.0 * esum);
        vector_kernel<<<(unsigned)n_vec, TRI_THREADS, smem_v, st>>>(t);
        check_launch("vector_kernel");
    }
    {
        ProfRange pr("ortho_kernel", st, 0.0, 0.0);
        ortho_kernel<<<(unsigned)n_vec, TRI_THREADS, smem_v, st>>>(t);
        check_launch("ortho_kernel");
    }

    // U = Q Z: Q column-major (Zc), Z column-major (A), U row-major
    std::vector<GemmProblem<double, double, double>> probs;
    for (size_t b = 0; b < dims.size(); ++b) {
        const int n = dims[b];
        GemmProblem<double, double, double> g{};
        g.A = d.Zc + moff[b];
        g.B = d.A + moff[b];
        g.C = d.U + moff[b];
        g.M = n;
        g.N = n;
        g.K = n;
        g.sa_i = 1;
        g.sa_k = n;
        g.sb_k = 1;
        g.sb_j = n;
        g.sc_i = n;
        g.sc_j = 1;
        probs.push_back(g);
    }
    size_t tiles_cap = 0;
    const size_t probs_cap = eigh_gemm_bytes(dims, &tiles_cap);
    launch_gemm_batch(probs, d.gemm_probs, probs_cap, d.gemm_tiles, tiles_cap, st);
}

// Complex Hermitian blocks: embedding, real eigensolve of the embedding,
// extraction of the complex eigenvectors (see cx_extract_kernel).
static void launch_eigh_complex(pgx_ctx* c) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    const int nb = P.nblocks;
    std::vector<int> d2(nb);
    std::vector<long> m2(nb), e2(nb);
    long msz2 = 0, esz2 = 0;
    for (int b = 0; b < nb; ++b) {
        d2[b] = 2 * P.dims[b];
        m2[b] = msz2;
        e2[b] = esz2;
        msz2 += (long)d2[b] * d2[b];
        esz2 += d2[b];
    }
    // dims | moff | eoff of the embedding, on the device
    const size_t off_m = (nb * sizeof(int) + 15) & ~size_t(15);
    P.cx_meta.reserve(off_m + 2 * nb * sizeof(long));
    int* dd2 = P.cx_meta.as<int>();
    long* dm2 = reinterpret_cast<long*>(P.cx_meta.as<char>() + off_m);
    long* de2 = dm2 + nb;
    h2d(dd2, d2.data(), nb * sizeof(int), st);
    h2d(dm2, m2.data(), nb * sizeof(long), st);
    h2d(de2, e2.data(), nb * sizeof(long), st);
    P.cx_H.reserve(msz2 * sizeof(double));
    P.cx_A.reserve(msz2 * sizeof(double));
    P.cx_Zc.reserve(msz2 * sizeof(double));
    P.cx_U.reserve(msz2 * sizeof(double));
    P.cx_E.reserve(esz2 * sizeof(double));
    P.cx_tri.reserve((3 * esz2) * sizeof(double) + 3 * esz2 * sizeof(int) + 64);
    P.cx_S.reserve(eigh_vec_scratch_doubles(d2) * sizeof(double));
    P.cx_items.reserve(eigh_item_bytes(d2));
    size_t tiles_b = 0;
    const size_t probs_b = eigh_gemm_bytes(d2, &tiles_b);
    P.cx_gemm.reserve(((probs_b + 255) & ~size_t(255)) + tiles_b);
    int dmax = 1;
    for (int x : P.dims) dmax = std::max(dmax, x);
    {
        dim3 g(std::min(ceil_div((long)dmax * dmax, 256), 1024), (unsigned)nb);
        cx_embed_kernel<<<g, 256, 0, st>>>(P.d_dims, P.d_moff, dm2, P.d_H, P.cx_H.as<double>());
        check_launch("cx_embed_kernel");
    }
    EighDev d;
    d.dims = dd2;
    d.moff = dm2;
    d.eoff = de2;
    d.H = P.cx_H.as<double>();
    d.A = P.cx_A.as<double>();
    d.Zc = P.cx_Zc.as<double>();
    d.tri = P.cx_tri.as<double>();
    d.lam = d.tri + 2 * esz2;
    d.sb = reinterpret_cast<int*>(d.lam + esz2);
    d.rank = d.sb + 2 * esz2;
    d.S = P.cx_S.as<double>();
    d.items = P.cx_items.p;
    d.gemm_probs = P.cx_gemm.p;
    d.gemm_tiles = P.cx_gemm.as<char>() + ((probs_b + 255) & ~size_t(255));
    d.U = P.cx_U.as<double>();
    d.E = P.cx_E.as<double>();
    d.status = P.d_status;
    for (int i = 0; i < 3; ++i) {
        d.aux[i] = c->aux[i];
        d.join[i] = c->join[i];
    }
    d.fork = c->fork;
    launch_eigh_raw(d, d2, m2, st);
    // pairs of the embedding agree to the eigensolver's accuracy, far inside
    // this clustering tolerance; distinct eigenvalues of H closer than it are
    // orthonormalised together
    std::vector<double> e(esz2);
    PGX_CUDA(cudaMemcpyAsync(e.data(), d.E, esz2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    double emax = 1.0;
    for (double x : e) emax = std::max(emax, std::fabs(x));
    cx_extract_kernel<<<nb, 128, 0, st>>>(P.d_dims, P.d_moff, P.d_eoff, dm2, de2, d.E, d.U, P.d_E,
                                          reinterpret_cast<cd*>(P.d_U), 1e-10 * emax, P.d_status);
    check_launch("cx_extract_kernel");
}

void launch_eigh(pgx_ctx* c) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    if (!c->fork) {
        PGX_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
        for (int i = 0; i < 3; ++i) {
            PGX_CUDA(cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking));
            PGX_CUDA(cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming));
        }
    }
    if (P.is_complex) {
        launch_eigh_complex(c);
        return;
    }
    // tri (2 sum d) | lam (sum d) | sb (2 sum d ints) | rank (sum d ints)
    const long e = std::max<long>(P.esize, 1);
    P.tri.reserve((2 * e + e) * sizeof(double) + 3 * e * sizeof(int) + 64);
    P.tri_items.reserve(eigh_item_bytes(P.dims));
    size_t tiles_b = 0;
    const size_t probs_b = eigh_gemm_bytes(P.dims, &tiles_b);
    P.eigh_gemm.reserve(((probs_b + 255) & ~size_t(255)) + tiles_b);
    P.eigh_scratch.reserve(eigh_vec_scratch_doubles(P.dims) * sizeof(double));
    EighDev d;
    d.dims = P.d_dims;
    d.moff = P.d_moff;
    d.eoff = P.d_eoff;
    d.H = P.d_H;
    d.A = P.d_work;
    d.Zc = P.d_work2;
    d.tri = P.tri.as<double>();
    d.lam = d.tri + 2 * e;
    d.sb = reinterpret_cast<int*>(d.lam + e);
    d.rank = d.sb + 2 * e;
    d.S = P.eigh_scratch.as<double>();
    d.items = P.tri_items.p;
    d.gemm_probs = P.eigh_gemm.p;
    d.gemm_tiles = P.eigh_gemm.as<char>() + ((probs_b + 255) & ~size_t(255));
    d.U = P.d_U;
    d.E = P.d_E;
    d.status = P.d_status;
    for (int i = 0; i < 3; ++i) {
        d.aux[i] = c->aux[i];
        d.join[i] = c->join[i];
    }
    d.fork = c->fork;
    launch_eigh_raw(d, P.dims, P.moff, st);
}

}  // namespace pgx
