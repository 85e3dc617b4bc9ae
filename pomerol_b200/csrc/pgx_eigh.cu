// K1: batched FP64 symmetric eigensolver.
//
// Replaces Eigen::SelfAdjointEigenSolver as called by HamiltonianPart::computeImpl
// (HamiltonianPart.cpp:90-102).  Stages:
//   1. Householder reduction to tridiagonal form T and explicit accumulation
//      of the orthogonal factor Q (Golub & Van Loan, "Matrix Computations",
//      4th ed., 8.3.1):
//      eigh_cluster_kernel, one thread-block cluster of 1-8 CTAs per block
//      with the matrix in distributed shared memory (blocks up to 464 states);
//      larger blocks: a blocked reduction (panels of 32 columns, trailing
//      updates and Q by GEMMs) over the whole GPU.  Q is stored column-major.
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

// ----------------------------------------------------------------------------
// Householder stage for blocks too large for a cluster's shared memory
// (n > 464): the blocked reduction of LAPACK's dsytrd / dlatrd (lower).
// Panels of BHH_NB columns.  Column j of the panel that starts at k is first
// brought up to date with the panel's earlier reflectors,
//   a = A(j:, j) - V W(j, :)^T - W V(j, :)^T,
// then reflected (v, tau; d_j = a_j, e_j = alpha) and
//   w = tau (A(j+1:, j+1:) v - V (W^T v) - W (V^T v)),  w -= (tau/2)(w.v) v,
// with A the matrix as it was at the start of the panel: the trailing matrix
// is only read per column (bhh_symv_kernel) and written once per panel,
// A(k+p:, k+p:) -= V W^T + W V^T, by one GEMM of inner size 2p.
// The reflectors stay in the columns of A below the diagonal (zeros above),
// and Q = H_0 ... H_{n-3} is formed panel by panel, from the last one, as
// Q(k+1:, k+1:) += V (-T) (V^T Q(k+1:, k+1:)), where T is the upper
// triangular factor of the panel's block reflector I - V T V^T (LAPACK
// dlarft).  Every such block of a problem advances in the same launches.
// The outputs (tridiagonal, column-major Q) are those of the cluster kernel.
constexpr int BHH_NB = 32;  // panel width
constexpr int BHH_COL_THREADS = 1024;
constexpr int BHH_SYMV_THREADS = 256;
constexpr int BHH_SYMV_ROWS = 32;  // trailing rows per symv CTA

struct BigArgs {
    const int* big;    // the large blocks, largest first
    const long* boff;  // per entry of `big`: scratch offset in S (doubles)
    int nact;          // entries of `big` this launch covers (a prefix)
    const int* dims;
    const long* moff;
    const long* eoff;
    double* A;    // per block n x n row-major working copy of H
    double* Zc;   // per block Q, column-major
    double* S;    // scratch
    double* tri;  // per block: d (n), e (n)
    int k;        // first column of the current panel
    int fin;      // column whose w is completed (-1: none)
    int col;      // column to reflect (-1: none)
};

// Scratch of one large block, in doubles: V and W (BHH_NB columns of n each),
// y (n), tau (n), then per panel its Gram matrix and -T (BHH_NB^2 each).
__host__ __device__ inline long bhh_panels(int n) { return n > 2 ? (n - 2 + BHH_NB - 1) / BHH_NB : 0; }
__host__ __device__ inline long bhh_scratch_doubles(int n) {
    return 2L * BHH_NB * n + 2L * n + 2 * bhh_panels(n) * BHH_NB * BHH_NB;
}

__global__ void __launch_bounds__(BHH_COL_THREADS) bhh_col_kernel(BigArgs g) {
    __shared__ double red[32];
    __shared__ double dots[2 * BHH_NB];
    __shared__ double sv[BHH_NB], sw[BHH_NB];
    __shared__ double hh[2];
    const int b = g.big[blockIdx.x];
    const int n = g.dims[b];
    double* A = g.A + g.moff[b];
    double* V = g.S + g.boff[blockIdx.x];  // column t at V + t n
    double* W = V + (long)BHH_NB * n;
    const double* y = W + (long)BHH_NB * n;
    double* tau = W + (long)BHH_NB * n + n;
    const long eo = g.eoff[b];
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    const int last = n - 3;  // the last column with a reflector
    // ---- complete w of column fin
    if (g.fin >= 0 && g.fin <= last) {
        const int f = g.fin, cf = f - g.k;
        const double* v = V + (long)cf * n;
        double* w = W + (long)cf * n;
        const double t = tau[f];
        if (t == 0.0) {
            for (int r = tid; r < n; r += nt) w[r] = 0.0;
        } else {
            // dots[2s] = W_s . v, dots[2s + 1] = V_s . v (v vanishes above row f + 1)
            for (int q = wid; q < 2 * cf; q += nw) {
                const double* x = ((q & 1) ? V : W) + (long)(q >> 1) * n;
                double acc = 0.0;
                for (int r = f + 1 + lane; r < n; r += 32) acc = fma(x[r], v[r], acc);
                acc = warp_sum(acc);
                if (lane == 0) dots[q] = acc;
            }
            __syncthreads();
            double part = 0.0;
            for (int r = tid; r < n; r += nt) {
                double wr = 0.0;
                if (r > f) {
                    double acc = y[r];
                    for (int s2 = 0; s2 < cf; ++s2)
                        acc -= V[(long)s2 * n + r] * dots[2 * s2] + W[(long)s2 * n + r] * dots[2 * s2 + 1];
                    wr = t * acc;
                    part = fma(wr, v[r], part);
                }
                w[r] = wr;
            }
            const double K = 0.5 * t * block_sum(part, red);  // its barriers order the writes of w above
            for (int r = f + 1 + tid; r < n; r += nt) w[r] -= K * v[r];
        }
        __syncthreads();
    }
    // ---- reflect column col
    if (g.col >= 0 && g.col <= last) {
        const int j = g.col, cc = j - g.k;
        for (int s2 = tid; s2 < cc; s2 += nt) {
            sv[s2] = V[(long)s2 * n + j];
            sw[s2] = W[(long)s2 * n + j];
        }
        __syncthreads();
        double* a = V + (long)cc * n;         // the updated column, then the reflector, in place
        const double* Arow = A + (long)j * n;  // row j holds column j (A symmetric)
        double part = 0.0;
        for (int r = tid; r < n; r += nt) {
            double x = 0.0;
            if (r >= j) {
                x = Arow[r];
                for (int s2 = 0; s2 < cc; ++s2) x -= V[(long)s2 * n + r] * sw[s2] + W[(long)s2 * n + r] * sv[s2];
                if (r >= j + 2) part = fma(x, x, part);
            }
            a[r] = x;
        }
        const double sigma = block_sum(part, red);
        if (tid == 0) {
            const double x0 = a[j + 1];
            double alpha = x0, tj = 0.0, v0 = 0.0;
            if (sigma != 0.0) {
                const double mu = sqrt(x0 * x0 + sigma);
                alpha = (x0 > 0.0) ? -mu : mu;  // v0 = x0 - alpha without cancellation
                v0 = x0 - alpha;
                tj = 2.0 / (sigma + v0 * v0);
            }
            hh[0] = tj;
            hh[1] = v0;
            g.tri[2 * eo + j] = a[j];
            g.tri[2 * eo + n + j] = alpha;
            tau[j] = tj;
        }
        __syncthreads();
        const double tj = hh[0], v0 = hh[1];
        for (int r = tid; r < n; r += nt) {
            const double vr = (tj != 0.0 && r > j) ? ((r == j + 1) ? v0 : a[r]) : 0.0;
            a[r] = vr;
            A[(long)r * n + j] = vr;  // column j of A: zeros down to the diagonal, then v
        }
    }
}

// y(j+1:) = A(j+1:, j+1:) v for column j = col of every active block; one
// warp per row, the CTAs of the active blocks in one flat grid.
__global__ void __launch_bounds__(BHH_SYMV_THREADS) bhh_symv_kernel(BigArgs g) {
    extern __shared__ double svec[];
    int q = blockIdx.x, bi = 0, m = 0;
    for (; bi < g.nact; ++bi) {
        m = g.dims[g.big[bi]] - g.col - 1;
        const int cnt = (m + BHH_SYMV_ROWS - 1) / BHH_SYMV_ROWS;
        if (q < cnt) break;
        q -= cnt;
    }
    if (bi >= g.nact) return;
    const int b = g.big[bi];
    const int n = g.dims[b], j = g.col, cc = j - g.k;
    const double* A = g.A + g.moff[b];
    const double* v = g.S + g.boff[bi] + (long)cc * n + (j + 1);
    double* y = g.S + g.boff[bi] + 2L * BHH_NB * n + (j + 1);
    for (int c = threadIdx.x; c < m; c += blockDim.x) svec[c] = v[c];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int rr = wid; rr < BHH_SYMV_ROWS; rr += BHH_SYMV_THREADS / 32) {
        const int r = q * BHH_SYMV_ROWS + rr;
        if (r >= m) break;
        const double* row = A + (long)(j + 1 + r) * n + (j + 1);
        double s0 = 0.0, s1 = 0.0;
        int c = lane;
        for (; c + 32 < m; c += 64) {
            s0 = fma(row[c], svec[c], s0);
            s1 = fma(row[c + 32], svec[c + 32], s1);
        }
        if (c < m) s0 = fma(row[c], svec[c], s0);
        const double sum = warp_sum(s0 + s1);
        if (lane == 0) y[r] = sum;
    }
}

// the last 2 x 2 of the tridiagonal, and Q = I, per large block
__global__ void bhh_finish_kernel(BigArgs g) {
    const int b = g.big[blockIdx.x];
    const int n = g.dims[b];
    const double* A = g.A + g.moff[b];
    double* Z = g.Zc + g.moff[b];
    const long eo = g.eoff[b];
    if (threadIdx.x == 0) {
        if (n >= 2) {
            g.tri[2 * eo + n - 2] = A[(long)(n - 2) * n + (n - 2)];
            g.tri[2 * eo + n + n - 2] = A[(long)(n - 1) * n + (n - 2)];
        }
        g.tri[2 * eo + n - 1] = A[(long)(n - 1) * n + (n - 1)];
        g.tri[2 * eo + n + n - 1] = 0.0;
    }
    for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) Z[i] = ((i / n) == (i % n)) ? 1.0 : 0.0;
}

// -T of every panel's block reflector from its Gram matrix G = V^T V (LAPACK
// dlarft, forward, columnwise): T_ii = tau_i, T(0:i, i) = -tau_i T(0:i, 0:i) G(0:i, i).
// One warp per (block, panel); lane t owns row t of T.
__global__ void bhh_tfactor_kernel(BigArgs g) {
    int q = blockIdx.x, bi = 0;
    for (; bi < g.nact; ++bi) {
        const int np = (int)bhh_panels(g.dims[g.big[bi]]);
        if (q < np) break;
        q -= np;
    }
    if (bi >= g.nact) return;
    const int n = g.dims[g.big[bi]];
    const int k = q * BHH_NB, p = min(BHH_NB, n - 2 - k);
    double* base = g.S + g.boff[bi];
    const double* tau = base + 2L * BHH_NB * n + n + k;
    const double* G = base + 2L * BHH_NB * n + 2L * n + (long)q * BHH_NB * BHH_NB;
    double* nT = base + 2L * BHH_NB * n + 2L * n + (bhh_panels(n) + q) * BHH_NB * BHH_NB;
    const int t = threadIdx.x;
    double row[BHH_NB];
#pragma unroll
    for (int i = 0; i < BHH_NB; ++i) row[i] = 0.0;
#pragma unroll
    for (int i = 0; i < BHH_NB; ++i) {
        if (i < p) {
            if (t == i) row[i] = tau[i];
            if (t < i) {
                double acc = 0.0;
#pragma unroll
                for (int s2 = 0; s2 < BHH_NB; ++s2)
                    if (s2 >= t && s2 < i) acc = fma(row[s2], G[s2 * BHH_NB + i], acc);
                row[i] = -tau[i] * acc;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < BHH_NB; ++i) nT[t * BHH_NB + i] = -row[i];
}

// ----------------------------------------------------------------------------
// Householder stage on a thread-block cluster (blocks whose matrix fits in
// the shared memory of up to 8 CTAs: 464 states at 220 KB per CTA).
//
// The C CTAs of a cluster hold the block's symmetric matrix in distributed
// shared memory, row r in CTA r mod C (cyclic, so the shrinking trailing
// matrix stays spread over all CTAs).  Every CTA also keeps its own copy of
// the current row k (the column below the diagonal), brought up to date
// locally, so one cluster barrier per step suffices.  Step k:
//   every CTA forms the Householder vector v, tau from its copy of row k,
//   computes p = tau B v on its own rows and its share of v.p (into the
//   buffers of this step's parity);
//   cluster barrier;
//   every CTA gathers all of p and the v.p shares, forms
//   w = p - (tau/2)(v.p) v, reads row k+1 from its owner (who leaves that
//   row alone in this step: it leaves the trailing matrix) and updates it
//   into its copy, and applies B -= v w^T + w v^T to its own rows r >= k+2.
// A CTA one step ahead writes the other parity's buffers, and cannot get two
// steps ahead before the others pass the barrier, so no reader is overrun.
// CTA 0 stores d_k, e_k and sqrt(tau) v (row k of V in global memory).
// Q = H_0 ... H_{n-3} is then formed from V with the CTAs owning columns
// j = c (mod C) of Q: a column's update needs only that column, so this
// phase has no cross-CTA traffic.  The outputs (tridiagonal, column-major Q)
// are those of the blocked large-block path.
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
    return (size_t)R * n + 3 * (size_t)n + 2 * (size_t)R + 2;
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
    double* cur = w + n;                    // n: row k, up to date (this CTA's copy)
    double* pb = cur + n;                   // 2 R: p of the steps of either parity
    double* dslot = pb + 2 * R;             // 2
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    const double* Hb = g.H + mo;
    double* V = g.V + mo;

    for (long idx = tid; idx < (long)nrows * n; idx += nt) {
        const int lr = (int)(idx / n), j = (int)(idx % n);
        slab[idx] = Hb[(long)(c + C * lr) * n + j];
    }
    for (int j = tid; j < n; j += nt) cur[j] = Hb[j];  // row 0
    __syncthreads();
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        double* p = pb + (k & 1) * R;
        double part = 0.0;
        for (int i = tid; i < m; i += nt) {
            const double x = cur[k + 1 + i];
            v[i] = x;
            if (i > 0) part += x * x;
        }
        const double sigma = block_sum(part, red);
        const double x0 = v[0];
        const double dk = cur[k];
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
            double sacc = 0.0;
            for (int j = lane; j < m; j += 32) sacc = fma(row[j], v[j], sacc);
            sacc = warp_sum(sacc) * tau;
            if (lane == 0) {
                p[lr] = sacc;
                dpart += v[c + C * lr - (k + 1)] * sacc;
            }
        }
        const double dsum = block_sum(dpart, red);
        if (tid == 0) dslot[k & 1] = dsum;
        cl.sync();  // p and the v.p shares of this step are complete in every CTA
        double dtot = 0.0;
        for (int q = 0; q < C; ++q) dtot += cl.map_shared_rank(dslot, q)[k & 1];
        const double K = 0.5 * tau * dtot;
        for (int i = tid; i < m; i += nt) {
            const int r = k + 1 + i;
            w[i] = cl.map_shared_rank(pb, r % C)[(k & 1) * R + r / C] - K * v[i];
        }
        __syncthreads();
        // row k+1, up to date through step k-1 in its owner's slab, updated into this CTA's copy
        {
            const double* nxt = cl.map_shared_rank(slab, (k + 1) % C) + (size_t)((k + 1) / C) * n;
            const double v1 = v[0], w1 = w[0];
            for (int i = tid; i < m; i += nt) cur[k + 1 + i] = nxt[k + 1 + i] - (v1 * w[i] + w1 * v[i]);
        }
        // own rows r >= k+2 (row k+1 is read by the other CTAs in this step)
        const int lr2 = (k + 2 - c + C - 1) / C;
        for (int lr = lr2 + wid; lr < nrows; lr += nw) {
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
        __syncthreads();  // cur and v are reused by the next step
    }
    cl.sync();
    if (c == 0 && tid == 0) {
        auto elem = [&](int r, int j) { return cl.map_shared_rank(slab, r % C)[(size_t)(r / C) * n + j]; };
        // row n-2 is this CTA's copy (its owner skipped it in the last step); row n-1 its owner's
        if (n >= 2) {
            g.tri[2 * eo + n - 2] = cur[n - 2];
            g.tri[2 * eo + n + n - 2] = cur[n - 1];
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
// The CTA's warp orthogonalises each chain whose head lies in its range:
// modified Gram-Schmidt (two passes) of every member against its close
// predecessors, the dot products and updates spread over the lanes (a chain
// of a symmetry multiplet can hold dozens of vectors of thousands of states).
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
    const int lane = threadIdx.x;
    const double ortol = CHAIN_TOL * tn;
    const int* sa = g.sb + 2 * eo;
    const int* sbe = sa + n;
    const int* rank = g.rank + eo;
    double* Zb = g.Z + mo;
    for (int j = it.j0; j < it.j1; ++j) {
        const int a = sa[j], b = sbe[j];
        if (j > a && lam[j] - lam[j - 1] <= ortol) continue;  // not the head of a chain
        bool ok = true;
        for (int jj = j + 1; jj <= b && lam[jj] - lam[jj - 1] <= ortol; ++jj) {
            double* z = Zb + (long)rank[jj] * n;
            for (int pass = 0; pass < 2 && ok; ++pass) {
                for (int pp = jj - 1; pp >= j && lam[jj] - lam[pp] <= ortol; --pp) {
                    const double* qv = Zb + (long)rank[pp] * n;
                    double dot = 0.0;
                    for (int i = a + lane; i <= b; i += TRI_THREADS) dot = fma(qv[i], z[i], dot);
                    dot = warp_sum(dot);
                    for (int i = a + lane; i <= b; i += TRI_THREADS) z[i] = fma(-dot, qv[i], z[i]);
                }
                double nn = 0.0;
                for (int i = a + lane; i <= b; i += TRI_THREADS) nn = fma(z[i], z[i], nn);
                nn = warp_sum(nn);
                if (!(nn > 0.0) || !isfinite(nn)) {
                    ok = false;
                } else {
                    const double inv = rsqrt(nn);
                    for (int i = a + lane; i <= b; i += TRI_THREADS) z[i] *= inv;
                }
            }
            __syncwarp();
        }
        if (!ok && lane == 0) atomicExch(g.status, PGX_ERR_NUMERIC);
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

constexpr int CL_NCLS = 5;
constexpr int CL_SIZES[CL_NCLS] = {1, 2, 4, 8, 16};
constexpr size_t CL_SMEM_MAX = 226 * 1024;  // dynamic shared memory per CTA (the static part is 256 bytes)

// The cluster class of an n x n block, or -1 (the block then takes the
// large-block path): the smallest cluster whose shared memory holds the
// block.  16 CTAs (a non-portable cluster size) only where 8 do not suffice
// (465 to 513 states): at 400 states the per-step cost is set by the cluster
// barriers, and 16-CTA clusters were measured slower than 8-CTA ones there.
static int cluster_class(int n) {
    if (n > CL_MAX_DIM) return -1;
    for (int i = 0; i < CL_NCLS; ++i)
        if (cluster_smem_doubles(n, CL_SIZES[i]) * sizeof(double) <= CL_SMEM_MAX) return i;
    return -1;
}

// doubles of vector_kernel scratch (EighDev::S); the large-block path uses
// the same buffer before the vector stage (a -1 scale vector, then one
// scratch per large block)
size_t eigh_vec_scratch_doubles(const std::vector<int>& dims) {
    size_t s = 0, big = 2 * BHH_NB;
    for (int n : dims) {
        s += 4 * (size_t)n * TRI_THREADS * ((n + TRI_THREADS - 1) / TRI_THREADS);
        if (cluster_class(n) < 0) big += (size_t)bhh_scratch_doubles(n);
    }
    return std::max<size_t>(std::max(s, big), 1);
}


// Householder stage plan: the block list of each cluster size (largest
// blocks first) and the blocks left to the single-CTA global-memory kernel.
struct HhPlan {
    std::vector<int> cls[CL_NCLS];
    std::vector<int> global;
};

static HhPlan hh_plan(const std::vector<int>& dims) {
    std::vector<int> order(dims.size());
    for (size_t b = 0; b < dims.size(); ++b) order[b] = (int)b;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return dims[x] > dims[y]; });
    HhPlan h;
    for (int b : order) {
        const int q = cluster_class(dims[b]);
        if (q < 0) h.global.push_back(b);
        else h.cls[q].push_back(b);
    }
    return h;
}

// the large blocks (beyond the cluster path), largest first
static std::vector<int> big_blocks(const std::vector<int>& dims) {
    std::vector<int> big;
    for (size_t b = 0; b < dims.size(); ++b)
        if (cluster_class(dims[b]) < 0) big.push_back((int)b);
    std::stable_sort(big.begin(), big.end(), [&](int x, int y) { return dims[x] > dims[y]; });
    return big;
}

// descriptor bytes: bisection items, one int per block (Householder lists);
// with large blocks also their scratch offsets and the column-index table of
// the panel updates
static size_t big_desc_bytes(const std::vector<int>& dims) {
    const size_t nb = big_blocks(dims).size();
    if (nb == 0) return 0;
    return 8 + nb * sizeof(long) + (size_t)BHH_NB * 4 * BHH_NB * sizeof(int);
}
size_t eigh_item_bytes(const std::vector<int>& dims) {
    std::vector<TriItem> items;
    tri_plan(dims, items);
    return items.size() * sizeof(TriItem) + dims.size() * sizeof(int) + big_desc_bytes(dims);
}

size_t eigh_gemm_bytes(const std::vector<int>& dims, size_t* tiles_bytes) {
    size_t np = dims.size();
    size_t panels = 0;
    for (int b : big_blocks(dims)) panels += (size_t)bhh_panels(dims[b]);
    np = std::max(np, panels);
    if (tiles_bytes) *tiles_bytes = gemm_index_bytes(np);
    return std::max<size_t>(np, 1) * sizeof(GemmProblem<double, double, double>);
}

// The large-block Householder path (see bhh_col_kernel) on stream st.
// big: the blocks, largest first; d_big / d_boff / d_kidx: their device list,
// scratch offsets and the panel-update column table (uploaded by the caller).
static void launch_big(const EighDev& d, const std::vector<int>& dims, const std::vector<long>& moff,
                       const std::vector<int>& big, const int* d_big, const long* d_boff, const int* d_kidx,
                       cudaStream_t st) {
    const int nbig = (int)big.size();
    std::vector<long> boff(nbig);
    long o = 2 * BHH_NB;
    for (int i = 0; i < nbig; ++i) {
        boff[i] = o;
        o += bhh_scratch_doubles(dims[big[i]]);
    }
    const int nmax = dims[big[0]];
    // blocks with a reflector in column j: a prefix of the list
    auto nact = [&](int j) {
        int c = 0;
        while (c < nbig && dims[big[c]] - 2 > j) ++c;
        return c;
    };
    BigArgs a{};
    a.big = d_big;
    a.boff = d_boff;
    a.dims = d.dims;
    a.moff = d.moff;
    a.eoff = d.eoff;
    a.A = d.A;
    a.Zc = d.Zc;
    a.S = d.S;
    a.tri = d.tri;
    double fl = 0.0, by = 0.0;
    for (int b : big) {
        const double n = dims[b];
        fl += 8.0 / 3.0 * n * n * n;
        by += 16.0 * n * n + 16.0 * n;
    }
    ProfRange pr("eigh_blocked_householder", st, fl, by);
    for (int b : big)
        PGX_CUDA(cudaMemcpyAsync(d.A + moff[b], d.H + moff[b], (size_t)dims[b] * dims[b] * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st));
    {
        double neg[2 * BHH_NB];
        for (double& x : neg) x = -1.0;
        h2d(d.S, neg, sizeof(neg), st);
    }
    PGX_CUDA(cudaFuncSetAttribute(bhh_symv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * nmax)));
    std::vector<GemmProblem<double, double, double>> probs;
    size_t tiles_cap = 0;
    const size_t probs_cap = eigh_gemm_bytes(dims, &tiles_cap);
    // ---- tridiagonalisation
    for (int k = 0; k < nmax - 2; k += BHH_NB) {
        a.k = k;
        const int jend = std::min(k + BHH_NB, nmax - 2);  // columns k .. jend - 1 of the largest block
        for (int j = k; j < jend; ++j) {
            a.fin = (j > k) ? j - 1 : -1;
            a.col = j;
            a.nact = nact(j > k ? j - 1 : j);
            {
                ProfRange r1("bhh_col_kernel", st, 0.0, 0.0);
                bhh_col_kernel<<<(unsigned)a.nact, BHH_COL_THREADS, 0, st>>>(a);
                check_launch("bhh_col_kernel");
            }
            a.fin = -1;
            a.nact = nact(j);
            long ctas = 0;
            double bytes = 0.0;
            for (int i = 0; i < a.nact; ++i) {
                const long m = dims[big[i]] - j - 1;
                ctas += (m + BHH_SYMV_ROWS - 1) / BHH_SYMV_ROWS;
                bytes += 8.0 * m * m;
            }
            ProfRange r2("bhh_symv_kernel", st, 0.0, bytes);
            bhh_symv_kernel<<<(unsigned)ctas, BHH_SYMV_THREADS, sizeof(double) * nmax, st>>>(a);
            check_launch("bhh_symv_kernel");
        }
        a.fin = jend - 1;
        a.col = -1;
        a.nact = nact(jend - 1);
        {
            ProfRange r1("bhh_col_kernel", st, 0.0, 0.0);
            bhh_col_kernel<<<(unsigned)a.nact, BHH_COL_THREADS, 0, st>>>(a);
            check_launch("bhh_col_kernel");
        }
        // A(k+p:, k+p:) -= V W^T + W V^T, p = the block's columns in this panel
        probs.clear();
        for (int i = 0; i < nact(k); ++i) {
            const int n = dims[big[i]];
            const int p = std::min(BHH_NB, n - 2 - k), kp = k + p, m = n - kp;
            if (m <= 0) continue;
            double* VW = d.S + boff[i] + kp;
            GemmProblem<double, double, double> g{};
            g.A = VW;
            g.B = VW;
            g.C = d.A + moff[big[i]] + (long)kp * n + kp;
            g.M = m;
            g.N = m;
            g.K = 2 * p;
            g.sa_i = 1;
            g.sa_k = n;
            g.sb_k = n;
            g.sb_j = 1;
            g.sc_i = n;
            g.sc_j = 1;
            g.a_kidx = d_kidx + (p - 1) * 4 * BHH_NB;
            g.b_kidx = g.a_kidx + 2 * BHH_NB;
            g.kscale = d.S;
            g.accumulate = 1;
            probs.push_back(g);
        }
        launch_gemm_batch(probs, d.gemm_probs, probs_cap, d.gemm_tiles, tiles_cap, st);
    }
    a.nact = nbig;
    bhh_finish_kernel<<<(unsigned)nbig, 256, 0, st>>>(a);
    check_launch("bhh_finish_kernel");
    // ---- Q: Gram matrices and -T of every panel, then the panels from the last
    probs.clear();
    long npan_total = 0;
    long npan_max = 0;
    for (int i = 0; i < nbig; ++i) {
        const int n = dims[big[i]];
        const long np = bhh_panels(n);
        npan_max = std::max(npan_max, np);
        npan_total += np;
        for (long q = 0; q < np; ++q) {
            const int k = (int)q * BHH_NB, p = std::min(BHH_NB, n - 2 - k), m = n - k - 1;
            const double* Vp = d.A + moff[big[i]] + (long)(k + 1) * n + k;
            GemmProblem<double, double, double> g{};
            g.A = Vp;  // V^T
            g.B = Vp;
            g.C = d.S + boff[i] + 2L * BHH_NB * n + 2L * n + q * BHH_NB * BHH_NB;
            g.M = p;
            g.N = p;
            g.K = m;
            g.sa_i = 1;
            g.sa_k = n;
            g.sb_k = n;
            g.sb_j = 1;
            g.sc_i = BHH_NB;
            g.sc_j = 1;
            probs.push_back(g);
        }
    }
    launch_gemm_batch(probs, d.gemm_probs, probs_cap, d.gemm_tiles, tiles_cap, st);
    a.nact = nbig;
    bhh_tfactor_kernel<<<(unsigned)npan_total, 32, 0, st>>>(a);
    check_launch("bhh_tfactor_kernel");
    for (long q = npan_max - 1; q >= 0; --q) {
        const int k = (int)q * BHH_NB;
        std::vector<GemmProblem<double, double, double>> py, pt, pu;
        for (int i = 0; i < nact(k); ++i) {
            const int n = dims[big[i]];
            const int p = std::min(BHH_NB, n - 2 - k), m = n - k - 1;
            const double* Vp = d.A + moff[big[i]] + (long)(k + 1) * n + k;
            double* Qs = d.Zc + moff[big[i]] + (long)(k + 1) * n + (k + 1);
            double* Y = d.S + boff[i];
            double* Y2 = Y + (long)BHH_NB * n;
            const double* nT = d.S + boff[i] + 2L * BHH_NB * n + 2L * n + (bhh_panels(n) + q) * BHH_NB * BHH_NB;
            GemmProblem<double, double, double> g{};
            g.A = Vp;  // Y = V^T Q
            g.sa_i = 1;
            g.sa_k = n;
            g.B = Qs;
            g.sb_k = 1;
            g.sb_j = n;
            g.C = Y;
            g.sc_i = n;
            g.sc_j = 1;
            g.M = p;
            g.N = m;
            g.K = m;
            py.push_back(g);
            GemmProblem<double, double, double> h{};  // Y2 = (-T) Y
            h.A = nT;
            h.sa_i = BHH_NB;
            h.sa_k = 1;
            h.B = Y;
            h.sb_k = n;
            h.sb_j = 1;
            h.C = Y2;
            h.sc_i = n;
            h.sc_j = 1;
            h.M = p;
            h.N = m;
            h.K = p;
            pt.push_back(h);
            GemmProblem<double, double, double> u{};  // Q += V Y2
            u.A = Vp;
            u.sa_i = n;
            u.sa_k = 1;
            u.B = Y2;
            u.sb_k = n;
            u.sb_j = 1;
            u.C = Qs;
            u.sc_i = 1;
            u.sc_j = n;
            u.M = m;
            u.N = m;
            u.K = p;
            u.accumulate = 1;
            pu.push_back(u);
        }
        launch_gemm_batch(py, d.gemm_probs, probs_cap, d.gemm_tiles, tiles_cap, st);
        launch_gemm_batch(pt, d.gemm_probs, probs_cap, d.gemm_tiles, tiles_cap, st);
        launch_gemm_batch(pu, d.gemm_probs, probs_cap, d.gemm_tiles, tiles_cap, st);
    }
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
    size_t cl_smem[CL_NCLS] = {0, 0, 0, 0, 0};
    PGX_CUDA(cudaFuncSetAttribute(eigh_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CL_SMEM_MAX));
    PGX_CUDA(cudaFuncSetAttribute(eigh_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    for (int q = CL_NCLS - 1; q >= 0; --q) {
        if (hp.cls[q].empty()) continue;
        for (int b : hp.cls[q]) cl_smem[q] = std::max(cl_smem[q], cluster_smem_doubles(dims[b], CL_SIZES[q]) * sizeof(double));
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
            // 16-CTA clusters not schedulable: their blocks go to 8-CTA clusters where they fit
            bool moved = q == 4;
            for (int b : hp.cls[q])
                moved = moved && cluster_smem_doubles(dims[b], 8) * sizeof(double) <= CL_SMEM_MAX;
            PGX_CHECK(moved, PGX_ERR_CUDA, "the eigensolver's thread-block clusters cannot be scheduled on this device");
            hp.cls[3].insert(hp.cls[3].end(), hp.cls[q].begin(), hp.cls[q].end());
            std::stable_sort(hp.cls[3].begin(), hp.cls[3].end(), [&](int x, int y) { return dims[x] > dims[y]; });
            hp.cls[q].clear();
            cl_smem[q] = 0;
        }
    }
    std::vector<int> lists(hp.global);
    size_t cl_off[CL_NCLS];
    for (int q = 0; q < CL_NCLS; ++q) {
        cl_off[q] = lists.size();
        lists.insert(lists.end(), hp.cls[q].begin(), hp.cls[q].end());
    }
    // large blocks: scratch offsets (doubles into S) and, per panel width p, the
    // column gathers of the panel update [V_0..V_p-1 W_0..W_p-1] and [W.. V..]
    const std::vector<int>& big = hp.global;
    const size_t lists_end = items.size() * sizeof(TriItem) + lists.size() * sizeof(int);
    const size_t boff_at = (lists_end + 7) & ~size_t(7);
    size_t host_bytes = lists_end;
    std::vector<long> boff;
    std::vector<int> kidx;
    if (!big.empty()) {
        long o = 2 * BHH_NB;
        for (int b : big) {
            boff.push_back(o);
            o += bhh_scratch_doubles(dims[b]);
        }
        for (int p = 1; p <= BHH_NB; ++p) {
            std::vector<int> ia(2 * BHH_NB, 0), ib(2 * BHH_NB, 0);
            for (int t = 0; t < p; ++t) {
                ia[t] = t;
                ia[p + t] = BHH_NB + t;
                ib[t] = BHH_NB + t;
                ib[p + t] = t;
            }
            kidx.insert(kidx.end(), ia.begin(), ia.end());
            kidx.insert(kidx.end(), ib.begin(), ib.end());
        }
        host_bytes = boff_at + boff.size() * sizeof(long) + kidx.size() * sizeof(int);
        PGX_CHECK(host_bytes <= eigh_item_bytes(dims), PGX_ERR_ARG, "eigensolver descriptor layout overflow");
    }
    std::vector<char> host(host_bytes);
    std::memcpy(host.data(), items.data(), items.size() * sizeof(TriItem));
    std::memcpy(host.data() + items.size() * sizeof(TriItem), lists.data(), lists.size() * sizeof(int));
    if (!big.empty()) {
        std::memcpy(host.data() + boff_at, boff.data(), boff.size() * sizeof(long));
        std::memcpy(host.data() + boff_at + boff.size() * sizeof(long), kidx.data(), kidx.size() * sizeof(int));
    }
    h2d(d.items, host.data(), host.size(), st);
    const int* d_lists = reinterpret_cast<const int*>(static_cast<const char*>(d.items) + items.size() * sizeof(TriItem));
    const long* d_boff = reinterpret_cast<const long*>(static_cast<const char*>(d.items) + boff_at);
    const int* d_kidx = reinterpret_cast<const int*>(static_cast<const char*>(d.items) + boff_at +
                                                     boff.size() * sizeof(long));

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
    const bool fork = d.aux[0] && d.aux[1] && d.aux[2] && d.aux[3] && d.fork;
    if (fork) {
        PGX_CUDA(cudaEventRecord(d.fork, st));
        for (int i = 0; i < 4; ++i) PGX_CUDA(cudaStreamWaitEvent(d.aux[i], d.fork, 0));
    }
    if (!big.empty()) launch_big(d, dims, moff, big, d_lists, d_boff, d_kidx, st);
    for (int q = 0; q < CL_NCLS; ++q) {
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
        static const char* names[CL_NCLS] = {"eigh_cluster_kernel<1>", "eigh_cluster_kernel<2>", "eigh_cluster_kernel<4>",
                                       "eigh_cluster_kernel<8>", "eigh_cluster_kernel<16>"};
        ProfRange pr(names[q], sq, fl, by);
        PGX_CUDA(cudaLaunchKernelEx(&cfg, eigh_cluster_kernel, ca));
        check_launch("eigh_cluster_kernel");
    }
    if (fork) {
        for (int i = 0; i < 4; ++i) {
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
    for (int i = 0; i < 4; ++i) {
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

void ensure_side_streams(pgx_ctx* c) {
    if (c->fork) return;
    PGX_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    for (int i = 0; i < 4; ++i) {
        PGX_CUDA(cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking));
        PGX_CUDA(cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming));
    }
}

void launch_eigh(pgx_ctx* c) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    ensure_side_streams(c);
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
    for (int i = 0; i < 4; ++i) {
        d.aux[i] = c->aux[i];
        d.join[i] = c->join[i];
    }
    d.fork = c->fork;
    launch_eigh_raw(d, P.dims, P.moff, st);
}

}  // namespace pgx
