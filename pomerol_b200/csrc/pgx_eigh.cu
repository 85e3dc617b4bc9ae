// K1: batched FP64 symmetric eigensolver, one CTA per symmetry block.
//
// Replaces Eigen::SelfAdjointEigenSolver as called by HamiltonianPart::computeImpl
// (HamiltonianPart.cpp:90-102).  Method (Golub & Van Loan, "Matrix Computations",
// 4th ed., sections 8.3.1 and 8.3.5): Householder reduction to tridiagonal form,
// explicit accumulation of the orthogonal factor, implicit QL iterations with
// Wilkinson shift whose Givens rotations are applied to the accumulated factor.
//
// Parallel layout inside a CTA:
//   * the Householder step's symmetric mat-vec and rank-2 update run over all
//     threads with coalesced column access (the trailing matrix is symmetric);
//   * the factor Q is stored column-major so that a Givens rotation on columns
//     (i, i+1) is a coalesced update over rows;
//   * each QL sweep's rotation sequence is produced by one thread into shared
//     memory and applied to all rows of Q in parallel (row r carries its
//     running value through the sweep, one load and one store per rotation);
//   * eigenvalues are sorted by a parallel rank computation.
// Convergence failure sets a device status word instead of trapping.

#include "pgx_common.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

constexpr int EIGH_THREADS = 512;
constexpr int QL_MAX_ITER = 90;

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

// Hypotenuse without overflow for the QL sweep (scaled form).
__device__ __forceinline__ double hyp(double a, double b) {
    double x = fabs(a), y = fabs(b);
    double m = fmax(x, y), n = fmin(x, y);
    if (m == 0.0) return 0.0;
    double r = n / m;
    return m * sqrt(1.0 + r * r);
}

struct EighArgs {
    const int* order;          // CTA -> block (largest first)
    const int* dims;
    const long* moff;          // matrix offset of block b (elements)
    const long* eoff;          // vector offset of block b
    const double* H;           // packed input blocks (row-major)
    double* A;                 // workspace copy (destroyed)
    double* Zc;                // workspace, column-major accumulated factor
    double* U;                 // output eigenvectors, row-major, columns = vectors
    double* E;                 // output eigenvalues, ascending per block
    int* status;               // set to PGX_ERR_NUMERIC on failure
};

__global__ void __launch_bounds__(EIGH_THREADS) eigh_kernel(EighArgs g) {
    extern __shared__ double sh[];
    __shared__ double red[32];
    __shared__ int s_state, s_m, s_nrot;

    const int b = g.order[blockIdx.x];
    const int n = g.dims[b];
    const long mo = g.moff[b], eo = g.eoff[b];
    const double* Hb = g.H + mo;
    double* A = g.A + mo;
    double* Z = g.Zc + mo;
    double* U = g.U + mo;
    double* E = g.E + eo;
    const int tid = threadIdx.x, nt = blockDim.x;

    double* v = sh;            // n   Householder vector   | later: cosines
    double* w = sh + n;        // n   p / w vectors        | later: sines
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
    // ---------------- implicit QL with Wilkinson shift ----------------
    double* cs = v;
    double* sn = w;
    const double eps = 2.220446049250313e-16;
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        while (true) {
            if (tid == 0) {
                int m = l;
                for (; m < n - 1; ++m) {
                    double dd = fabs(dg[m]) + fabs(dg[m + 1]);
                    if (fabs(ed[m]) <= eps * dd) break;
                }
                if (m == l) {
                    s_state = 1;
                } else if (++iter > QL_MAX_ITER) {
                    s_state = 2;
                } else {
                    double g = (dg[l + 1] - dg[l]) / (2.0 * ed[l]);
                    double r = hyp(g, 1.0);
                    g = dg[m] - dg[l] + ed[l] / (g + copysign(r, g));
                    double s = 1.0, c = 1.0, p = 0.0;
                    int i = m - 1, nrot = 0;
                    bool underflow = false;
                    for (; i >= l; --i) {
                        double f = s * ed[i], bb = c * ed[i];
                        r = hyp(f, g);
                        ed[i + 1] = r;
                        if (r == 0.0) {
                            dg[i + 1] -= p;
                            ed[m] = 0.0;
                            underflow = true;
                            break;
                        }
                        s = f / r;
                        c = g / r;
                        g = dg[i + 1] - p;
                        r = (dg[i] - g) * s + 2.0 * c * bb;
                        p = s * r;
                        dg[i + 1] = g + p;
                        g = c * r - bb;
                        cs[nrot] = c;
                        sn[nrot] = s;
                        ++nrot;
                    }
                    if (!underflow) {
                        dg[l] -= p;
                        ed[l] = g;
                        ed[m] = 0.0;
                    }
                    s_m = m;
                    s_nrot = nrot;
                    s_state = 0;
                }
            }
            __syncthreads();
            const int st = s_state;
            if (st == 2) {
                if (tid == 0) atomicExch(g.status, PGX_ERR_NUMERIC);
                return;
            }
            if (st == 1) break;
            const int m = s_m, nrot = s_nrot;
            // rotations at i = m-1, m-2, ..., m-nrot on columns (i, i+1)
            // columns m-1-q are loaded eight at a time before the stores of
            // the same group, so the loads overlap instead of waiting on them
            for (int r = tid; r < n; r += nt) {
                double carry = Z[(long)m * n + r];
                for (int q0 = 0; q0 < nrot; q0 += 8) {
                    double zi[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (q0 + u < nrot) zi[u] = Z[(long)(m - 1 - q0 - u) * n + r];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        if (q0 + u < nrot) {
                            const double s = sn[q0 + u], c = cs[q0 + u];
                            Z[(long)(m - q0 - u) * n + r] = s * zi[u] + c * carry;
                            carry = c * zi[u] - s * carry;
                        }
                    }
                }
                if (nrot > 0) Z[(long)(m - nrot) * n + r] = carry;
            }
            __syncthreads();
        }
    }
    // ---------------- sort ascending (rank) and write E, U (row-major) ----------------
    for (int i = tid; i < n; i += nt) {
        const double di = dg[i];
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const double dj = dg[j];
            rank += (dj < di) || (dj == di && j < i);
        }
        ed[i] = (double)rank;  // reuse as rank storage
        E[rank] = di;
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {
        const int rank = (int)ed[i];
        const double* col = Z + (long)i * n;
        for (int r = tid; r < n; r += nt) U[(long)r * n + rank] = col[r];
    }
}

}  // namespace

void launch_eigh(Problem& P, cudaStream_t st) {
    const size_t smem = 4 * sizeof(double) * (size_t)std::max(P.dmax, 1);
    PGX_CHECK(smem <= 200 * 1024, PGX_ERR_ARG, "block too large for the single-CTA eigensolver (d > 6400)");
    PGX_CUDA(cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EighArgs a;
    a.order = P.d_order;
    a.dims = P.d_dims;
    a.moff = P.d_moff;
    a.eoff = P.d_eoff;
    a.H = P.d_H;
    a.A = P.d_work;
    a.Zc = P.d_work2;
    a.U = P.d_U;
    a.E = P.d_E;
    a.status = P.d_status;
    eigh_kernel<<<P.nblocks, EIGH_THREADS, smem, st>>>(a);
    check_launch("eigh_kernel");
}

}  // namespace pgx
