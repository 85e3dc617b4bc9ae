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
    // hand the tridiagonal (diagonal, sub-diagonal) to the QL stage
    for (int i = tid; i < n; i += nt) {
        g.tri[2 * eo + i] = dg[i];
        g.tri[2 * eo + n + i] = ed[i];
    }
}

// Implicit QL with Wilkinson shift on the tridiagonal of one block, applied to
// a slice of rows of the accumulated factor held in shared memory.  Rows of
// Q evolve independently under right-multiplication by Givens rotations, so a
// large block is split over many CTAs; each CTA regenerates the (identical)
// rotation sequence with one thread and applies it to its rows.  The rows
// then give the eigenvectors, sorted by a rank computation.
struct QlItem {
    int block, row0, nrows, pad;
};

struct QlArgs {
    const QlItem* items;
    const int* dims;
    const long* moff;
    const long* eoff;
    const double* Zc;   // column-major factor per block
    const double* tri;  // per block: n diagonal then n sub-diagonal entries
    double* U;
    double* E;
    int* status;
};

__global__ void __launch_bounds__(128) ql_rows_kernel(QlArgs g) {
    extern __shared__ double sh[];
    __shared__ int s_state, s_m, s_nrot;
    const QlItem it = g.items[blockIdx.x];
    const int n = g.dims[it.block], nr = it.nrows, row0 = it.row0;
    const long mo = g.moff[it.block], eo = g.eoff[it.block];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ld = n + 1;  // odd row stride: rows of different threads fall in different banks
    double* dg = sh;
    double* ed = sh + n;
    double* cs = sh + 2 * n;
    double* sn = sh + 3 * n;
    double* Zs = sh + 4 * n;  // nr x ld
    for (int i = tid; i < n; i += nt) {
        dg[i] = g.tri[2 * eo + i];
        ed[i] = g.tri[2 * eo + n + i];
    }
    const double* Zc = g.Zc + mo;
    for (long e = tid; e < (long)nr * n; e += nt) {
        const int r = (int)(e % nr), j = (int)(e / nr);
        Zs[r * ld + j] = Zc[(long)j * n + row0 + r];
    }
    __syncthreads();
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
                    // one reciprocal square root per rotation keeps the
                    // dependent chain short (the sweep is sequential);
                    // d[i+1] of this step is the d[i] loaded one step earlier
                    double d_hi = dg[m];
                    for (; i >= l; --i) {
                        const double ei = ed[i], d_lo = dg[i];
                        const double f = s * ei, bb = c * ei;
                        const double r2 = fma(f, f, g * g);
                        if (r2 == 0.0) {
                            ed[i + 1] = 0.0;
                            dg[i + 1] = d_hi - p;
                            ed[m] = 0.0;
                            underflow = true;
                            break;
                        }
                        const double rinv = rsqrt(r2);
                        ed[i + 1] = r2 * rinv;
                        s = f * rinv;
                        c = g * rinv;
                        g = d_hi - p;
                        r = (d_lo - g) * s + 2.0 * c * bb;
                        p = s * r;
                        dg[i + 1] = g + p;
                        g = c * r - bb;
                        cs[nrot] = c;
                        sn[nrot] = s;
                        ++nrot;
                        d_hi = d_lo;
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
            // rotations at i = m-1, ..., m-nrot on columns (i, i+1) of each row
            for (int r = tid; r < nr; r += nt) {
                double* row = Zs + r * ld;
                double carry = row[m];
                for (int q = 0; q < nrot; ++q) {
                    const double zi = row[m - 1 - q], s = sn[q], c = cs[q];
                    row[m - q] = s * zi + c * carry;
                    carry = c * zi - s * carry;
                }
                if (nrot > 0) row[m - nrot] = carry;
            }
            __syncthreads();
        }
    }
    // ---------------- sort ascending (rank) and write E, U (row-major) ----------------
    int* rank = reinterpret_cast<int*>(cs);
    for (int i = tid; i < n; i += nt) {
        const double di = dg[i];
        int rk = 0;
        for (int j = 0; j < n; ++j) {
            const double dj = dg[j];
            rk += (dj < di) || (dj == di && j < i);
        }
        rank[i] = rk;
        if (row0 == 0) g.E[eo + rk] = di;
    }
    __syncthreads();
    double* U = g.U + mo;
    for (long e = tid; e < (long)nr * n; e += nt) {
        const int r = (int)(e / n), j = (int)(e % n);
        U[(long)(row0 + r) * n + rank[j]] = Zs[r * ld + j];
    }
}

}  // namespace

// QL work items of a block list: row slices sized to fill ~200 KB of shared
// memory per CTA, largest blocks first.  Returns the dynamic shared memory
// the QL kernel needs.
static long ql_plan(const std::vector<int>& dims, std::vector<QlItem>& items) {
    const long cap = 200L * 1024 / sizeof(double);
    std::vector<int> order(dims.size());
    for (size_t b = 0; b < dims.size(); ++b) order[b] = (int)b;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return dims[x] > dims[y]; });
    long smem_ql = 0;
    for (int b : order) {
        const long n = dims[b];
        const long rows = std::max<long>(1, std::min<long>(n, (cap - 4 * n) / (n + 1)));
        PGX_CHECK(4 * n + rows * (n + 1) <= cap, PGX_ERR_ARG, "block too large for the QL stage");
        for (long r0 = 0; r0 < n; r0 += rows) {
            const int nr = (int)std::min(rows, n - r0);
            items.push_back(QlItem{b, (int)r0, nr, 0});
            smem_ql = std::max(smem_ql, (4 * n + (long)nr * (n + 1)) * (long)sizeof(double));
        }
    }
    return smem_ql;
}

size_t eigh_ql_item_bytes(const std::vector<int>& dims) {
    std::vector<QlItem> items;
    ql_plan(dims, items);
    return items.size() * sizeof(QlItem);
}

// Both eigensolver stages on caller-provided device buffers (no allocation).
// `items_dev` must hold eigh_ql_item_bytes(dims) bytes; the function waits for
// the stream before returning because the host item list is staged from it.
void launch_eigh_raw(const EighDev& d, const std::vector<int>& dims, cudaStream_t st) {
    int dmax = 1;
    for (int x : dims) dmax = std::max(dmax, x);
    const size_t smem = 4 * sizeof(double) * (size_t)dmax;
    PGX_CHECK(smem <= 200 * 1024, PGX_ERR_ARG, "block too large for the single-CTA eigensolver (d > 6400)");
    PGX_CUDA(cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EighArgs a;
    a.order = d.order;
    a.dims = d.dims;
    a.moff = d.moff;
    a.eoff = d.eoff;
    a.H = d.H;
    a.A = d.A;
    a.Zc = d.Zc;
    a.tri = d.tri;
    eigh_kernel<<<(unsigned)dims.size(), EIGH_THREADS, smem, st>>>(a);
    check_launch("eigh_kernel");
    std::vector<QlItem> items;
    const long smem_ql = ql_plan(dims, items);
    PGX_CUDA(cudaMemcpyAsync(d.items, items.data(), items.size() * sizeof(QlItem), cudaMemcpyHostToDevice, st));
    PGX_CUDA(cudaFuncSetAttribute(ql_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_ql));
    QlArgs q;
    q.items = static_cast<const QlItem*>(d.items);
    q.dims = d.dims;
    q.moff = d.moff;
    q.eoff = d.eoff;
    q.Zc = d.Zc;
    q.tri = d.tri;
    q.U = d.U;
    q.E = d.E;
    q.status = d.status;
    ql_rows_kernel<<<(unsigned)items.size(), 128, smem_ql, st>>>(q);
    check_launch("ql_rows_kernel");
    PGX_CUDA(cudaStreamSynchronize(st));  // the host item list goes out of scope
}

void launch_eigh(Problem& P, cudaStream_t st) {
    P.tri.reserve(2 * std::max<long>(P.esize, 1) * sizeof(double));
    P.ql_items.reserve(eigh_ql_item_bytes(P.dims));
    EighDev d;
    d.order = P.d_order;
    d.dims = P.d_dims;
    d.moff = P.d_moff;
    d.eoff = P.d_eoff;
    d.H = P.d_H;
    d.A = P.d_work;
    d.Zc = P.d_work2;
    d.tri = P.tri.as<double>();
    d.items = P.ql_items.p;
    d.U = P.d_U;
    d.E = P.d_E;
    d.status = P.d_status;
    launch_eigh_raw(d, P.dims, st);
}

}  // namespace pgx
