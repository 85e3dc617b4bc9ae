// K5 Boltzmann weights, K2 operator rotation, K3 pair-Lehmann sums (G, chi, <A>).
//
// Reference counterparts:
//   weights   DensityMatrixPart.cpp:23-50, DensityMatrix.cpp:38-92, Hamiltonian.cpp:125-130
//   rotation  MonomialOperatorPart.cpp:48-111 (O' = U_L^dagger (O U_R)), FieldOperatorContainer.cpp:22-37
//   G         GreensFunctionPart.cpp:65-110 (residues, poles) and GreensFunction.hpp:123-136 (sum)
//   chi       SusceptibilityPart.cpp:76-127, SusceptibilityPart.hpp:212-220, Susceptibility.hpp:143-158
//   <A>       EnsembleAverage.cpp:27-67

#include <cfloat>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Single-CTA weights: E0 = min E, w = exp(-beta (E - E0)), Z = sum w, w /= Z.
// One CTA keeps the reduction order fixed (deterministic Z).
__global__ void __launch_bounds__(1024) weights_kernel(const double* E, double* w, long n, double beta,
                                                        double* out3) {
    __shared__ double red[32];
    __shared__ double s_e0, s_z;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double m = DBL_MAX;
    for (long i = tid; i < n; i += blockDim.x) m = fmin(m, E[i]);
    m = warp_min(m);
    if (lane == 0) red[wid] = m;
    __syncthreads();
    if (wid == 0) {
        double r = (lane < (int)(blockDim.x >> 5)) ? red[lane] : DBL_MAX;
        r = warp_min(r);
        if (lane == 0) s_e0 = r;
    }
    __syncthreads();
    const double e0 = s_e0;
    double s = 0.0;
    for (long i = tid; i < n; i += blockDim.x) {
        const double x = exp(-beta * (E[i] - e0));
        w[i] = x;
        s += x;
    }
    s = warp_sum(s);
    __syncthreads();
    if (lane == 0) red[wid] = s;
    __syncthreads();
    if (wid == 0) {
        double r = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
        r = warp_sum(r);
        if (lane == 0) s_z = r;
    }
    __syncthreads();
    const double inv = 1.0 / s_z;
    for (long i = tid; i < n; i += blockDim.x) w[i] *= inv;
    if (tid == 0) {
        out3[0] = e0;
        out3[1] = s_z;
    }
}

__global__ void retained_kernel(const double* w, const long* eoff, const int* dims, int nblocks, double tol,
                                int* flags) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    int r = 0;
    for (int i = 0; i < dims[b]; ++i) r |= (w[eoff[b] + i] > tol);
    flags[b] = r;
}

// Transposed (conjugated) copy of every part: dst_p = src_p^dagger.
template <typename T>
__global__ void adjoint_kernel(const T* src, T* dst, const long* soff, const long* doff, const int* rows,
                               const int* cols, int nparts) {
    const int p = blockIdx.y;
    if (p >= nparts) return;
    const long n = (long)rows[p] * cols[p];
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const long i = e / cols[p], j = e % cols[p];  // src (i, j) -> dst (j, i)
        T v = src[soff[p] + e];
        if constexpr (is_cd<T>::value) v = conj(v);
        dst[doff[p] + j * rows[p] + i] = v;
    }
}

// Pair-term description for G / chi: part q uses F1 (left=outer, d_o x d_i)
// and F2 (left=inner, right=outer, d_i x d_o).
struct PairPart {
    long f1, f2;       // element offsets of the two rotated matrices
    long eo, ei;       // vector offsets of outer / inner blocks
    int d_o, d_i;
    long term0;        // first term slot
    long model;        // model of the part (0 with a single model): its zero-pole slot
};

// Residues and poles.  mode 0: G (R = F1 F2 (w_o + w_i)); mode 1: chi
// (zero poles accumulate into zero[], R = A B (w_o - w_i)).
template <typename T>
__global__ void pair_terms_kernel(const PairPart* parts, int nparts, const T* m1, const T* m2, const double* E,
                                  const double* w, double coef_tol, double pole_res, int mode, cd* R, double* P,
                                  double* zero) {
    const int q = blockIdx.y;
    if (q >= nparts) return;
    const PairPart pp = parts[q];
    const long n = (long)pp.d_o * pp.d_i;
    double zx = 0.0, zy = 0.0;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int a = (int)(e / pp.d_i), b = (int)(e % pp.d_i);
        const cd ab = tocd(m1[pp.f1 + e]) * tocd(m2[pp.f2 + (long)b * pp.d_o + a]);
        const double wo = w[pp.eo + a], wi = w[pp.ei + b];
        const double pole = E[pp.ei + b] - E[pp.eo + a];
        cd r;
        if (mode == 0) {
            r = ab * (wo + wi);
        } else {
            if (fabs(pole) < pole_res) {
                zx += ab.x * wo;
                zy += ab.y * wo;
                r = cd{0.0, 0.0};
            } else {
                r = ab * (wo - wi);
            }
        }
        if (sqrt(abs2(r)) <= coef_tol) r = cd{0.0, 0.0};
        R[pp.term0 + e] = r;
        P[pp.term0 + e] = pole;
    }
    if (mode == 1) {
        zx = warp_sum(zx);
        zy = warp_sum(zy);
        if ((threadIdx.x & 31) == 0 && (zx != 0.0 || zy != 0.0)) {
            atomicAdd(zero + 2 * pp.model, zx);
            atomicAdd(zero + 2 * pp.model + 1, zy);
        }
    }
}

// out[z] += sign * sum_t R_t / (z - P_t).  CTA = (term chunk, z tile of
// blockDim): the chunks run along x, whose grid limit holds every term list.
constexpr int EVAL_THREADS = 128, EVAL_CHUNK = 1024;
__global__ void __launch_bounds__(EVAL_THREADS) pair_eval_kernel(const cd* R, const double* P, long nterms,
                                                                  const cd* z, int nz, double sign, cd* out) {
    __shared__ cd sR[EVAL_CHUNK];
    __shared__ double sP[EVAL_CHUNK];
    const long t0 = (long)blockIdx.x * EVAL_CHUNK;
    const int cnt = (int)min((long)EVAL_CHUNK, nterms - t0);
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
        sR[i] = R[t0 + i];
        sP[i] = P[t0 + i];
    }
    __syncthreads();
    const int iz = blockIdx.y * blockDim.x + threadIdx.x;
    if (iz >= nz) return;
    const cd zz = z[iz];
    double ax = 0.0, ay = 0.0;
    for (int i = 0; i < cnt; ++i) {
        const cd r = sR[i];
        if (r.x == 0.0 && r.y == 0.0) continue;
        const cd q = r * inv(cd{zz.x - sP[i], zz.y});
        ax += q.x;
        ay += q.y;
    }
    atomicAdd(&out[iz].x, sign * ax);
    atomicAdd(&out[iz].y, sign * ay);
}

// Independent models: out[m][z] += sign * sum over the terms of model m of
// R_t / (z_m - P_t).  CTA = (chunk of one model's terms, z tile): the chunks
// run along x, whose grid limit (2^31 - 1) holds every term list.
struct EvalChunk {
    long t0;
    int cnt, model;
};
__global__ void __launch_bounds__(EVAL_THREADS) pair_eval_models_kernel(const cd* R, const double* P,
                                                                         const EvalChunk* chunks, const cd* z, int nz,
                                                                         double sign, cd* out) {
    __shared__ cd sR[EVAL_CHUNK];
    __shared__ double sP[EVAL_CHUNK];
    const EvalChunk ch = chunks[blockIdx.x];
    for (int i = threadIdx.x; i < ch.cnt; i += blockDim.x) {
        sR[i] = R[ch.t0 + i];
        sP[i] = P[ch.t0 + i];
    }
    __syncthreads();
    const int iz = blockIdx.y * blockDim.x + threadIdx.x;
    if (iz >= nz) return;
    const long o = (long)ch.model * nz + iz;
    const cd zz = z[o];
    double ax = 0.0, ay = 0.0;
    for (int i = 0; i < ch.cnt; ++i) {
        const cd r = sR[i];
        if (r.x == 0.0 && r.y == 0.0) continue;
        const cd q = r * inv(cd{zz.x - sP[i], zz.y});
        ax += q.x;
        ay += q.y;
    }
    atomicAdd(&out[o].x, sign * ax);
    atomicAdd(&out[o].y, sign * ay);
}

// Weights of every model on its own states [s[m], s[m+1]) at its own beta:
// E0_m = min E, w = exp(-beta_m (E - E0_m)) / Z_m.  One CTA per model (fixed
// reduction order, as weights_kernel).
__global__ void __launch_bounds__(1024) weights_models_kernel(const double* E, double* w, const long* s,
                                                               const double* beta, double* e0z) {
    __shared__ double red[32];
    __shared__ double s_e0, s_z;
    const int m = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const long a = s[m], b = s[m + 1];
    const double bt = beta[m];
    double mn = DBL_MAX;
    for (long i = a + tid; i < b; i += blockDim.x) mn = fmin(mn, E[i]);
    mn = warp_min(mn);
    if (lane == 0) red[wid] = mn;
    __syncthreads();
    if (wid == 0) {
        double r = (lane < (int)(blockDim.x >> 5)) ? red[lane] : DBL_MAX;
        r = warp_min(r);
        if (lane == 0) s_e0 = r;
    }
    __syncthreads();
    const double e0 = s_e0;
    double sum = 0.0;
    for (long i = a + tid; i < b; i += blockDim.x) {
        const double x = exp(-bt * (E[i] - e0));
        w[i] = x;
        sum += x;
    }
    sum = warp_sum(sum);
    __syncthreads();
    if (lane == 0) red[wid] = sum;
    __syncthreads();
    if (wid == 0) {
        double r = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
        r = warp_sum(r);
        if (lane == 0) s_z = r;
    }
    __syncthreads();
    const double zs = s_z;
    for (long i = a + tid; i < b; i += blockDim.x) w[i] /= zs;
    if (tid == 0) {
        e0z[2 * m] = e0;
        e0z[2 * m + 1] = zs;
    }
}

template <typename T>
__global__ void ensemble_kernel(const T* mat, const long* offs, const long* eo, const int* dims, int nparts,
                                const double* w, double* out) {
    const int q = blockIdx.x;
    if (q >= nparts) return;
    double sx = 0.0, sy = 0.0;
    const int d = dims[q];
    for (int a = threadIdx.x; a < d; a += blockDim.x) {
        const cd v = tocd(mat[offs[q] + (long)a * d + a]) * w[eo[q] + a];
        sx += v.x;
        sy += v.y;
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, sx);
        atomicAdd(out + 1, sy);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
void launch_weights(Problem& P, double beta, cudaStream_t st) {
    double* tmp = P.status.as<double>() + 1;  // status buffer holds 4 doubles after the int slot
    weights_kernel<<<1, 1024, 0, st>>>(P.d_E, P.d_w, P.esize, beta, tmp);
    check_launch("weights_kernel");
    double h[2];
    P.w_host.resize(P.esize);
    PGX_CUDA(cudaMemcpyAsync(h, tmp, sizeof(h), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaMemcpyAsync(P.w_host.data(), P.d_w, P.esize * sizeof(double), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    P.E0 = h[0];
    P.Z = h[1];
}

void launch_retained(Problem& P, double tol, int* d_flags, cudaStream_t st) {
    retained_kernel<<<ceil_div(P.nblocks, 128), 128, 0, st>>>(P.d_w, P.d_eoff, P.d_dims, P.nblocks, tol, d_flags);
    check_launch("retained_kernel");
}

void rotate_operator(Problem& P, Operator& op, cudaStream_t st) {
    // O'(n, m) = sum_k conj(U_L[t_k, n]) * coef_k * U_R[k, m] over states k of
    // the right block with t_k >= 0: a GEMM whose reduction index gathers rows.
    const int np = (int)op.parts.size();
    const size_t esz = P.is_complex ? sizeof(cd) : sizeof(double);
    op.mat.reserve(std::max<long>(op.total, 1) * esz);
    DevBuf& probs_b = P.op_probs;
    DevBuf& tiles_b = P.op_tiles;
    tiles_b.reserve(gemm_index_bytes(op.parts.size()));
    const int* kA = op.target.as<int>();
    const int* kB = kA + op.act_off.back();
    const double* ks = op.coef.as<double>();
    if (!P.is_complex) {
        std::vector<GemmProblem<double, double, double>> probs;
        for (int q = 0; q < np; ++q) {
            const OpPart& pt = op.parts[q];
            GemmProblem<double, double, double> g{};
            g.A = P.d_U + P.moff[pt.left];
            g.B = P.d_U + P.moff[pt.right];
            g.C = op.mat.as<double>() + pt.off;
            g.M = pt.dl;
            g.N = pt.dr;
            g.K = (int)(op.act_off[q + 1] - op.act_off[q]);
            g.sa_i = 1;
            g.sa_k = pt.dl;
            g.sb_k = pt.dr;
            g.sb_j = 1;
            g.sc_i = pt.dr;
            g.sc_j = 1;
            g.a_kidx = kA + op.act_off[q];
            g.b_kidx = kB + op.act_off[q];
            g.kscale = ks + op.act_off[q];
            probs.push_back(g);
        }
        PGX_CUDA(cudaMemsetAsync(op.mat.p, 0, op.total * esz, st));
        probs_b.reserve(probs.size() * sizeof(probs[0]));
        launch_gemm_batch(probs, probs_b.p, probs_b.bytes, tiles_b.p, tiles_b.bytes, st);
    } else {
        std::vector<GemmProblem<cd, cd, cd>> probs;
        const cd* U = reinterpret_cast<const cd*>(P.d_U);
        for (int q = 0; q < np; ++q) {
            const OpPart& pt = op.parts[q];
            GemmProblem<cd, cd, cd> g{};
            g.A = U + P.moff[pt.left];
            g.B = U + P.moff[pt.right];
            g.C = op.mat.as<cd>() + pt.off;
            g.M = pt.dl;
            g.N = pt.dr;
            g.K = (int)(op.act_off[q + 1] - op.act_off[q]);
            g.sa_i = 1;
            g.sa_k = pt.dl;
            g.sb_k = pt.dr;
            g.sb_j = 1;
            g.sc_i = pt.dr;
            g.sc_j = 1;
            g.a_kidx = kA + op.act_off[q];
            g.b_kidx = kB + op.act_off[q];
            g.kscale = ks + op.act_off[q];
            g.conj_a = 1;
            probs.push_back(g);
        }
        PGX_CUDA(cudaMemsetAsync(op.mat.p, 0, op.total * esz, st));
        probs_b.reserve(probs.size() * sizeof(probs[0]));
        launch_gemm_batch(probs, probs_b.p, probs_b.bytes, tiles_b.p, tiles_b.bytes, st);
    }
    op.rotated = true;
    op.is_complex = P.is_complex;
}

void adjoint_operator(Problem& P, const Operator& src, Operator& dst, cudaStream_t st) {
    const int np = (int)src.parts.size();
    dst.parts.clear();
    long off = 0;
    for (const auto& sp : src.parts) {
        dst.parts.push_back(OpPart{sp.left, sp.right, sp.dr, sp.dl, off});
        off += (long)sp.dl * sp.dr;
    }
    dst.total = off;
    dst.by_left.assign(P.nblocks, -1);
    dst.by_right.assign(P.nblocks, -1);
    for (int q = 0; q < np; ++q) {
        dst.by_left[dst.parts[q].left] = q;
        dst.by_right[dst.parts[q].right] = q;
    }
    const size_t esz = P.is_complex ? sizeof(cd) : sizeof(double);
    dst.mat.reserve(std::max<long>(off, 1) * esz);
    std::vector<long> so(np), dof(np);
    std::vector<int> rows(np), cols(np);
    int maxe = 1;
    for (int q = 0; q < np; ++q) {
        so[q] = src.parts[q].off;
        dof[q] = dst.parts[q].off;
        rows[q] = src.parts[q].dl;
        cols[q] = src.parts[q].dr;
        maxe = std::max(maxe, rows[q] * cols[q]);
    }
    DevBuf& meta = P.op_meta;
    meta.reserve(np * (2 * sizeof(long) + 2 * sizeof(int)) + 64);
    char* m = meta.as<char>();
    h2d(m, so.data(), np * sizeof(long), st);
    h2d(m + np * sizeof(long), dof.data(), np * sizeof(long), st);
    h2d(m + 2 * np * sizeof(long), rows.data(), np * sizeof(int), st);
    h2d(m + 2 * np * sizeof(long) + np * sizeof(int), cols.data(), np * sizeof(int), st);
    if (np > 0) {
        dim3 grid(std::min(ceil_div(maxe, 256), 1024), np);
        const long* dso = reinterpret_cast<const long*>(m);
        const long* ddo = dso + np;
        const int* drows = reinterpret_cast<const int*>(ddo + np);
        const int* dcols = drows + np;
        if (P.is_complex)
            adjoint_kernel<cd><<<grid, 256, 0, st>>>(src.mat.as<cd>(), dst.mat.as<cd>(), dso, ddo, drows, dcols, np);
        else
            adjoint_kernel<double><<<grid, 256, 0, st>>>(src.mat.as<double>(), dst.mat.as<double>(), dso, ddo, drows,
                                                         dcols, np);
        check_launch("adjoint_kernel");
    }
    dst.rotated = true;
    dst.is_complex = P.is_complex;
}

// ---------------------------------------------------------------------------
static void run_pair(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                     const double* z, double pole_res, double coef_tol, int mode, double sign, double beta,
                     double* out, double* zero_out) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    PGX_CHECK(op1 >= 0 && op1 < (int)P.ops.size() && op2 >= 0 && op2 < (int)P.ops.size(), PGX_ERR_ARG,
              "bad operator id");
    const Operator& A = P.ops[op1];
    const Operator& B = P.ops[op2];
    PGX_CHECK(A.rotated && B.rotated && P.have_w, PGX_ERR_STATE, "operators must be rotated and weights computed");
    std::vector<PairPart> pp;
    long nterms = 0;
    for (int q = 0; q < nparts; ++q) {
        const int o = outer[q], i = inner[q];
        PGX_CHECK(o >= 0 && o < P.nblocks && i >= 0 && i < P.nblocks, PGX_ERR_ARG, "bad block");
        const int pa = A.by_left[o], pb = B.by_right[o];
        PGX_CHECK(pa >= 0 && pb >= 0 && A.parts[pa].right == i && B.parts[pb].left == i, PGX_ERR_ARG,
                  "blocks do not form a pair part");
        PairPart x{A.parts[pa].off, B.parts[pb].off, P.eoff[o], P.eoff[i], P.dims[o], P.dims[i], nterms, 0};
        nterms += (long)x.d_o * x.d_i;
        pp.push_back(x);
    }
    DevBuf& bR = c->scratch[0];
    DevBuf& bP = c->scratch[1];
    DevBuf& bparts = c->scratch[2];
    DevBuf& bz = c->scratch[3];
    DevBuf& bout = c->scratch[4];
    bR.reserve(std::max<long>(nterms, 1) * sizeof(cd));
    bP.reserve(std::max<long>(nterms, 1) * sizeof(double));
    bparts.reserve(std::max<size_t>(pp.size(), 1) * sizeof(PairPart));
    bz.reserve(std::max(nz, 1) * sizeof(cd));
    bout.reserve((std::max(nz, 1) + 1) * sizeof(cd));
    if (!pp.empty())
        h2d(bparts.p, pp.data(), pp.size() * sizeof(PairPart), st);
    if (nz > 0) h2d(bz.p, z, nz * sizeof(cd), st);
    PGX_CUDA(cudaMemsetAsync(bout.p, 0, (nz + 1) * sizeof(cd), st));
    cd* d_out = bout.as<cd>();
    double* d_zero = reinterpret_cast<double*>(d_out + nz);
    if (nterms > 0) {
        long maxn = 1;
        for (auto& x : pp) maxn = std::max(maxn, (long)x.d_o * x.d_i);
        dim3 g1(std::min(ceil_div(maxn, 256), 512), (unsigned)pp.size());
        if (P.is_complex)
            pair_terms_kernel<cd><<<g1, 256, 0, st>>>(bparts.as<PairPart>(), (int)pp.size(), A.mat.as<cd>(),
                                                      B.mat.as<cd>(), P.d_E, P.d_w, coef_tol, pole_res, mode,
                                                      bR.as<cd>(), bP.as<double>(), d_zero);
        else
            pair_terms_kernel<double><<<g1, 256, 0, st>>>(bparts.as<PairPart>(), (int)pp.size(), A.mat.as<double>(),
                                                          B.mat.as<double>(), P.d_E, P.d_w, coef_tol, pole_res, mode,
                                                          bR.as<cd>(), bP.as<double>(), d_zero);
        check_launch("pair_terms_kernel");
        if (nz > 0) {
            PGX_CHECK(ceil_div(nz, EVAL_THREADS) < 65536, PGX_ERR_ARG, "too many frequencies for one call");
            dim3 g2((unsigned)((nterms + EVAL_CHUNK - 1) / EVAL_CHUNK), ceil_div(nz, EVAL_THREADS));
            pair_eval_kernel<<<g2, EVAL_THREADS, 0, st>>>(bR.as<cd>(), bP.as<double>(), nterms, bz.as<cd>(), nz, sign,
                                                          d_out);
            check_launch("pair_eval_kernel");
        }
    }
    std::vector<cd> h(nz + 1);
    PGX_CUDA(cudaMemcpyAsync(h.data(), bout.p, (nz + 1) * sizeof(cd), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    const cd zero = h[nz];
    for (int k = 0; k < nz; ++k) {
        cd v = h[k];
        if (mode == 1) {
            const double az = std::sqrt(z[2 * k] * z[2 * k] + z[2 * k + 1] * z[2 * k + 1]);
            if (az <= DBL_EPSILON) v = v + zero * beta;
        }
        out[2 * k] = v.x;
        out[2 * k + 1] = v.y;
    }
    if (zero_out) {
        zero_out[0] = zero.x;
        zero_out[1] = zero.y;
    }
}

// ---------------------------------------------------------------------------
// Independent models in one context.
void set_models(Problem& P, int nmodels, const int32_t* first, const double* beta) {
    PGX_CHECK(P.nblocks > 0, PGX_ERR_STATE, "pgx_set_blocks first");
    PGX_CHECK(nmodels >= 1 && first && beta, PGX_ERR_ARG, "bad model description");
    PGX_CHECK(first[0] == 0 && first[nmodels] == P.nblocks, PGX_ERR_ARG, "models must cover the blocks in order");
    for (int m = 0; m < nmodels; ++m) {
        PGX_CHECK(first[m + 1] > first[m], PGX_ERR_ARG, "every model needs at least one block");
        PGX_CHECK(beta[m] > 0.0, PGX_ERR_ARG, "beta must be positive");
    }
    P.nmodels = nmodels;
    P.model_first.assign(first, first + nmodels + 1);
    P.model_beta.assign(beta, beta + nmodels);
    P.block_model.assign(P.nblocks, 0);
    for (int m = 0; m < nmodels; ++m)
        for (int b = first[m]; b < first[m + 1]; ++b) P.block_model[b] = m;
    P.have_w = false;
}

void launch_weights_models(Problem& P, cudaStream_t st) {
    PGX_CHECK(P.nmodels > 0, PGX_ERR_STATE, "pgx_set_models first");
    const int nm = P.nmodels;
    std::vector<long> s(nm + 1);
    for (int m = 0; m <= nm; ++m) s[m] = (P.model_first[m] < P.nblocks) ? P.eoff[P.model_first[m]] : P.esize;
    const size_t b_s = ((nm + 1) * sizeof(long) + 255) & ~size_t(255), b_b = (nm * sizeof(double) + 255) & ~size_t(255);
    P.model_buf.reserve(b_s + b_b + 2 * nm * sizeof(double));
    char* base = P.model_buf.as<char>();
    long* d_s = reinterpret_cast<long*>(base);
    double* d_beta = reinterpret_cast<double*>(base + b_s);
    double* d_e0z = reinterpret_cast<double*>(base + b_s + b_b);
    h2d(d_s, s.data(), (nm + 1) * sizeof(long), st);
    h2d(d_beta, P.model_beta.data(), nm * sizeof(double), st);
    {
        ProfRange pr("weights_models_kernel", st, 0.0, 24.0 * P.esize);
        weights_models_kernel<<<nm, 1024, 0, st>>>(P.d_E, P.d_w, d_s, d_beta, d_e0z);
        check_launch("weights_models_kernel");
    }
    std::vector<double> h(2 * nm);
    P.w_host.resize(P.esize);
    PGX_CUDA(cudaMemcpyAsync(h.data(), d_e0z, 2 * nm * sizeof(double), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaMemcpyAsync(P.w_host.data(), P.d_w, P.esize * sizeof(double), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    P.model_E0.resize(nm);
    P.model_Z.resize(nm);
    for (int m = 0; m < nm; ++m) {
        P.model_E0[m] = h[2 * m];
        P.model_Z[m] = h[2 * m + 1];
    }
}

// The pair sums of run_pair for every model at once: each part belongs to the
// model of its outer block; z and out are nmodels x nz (model-major), each
// model summed over its own parts at its own frequencies.
static void run_pair_models(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner,
                            int nz, const double* z, double pole_res, double coef_tol, int mode, double sign,
                            double* out, double* zero_out) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    PGX_CHECK(P.nmodels > 0 && P.w_models && P.have_w, PGX_ERR_STATE, "pgx_set_models and pgx_weights_models first");
    PGX_CHECK(op1 >= 0 && op1 < (int)P.ops.size() && op2 >= 0 && op2 < (int)P.ops.size(), PGX_ERR_ARG,
              "bad operator id");
    const Operator& A = P.ops[op1];
    const Operator& B = P.ops[op2];
    PGX_CHECK(A.rotated && B.rotated, PGX_ERR_STATE, "operators must be rotated");
    const int nm = P.nmodels;
    // parts grouped by model, their terms contiguous
    std::vector<int> order(nparts);
    for (int q = 0; q < nparts; ++q) {
        PGX_CHECK(outer[q] >= 0 && outer[q] < P.nblocks && inner[q] >= 0 && inner[q] < P.nblocks, PGX_ERR_ARG,
                  "bad block");
        PGX_CHECK(P.block_model[outer[q]] == P.block_model[inner[q]], PGX_ERR_ARG, "a part joins two models");
        order[q] = q;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return P.block_model[outer[x]] < P.block_model[outer[y]]; });
    std::vector<PairPart> pp;
    std::vector<EvalChunk> chunks;
    long nterms = 0;
    for (int q : order) {
        const int o = outer[q], i = inner[q];
        const int pa = A.by_left[o], pb = B.by_right[o];
        PGX_CHECK(pa >= 0 && pb >= 0 && A.parts[pa].right == i && B.parts[pb].left == i, PGX_ERR_ARG,
                  "blocks do not form a pair part");
        const long m = P.block_model[o];
        PairPart x{A.parts[pa].off, B.parts[pb].off, P.eoff[o], P.eoff[i], P.dims[o], P.dims[i], nterms, m};
        const long n = (long)x.d_o * x.d_i;
        for (long t = 0; t < n; t += EVAL_CHUNK)  // chunks never straddle two parts, so never two models
            chunks.push_back(EvalChunk{nterms + t, (int)std::min<long>(EVAL_CHUNK, n - t), (int)m});
        nterms += n;
        pp.push_back(x);
    }
    PGX_CHECK(chunks.size() < (1u << 31) && ceil_div(nz, EVAL_THREADS) < 65536, PGX_ERR_ARG,
              "too many Lehmann terms or frequencies for one call");
    DevBuf& bR = c->scratch[0];
    DevBuf& bP = c->scratch[1];
    DevBuf& bparts = c->scratch[2];
    DevBuf& bz = c->scratch[3];
    DevBuf& bout = c->scratch[4];
    DevBuf& bch = c->scratch[5];
    const long nzt = (long)nm * nz;
    bR.reserve(std::max<long>(nterms, 1) * sizeof(cd));
    bP.reserve(std::max<long>(nterms, 1) * sizeof(double));
    bparts.reserve(std::max<size_t>(pp.size(), 1) * sizeof(PairPart));
    bch.reserve(std::max<size_t>(chunks.size(), 1) * sizeof(EvalChunk));
    bz.reserve(std::max<long>(nzt, 1) * sizeof(cd));
    bout.reserve((std::max<long>(nzt, 1) + nm) * sizeof(cd));
    if (!pp.empty()) {
        h2d(bparts.p, pp.data(), pp.size() * sizeof(PairPart), st);
        h2d(bch.p, chunks.data(), chunks.size() * sizeof(EvalChunk), st);
    }
    if (nzt > 0) h2d(bz.p, z, nzt * sizeof(cd), st);
    PGX_CUDA(cudaMemsetAsync(bout.p, 0, (nzt + nm) * sizeof(cd), st));
    cd* d_out = bout.as<cd>();
    double* d_zero = reinterpret_cast<double*>(d_out + nzt);
    if (nterms > 0) {
        long maxn = 1;
        for (auto& x : pp) maxn = std::max(maxn, (long)x.d_o * x.d_i);
        dim3 g1(std::min(ceil_div(maxn, 256), 512), (unsigned)pp.size());
        {
            ProfRange pr("pair_terms_kernel", st, 0.0, 40.0 * nterms);
            if (P.is_complex)
                pair_terms_kernel<cd><<<g1, 256, 0, st>>>(bparts.as<PairPart>(), (int)pp.size(), A.mat.as<cd>(),
                                                          B.mat.as<cd>(), P.d_E, P.d_w, coef_tol, pole_res, mode,
                                                          bR.as<cd>(), bP.as<double>(), d_zero);
            else
                pair_terms_kernel<double><<<g1, 256, 0, st>>>(bparts.as<PairPart>(), (int)pp.size(),
                                                              A.mat.as<double>(), B.mat.as<double>(), P.d_E, P.d_w,
                                                              coef_tol, pole_res, mode, bR.as<cd>(), bP.as<double>(),
                                                              d_zero);
            check_launch("pair_terms_kernel");
        }
        if (nz > 0) {
            dim3 g2((unsigned)chunks.size(), ceil_div(nz, EVAL_THREADS));
            ProfRange pr("pair_eval_models_kernel", st, 12.0 * (double)nterms * nz, 24.0 * nterms);
            pair_eval_models_kernel<<<g2, EVAL_THREADS, 0, st>>>(bR.as<cd>(), bP.as<double>(), bch.as<EvalChunk>(),
                                                                 bz.as<cd>(), nz, sign, d_out);
            check_launch("pair_eval_models_kernel");
        }
    }
    std::vector<cd> h(nzt + nm);
    PGX_CUDA(cudaMemcpyAsync(h.data(), bout.p, (nzt + nm) * sizeof(cd), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    for (int m = 0; m < nm; ++m) {
        const cd zero = h[nzt + m];
        for (int k = 0; k < nz; ++k) {
            const long o = (long)m * nz + k;
            cd v = h[o];
            if (mode == 1) {
                const double az = std::sqrt(z[2 * o] * z[2 * o] + z[2 * o + 1] * z[2 * o + 1]);
                if (az <= DBL_EPSILON) v = v + zero * P.model_beta[m];
            }
            out[2 * o] = v.x;
            out[2 * o + 1] = v.y;
        }
        if (zero_out) {
            zero_out[2 * m] = zero.x;
            zero_out[2 * m + 1] = zero.y;
        }
    }
}

void run_gf_models(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                   const double* z, double coef_tol, double* out) {
    run_pair_models(c, op1, op2, nparts, outer, inner, nz, z, 0.0, coef_tol, 0, 1.0, out, nullptr);
}

void run_susc_models(pgx_ctx* c, int opA, int opB, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                     const double* z, double pole_res, double coef_tol, double* out, double* zero_pole) {
    run_pair_models(c, opA, opB, nparts, outer, inner, nz, z, pole_res, coef_tol, 1, -1.0, out, zero_pole);
}

void run_gf(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner, int nz,
            const double* z, double coef_tol, double* out) {
    run_pair(c, op1, op2, nparts, outer, inner, nz, z, 0.0, coef_tol, 0, 1.0, 0.0, out, nullptr);
}

void run_susc(pgx_ctx* c, int opA, int opB, int nparts, const int32_t* outer, const int32_t* inner, int nz,
              const double* z, double pole_res, double coef_tol, double beta, double* out, double* zero_pole) {
    run_pair(c, opA, opB, nparts, outer, inner, nz, z, pole_res, coef_tol, 1, -1.0, beta, out, zero_pole);
}

void run_ensemble_average(pgx_ctx* c, int op, double* out) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    PGX_CHECK(op >= 0 && op < (int)P.ops.size(), PGX_ERR_ARG, "bad operator id");
    const Operator& A = P.ops[op];
    PGX_CHECK(A.rotated && P.have_w, PGX_ERR_STATE, "operator must be rotated and weights computed");
    std::vector<long> offs, eo;
    std::vector<int> dims;
    for (const auto& pt : A.parts) {
        if (pt.left != pt.right) continue;
        if (!P.retained.empty() && !P.retained[pt.left]) continue;
        offs.push_back(pt.off);
        eo.push_back(P.eoff[pt.left]);
        dims.push_back(pt.dl);
    }
    const int n = (int)offs.size();
    DevBuf& meta = c->scratch[5];
    meta.reserve(n * (2 * sizeof(long) + sizeof(int)) + 2 * sizeof(double) + 64);
    char* m = meta.as<char>();
    double* d_out = reinterpret_cast<double*>(m);
    long* d_offs = reinterpret_cast<long*>(m + 16);
    long* d_eo = d_offs + n;
    int* d_dims = reinterpret_cast<int*>(d_eo + n);
    PGX_CUDA(cudaMemsetAsync(d_out, 0, 2 * sizeof(double), st));
    if (n > 0) {
        h2d(d_offs, offs.data(), n * sizeof(long), st);
        h2d(d_eo, eo.data(), n * sizeof(long), st);
        h2d(d_dims, dims.data(), n * sizeof(int), st);
        if (P.is_complex)
            ensemble_kernel<cd><<<n, 128, 0, st>>>(A.mat.as<cd>(), d_offs, d_eo, d_dims, n, P.d_w, d_out);
        else
            ensemble_kernel<double><<<n, 128, 0, st>>>(A.mat.as<double>(), d_offs, d_eo, d_dims, n, P.d_w, d_out);
        check_launch("ensemble_kernel");
    }
    PGX_CUDA(cudaMemcpyAsync(out, d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
}

}  // namespace pgx
