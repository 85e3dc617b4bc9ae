// Reverse-mode derivative of a single-particle Green's function (pgx_gf_vjp)
// or a susceptibility (pgx_susc_vjp) through the exact-diagonalisation chain.
// The reference computes no derivatives; this follows the forward path of
// pgx_gf backwards (for chi the residue is -(w_a - w_b) A B, and a zero-pole
// pair adds beta A B w_a at z = 0, see pair_vjp_kernel):
//
//   G(z_n) = sum_{parts} sum_{a in o, b in i} A_ab B_ba (w_a + w_b) R_ab(n),
//   R_ab(n) = 1 / (z_n - (E_b - E_a)),  A = U_o^T C1 U_i,  B = U_i^T C2 U_o,
//   w_s = exp(-beta E_s) / sum_t exp(-beta E_t),  H_b = U_b diag(E_b) U_b^T.
//
// With dL = Re sum_n lambda_n dG(z_n), P_ab = sum_n lambda_n R_ab(n) and
// Q_ab = sum_n lambda_n R_ab(n)^2:
//   dL/dA_ab = B_ba (w_a + w_b) Re P_ab,   dL/dB_ba = A_ab (w_a + w_b) Re P_ab,
//   dL/dw_a, dL/dw_b += A_ab B_ba Re P_ab,
//   dL/dE_b += A_ab B_ba (w_a + w_b) Re Q_ab = -dL/dE_a (same pair),
//   dL/dE_t += -beta w_t (dL/dw_t - sum_s w_s dL/dw_s)      (normalised weights),
// the rotated operators O' = U_L^T O U_R with O|k> = c_k |t_k> give
//   dL/dU_L[t_k, :] += c_k (U_R O'bar^T)[k, :],  dL/dU_R[k, :] += c_k (U_L O'bar)[t_k, :],
// and the symmetric eigendecomposition gives (Giles, "Collected matrix
// derivative results for forward and reverse mode algorithmic
// differentiation", 2008, sec. 3.1)
//   Hbar = U (diag(Ebar) + F o (U^T Ubar)) U^T,  F_ij = 1 / (E_j - E_i), i != j,
// symmetrised; F is set to zero between eigenvalues closer than 1e-10 max|E|
// (G does not depend on the basis inside a degenerate subspace, so those
// terms cancel).  Finally dL/dc_t = sum over columns j of the terms' Fock
// action sign * Hbar_sym[o][j], the transpose of the Hamiltonian assembly.

#include <cfloat>
#include <cmath>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

struct VjpPart {
    long f1, f2;  // element offsets of the rotated parts of op1 (o -> rows) and op2
    long eo, ei;  // vector offsets of outer / inner blocks
    int d_o, d_i;
};

// one thread per (a, b) element of a pair part; real operators.  mode 0: G,
// residue (w_a + w_b) A B.  mode 1: chi, residue -(w_a - w_b) A B away from
// the zero pole; a pair with |pole| < pole_res adds beta A B w_a at z = 0
// only (zre = Re of the sum of lambda over the zero frequencies), as the
// forward sum does.
__global__ void pair_vjp_kernel(const VjpPart* parts, const double* m1, const double* m2, const double* E,
                                const double* w, const cd* z, const cd* lam, int nz, double* g1, double* g2,
                                double* wbar, double* Ebar, int mode, double pole_res, double beta, double zre) {
    const VjpPart pp = parts[blockIdx.y];
    const long n = (long)pp.d_o * pp.d_i;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int a = (int)(e / pp.d_i), b = (int)(e % pp.d_i);
        const double A = m1[pp.f1 + e], B = m2[pp.f2 + (long)b * pp.d_o + a];
        if (A == 0.0 && B == 0.0) continue;
        const double wo = w[pp.eo + a], wi = w[pp.ei + b];
        const double pole = E[pp.ei + b] - E[pp.eo + a];
        if (mode == 1 && fabs(pole) < pole_res) {
            const double f = beta * zre;
            if (f != 0.0) {
                atomicAdd(&g1[pp.f1 + e], B * wo * f);
                atomicAdd(&g2[pp.f2 + (long)b * pp.d_o + a], A * wo * f);
                if (A * B != 0.0) atomicAdd(&wbar[pp.eo + a], A * B * f);
            }
            continue;
        }
        const double s = mode ? -(wo - wi) : wo + wi;
        double Px = 0.0, Qx = 0.0;
        for (int t = 0; t < nz; ++t) {
            const cd R = inv(cd{z[t].x - pole, z[t].y});
            const cd lr = lam[t] * R;
            Px += lr.x;
            Qx += (lr * R).x;
        }
        atomicAdd(&g1[pp.f1 + e], B * s * Px);
        atomicAdd(&g2[pp.f2 + (long)b * pp.d_o + a], A * s * Px);
        const double ab = A * B;
        if (ab != 0.0) {
            atomicAdd(&wbar[pp.eo + a], mode ? -ab * Px : ab * Px);  // d s / d w_a = 1 (G) or -1 (chi)
            atomicAdd(&wbar[pp.ei + b], ab * Px);
            const double de = ab * s * Qx;
            atomicAdd(&Ebar[pp.ei + b], de);
            atomicAdd(&Ebar[pp.eo + a], -de);
        }
    }
}

// Ebar_t += -beta w_t (wbar_t - sum_s w_s wbar_s), and emax = max(1, max_s |E_s|)
// (the scale of the degeneracy test); one CTA
__global__ void weight_vjp_kernel(const double* w, const double* wbar, const double* E, double* Ebar, long n,
                                  double beta, double* emax) {
    __shared__ double red[32], redm[32];
    double part = 0.0, m = 1.0;
    for (long s = threadIdx.x; s < n; s += blockDim.x) {
        part += w[s] * wbar[s];
        m = fmax(m, fabs(E[s]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        part += __shfl_xor_sync(0xffffffffu, part, o);
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = part;
        redm[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    double S = 0.0, M = 1.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
        S += red[k];
        M = fmax(M, redm[k]);
    }
    if (threadIdx.x == 0) *emax = M;
    for (long t = threadIdx.x; t < n; t += blockDim.x) Ebar[t] += -beta * w[t] * (wbar[t] - S);
}

// gradient of an adjoint operator's parts added, transposed, to its source's
struct TransPart {
    long off_adj, off_src;
    int dl, dr;  // of the adjoint part
};
__global__ void transpose_add_kernel(const TransPart* parts, const double* gadj, double* gsrc) {
    const TransPart p = parts[blockIdx.y];
    const long n = (long)p.dl * p.dr;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e / p.dr), j = (int)(e % p.dr);
        gsrc[p.off_src + (long)j * p.dl + i] += gadj[p.off_adj + e];
    }
}

// dL/dU from the gradient of a rotated operator's parts, through its Fock
// action (entries act[q]..act[q+1] of part q: target t, source k, coefficient)
struct ScatPart {
    long a0, a1;           // Fock-action entries of the part
    long m1, m2;           // offsets of U_R Obar^T (dr x dl) and U_L Obar (dl x dr) in the workspace
    long uL, uR;           // matrix offsets of the left / right blocks
    int dl, dr;
};
__global__ void uscatter_kernel(const ScatPart* parts, const int* tgt, const int* src, const double* coef,
                                const double* W, double* Ubar) {
    const ScatPart p = parts[blockIdx.y];
    const long ne = p.a1 - p.a0;
    const int w = max(p.dl, p.dr);
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < ne * w; x += (long)gridDim.x * blockDim.x) {
        const long e = p.a0 + x / w;
        const int col = (int)(x % w);
        const int t = tgt[e], k = src[e];
        const double c = coef[e];
        if (col < p.dl) atomicAdd(&Ubar[p.uL + (long)t * p.dl + col], c * W[p.m1 + (long)k * p.dl + col]);
        if (col < p.dr) atomicAdd(&Ubar[p.uR + (long)k * p.dr + col], c * W[p.m2 + (long)t * p.dr + col]);
    }
}

// X = F o W + diag(Ebar) on every block, F_ij = 1/(E_j - E_i) unless
// |E_j - E_i| <= rel * emax
__global__ void eig_adjoint_kernel(const int* dims, const long* moff, const long* eoff, const double* E,
                                   const double* Ebar, const double* W, double* X, double rel, const double* emax) {
    const int b = blockIdx.y, d = dims[b];
    const double tol = rel * *emax;
    const long mo = moff[b], eo = eoff[b];
    const long n = (long)d * d;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e / d), j = (int)(e % d);
        double v;
        if (i == j) {
            v = Ebar[eo + i];
        } else {
            const double gap = E[eo + j] - E[eo + i];
            v = (fabs(gap) > tol) ? W[mo + e] / gap : 0.0;
        }
        X[mo + e] = v;
    }
}

// dL/dc_t = sum over block columns j of sign * (Hbar[o][j] + Hbar[j][o]) / 2,
// with O_t |s_j> = sign |o> (the Fock action of pgx_assemble_hamiltonian)
__global__ void term_grad_kernel(const int* ops, int nterms, const uint64_t* fock, long nstates, const int* sb,
                                 const int* si, const int* dims, const long* moff, const double* Hbar, double* dterm) {
    const long col = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (col >= nstates) return;
    const uint64_t s0 = fock[col];
    const int b = sb[s0], j = si[s0];
    const long d = dims[b];
    const double* Hb = Hbar + moff[b];
    for (int t = 0; t < nterms; ++t) {
        const int* op = ops + t * PGX_TERM_OPS;
        uint64_t s = s0;
        double sign = 1.0;
        bool ok = true;
        for (int k = PGX_TERM_OPS - 1; k >= 0 && ok; --k) {
            const int o = op[k];
            if (o < 0) continue;
            const uint64_t mask = 1ull << (o >> 1);
            const bool occ = (s & mask) != 0;
            if ((o & 1) == (int)occ) {
                ok = false;
                break;
            }
            if (__popcll(s & (mask - 1)) & 1) sign = -sign;
            s ^= mask;
        }
        if (!ok || sb[s] != b) continue;
        const long i = si[s];
        atomicAdd(&dterm[t], sign * 0.5 * (Hb[i * d + j] + Hb[(long)j * d + i]));
    }
}

}  // namespace

static void run_pair_vjp(pgx_ctx* c, int mode, int op1, int op2, int nparts, const int32_t* outer,
                         const int32_t* inner, int nz, const double* z, double pole_res, const double* lambda,
                         double* dterm, double* dE) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    PGX_CHECK(!P.is_complex, PGX_ERR_ARG, "pgx_gf_vjp: real Hamiltonians only");
    PGX_CHECK(P.have_asm && P.have_H, PGX_ERR_STATE, "pgx_gf_vjp needs a Hamiltonian from pgx_assemble_hamiltonian");
    PGX_CHECK(op1 >= 0 && op1 < (int)P.ops.size() && op2 >= 0 && op2 < (int)P.ops.size(), PGX_ERR_ARG,
              "bad operator id");
    const Operator& A = P.ops[op1];
    const Operator& B = P.ops[op2];
    PGX_CHECK(A.rotated && B.rotated && P.have_w && P.have_eig, PGX_ERR_STATE,
              "operators must be rotated and weights computed");
    // operator whose Fock action defines op (itself, or the source of an adjoint)
    auto root_of = [&](int op) {
        const Operator& o = P.ops[op];
        if (!o.act_off.empty()) return op;
        PGX_CHECK(o.adj_src >= 0 && o.adj_src < (int)P.ops.size() && !P.ops[o.adj_src].act_off.empty() &&
                      P.ops[o.adj_src].rotated,
                  PGX_ERR_ARG, "pgx_gf_vjp: operators must be defined by a Fock action or be adjoints of such");
        return o.adj_src;
    };
    PGX_CHECK(P.nblocks < 65536 && nparts >= 0 && nparts < 65536 && nz >= 0 && (nz == 0 || (z && lambda)) && dterm,
              PGX_ERR_ARG, "pgx_gf_vjp: bad arguments");
    const int r1 = root_of(op1), r2 = root_of(op2);
    std::vector<int> roots{r1};
    if (r2 != r1) roots.push_back(r2);
    std::vector<VjpPart> pp;
    for (int q = 0; q < nparts; ++q) {
        const int o = outer[q], i = inner[q];
        PGX_CHECK(o >= 0 && o < P.nblocks && i >= 0 && i < P.nblocks, PGX_ERR_ARG, "bad block");
        const int pa = A.by_left[o], pb = B.by_right[o];
        PGX_CHECK(pa >= 0 && pb >= 0 && A.parts[pa].right == i && B.parts[pb].left == i, PGX_ERR_ARG,
                  "blocks do not form a pair part");
        pp.push_back(VjpPart{A.parts[pa].off, B.parts[pb].off, P.eoff[o], P.eoff[i], P.dims[o], P.dims[i]});
    }
    // workspace (doubles): g1 | g2 | groot[0..1] | M1M2 | Ebar | wbar | Ubar | W | X | T
    long o_g1 = 0, o_g2 = o_g1 + std::max<long>(A.total, 1), o_gr = o_g2 + std::max<long>(B.total, 1);
    std::vector<long> o_groot;
    long o = o_gr;
    long mm = 1;
    for (int r : roots) {
        o_groot.push_back(o);
        o += std::max<long>(P.ops[r].total, 1);
        mm = std::max(mm, 2 * P.ops[r].total);
    }
    const long o_mm = o, o_Eb = o_mm + mm, o_wb = o_Eb + P.esize, o_Ub = o_wb + P.esize, o_W = o_Ub + P.msize,
               o_X = o_W + P.msize, o_T = o_X + P.msize, o_em = o_T + P.msize, total = o_em + 1;
    P.vjp_buf.reserve(total * sizeof(double));
    double* ws = P.vjp_buf.as<double>();
    PGX_CUDA(cudaMemsetAsync(ws, 0, total * sizeof(double), st));
    double *g1 = ws + o_g1, *g2 = ws + o_g2, *Eb = ws + o_Eb, *wb = ws + o_wb, *Ub = ws + o_Ub, *W = ws + o_W,
           *X = ws + o_X, *T = ws + o_T, *MM = ws + o_mm;
    // ---- Lehmann sum
    DevBuf& meta = c->scratch[2];
    const size_t b_parts = std::max<size_t>(pp.size(), 1) * sizeof(VjpPart);
    const size_t b_z = (size_t)std::max(nz, 1) * sizeof(cd);
    meta.reserve(((b_parts + 255) & ~size_t(255)) + 2 * ((b_z + 255) & ~size_t(255)));
    VjpPart* d_pp = meta.as<VjpPart>();
    cd* d_z = reinterpret_cast<cd*>(meta.as<char>() + ((b_parts + 255) & ~size_t(255)));
    cd* d_lam = reinterpret_cast<cd*>(reinterpret_cast<char*>(d_z) + ((b_z + 255) & ~size_t(255)));
    if (!pp.empty() && nz > 0) {
        h2d(d_pp, pp.data(), pp.size() * sizeof(VjpPart), st);
        h2d(d_z, z, nz * sizeof(cd), st);
        h2d(d_lam, lambda, nz * sizeof(cd), st);
        long maxn = 1;
        double nel = 0.0;
        for (auto& x : pp) {
            maxn = std::max(maxn, (long)x.d_o * x.d_i);
            nel += (double)x.d_o * x.d_i;
        }
        dim3 g(std::min(ceil_div(maxn, 256), 256), (unsigned)pp.size());
        // per (a, b, z): complex reciprocal (8), lambda R (6), lambda R^2 (6) and two sums
        ProfRange pr("pair_vjp_kernel", st, 22.0 * nel * nz, 56.0 * nel);
        // chi's zero-pole terms act at z = 0 only (the same test as the forward sum)
        double zre = 0.0;
        for (int t = 0; t < nz; ++t)
            if (std::sqrt(z[2 * t] * z[2 * t] + z[2 * t + 1] * z[2 * t + 1]) <= DBL_EPSILON) zre += lambda[2 * t];
        pair_vjp_kernel<<<g, 256, 0, st>>>(d_pp, A.mat.as<double>(), B.mat.as<double>(), P.d_E, P.d_w, d_z, d_lam, nz,
                                           g1, g2, wb, Eb, mode, pole_res, P.beta, zre);
        check_launch("pair_vjp_kernel");
    }
    {
        ProfRange pr("weight_vjp_kernel", st, 0.0, 40.0 * P.esize);
        weight_vjp_kernel<<<1, 1024, 0, st>>>(P.d_w, wb, P.d_E, Eb, P.esize, P.beta, ws + o_em);
        check_launch("weight_vjp_kernel");
    }
    // ---- operator parts -> gradient of their defining operator
    auto add_to_root = [&](int op, const double* g, int slot) {
        const Operator& x = P.ops[op];
        const int r = root_of(op);
        double* gr = ws + o_groot[r == r1 ? 0 : 1];
        const Operator& s = P.ops[r];
        // the same operator: identity map; an adjoint: part q of op is the transpose of part q of r
        std::vector<TransPart> tp;
        long maxe = 1;
        for (size_t q = 0; q < x.parts.size(); ++q) {
            const OpPart& a = x.parts[q];
            if (r == op)
                tp.push_back(TransPart{a.off, a.off, 1, a.dl * a.dr});
            else
                tp.push_back(TransPart{a.off, s.parts[q].off, a.dl, a.dr});
            maxe = std::max(maxe, (long)a.dl * a.dr);
        }
        if (tp.empty()) return;
        DevBuf& tb = c->scratch[slot];
        tb.reserve(tp.size() * sizeof(TransPart));
        h2d(tb.p, tp.data(), tp.size() * sizeof(TransPart), st);
        dim3 gg(std::min(ceil_div(maxe, 256), 256), (unsigned)tp.size());
        ProfRange pr("transpose_add_kernel", st, 0.0, 24.0 * x.total);
        transpose_add_kernel<<<gg, 256, 0, st>>>(tb.as<TransPart>(), g, gr);
        check_launch("transpose_add_kernel");
    };
    add_to_root(op1, g1, 5);
    add_to_root(op2, g2, 6);
    // ---- rotated-operator gradients -> dL/dU
    for (size_t ri = 0; ri < roots.size(); ++ri) {
        const Operator& x = P.ops[roots[ri]];
        const double* gx = ws + o_groot[ri];
        std::vector<GemmProblem<double, double, double>> probs;
        std::vector<ScatPart> sp;
        long m = 0, maxw = 1;
        for (size_t q = 0; q < x.parts.size(); ++q) {
            const OpPart& pt = x.parts[q];
            const int dl = pt.dl, dr = pt.dr;
            const double* UL = P.d_U + P.moff[pt.left];
            const double* UR = P.d_U + P.moff[pt.right];
            const double* Ob = gx + pt.off;
            GemmProblem<double, double, double> g1p{};  // M1 = U_R Obar^T (dr x dl)
            g1p.A = UR;
            g1p.B = Ob;
            g1p.C = MM + m;
            g1p.M = dr;
            g1p.N = dl;
            g1p.K = dr;
            g1p.sa_i = dr;
            g1p.sa_k = 1;
            g1p.sb_k = 1;
            g1p.sb_j = dr;
            g1p.sc_i = dl;
            g1p.sc_j = 1;
            probs.push_back(g1p);
            GemmProblem<double, double, double> g2p{};  // M2 = U_L Obar (dl x dr)
            g2p.A = UL;
            g2p.B = Ob;
            g2p.C = MM + m + (long)dr * dl;
            g2p.M = dl;
            g2p.N = dr;
            g2p.K = dl;
            g2p.sa_i = dl;
            g2p.sa_k = 1;
            g2p.sb_k = dr;
            g2p.sb_j = 1;
            g2p.sc_i = dr;
            g2p.sc_j = 1;
            probs.push_back(g2p);
            sp.push_back(ScatPart{x.act_off[q], x.act_off[q + 1], m, m + (long)dr * dl, P.moff[pt.left],
                                  P.moff[pt.right], dl, dr});
            maxw = std::max(maxw, (x.act_off[q + 1] - x.act_off[q]) * std::max(dl, dr));
            m += 2L * dr * dl;
        }
        if (probs.empty()) continue;
        c->scratch[7].reserve(probs.size() * sizeof(probs[0]));
        c->scratch[8].reserve(gemm_index_bytes(probs.size()));
        launch_gemm_batch(probs, c->scratch[7].p, c->scratch[7].bytes, c->scratch[8].p, c->scratch[8].bytes, st);
        DevBuf& sb = c->scratch[9 + (int)ri];
        sb.reserve(sp.size() * sizeof(ScatPart));
        h2d(sb.p, sp.data(), sp.size() * sizeof(ScatPart), st);
        const int* kA = x.target.as<int>();
        const int* kB = kA + x.act_off.back();
        dim3 gg(std::min(ceil_div(maxw, 256), 1024), (unsigned)sp.size());
        // per Fock-action entry and column: two products read, two gradient rows updated
        double nel = 0.0;
        for (const auto& q : sp) nel += (double)(q.a1 - q.a0) * (q.dl + q.dr);
        ProfRange pr("uscatter_kernel", st, 2.0 * nel, 24.0 * nel);
        uscatter_kernel<<<gg, 256, 0, st>>>(sb.as<ScatPart>(), kA, kB, x.coef.as<double>(), MM, Ub);
        check_launch("uscatter_kernel");
    }
    // ---- eigendecomposition adjoint: W = U^T Ubar, X = F o W + diag(Ebar), Hbar = U X U^T
    {
        std::vector<GemmProblem<double, double, double>> pw, pt, ph;
        for (int b = 0; b < P.nblocks; ++b) {
            const int d = P.dims[b];
            const long mo = P.moff[b];
            GemmProblem<double, double, double> g{};
            g.M = g.N = g.K = d;
            g.sc_i = d;
            g.sc_j = 1;
            g.A = P.d_U + mo;  // U^T
            g.sa_i = 1;
            g.sa_k = d;
            g.B = Ub + mo;
            g.sb_k = d;
            g.sb_j = 1;
            g.C = W + mo;
            pw.push_back(g);
            g.A = P.d_U + mo;  // U X
            g.sa_i = d;
            g.sa_k = 1;
            g.B = X + mo;
            g.C = T + mo;
            pt.push_back(g);
            g.A = T + mo;  // (U X) U^T
            g.B = P.d_U + mo;
            g.sb_k = 1;
            g.sb_j = d;
            g.C = W + mo;  // W is free again: Hbar
            ph.push_back(g);
        }
        c->scratch[7].reserve(pw.size() * sizeof(pw[0]));
        c->scratch[8].reserve(gemm_index_bytes(pw.size()));
        launch_gemm_batch(pw, c->scratch[7].p, c->scratch[7].bytes, c->scratch[8].p, c->scratch[8].bytes, st);
        int dmax = 1;
        for (int d : P.dims) dmax = std::max(dmax, d);
        dim3 gg(std::min(ceil_div((long)dmax * dmax, 256), 1024), (unsigned)P.nblocks);
        {
            ProfRange pr("eig_adjoint_kernel", st, 0.0, 24.0 * P.msize);
            eig_adjoint_kernel<<<gg, 256, 0, st>>>(P.d_dims, P.d_moff, P.d_eoff, P.d_E, Eb, W, X, 1e-10, ws + o_em);
            check_launch("eig_adjoint_kernel");
        }
        launch_gemm_batch(pt, c->scratch[7].p, c->scratch[7].bytes, c->scratch[8].p, c->scratch[8].bytes, st);
        launch_gemm_batch(ph, c->scratch[7].p, c->scratch[7].bytes, c->scratch[8].p, c->scratch[8].bytes, st);
    }
    // ---- term gradients
    DevBuf& db = c->scratch[11];
    db.reserve(std::max(P.asm_nterms, 1) * sizeof(double));
    PGX_CUDA(cudaMemsetAsync(db.p, 0, std::max(P.asm_nterms, 1) * sizeof(double), st));
    if (P.asm_nterms > 0) {
        {
            ProfRange pr("term_grad_kernel", st, 0.0, 8.0 * P.esize * (2.0 + P.asm_nterms));
            term_grad_kernel<<<ceil_div(P.esize, 128), 128, 0, st>>>(P.d_asm_ops, P.asm_nterms, P.d_asm_fock,
                                                                     P.esize, P.d_asm_sb, P.d_asm_si, P.d_dims,
                                                                     P.d_moff, W, db.as<double>());
            check_launch("term_grad_kernel");
        }
        PGX_CUDA(cudaMemcpyAsync(dterm, db.p, P.asm_nterms * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    if (dE) PGX_CUDA(cudaMemcpyAsync(dE, Eb, P.esize * sizeof(double), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
}

void run_gf_vjp(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                const double* z, const double* lambda, double* dterm, double* dE) {
    run_pair_vjp(c, 0, op1, op2, nparts, outer, inner, nz, z, 0.0, lambda, dterm, dE);
}

void run_susc_vjp(pgx_ctx* c, int opA, int opB, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                  const double* z, double pole_res, const double* lambda, double* dterm, double* dE) {
    run_pair_vjp(c, 1, opA, opB, nparts, outer, inner, nz, z, pole_res, lambda, dterm, dE);
}

}  // namespace pgx
