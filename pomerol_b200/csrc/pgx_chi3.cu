// Three-point fermion-boson susceptibility (pgx_chi3).
//
// The reference (ThreePointSusceptibilityPart.cpp:243-342) walks every state
// triple (i, j, k) of a part <i|F1|j><j|F2|k><k|B|i>, B = B1 B2, builds three
// term lists and evaluates every term at every frequency duplet.  Here the
// same sum is factorised over matrix products.  With C = pf F1_ij F2_jk B_ki,
// E_ab = E_a - E_b, m_ik = [|E_ik| > PoleResolution], Om = z1 - xi z2, the
// part contributes (not swapped / swapped)
//   fermion-fermion  spp C (w_i + w_j + m_ik (w_k - w_i)) / ((z1 - E_ij)(z2 - sig E_jk))
//                    spp C (w_i + w_j)                   / ((z1 - E_jk)(z2 - sig E_ij))
//   fermion-boson    m_ik C (w_k - w_i) / ((z1 - E_ij)(Om - E_ik))
//                   -m_ik C (w_k - w_i) / ((z1 - E_jk)(Om - E_ik))
//   resonant         (1 - m_ik) [|Om| <= res] (-beta C w_i) / (z1 + E_jk)
//                    (1 - m_ik) [|Om| <= res] ( beta C w_i) / (z1 - E_jk)
// (pf, spp, sig, xi: signs fixed by the channel and the swap, as in
// addMultiterm).  Each family is a contraction over two of the three state
// indices of matrices that carry one frequency each:
//   fermion-fermion  sum_{k,j} [sum_i W_ki F1_ij / (z - E_ij)] [F2_jk / (z' - E_jk)]
//   fermion-boson    sum_{i,k} [sum_j F1_ij F2_jk / (z1 - E..)] [B'_ki / (Om - E_ik)]
//   resonant         sum_{k,j} [sum_i B''_ki F1_ij] [F2_jk / (z1 -+ E_jk)]
// so every part becomes (1) frequency-batched GEMMs with the dressing fused
// into the operand loads, writing one row (or column) per frequency of a
// matrix L (or R) whose inner index runs over the flattened (k, j) or (i, k)
// pairs of all parts, (2) a materialised dressed matrix for the other side,
// and (3) one split-K GEMM L R over all parts at once, whose result is the
// (z1, z2) or (z1, Om) table.  A final kernel gathers the requested duplets.

#include <map>
#include <utility>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

template <typename T> struct Chi3Dev {
    const T* F1;   // d1 x d2 rotated part <i|F1|j>
    const T* F2;   // d2 x d3 rotated part <j|F2|k>
    T* Bm;         // d3 x d1, B1 B2
    T* Lhs;        // d3 x 2 d1: [B_ki w'_ki | B_ki]
    T* S1;         // 2 d1 x d2: [F1_ij ; F1_ij w_j]
    double* E2r;   // 2 d1: [E_i ; E_i]
    T* BF;         // d1 x d3: m_ik B_ki (w_k - w_i), (i, k) layout
    T* BR;         // d3 x d1: (1 - m_ik) B_ki w_i
    T* R0;         // d3 x d2: BR F1
    const double *Ei, *Ej, *Ek, *wi, *wj, *wk;
    int d1, d2, d3, swapped;
    long offN, offF;      // column offsets of the part in L / R and LF / RF
    double cN, cF, cR;    // scalar prefactors of the three families
};

template <typename T> __device__ __forceinline__ T mul(T a, double s) { return a * s; }

__device__ __forceinline__ double lane_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T> __global__ void chi3_prep_kernel(const Chi3Dev<T>* parts, double res) {
    const Chi3Dev<T> p = parts[blockIdx.y];
    const long n1 = (long)p.d3 * p.d1, n2 = 2L * p.d1 * p.d2;
    const long n = n1 > n2 ? n1 : n2;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        if (e < n1) {
            const int k = (int)(e / p.d1), i = (int)(e % p.d1);
            const T b = p.Bm[e];
            const bool nonres = fabs(p.Ei[i] - p.Ek[k]) > res;
            const double wt = (!p.swapped && nonres) ? p.wk[k] : p.wi[i];
            p.Lhs[(long)k * 2 * p.d1 + i] = mul(b, wt);
            p.Lhs[(long)k * 2 * p.d1 + p.d1 + i] = b;
            p.BF[(long)i * p.d3 + k] = nonres ? mul(b, p.wk[k] - p.wi[i]) : mul(b, 0.0);
            p.BR[e] = nonres ? mul(b, 0.0) : mul(b, p.wi[i]);
        }
        if (e < n2) {
            const long half = (long)p.d1 * p.d2;
            const long f = e < half ? e : e - half;
            const int j = (int)(f % p.d2);
            p.S1[e] = e < half ? p.F1[f] : mul(p.F1[f], p.wj[j]);
        }
        if (e < 2L * p.d1) p.E2r[e] = p.Ei[e < p.d1 ? e : e - p.d1];
    }
}

// The side of the fermion-fermion contraction that is dressed with one
// frequency per row / column: F2_jk / (z - E_jk), z = sig z2 into R (not
// swapped, columns = z2) or z = z1 into L (swapped, rows = z1).
template <typename T>
__global__ void chi3_dress_ff_kernel(const Chi3Dev<T>* parts, const cd* Z1, int N1, const cd* sZ2, int N2, cd* L,
                                     cd* R, long KN) {
    const Chi3Dev<T> p = parts[blockIdx.y];
    const long nkj = (long)p.d3 * p.d2;
    const int nf = p.swapped ? N1 : N2;
    const long n = nkj * nf;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        long kj;
        int b;
        if (p.swapped) {  // L row b, contiguous in kj
            kj = e % nkj;
            b = (int)(e / nkj);
        } else {  // R row kj, contiguous in b
            kj = e / nf;
            b = (int)(e % nf);
        }
        const int k = (int)(kj / p.d2), j = (int)(kj % p.d2);
        const cd z = p.swapped ? Z1[b] : sZ2[b];
        const cd v = tocd(p.F2[(long)j * p.d3 + k]) * inv(cd{z.x - (p.Ej[j] - p.Ek[k]), z.y}) * p.cN;
        if (p.swapped)
            L[(long)b * KN + p.offN + kj] = v;
        else
            R[(p.offN + kj) * N2 + b] = v;
    }
}

// RF[(i, k), Om] = cF m_ik B_ki (w_k - w_i) / (Om - E_ik)
template <typename T>
__global__ void chi3_dress_fb_kernel(const Chi3Dev<T>* parts, const cd* ZO, int NO, cd* RF) {
    const Chi3Dev<T> p = parts[blockIdx.y];
    const long n = (long)p.d1 * p.d3 * NO;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const long ik = e / NO;
        const int b = (int)(e % NO);
        const int i = (int)(ik / p.d3), k = (int)(ik % p.d3);
        const cd x = tocd(p.BF[ik]);
        cd v{0.0, 0.0};
        if (x.x != 0.0 || x.y != 0.0) v = x * inv(cd{ZO[b].x - (p.Ei[i] - p.Ek[k]), ZO[b].y}) * p.cF;
        RF[(p.offF + ik) * NO + b] = v;
    }
}

// RES[b] += cR sum_{k,j} R0_kj F2_jk / (z1_b - P_jk), P = -E_jk (not swapped) or E_jk;
// one CTA per (part, frequency)
template <typename T>
__global__ void chi3_resonant_kernel(const Chi3Dev<T>* parts, const cd* Z1, cd* RES) {
    const Chi3Dev<T> p = parts[blockIdx.y];
    const cd z = Z1[blockIdx.x];
    const long n = (long)p.d3 * p.d2;
    cd acc{0.0, 0.0};
    for (long kj = threadIdx.x; kj < n; kj += blockDim.x) {
        const int k = (int)(kj / p.d2), j = (int)(kj % p.d2);
        const cd r = tocd(p.R0[kj]);
        if (r.x == 0.0 && r.y == 0.0) continue;
        const double Ejk = p.Ej[j] - p.Ek[k];
        const double P = p.swapped ? Ejk : -Ejk;
        acc = acc + r * tocd(p.F2[(long)j * p.d3 + k]) * inv(cd{z.x - P, z.y});
    }
    __shared__ cd red[32];
    acc.x = lane_sum(acc.x);
    acc.y = lane_sum(acc.y);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        cd s{0.0, 0.0};
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s = s + red[w];
        atomicAdd(&RES[blockIdx.x].x, s.x * p.cR);
        atomicAdd(&RES[blockIdx.x].y, s.y * p.cR);
    }
}

// OUT[e] += sum_s partial[s][e]
__global__ void chi3_reduce_kernel(const cd* partial, int nsplit, long mn, cd* out) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < mn; e += (long)gridDim.x * blockDim.x) {
        cd s = out[e];
        for (int q = 0; q < nsplit; ++q) s = s + partial[q * mn + e];
        out[e] = s;
    }
}

struct DupletIdx {
    int i1, i2, io, res;
};
__global__ void chi3_gather_kernel(const DupletIdx* q, int n, const cd* OUTN, int N2, const cd* OUTF, int NO,
                                   const cd* RES, cd* out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const DupletIdx d = q[t];
    cd v = OUTN[(long)d.i1 * N2 + d.i2] + OUTF[(long)d.i1 * NO + d.io];
    if (d.res) v = v + RES[d.i1];
    out[t] = v;
}

// distinct values of a complex list (exact bits), in order of first appearance
int distinct_index(const std::vector<cd>& v, std::vector<cd>& uniq, std::vector<int>& idx) {
    std::map<std::pair<double, double>, int> seen;
    idx.resize(v.size());
    for (size_t q = 0; q < v.size(); ++q) {
        auto key = std::make_pair(v[q].x, v[q].y);
        auto it = seen.find(key);
        if (it == seen.end()) {
            it = seen.emplace(key, (int)uniq.size()).first;
            uniq.push_back(v[q]);
        }
        idx[q] = it->second;
    }
    return (int)uniq.size();
}

// C (M x N) += A (M x K) B (K x N), row-major, split over K into partial
// products that a reduction adds up
void split_k_gemm(const cd* A, const cd* B, int M, int N, long K, cd* C, DevBuf& partial, DevBuf& probs,
                  DevBuf& index, cudaStream_t st) {
    if (K <= 0 || M <= 0 || N <= 0) return;
    const long kc = std::max<long>(256, (K + 591) / 592);
    const long nfull = K / kc, rem = K - nfull * kc;
    const int nsplit = (int)(nfull + (rem > 0 ? 1 : 0));
    const long mn = (long)M * N;
    partial.reserve(nsplit * mn * sizeof(cd));
    cd* P = partial.as<cd>();
    std::vector<GemmProblem<cd, cd, cd>> pr;
    GemmProblem<cd, cd, cd> g{};
    g.M = M;
    g.N = N;
    g.sa_i = K;
    g.sa_k = 1;
    g.sb_k = N;
    g.sb_j = 1;
    g.sc_i = N;
    g.sc_j = 1;
    if (nfull > 0) {
        g.A = A;
        g.B = B;
        g.C = P;
        g.K = (int)kc;
        g.nb = (int)nfull;
        g.ba = kc;
        g.bb = kc * N;
        g.bc = mn;
        pr.push_back(g);
    }
    if (rem > 0) {
        g.A = A + nfull * kc;
        g.B = B + nfull * kc * N;
        g.C = P + nfull * mn;
        g.K = (int)rem;
        g.nb = 1;
        g.ba = g.bb = g.bc = 0;
        pr.push_back(g);
    }
    probs.reserve(pr.size() * sizeof(pr[0]));
    index.reserve(gemm_index_bytes(pr.size()));
    launch_gemm_batch(pr, probs.p, probs.bytes, index.p, index.bytes, st);
    ProfRange r("chi3_reduce_kernel", st, 2.0 * nsplit * mn, 16.0 * (nsplit + 2) * mn);
    chi3_reduce_kernel<<<std::min(ceil_div(mn, 256), 1024), 256, 0, st>>>(P, nsplit, mn, C);
    check_launch("chi3_reduce_kernel");
}

template <typename T>
void run_chi3_t(pgx_ctx* c, int channel, int nparts, const pgx_chi3_part* parts, int nfreq, const double* z,
                double res, double* out) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    const int xi = channel == PGX_PP ? -1 : 1;
    const double sig = channel == PGX_PP ? 1.0 : -1.0, spp = channel == PGX_PP ? -1.0 : 1.0;
    // ---- duplets: distinct z1, sig z2 and Om = z1 - xi z2
    std::vector<cd> z1(nfreq), sz2(nfreq), om(nfreq);
    for (int q = 0; q < nfreq; ++q) {
        z1[q] = cd{z[4 * q], z[4 * q + 1]};
        sz2[q] = cd{sig * z[4 * q + 2], sig * z[4 * q + 3]};
        om[q] = cd{z[4 * q] - xi * z[4 * q + 2], z[4 * q + 1] - xi * z[4 * q + 3]};
    }
    std::vector<cd> Z1, SZ2, ZO;
    std::vector<int> i1, i2, io;
    const int N1 = distinct_index(z1, Z1, i1), N2 = distinct_index(sz2, SZ2, i2), NO = distinct_index(om, ZO, io);
    std::vector<DupletIdx> dq(nfreq);
    bool any_res = false;
    for (int q = 0; q < nfreq; ++q) {
        const bool r = std::sqrt(om[q].x * om[q].x + om[q].y * om[q].y) <= res;
        any_res = any_res || r;
        dq[q] = DupletIdx{i1[q], i2[q], io[q], r ? 1 : 0};
    }
    // negated frequency lists for the fused dressing 1 / (-z - (E_b - E_a))
    std::vector<cd> nZ1(N1), nSZ2(N2);
    for (int b = 0; b < N1; ++b) nZ1[b] = cd{-Z1[b].x, -Z1[b].y};
    for (int b = 0; b < N2; ++b) nSZ2[b] = cd{-SZ2[b].x, -SZ2[b].y};
    // ---- parts: validation and sizes
    struct Host {
        const OpPart *f1, *f2, *b1, *b2;
        const Operator *F1, *F2, *B1, *B2;
        int blk[4];
        int swapped;
    };
    std::vector<Host> hp;
    auto find_part = [&](int opid, int left, int right) -> std::pair<const Operator*, const OpPart*> {
        PGX_CHECK(opid >= 0 && opid < (int)P.ops.size(), PGX_ERR_ARG, "bad operator id");
        const Operator& o = P.ops[opid];
        PGX_CHECK(o.rotated, PGX_ERR_STATE, "operators must be rotated");
        PGX_CHECK(left >= 0 && left < P.nblocks && right >= 0 && right < P.nblocks, PGX_ERR_ARG, "bad block");
        const int q = o.by_left[left];
        PGX_CHECK(q >= 0 && o.parts[q].right == right, PGX_ERR_ARG, "blocks do not form a 3-point part");
        return {&o, &o.parts[q]};
    };
    for (int q = 0; q < nparts; ++q) {
        const pgx_chi3_part& x = parts[q];
        Host h;
        std::copy(x.block, x.block + 4, h.blk);
        auto a = find_part(x.f1, x.block[0], x.block[1]);
        auto b = find_part(x.f2, x.block[1], x.block[2]);
        auto cc = find_part(x.b1, x.block[2], x.block[3]);
        auto d = find_part(x.b2, x.block[3], x.block[0]);
        h.F1 = a.first;
        h.f1 = a.second;
        h.F2 = b.first;
        h.f2 = b.second;
        h.B1 = cc.first;
        h.b1 = cc.second;
        h.B2 = d.first;
        h.b2 = d.second;
        h.swapped = x.swapped ? 1 : 0;
        hp.push_back(h);
    }
    // ---- result tables (persist over part groups)
    DevBuf& tab = c->scratch[0];
    const long nOUTN = (long)N1 * N2, nOUTF = (long)N1 * NO;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t b_outn = al(nOUTN * sizeof(cd)), b_outf = al(nOUTF * sizeof(cd)), b_res = al(N1 * sizeof(cd)),
                 b_z = al(std::max(N1, 1) * sizeof(cd)), b_z2 = al(std::max(N2, 1) * sizeof(cd)),
                 b_zo = al(std::max(NO, 1) * sizeof(cd)), b_dq = al(std::max(nfreq, 1) * sizeof(DupletIdx)),
                 b_out = al(std::max(nfreq, 1) * sizeof(cd));
    tab.reserve(b_outn + b_outf + b_res + 2 * b_z + 2 * b_z2 + b_zo + b_dq + b_out);
    char* tp = tab.as<char>();
    cd* OUTN = reinterpret_cast<cd*>(tp);
    cd* OUTF = reinterpret_cast<cd*>(tp + b_outn);
    cd* RES = reinterpret_cast<cd*>(tp + b_outn + b_outf);
    cd* dZ1 = reinterpret_cast<cd*>(tp + b_outn + b_outf + b_res);
    cd* dnZ1 = reinterpret_cast<cd*>(reinterpret_cast<char*>(dZ1) + b_z);
    cd* dSZ2 = reinterpret_cast<cd*>(reinterpret_cast<char*>(dnZ1) + b_z);
    cd* dnSZ2 = reinterpret_cast<cd*>(reinterpret_cast<char*>(dSZ2) + b_z2);
    cd* dZO = reinterpret_cast<cd*>(reinterpret_cast<char*>(dnSZ2) + b_z2);
    DupletIdx* dDQ = reinterpret_cast<DupletIdx*>(reinterpret_cast<char*>(dZO) + b_zo);
    cd* dOut = reinterpret_cast<cd*>(reinterpret_cast<char*>(dDQ) + b_dq);
    PGX_CUDA(cudaMemsetAsync(tp, 0, b_outn + b_outf + b_res, st));
    if (nfreq > 0) {
        h2d(dZ1, Z1.data(), N1 * sizeof(cd), st);
        h2d(dnZ1, nZ1.data(), N1 * sizeof(cd), st);
        h2d(dSZ2, SZ2.data(), N2 * sizeof(cd), st);
        h2d(dnSZ2, nSZ2.data(), N2 * sizeof(cd), st);
        h2d(dZO, ZO.data(), NO * sizeof(cd), st);
        h2d(dDQ, dq.data(), nfreq * sizeof(DupletIdx), st);
    }
    // ---- parts in groups whose frequency-dependent matrices fit the budget
    const double budget = 4.0e9;
    size_t q0 = 0;
    while (q0 < hp.size() && nfreq > 0) {
        size_t q1 = q0;
        double bytes = 0.0;
        while (q1 < hp.size()) {
            const Host& h = hp[q1];
            const double d1 = h.f1->dl, d2 = h.f1->dr, d3 = h.f2->dr;
            const double add = 16.0 * ((N1 + N2) * d2 * d3 + (N1 + NO) * d1 * d3);
            if (q1 > q0 && bytes + add > budget) break;
            bytes += add;
            ++q1;
        }
        // per-part constant buffers and column offsets
        std::vector<Chi3Dev<T>> dv;
        long KN = 0, KF = 0;
        size_t small = 0;
        for (size_t q = q0; q < q1; ++q) {
            const Host& h = hp[q];
            const int d1 = h.f1->dl, d2 = h.f1->dr, d3 = h.f2->dr;
            Chi3Dev<T> x{};
            x.d1 = d1;
            x.d2 = d2;
            x.d3 = d3;
            x.swapped = h.swapped;
            x.offN = KN;
            x.offF = KF;
            KN += (long)d2 * d3;
            KF += (long)d1 * d3;
            const double pf = ((channel == PGX_PH) == (h.swapped != 0)) ? 1.0 : -1.0;
            x.cN = -spp * pf * sig;
            x.cF = h.swapped ? pf : -pf;
            x.cR = h.swapped ? P.beta * pf : -P.beta * pf;
            x.F1 = h.F1->mat.as<T>() + h.f1->off;
            x.F2 = h.F2->mat.as<T>() + h.f2->off;
            x.Ei = P.d_E + P.eoff[h.blk[0]];
            x.Ej = P.d_E + P.eoff[h.blk[1]];
            x.Ek = P.d_E + P.eoff[h.blk[2]];
            x.wi = P.d_w + P.eoff[h.blk[0]];
            x.wj = P.d_w + P.eoff[h.blk[1]];
            x.wk = P.d_w + P.eoff[h.blk[2]];
            // Bm, Lhs, S1, E2r, BF, BR, R0, each 256-byte aligned (the layout below)
            small += al((size_t)d3 * d1 * sizeof(T)) + al((size_t)d3 * 2 * d1 * sizeof(T)) +
                     al((size_t)2 * d1 * d2 * sizeof(T)) + al((size_t)2 * d1 * sizeof(double)) +
                     al((size_t)d1 * d3 * sizeof(T)) + al((size_t)d3 * d1 * sizeof(T)) + al((size_t)d3 * d2 * sizeof(T));
            dv.push_back(x);
        }
        DevBuf& sb = P.chi3_small;
        sb.reserve(std::max<size_t>(small, 256));
        {
            char* base = sb.as<char>();
            size_t o = 0;
            auto take = [&](size_t n) {
                char* r = base + o;
                o = al(o + n);
                return r;
            };
            for (auto& x : dv) {
                x.Bm = reinterpret_cast<T*>(take((size_t)x.d3 * x.d1 * sizeof(T)));
                x.Lhs = reinterpret_cast<T*>(take((size_t)x.d3 * 2 * x.d1 * sizeof(T)));
                x.S1 = reinterpret_cast<T*>(take((size_t)2 * x.d1 * x.d2 * sizeof(T)));
                x.E2r = reinterpret_cast<double*>(take((size_t)2 * x.d1 * sizeof(double)));
                x.BF = reinterpret_cast<T*>(take((size_t)x.d1 * x.d3 * sizeof(T)));
                x.BR = reinterpret_cast<T*>(take((size_t)x.d3 * x.d1 * sizeof(T)));
                x.R0 = reinterpret_cast<T*>(take((size_t)x.d3 * x.d2 * sizeof(T)));
            }
            PGX_CHECK(o <= sb.bytes, PGX_ERR_ARG, "chi3 workspace layout overflow");
        }
        DevBuf& big = P.chi3_big;
        const size_t b_L = al(KN * N1 * sizeof(cd)), b_R = al(KN * N2 * sizeof(cd)), b_LF = al(KF * N1 * sizeof(cd)),
                     b_RF = al(KF * NO * sizeof(cd));
        big.reserve(b_L + b_R + b_LF + b_RF);
        cd* L = big.as<cd>();
        cd* R = reinterpret_cast<cd*>(big.as<char>() + b_L);
        cd* LF = reinterpret_cast<cd*>(big.as<char>() + b_L + b_R);
        cd* RF = reinterpret_cast<cd*>(big.as<char>() + b_L + b_R + b_LF);
        DevBuf& dparts = c->scratch[1];
        dparts.reserve(dv.size() * sizeof(Chi3Dev<T>));
        h2d(dparts.p, dv.data(), dv.size() * sizeof(Chi3Dev<T>), st);
        const Chi3Dev<T>* dp = dparts.as<Chi3Dev<T>>();
        // (1) B = B1 B2
        {
            std::vector<GemmProblem<T, T, T>> pr;
            for (size_t q = q0; q < q1; ++q) {
                const Host& h = hp[q];
                const Chi3Dev<T>& x = dv[q - q0];
                GemmProblem<T, T, T> g{};
                g.A = h.B1->mat.as<T>() + h.b1->off;  // d3 x dm
                g.B = h.B2->mat.as<T>() + h.b2->off;  // dm x d1
                g.C = x.Bm;
                g.M = x.d3;
                g.N = x.d1;
                g.K = h.b1->dr;
                g.sa_i = h.b1->dr;
                g.sa_k = 1;
                g.sb_k = x.d1;
                g.sb_j = 1;
                g.sc_i = x.d1;
                g.sc_j = 1;
                pr.push_back(g);
            }
            c->scratch[2].reserve(pr.size() * sizeof(pr[0]));
            c->scratch[3].reserve(gemm_index_bytes(pr.size()));
            launch_gemm_batch(pr, c->scratch[2].p, c->scratch[2].bytes, c->scratch[3].p, c->scratch[3].bytes, st);
        }
        long maxe = 1;
        for (auto& x : dv) maxe = std::max(maxe, std::max((long)x.d3 * x.d1, 2L * x.d1 * x.d2));
        {
            ProfRange pr("chi3_prep_kernel", st, 0.0, 0.0);
            chi3_prep_kernel<T><<<dim3(std::min(ceil_div(maxe, 256), 512), (unsigned)dv.size()), 256, 0, st>>>(dp,
                                                                                                          res);
            check_launch("chi3_prep_kernel");
        }
        // (2) frequency-batched dressed GEMMs
        {
            std::vector<GemmProblem<T, Dressed<T>, cd>> pa;  // fermion-fermion sides; swapped fermion-boson
            std::vector<GemmProblem<Dressed<T>, T, cd>> pb;  // fermion-boson, not swapped
            for (const auto& x : dv) {
                GemmProblem<T, Dressed<T>, cd> g{};
                g.A = x.Lhs;
                g.B = x.S1;
                g.M = x.d3;
                g.N = x.d2;
                g.K = 2 * x.d1;
                g.sa_i = 2L * x.d1;
                g.sa_k = 1;
                g.sb_k = x.d2;
                g.sb_j = 1;
                g.dEa = x.E2r;
                g.dEb = x.Ej;
                if (!x.swapped) {  // L row b = z1_b
                    g.C = L + x.offN;
                    g.sc_i = x.d2;
                    g.sc_j = 1;
                    g.nb = N1;
                    g.bc = KN;
                    g.dzs = dnZ1;
                } else {  // R column b = z2_b
                    g.C = R + x.offN * N2;
                    g.sc_i = (long)x.d2 * N2;
                    g.sc_j = N2;
                    g.nb = N2;
                    g.bc = 1;
                    g.dzs = dnSZ2;
                }
                pa.push_back(g);
                if (x.swapped) {  // F1 (F2 / (z1 - E_jk)) into LF row b
                    GemmProblem<T, Dressed<T>, cd> f{};
                    f.A = x.F1;
                    f.B = x.F2;
                    f.M = x.d1;
                    f.N = x.d3;
                    f.K = x.d2;
                    f.sa_i = x.d2;
                    f.sa_k = 1;
                    f.sb_k = x.d3;
                    f.sb_j = 1;
                    f.dEa = x.Ej;
                    f.dEb = x.Ek;
                    f.C = LF + x.offF;
                    f.sc_i = x.d3;
                    f.sc_j = 1;
                    f.nb = N1;
                    f.bc = KF;
                    f.dzs = dnZ1;
                    pa.push_back(f);
                } else {  // (F1 / (z1 - E_ij)) F2 into LF row b
                    GemmProblem<Dressed<T>, T, cd> f{};
                    f.A = x.F1;
                    f.B = x.F2;
                    f.M = x.d1;
                    f.N = x.d3;
                    f.K = x.d2;
                    f.sa_i = x.d2;
                    f.sa_k = 1;
                    f.sb_k = x.d3;
                    f.sb_j = 1;
                    f.dEa = x.Ei;
                    f.dEb = x.Ej;
                    f.C = LF + x.offF;
                    f.sc_i = x.d3;
                    f.sc_j = 1;
                    f.nb = N1;
                    f.bc = KF;
                    f.dzs = dnZ1;
                    pb.push_back(f);
                }
            }
            c->scratch[2].reserve(pa.size() * sizeof(pa[0]));
            c->scratch[3].reserve(gemm_index_bytes(pa.size()));
            launch_gemm_batch(pa, c->scratch[2].p, c->scratch[2].bytes, c->scratch[3].p, c->scratch[3].bytes, st);
            c->scratch[4].reserve(std::max<size_t>(pb.size(), 1) * sizeof(GemmProblem<Dressed<T>, T, cd>));
            c->scratch[5].reserve(gemm_index_bytes(pb.size()));
            launch_gemm_batch(pb, c->scratch[4].p, c->scratch[4].bytes, c->scratch[5].p, c->scratch[5].bytes, st);
        }
        // (3) materialised dressed sides
        long maxff = 1, maxfb = 1;
        for (auto& x : dv) {
            maxff = std::max(maxff, (long)x.d3 * x.d2 * (x.swapped ? N1 : N2));
            maxfb = std::max(maxfb, (long)x.d1 * x.d3 * NO);
        }
        {
            ProfRange pr("chi3_dress_kernel", st, 0.0, 16.0 * (double)(KN * std::max(N1, N2) + KF * NO));
            chi3_dress_ff_kernel<T><<<dim3(std::min(ceil_div(maxff, 256), 1024), (unsigned)dv.size()), 256, 0, st>>>(
                dp, dZ1, N1, dSZ2, N2, L, R, KN);
            check_launch("chi3_dress_ff_kernel");
            chi3_dress_fb_kernel<T><<<dim3(std::min(ceil_div(maxfb, 256), 1024), (unsigned)dv.size()), 256, 0, st>>>(
                dp, dZO, NO, RF);
            check_launch("chi3_dress_fb_kernel");
        }
        // (4) resonant terms
        if (any_res) {
            std::vector<GemmProblem<T, T, T>> pr;
            for (const auto& x : dv) {
                GemmProblem<T, T, T> g{};
                g.A = x.BR;
                g.B = x.F1;
                g.C = x.R0;
                g.M = x.d3;
                g.N = x.d2;
                g.K = x.d1;
                g.sa_i = x.d1;
                g.sa_k = 1;
                g.sb_k = x.d2;
                g.sb_j = 1;
                g.sc_i = x.d2;
                g.sc_j = 1;
                pr.push_back(g);
            }
            c->scratch[6].reserve(pr.size() * sizeof(pr[0]));
            c->scratch[7].reserve(gemm_index_bytes(pr.size()));
            launch_gemm_batch(pr, c->scratch[6].p, c->scratch[6].bytes, c->scratch[7].p, c->scratch[7].bytes, st);
            ProfRange rr("chi3_resonant_kernel", st, 0.0, 0.0);
            chi3_resonant_kernel<T><<<dim3((unsigned)N1, (unsigned)dv.size()), 256, 0, st>>>(dp, dZ1, RES);
            check_launch("chi3_resonant_kernel");
        }
        // (5) contractions over all parts of the group
        split_k_gemm(L, R, N1, N2, KN, OUTN, c->scratch[8], c->scratch[9], c->scratch[10], st);
        split_k_gemm(LF, RF, N1, NO, KF, OUTF, c->scratch[8], c->scratch[9], c->scratch[10], st);
        q0 = q1;
    }
    if (nfreq > 0) {
        chi3_gather_kernel<<<ceil_div(nfreq, 128), 128, 0, st>>>(dDQ, nfreq, OUTN, N2, OUTF, NO, RES, dOut);
        check_launch("chi3_gather_kernel");
        PGX_CUDA(cudaMemcpyAsync(out, dOut, nfreq * sizeof(cd), cudaMemcpyDeviceToHost, st));
    }
    PGX_CUDA(cudaStreamSynchronize(st));
}

}  // namespace

void run_chi3(pgx_ctx* c, int channel, int nparts, const pgx_chi3_part* parts, int nfreq, const double* z,
              double pole_res, double* out) {
    Problem& P = c->P;
    PGX_CHECK(channel == PGX_PP || channel == PGX_PH || channel == PGX_XPH, PGX_ERR_ARG, "bad channel");
    PGX_CHECK(P.have_w, PGX_ERR_STATE, "pgx_weights first");
    PGX_CHECK(P.nblocks < 65536 && nparts < 65536, PGX_ERR_ARG, "too many parts");
    if (P.is_complex)
        run_chi3_t<cd>(c, channel, nparts, parts, nfreq, z, pole_res, out);
    else
        run_chi3_t<double>(c, channel, nparts, parts, nfreq, z, pole_res, out);
}

}  // namespace pgx
