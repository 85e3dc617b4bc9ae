// K4, weight-anchored form of the G2 Lehmann sum.
//
// Every sub-term of TwoParticleGFPart::addMultiterm (TwoParticleGFPart.cpp:277-297)
// is a product of the matrix element M and ONE Boltzmann weight once the weight
// sums are split: -M(w2+w3) -> w2 and w3 parts, M(w1+w4) -> w1 and w4 parts, the
// resonant z1z2 term -> w1 (delta: beta w1, else -w1/D) and w3 (w3/D), the z2z3
// term -> w2 (delta: -beta w2, else w2/D) and w4 (-w4/D).  Each part only needs
// the states of its weighted ("anchor") index whose weight exceeds the anchor
// threshold; the other three indices are summed completely.  The dropped
// contribution is bounded by threshold * d * (beta/pi)^3 per chain, the same
// order as the reference's own CoefficientTolerance filter (:241, :283-297).
//
// With A(z1) = O1 / (z1 - (E2 - E1)), C(z3) = O3 / (z3 - (E4 - E3)) and H_b the
// anchor states of block b, the eight anchored sub-terms are
//   T1a  -s  w2 sum_3 O2[h,3] / (z2 - (E3 - E2h)) [C(z3) X4 A(z1)[:,h]]_3
//   T1b  -s  w3 sum_2 O2[2,h] / (z2 - (E3h - E2)) [C(z3)[h,:] X4 A(z1)]_2
//   T2a   s  w1 sum_4 X4[4,h] / (Z - (E4 - E1h))  [A(z1)[h,:] O2 C(z3)]_4
//   T2b   s  w4 sum_1 X4[h,1] / (Z - (E4h - E1))  [A(z1) O2 C(z3)[:,h]]_1
//   T3a   s  sum_3 [A(z1)[h,:] O2]_3 [C(z3) X4[:,h]]_3 (delta ? beta w1 : -w1/D)
//   T3b   s  sum_1 [A(z1) O2[:,h]]_1 [C(z3)[h,:] X4]_1 (delta ? 0 : w3/D)
//   T4a   s  sum_4 [O2[h,:] C(z3)]_4 [X4 A(z1)[:,h]]_4 (delta ? -beta w2 : w2/D)
//   T4b   s  sum_2 [O2 C(z3)[:,h]]_2 [X4[h,:] A(z1)]_2 (delta ? 0 : -w4/D)
// (Z = z1+z2+z3, D = s - (E_b - E_a) with s = z1+z2 for T3 and z2+z3 for T4).
// Stages, each one launch for a batch of chains: anchored products per
// frequency (gather GEMMs); products per (z1, z3) stacked into GEMMs over all
// anchors; contractions per triple (warp per (sub-term, (z1, z3) group),
// resonant delta test in FP64).  A(z1) and C(z3) are never stored: the GEMM
// tile loads dress O1 and O3 with the frequency as they read them.

#include <array>
#include <map>
#include <set>
#include <tuple>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

struct DTerm {
    const void* VA;
    long a1, a3, ah, ak;
    const void* VB;
    long b1, b3, bh, bk;
    const double *Ek, *Eh, *wh;
    const int* hot;       // anchor states (inner indices) of the anchor block
    const int* gi1;       // per group: index of z1 in the plan
    const int* gi3;       // per group: index of z3 in the plan
    int nh, nk;
    int va_cplx, vb_cplx; // operand element types
    int va_hstate, vb_hstate;  // h stride applies to the anchor's state index instead of its position
    int use_delta;
    double sgn, cdelta, cnum, pref;
    // host side only: the plan and the frequency sum (0: z2, 1: z1+z2+z3,
    // 2: z1+z2, 3: z2+z3) of the sub-term
    int plan, sidx;
};

__device__ __forceinline__ cd load_v(const void* p, int cplx, long idx) {
    return cplx ? static_cast<const cd*>(p)[idx] : cd{static_cast<const double*>(p)[idx], 0.0};
}

// ---- contractions as products
// For one sub-term, the (z1, z3) groups of a plan whose triples carry the same
// list of frequency sums s_j form a class.  Over a class the contraction is a
// complex product
//   out[t(g, j)] += pref * sum_{h, k} AB[g, (h, k)] K[(h, k), j]
// with AB[g, (h, k)] = VA(g, h, k) VB(g, h, k) (the two anchored operand
// arrays, multiplied as the tile is loaded) and the Lehmann kernel
//   K[(h, k), j] = delta ? cdelta beta w_h : cnum w_h / (s_j - sgn (E_k - E_h)),
// delta = |s_j - sgn (E_k - E_h)| <= PoleResolution (FP64, the reference's
// rule for resonant terms).  K is formed once per tile element and used by
// every row of the tile; the rows of a T1 class are all (z1, z3) groups, those
// of T2, T3, T4 classes the groups with equal z1 + z3, z1 or z3.  A work item
// is one tile of rows of a class over a range of anchors; items of the same
// outputs add their results with atomics.
struct CClass {
    int term;          // index into the DTerm list
    int nrows, ncols;  // rows (groups) and columns (frequency sums) of the class
    const cd* s;       // ncols frequency sums
    const int* rows;   // nrows group indices
    const int* slots;  // nrows x ncols triple ids (row-major), -1 where absent
};
struct CItem {
    int cls, row0, h0, h1;
};

constexpr int CG_NX = 8;
// rows per thread: 4 in 64-row tiles (16 thread rows), BM / 8 below (8 thread rows)
__host__ __device__ constexpr int cg_tm(int bm) { return bm >= 64 ? 4 : bm / 8; }

// One CTA per work item: BM rows x BN columns, (BM / TM) x CG_NX threads,
// each a TM x (BN / CG_NX) block of complex accumulators.  The next k-tile's
// operand loads are issued into registers before the current tile's products.
template <int BM, int BN>
__global__ void __launch_bounds__((BM / cg_tm(BM)) * CG_NX)
    contract_gemm_kernel(const DTerm* __restrict__ terms, const CClass* __restrict__ classes,
                         const CItem* __restrict__ items, double beta, double tol2, cd* __restrict__ out) {
    constexpr int CG_TM = cg_tm(BM);
    constexpr int NY = BM / CG_TM, NT = NY * CG_NX, TN = BN / CG_NX;
    // k-tile depth: 16, or 8 where two 16-deep buffers would pass 48 KB
    constexpr int CG_BK = (BM * BN > 64 * 24) ? 8 : 16;
    constexpr int LA = (BM * CG_BK + NT - 1) / NT, LB = (BN * CG_BK + NT - 1) / NT;
    __shared__ cd As[2][CG_BK][BM + 1];
    __shared__ cd Bs[2][CG_BK][BN + 1];
    __shared__ cd s_s[BN];
    __shared__ long s_oa[BM], s_ob[BM];
    __shared__ DTerm s_term;  // the sub-term's descriptor, read once per CTA
    const CItem it = items[blockIdx.x];
    const CClass cc = classes[it.cls];
    const DTerm& d = s_term;
    const int tid = threadIdx.x, tx = tid % CG_NX, ty = tid / CG_NX;
    if (tid == 0) s_term = terms[cc.term];
    __syncthreads();
    const int nrows = min(BM, cc.nrows - it.row0);
    for (int j = tid; j < BN; j += NT) s_s[j] = j < cc.ncols ? cc.s[j] : cd{0.0, 0.0};
    for (int r = tid; r < BM; r += NT) {
        long oa = 0, ob = 0;
        if (r < nrows) {
            const int g = cc.rows[it.row0 + r];
            const long i1 = d.gi1[g], i3 = d.gi3[g];
            oa = i1 * d.a1 + i3 * d.a3;
            ob = i1 * d.b1 + i3 * d.b3;
        }
        s_oa[r] = oa;
        s_ob[r] = ob;
    }
    cd acc[CG_TM][TN];
#pragma unroll
    for (int a = 0; a < CG_TM; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) acc[a][b] = cd{0.0, 0.0};
    __syncthreads();

    const int nk = d.nk;
    const int ktiles = (nk + CG_BK - 1) / CG_BK;
    const long nsteps = (long)(it.h1 - it.h0) * ktiles;
    // Operands of step q (anchor h0 + q / ktiles, k-tile q % ktiles): fetch()
    // issues the global loads of the raw values into registers before the
    // current step's products; finish() forms VA VB and the Lehmann kernel from
    // them and stores the tiles after the products, so the loads' latency is
    // covered by the inner loop instead of stalling ahead of it.
    cd rx[LA], ry[LA];
    double rek[LB];
    double r_eh = 0.0, r_w = 0.0;
    auto fetch = [&](long q) {
        const int h = it.h0 + (int)(q / ktiles), k0 = (int)(q % ktiles) * CG_BK;
        const int hs = d.hot[h];
        const long oah = (long)(d.va_hstate ? hs : h) * d.ah, obh = (long)(d.vb_hstate ? hs : h) * d.bh;
#pragma unroll
        for (int u = 0; u < LA; ++u) {
            const int l = tid + u * NT;
            cd x{0.0, 0.0}, y{0.0, 0.0};
            if (l < BM * CG_BK) {
                const int r = l / CG_BK, kk = l % CG_BK, k = k0 + kk;
                if (r < nrows && k < nk) {
                    x = load_v(d.VA, d.va_cplx, s_oa[r] + oah + (long)k * d.ak);
                    y = load_v(d.VB, d.vb_cplx, s_ob[r] + obh + (long)k * d.bk);
                }
            }
            rx[u] = x;
            ry[u] = y;
        }
        r_eh = d.Eh[hs];
        r_w = d.wh[hs];
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int l = tid + u * NT;
            double ek = 0.0;
            if (l < BN * CG_BK) {
                const int k = k0 + l / BN;
                if (k < nk) ek = d.Ek[k];
            }
            rek[u] = ek;
        }
    };
    auto finish = [&](long q, int buf) {
        const int k0 = (int)(q % ktiles) * CG_BK;
#pragma unroll
        for (int u = 0; u < LA; ++u) {
            const int l = tid + u * NT;
            if (l < BM * CG_BK) As[buf][l % CG_BK][l / CG_BK] = rx[u] * ry[u];
        }
        const double cw = d.cnum * r_w, cdl = d.cdelta * beta * r_w;
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int l = tid + u * NT;
            if (l < BN * CG_BK) {
                const int kk = l / BN, j = l % BN, k = k0 + kk;
                cd v{0.0, 0.0};
                if (k < nk && j < cc.ncols) {
                    const cd sv = s_s[j];
                    const double dx = sv.x - d.sgn * (rek[u] - r_eh);
                    const double m2 = fma(dx, dx, sv.y * sv.y);
                    if (d.use_delta && m2 <= tol2) {
                        v = cd{cdl, 0.0};
                    } else {
                        const double rr = cw * recip_pos(m2);
                        v = cd{dx * rr, -sv.y * rr};
                    }
                }
                Bs[buf][kk][j] = v;
            }
        }
    };
    if (nsteps > 0) {
        fetch(0);
        finish(0, 0);
    }
    __syncthreads();
    int buf = 0;
    for (long q = 0; q < nsteps; ++q) {
        const bool more = q + 1 < nsteps;
        if (more) fetch(q + 1);
#pragma unroll
        for (int kk = 0; kk < CG_BK; ++kk) {
            cd a[CG_TM], b[TN];
#pragma unroll
            for (int u = 0; u < CG_TM; ++u) a[u] = As[buf][kk][ty + NY * u];
#pragma unroll
            for (int u = 0; u < TN; ++u) b[u] = Bs[buf][kk][tx + CG_NX * u];
#pragma unroll
            for (int qa = 0; qa < CG_TM; ++qa)
#pragma unroll
                for (int qb = 0; qb < TN; ++qb) {
                    acc[qa][qb].x = fma(a[qa].x, b[qb].x, acc[qa][qb].x);
                    acc[qa][qb].x = fma(-a[qa].y, b[qb].y, acc[qa][qb].x);
                    acc[qa][qb].y = fma(a[qa].x, b[qb].y, acc[qa][qb].y);
                    acc[qa][qb].y = fma(a[qa].y, b[qb].x, acc[qa][qb].y);
                }
        }
        if (more) finish(q + 1, buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int qa = 0; qa < CG_TM; ++qa) {
        const int r = ty + NY * qa;
        if (r >= nrows) continue;
#pragma unroll
        for (int qb = 0; qb < TN; ++qb) {
            const int j = tx + CG_NX * qb;
            if (j >= cc.ncols) continue;
            const int t = cc.slots[(long)(it.row0 + r) * cc.ncols + j];
            const double x = acc[qa][qb].x, y = acc[qa][qb].y;
            if (t >= 0 && (x != 0.0 || y != 0.0)) {
                atomicAdd(&out[t].x, d.pref * x);
                atomicAdd(&out[t].y, d.pref * y);
            }
        }
    }
}

// Column widths of the contraction tiles; a class with more columns is split
// into column chunks of at most CG_BN_MAX.
constexpr int CG_NBN = 4, CG_BN_MAX = 32;
constexpr int CG_BNS[CG_NBN] = {8, 16, 24, 32};

template <int BM, int BN>
void launch_contract_t(unsigned n, cudaStream_t st, const DTerm* t, const CClass* c, const CItem* i, double beta,
                       double tol2, cd* out) {
    contract_gemm_kernel<BM, BN><<<n, (BM / cg_tm(BM)) * CG_NX, 0, st>>>(t, c, i, beta, tol2, out);
}

template <int BM>
void launch_contract_m(int BN, unsigned n, cudaStream_t st, const DTerm* t, const CClass* c, const CItem* i,
                       double beta, double tol2, cd* out) {
    if (BN == 8) launch_contract_t<BM, 8>(n, st, t, c, i, beta, tol2, out);
    else if (BN == 16) launch_contract_t<BM, 16>(n, st, t, c, i, beta, tol2, out);
    else if (BN == 24) launch_contract_t<BM, 24>(n, st, t, c, i, beta, tol2, out);
    else launch_contract_t<BM, 32>(n, st, t, c, i, beta, tol2, out);
}

// Row-tile heights of the contraction (a class takes the smallest that holds
// its rows, 64-row tiles above 32 rows).
constexpr int CG_NBM = 5;
constexpr int CG_BMS[CG_NBM] = {8, 16, 24, 32, 64};

void launch_contract(int BM, int BN, unsigned n, cudaStream_t st, const DTerm* t, const CClass* c, const CItem* i,
                     double beta, double tol2, cd* out) {
    switch (BM) {
        case 8: launch_contract_m<8>(BN, n, st, t, c, i, beta, tol2, out); break;
        case 16: launch_contract_m<16>(BN, n, st, t, c, i, beta, tol2, out); break;
        case 24: launch_contract_m<24>(BN, n, st, t, c, i, beta, tol2, out); break;
        case 32: launch_contract_m<32>(BN, n, st, t, c, i, beta, tol2, out); break;
        default: launch_contract_m<64>(BN, n, st, t, c, i, beta, tol2, out); break;
    }
}

// Frequencies of one permutation of a G2 part: triple t as (z1', z2', z3')
// = the permuted (z1, z2, -z3), with z1' dressing O1 and z3' dressing O3.
inline void perm_freqs(const double* z, int t, const int perm[3], cd& a, cd& b, cd& c) {
    const cd F[3] = {cd{z[6 * t], z[6 * t + 1]}, cd{z[6 * t + 2], z[6 * t + 3]}, cd{-z[6 * t + 4], -z[6 * t + 5]}};
    a = F[perm[0]];
    b = F[perm[1]];
    c = F[perm[2]];
}

struct KeyC {
    double a, b;
    bool operator<(const KeyC& o) const { return std::tie(a, b) < std::tie(o.a, o.b); }
};

// Per triple id (every triple of the call), the four frequency sums the
// contractions use under one permutation: z2', z1'+z2'+z3', z1'+z2', z2'+z3'.
struct PermSums {
    DevBuf buf;
    std::vector<cd> h;  // host copy: sum k of triple t at h[k * nfreq + t]
    int nfreq = 0;
    const cd* ds[4] = {nullptr, nullptr, nullptr, nullptr};
};

void build_sums(PermSums& ps, const int perm[3], int nfreq, const double* z, cudaStream_t st) {
    std::vector<cd> h(4 * (size_t)nfreq);
    for (int t = 0; t < nfreq; ++t) {
        cd a, b, c;
        perm_freqs(z, t, perm, a, b, c);
        h[t] = b;
        h[nfreq + t] = a + b + c;
        h[2 * (size_t)nfreq + t] = a + b;
        h[3 * (size_t)nfreq + t] = b + c;
    }
    ps.buf.reserve(std::max<size_t>(h.size(), 1) * sizeof(cd));
    if (!h.empty()) h2d(ps.buf.p, h.data(), h.size() * sizeof(cd), st);
    for (int k = 0; k < 4; ++k) ps.ds[k] = ps.buf.as<cd>() + (size_t)k * nfreq;
    ps.h = std::move(h);
    ps.nfreq = nfreq;
}

// Distinct z1' and z3' of all triples of a call under one permutation, in
// order of first appearance, and each triple's index into them.
struct PermIndex {
    std::vector<cd> Z1, Z3;
    std::vector<int> j1, j3;
};

void index_perm(PermIndex& ix, const int perm[3], int nfreq, const double* z) {
    std::map<KeyC, int> m1, m3;
    ix.j1.resize(nfreq);
    ix.j3.resize(nfreq);
    for (int t = 0; t < nfreq; ++t) {
        cd a, b, c;
        perm_freqs(z, t, perm, a, b, c);
        auto x1 = m1.emplace(KeyC{a.x, a.y}, (int)ix.Z1.size());
        if (x1.second) ix.Z1.push_back(a);
        auto x3 = m3.emplace(KeyC{c.x, c.y}, (int)ix.Z3.size());
        if (x3.second) ix.Z3.push_back(c);
        ix.j1[t] = x1.first->second;
        ix.j3[t] = x3.first->second;
    }
}

// The triples of one tile of a permutation's (z1', z3') plane: z1' indices
// [o1, o1 + n1) and z3' indices [o3, o3 + n3) of its PermIndex, the triples
// grouped by (z1', z3'), each group one warp's work in the contraction.
struct APlan {
    std::vector<cd> Z1, Z3;
    std::vector<int> gt, goff, gi1, gi3;  // triple ids grouped by (i1, i3)
    DevBuf buf;
    cd *dZ1 = nullptr, *dZ3 = nullptr;
    const cd* ds[4] = {nullptr, nullptr, nullptr, nullptr};  // the permutation's sums
    int *dgt = nullptr, *dgoff = nullptr, *dgi1 = nullptr, *dgi3 = nullptr;
    const PermSums* sums = nullptr;
    // contraction classes per frequency sum (built on first use), device
    // pointers in `cls` (term unset), storage in cbuf
    bool have_cls[4] = {false, false, false, false};
    std::vector<CClass> cls[4];
    DevBuf cbuf[4];
};

// Contraction classes of one plan for frequency sum k: the (z1, z3) groups
// whose triples carry the same sums (compared after rounding to 2^-46 of the
// largest |s|, so sums equal up to rounding share a class; the class uses its
// first group's values), columns ordered by sum, split into chunks of at most
// CG_BN_MAX columns.
void build_classes(APlan& pl, int k, cudaStream_t st) {
    if (pl.have_cls[k]) return;
    const PermSums& ps = *pl.sums;
    const cd* sv = ps.h.data() + (size_t)k * ps.nfreq;
    double smax = 0.0;
    for (int t : pl.gt) smax = std::max(smax, std::max(std::fabs(sv[t].x), std::fabs(sv[t].y)));
    const double q = smax > 0.0 ? std::ldexp(smax, -46) : 1.0;
    using Key = std::vector<std::pair<long long, long long>>;
    struct HC {
        std::vector<cd> s;
        std::vector<int> rows, slots;
    };
    std::map<Key, int> idx;
    std::vector<HC> hc;
    const int ng = (int)pl.gi1.size();
    std::vector<std::tuple<long long, long long, int>> el;
    for (int g = 0; g < ng; ++g) {
        el.clear();
        for (int u = pl.goff[g]; u < pl.goff[g + 1]; ++u) {
            const int t = pl.gt[u];
            el.emplace_back(std::llround(sv[t].x / q), std::llround(sv[t].y / q), t);
        }
        std::sort(el.begin(), el.end());
        Key key;
        key.reserve(el.size());
        for (auto& e : el) key.emplace_back(std::get<0>(e), std::get<1>(e));
        auto it = idx.find(key);
        if (it == idx.end()) {
            it = idx.emplace(std::move(key), (int)hc.size()).first;
            hc.emplace_back();
            for (auto& e : el) hc.back().s.push_back(sv[std::get<2>(e)]);
        }
        HC& c = hc[it->second];
        c.rows.push_back(g);
        for (auto& e : el) c.slots.push_back(std::get<2>(e));
    }
    // Classes of few rows (such as the z1 + z3 classes of the T2 sub-terms
    // near the grid's corners) make 8- or 16-row tiles that leave the FP64 pipe
    // idle.  Consecutive ones, in the order of their sum lists, are merged while
    // the union of their sums stays within CG_BN_MAX columns and their rows
    // within 64; a merged row holds -1 in the columns that are not its own, so
    // its tile computes those products and drops them.
    std::vector<HC> merged;
    {
        using QK = std::pair<long long, long long>;
        auto qk = [&](cd v) { return QK{std::llround(v.x / q), std::llround(v.y / q)}; };
        // groups of consecutive small classes under a row cap (sums within CG_BN_MAX)
        auto split_run = [&](const std::vector<int>& run, int cap) {
            std::vector<std::vector<int>> out;
            std::set<QK> uni;
            int rows = 0;
            for (int ci : run) {
                std::set<QK> u2 = uni;
                for (const cd& v : hc[ci].s) u2.insert(qk(v));
                const int r = (int)hc[ci].rows.size();
                if (!out.empty() && !out.back().empty() && ((int)u2.size() > CG_BN_MAX || rows + r > cap)) {
                    out.emplace_back();
                    uni.clear();
                    for (const cd& v : hc[ci].s) uni.insert(qk(v));
                    rows = 0;
                } else {
                    if (out.empty()) out.emplace_back();
                    uni = std::move(u2);
                }
                out.back().push_back(ci);
                rows += r;
            }
            return out;
        };
        auto emit = [&](const std::vector<int>& group) {
            if (group.size() == 1) {
                merged.push_back(std::move(hc[group[0]]));
                return;
            }
            std::map<QK, int> col;
            std::map<QK, cd> uni;
            for (int ci : group)
                for (const cd& v : hc[ci].s) uni.emplace(qk(v), v);
            HC m;
            for (auto& e : uni) {
                col[e.first] = (int)m.s.size();
                m.s.push_back(e.second);
            }
            const int w = (int)m.s.size();
            for (int ci : group) {
                const HC& c = hc[ci];
                const int nc = (int)c.s.size();
                for (size_t r = 0; r < c.rows.size(); ++r) {
                    m.rows.push_back(c.rows[r]);
                    const size_t base = m.slots.size();
                    m.slots.resize(base + w, -1);
                    for (int j = 0; j < nc; ++j) m.slots[base + col[qk(c.s[j])]] = c.slots[r * nc + j];
                }
            }
            merged.push_back(std::move(m));
        };
        // a run of consecutive small classes is cut into as few groups as 64
        // rows allow, then re-cut with the rows spread evenly over that many
        // groups, so that no group is left with a few rows
        auto flush_run = [&](std::vector<int>& run) {
            if (run.empty()) return;
            int total = 0, big = 0;
            for (int ci : run) {
                total += (int)hc[ci].rows.size();
                big = std::max(big, (int)hc[ci].rows.size());
            }
            const int ng = (int)split_run(run, 64).size();
            const int cap = std::max(big, (total + ng - 1) / ng);
            for (const auto& g : split_run(run, cap)) emit(g);
            run.clear();
        };
        std::vector<int> run;
        for (auto& e : idx) {  // classes in the order of their sum lists
            const int ci = e.second;
            const HC& c = hc[ci];
            std::set<QK> own;
            for (const cd& v : c.s) own.insert(qk(v));
            // large classes, and classes holding one sum twice (one column each
            // in a merged class would collide), stay as they are
            if (c.rows.size() > 16 || own.size() != c.s.size()) {
                flush_run(run);
                emit({ci});
                continue;
            }
            run.push_back(ci);
        }
        flush_run(run);
    }
    // column chunks, then one device buffer for every class of this sum
    std::vector<HC> fin;
    for (HC& c : merged) {
        const int nc = (int)c.s.size(), nr = (int)c.rows.size();
        for (int j0 = 0; j0 < nc; j0 += CG_BN_MAX) {
            const int w = std::min(CG_BN_MAX, nc - j0);
            HC f;
            f.s.assign(c.s.begin() + j0, c.s.begin() + j0 + w);
            f.rows = c.rows;
            f.slots.resize((size_t)nr * w);
            for (int r = 0; r < nr; ++r)
                for (int j = 0; j < w; ++j) f.slots[(size_t)r * w + j] = c.slots[(size_t)r * nc + j0 + j];
            fin.push_back(std::move(f));
        }
    }
    auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
    size_t bytes = 0;
    for (const HC& f : fin) bytes += al(f.s.size() * sizeof(cd)) + al(f.rows.size() * sizeof(int)) + al(f.slots.size() * sizeof(int));
    pl.cbuf[k].reserve(std::max<size_t>(bytes, 16));
    std::vector<char> host(std::max<size_t>(bytes, 16));
    char* dev = pl.cbuf[k].as<char>();
    size_t o = 0;
    for (const HC& f : fin) {
        CClass c{};
        c.term = -1;
        c.nrows = (int)f.rows.size();
        c.ncols = (int)f.s.size();
        std::memcpy(host.data() + o, f.s.data(), f.s.size() * sizeof(cd));
        c.s = reinterpret_cast<const cd*>(dev + o);
        o += al(f.s.size() * sizeof(cd));
        std::memcpy(host.data() + o, f.rows.data(), f.rows.size() * sizeof(int));
        c.rows = reinterpret_cast<const int*>(dev + o);
        o += al(f.rows.size() * sizeof(int));
        std::memcpy(host.data() + o, f.slots.data(), f.slots.size() * sizeof(int));
        c.slots = reinterpret_cast<const int*>(dev + o);
        o += al(f.slots.size() * sizeof(int));
        pl.cls[k].push_back(c);
    }
    if (bytes) h2d(dev, host.data(), bytes, st);
    pl.have_cls[k] = true;
}

void build_aplan(APlan& pl, const std::vector<int>& tids, const PermIndex& ix, int o1, int n1, int o3, int n3,
                 const PermSums& ps, cudaStream_t st) {
    pl.Z1.assign(ix.Z1.begin() + o1, ix.Z1.begin() + o1 + n1);
    pl.Z3.assign(ix.Z3.begin() + o3, ix.Z3.begin() + o3 + n3);
    const size_t nt = tids.size();
    pl.gt = tids;
    std::stable_sort(pl.gt.begin(), pl.gt.end(), [&](int x, int y) {
        return std::make_pair(ix.j1[x], ix.j3[x]) < std::make_pair(ix.j1[y], ix.j3[y]);
    });
    for (size_t q = 0; q < nt; ++q) {
        const int t = pl.gt[q];
        if (q == 0 || ix.j1[t] != ix.j1[pl.gt[q - 1]] || ix.j3[t] != ix.j3[pl.gt[q - 1]]) {
            pl.goff.push_back((int)q);
            pl.gi1.push_back(ix.j1[t] - o1);
            pl.gi3.push_back(ix.j3[t] - o3);
        }
    }
    pl.goff.push_back((int)nt);
    for (int k = 0; k < 4; ++k) pl.ds[k] = ps.ds[k];
    pl.sums = &ps;
    const size_t ng = pl.gi1.size();
    pl.buf.reserve((size_t)(n1 + n3) * sizeof(cd) + (nt + 3 * ng + 1) * sizeof(int) + 256);
    char* p = pl.buf.as<char>();
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 15) & ~size_t(15);
        return r;
    };
    pl.dZ1 = reinterpret_cast<cd*>(take((size_t)n1 * sizeof(cd)));
    pl.dZ3 = reinterpret_cast<cd*>(take((size_t)n3 * sizeof(cd)));
    pl.dgt = reinterpret_cast<int*>(take(nt * sizeof(int)));
    pl.dgoff = reinterpret_cast<int*>(take((ng + 1) * sizeof(int)));
    pl.dgi1 = reinterpret_cast<int*>(take(ng * sizeof(int)));
    pl.dgi3 = reinterpret_cast<int*>(take(ng * sizeof(int)));
    auto up = [&](void* d, const void* h, size_t b) {
        if (b) h2d(d, h, b, st);
    };
    up(pl.dZ1, pl.Z1.data(), (size_t)n1 * sizeof(cd));
    up(pl.dZ3, pl.Z3.data(), (size_t)n3 * sizeof(cd));
    up(pl.dgt, pl.gt.data(), nt * sizeof(int));
    up(pl.dgoff, pl.goff.data(), (ng + 1) * sizeof(int));
    up(pl.dgi1, pl.gi1.data(), ng * sizeof(int));
    up(pl.dgi3, pl.gi3.data(), ng * sizeof(int));
}

// Workspace of one chain inside a batch (element offsets into one cd pool).
struct ChainWs {
    long Lc, Lr, Pr, Pc, Rho, Qc, Rr, Rc, V1a, V1b, V2a, V2b, end;
};

// Frequency dressing of a Lehmann factor: the operator block (rows in block
// Sa, columns in Sb) divided elementwise by z - (E_Sb - E_Sa), with z taken
// per batch item from the plan's frequency list.
struct Dress {
    const double *Ea, *Eb;
    const cd* z;
};

// One product per frequency of a list (nb items): only the output moves, by
// bc elements per item; the dressed operand takes the item's frequency.
template <typename TA, typename TB>
GemmProblem<TA, TB, cd> gp(const typename src_t<TA>::type* A, long sai, long sak, const typename src_t<TB>::type* B,
                           long sbk, long sbj, cd* C, long sci, int M, int N, int K, const int* aii, const int* bjj,
                           Dress dr, int nb, long bc, long scj = 1) {
    GemmProblem<TA, TB, cd> g{};
    g.A = A;
    g.B = B;
    g.C = C;
    g.M = M;
    g.N = N;
    g.K = K;
    g.sa_i = sai;
    g.sa_k = sak;
    g.sb_k = sbk;
    g.sb_j = sbj;
    g.sc_i = sci;
    g.sc_j = scj;
    g.a_iidx = aii;
    g.b_jidx = bjj;
    g.dEa = dr.Ea;
    g.dEb = dr.Eb;
    g.dzs = dr.z;
    g.nb = nb;
    g.bc = bc;
    return g;
}

}  // namespace

template <typename T>
static void run_batch(pgx_ctx* c, const std::vector<int>& idx, const std::vector<int>& bplan,
                      const std::vector<ChainWs>& wsl, const pgx_g2_part* parts, std::vector<APlan>& plans,
                      const std::vector<std::array<int, 4>>& rs, cd* pool, const int* d_hot,
                      const std::vector<long>& hot_off, double pole_res, int split, const std::vector<int>& bdig,
                      cd* d_out) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    constexpr bool TC = is_cd<T>::value;
    // ---- anchored products per frequency and stacked products per (z1, z3);
    // A1(z1) = O1 / (z1 - (E2 - E1)) and C3(z3) = O3 / (z3 - (E4 - E3)) are
    // dressed inside the GEMM tile loads (Dressed<T> operands)
    using DT = Dressed<T>;
    std::vector<GemmProblem<T, DT, cd>> pa;   // operator x dressed
    std::vector<GemmProblem<DT, T, cd>> pb;   // dressed x operator
    std::vector<GemmProblem<DT, cd, cd>> pc;  // dressed x stacked anchors (per z1 or z3)
    std::vector<GemmProblem<cd, DT, cd>> pd;  // stacked anchors x dressed
    // digits of each split product: those of its anchor block (bdig)
    std::vector<int> pa_d, pb_d, pc_d, pd_d;
    auto push = [&](auto& list, std::vector<int>& digs, int anchor_block, const auto& prob) {
        list.push_back(prob);
        digs.push_back(bdig.empty() ? split : bdig[anchor_block]);
    };
    for (size_t j = 0; j < idx.size(); ++j) {
        const int q = idx[j];
        const pgx_g2_part& g = parts[q];
        const APlan& pl = plans[bplan[j]];
        const ChainWs& w = wsl[j];
        const int S1 = g.block[0], S2 = g.block[1], S3 = g.block[2], S4 = g.block[3];
        const int d1 = P.dims[S1], d2 = P.dims[S2], d3 = P.dims[S3], d4 = P.dims[S4];
        const int r1 = rs[q][0], r2 = rs[q][1], r3 = rs[q][2], r4 = rs[q][3];
        const int N1 = (int)pl.Z1.size(), N3 = (int)pl.Z3.size();
        const Operator &o1 = P.ops[g.op[0]], &o2 = P.ops[g.op[1]], &o3 = P.ops[g.op[2]], &o4 = P.ops[g.op[3]];
        const T* O1 = o1.mat.as<T>() + o1.parts[o1.by_left[S1]].off;
        const T* O2 = o2.mat.as<T>() + o2.parts[o2.by_left[S2]].off;
        const T* O3 = o3.mat.as<T>() + o3.parts[o3.by_left[S3]].off;
        const T* X4 = o4.mat.as<T>() + o4.parts[o4.by_left[S4]].off;
        const double *E1 = P.d_E + P.eoff[S1], *E2 = P.d_E + P.eoff[S2], *E3 = P.d_E + P.eoff[S3],
                     *E4 = P.d_E + P.eoff[S4];
        const int *H1 = d_hot + hot_off[S1], *H2 = d_hot + hot_off[S2], *H3 = d_hot + hot_off[S3], *H4 = d_hot + hot_off[S4];
        const Dress A1{E1, E2, pl.dZ1};  // A1(z1) = O1 dressed with z1: d1 x d2, row-major
        const Dress C3{E3, E4, pl.dZ3};  // C3(z3) = O3 dressed with z3: d3 x d4, row-major
        // anchored products, one item per z1 (or z3)
        // outputs that the contractions read along k are stored k-contiguous
        if (r2) push(pa, pa_d, S2, gp<T, DT>(X4, d1, 1, O1, d2, 1, pool + w.Lc, 1, d4, r2, d1, nullptr, H2, A1, N1,
                                       (long)r2 * d4, d4));                               // Lc = X4 A1[:,H2]: [(i1,h)][k]
        if (r4) push(pa, pa_d, S4, gp<T, DT>(X4, d1, 1, O1, d2, 1, pool + w.Lr, d2, r4, d2, d1, H4, nullptr, A1, N1,
                                       (long)r4 * d2));                                   // Lr = X4[H4,:] A1
        if (r1) push(pb, pb_d, S1, gp<DT, T>(O1, d2, 1, O2, d3, 1, pool + w.Pr, d3, r1, d3, d2, H1, nullptr, A1, N1,
                                       (long)r1 * d3));                                   // Pr = A1[H1,:] O2
        if (r3) push(pb, pb_d, S3, gp<DT, T>(O1, d2, 1, O2, d3, 1, pool + w.Pc, 1, d1, r3, d2, nullptr, H3, A1, N1,
                                       (long)d1 * r3, d1));                               // Pc = A1 O2[:,H3]: [i1][h][k]
        if (r3) push(pb, pb_d, S3, gp<DT, T>(O3, d4, 1, X4, d1, 1, pool + w.Rho, d1, r3, d1, d4, H3, nullptr, C3, N3,
                                       (long)r3 * d1));                                   // rho = C3[H3,:] X4
        if (r1) push(pb, pb_d, S1, gp<DT, T>(O3, d4, 1, X4, d1, 1, pool + w.Qc, 1, d3, r1, d4, nullptr, H1, C3, N3,
                                       (long)d3 * r1, d3));                               // Qc = C3 X4[:,H1]: [i3][h][k]
        if (r2) push(pa, pa_d, S2, gp<T, DT>(O2, d3, 1, O3, d4, 1, pool + w.Rr, d4, r2, d4, d3, H2, nullptr, C3, N3,
                                       (long)r2 * d4));                                   // Rr = O2[H2,:] C3
        if (r4) push(pa, pa_d, S4, gp<T, DT>(O2, d3, 1, O3, d4, 1, pool + w.Rc, 1, d2, r4, d3, nullptr, H4, C3, N3,
                                       (long)r4 * d2, d2));                               // Rc = O2 C3[:,H4]: [(i3,h)][k]
        // products over (z1, z3): anchors of all frequencies stacked as columns / rows
        if (r2) push(pc, pc_d, S2, gp<DT, cd>(O3, d4, 1, pool + w.Lc, 1, d4, pool + w.V1a, 1, d3, N1 * r2, d4, nullptr,
                                        nullptr, C3, N3, (long)d3 * N1 * r2, d3));  // V1a = C3 LcAll: [i3][(i1,h)][k]
        if (r1) push(pd, pd_d, S1, gp<cd, DT>(pool + w.Pr, d3, 1, O3, d4, 1, pool + w.V2a, d4, N1 * r1, d4, d3, nullptr, nullptr,
                                        C3, N3, (long)N1 * r1 * d4));                         // V2a = PrAll C3
        if (r3) push(pd, pd_d, S3, gp<cd, DT>(pool + w.Rho, d1, 1, O1, d2, 1, pool + w.V1b, d2, N3 * r3, d2, d1, nullptr, nullptr,
                                        A1, N1, (long)N3 * r3 * d2));                         // V1b = rhoAll A1
        if (r4) push(pc, pc_d, S4, gp<DT, cd>(O1, d2, 1, pool + w.Rc, 1, d2, pool + w.V2b, 1, d1, N3 * r4, d2, nullptr,
                                        nullptr, A1, N1, (long)d1 * N3 * r4, d1));  // V2b = A1 RcAll: [i1][(i3,h)][k]
    }
    // descriptor buffers: one region per product list, sized once for the
    // largest list before any launch, so that lists on different streams do
    // not share one
    const long nprob = std::max<long>(1, (long)std::max({pa.size(), pb.size(), pc.size(), pd.size()}));
    const size_t preg = ((size_t)nprob * sizeof(GemmProblem<cd, cd, cd>) + 255) & ~size_t(255);
    const size_t ireg = (gemm_index_bytes(nprob) + 255) & ~size_t(255);
    c->scratch[7].reserve(4 * preg);
    c->scratch[8].reserve(4 * ireg);
    auto launch_on = [&](auto& probs, int region, cudaStream_t s2) {
        if (probs.empty()) return;
        launch_gemm_batch(probs, c->scratch[7].as<char>() + region * preg, preg, c->scratch[8].as<char>() + region * ireg,
                          ireg, s2);
    };
    // The stacked products read Lc, Pr, rho and Rc written by the first two
    // lists.  With `split` slices, products of at least g2_split_min_macs
    // complex multiply-adds (default 1e9) go to the int8 tensor cores: smaller
    // ones, such as every product of a 400-state block, run faster on the FP64
    // tiles than their digit preparation and 128 x 256 tile padding allow.
    // Complex Hamiltonians keep the anchored products in FP64.
    auto launch_split = [&](auto& probs, const std::vector<int>& digs, int region) {
        std::remove_reference_t<decltype(probs)> rest;
        for (size_t i = 0; i < probs.size(); ++i) {
            const auto& g = probs[i];
            const double macs = (double)g.M * g.N * g.K * std::max(g.nb, 1);
            if (macs < c->g2_split_min_macs) {
                rest.push_back(g);
                continue;
            }
            oz_zgemm(g, digs[i], c->oz, st);
        }
        launch_on(rest, region, st);
    };
    if (split) {  // the split products share one workspace: one stream
        if constexpr (TC) {
            launch_on(pa, 0, st);
            launch_on(pb, 1, st);
        } else {
            launch_split(pa, pa_d, 0);
            launch_split(pb, pb_d, 1);
        }
        launch_split(pc, pc_d, 2);
        launch_split(pd, pd_d, 3);
    } else {
        // pa and pb are independent, and so are pc and pd (each needs both of
        // the first pair): each pair runs on two side streams at once
        ensure_side_streams(c);
        cudaStream_t s0 = c->aux[0], s1 = c->aux[1];
        PGX_CUDA(cudaEventRecord(c->fork, st));
        PGX_CUDA(cudaStreamWaitEvent(s0, c->fork, 0));
        PGX_CUDA(cudaStreamWaitEvent(s1, c->fork, 0));
        SideJoin join(c, st, 2);  // st waits for both side streams on every exit
        launch_on(pa, 0, s0);
        launch_on(pb, 1, s1);
        PGX_CUDA(cudaEventRecord(c->join[0], s0));
        PGX_CUDA(cudaEventRecord(c->join[1], s1));
        PGX_CUDA(cudaStreamWaitEvent(s0, c->join[1], 0));
        PGX_CUDA(cudaStreamWaitEvent(s1, c->join[0], 0));
        launch_on(pc, 2, s0);
        launch_on(pd, 3, s1);
    }
    // ---- contractions per triple
    std::vector<DTerm> dt;
    for (size_t j = 0; j < idx.size(); ++j) {
        const int q = idx[j];
        const pgx_g2_part& g = parts[q];
        const APlan& pl = plans[bplan[j]];
        const ChainWs& w = wsl[j];
        const int S[4] = {g.block[0], g.block[1], g.block[2], g.block[3]};
        const int d1 = P.dims[S[0]], d2 = P.dims[S[1]], d3 = P.dims[S[2]], d4 = P.dims[S[3]];
        const int r1 = rs[q][0], r2 = rs[q][1], r3 = rs[q][2], r4 = rs[q][3];
        const long N1 = (long)pl.Z1.size(), N3 = (long)pl.Z3.size();
        const Operator &o2 = P.ops[g.op[1]], &o4 = P.ops[g.op[3]];
        const T* O2 = o2.mat.as<T>() + o2.parts[o2.by_left[S[1]]].off;
        const T* X4 = o4.mat.as<T>() + o4.parts[o4.by_left[S[3]]].off;
        const double* E[4];
        const double* W[4];
        for (int k = 0; k < 4; ++k) {
            E[k] = P.d_E + P.eoff[S[k]];
            W[k] = P.d_w + P.eoff[S[k]];
        }
        const double sign = g.sign;
        auto base = [&](int anchor, int nh, int nk, int kb, double sgn, int sidx, int use_delta, double cd_, double cn,
                        double pref) {
            DTerm d{};
            d.Ek = E[kb];
            d.Eh = E[anchor];
            d.wh = W[anchor];
            d.hot = d_hot + hot_off[S[anchor]];
            d.nh = nh;
            d.nk = nk;
            d.gi1 = pl.dgi1;
            d.gi3 = pl.dgi3;
            d.plan = bplan[j];
            d.sidx = sidx;
            d.sgn = sgn;
            d.use_delta = use_delta;
            d.cdelta = cd_;
            d.cnum = cn;
            d.pref = pref;
            return d;
        };
        const int opc = TC ? 1 : 0;
        if (r2) {  // T1a: va = O2[h,k] (state h), vb = V1a[i3][(i1,h)][k]
            DTerm d = base(1, r2, d3, 2, +1.0, 0, 0, 0.0, 1.0, -sign);
            d.VA = O2; d.va_cplx = opc; d.va_hstate = 1; d.ah = d3; d.ak = 1;
            d.VB = pool + w.V1a; d.vb_cplx = 1; d.b3 = (long)d3 * N1 * r2; d.bk = 1; d.b1 = (long)r2 * d3; d.bh = d3;
            dt.push_back(d);
            // T4a: va = Rr[i3][h][k], vb = Lc[(i1,h)][k]
            DTerm e = base(1, r2, d4, 3, +1.0, 3, 1, -1.0, 1.0, sign);
            e.VA = pool + w.Rr; e.va_cplx = 1; e.a3 = (long)r2 * d4; e.ah = d4; e.ak = 1;
            e.VB = pool + w.Lc; e.vb_cplx = 1; e.bk = 1; e.b1 = (long)r2 * d4; e.bh = d4;
            dt.push_back(e);
        }
        if (r3) {  // T1b: va = O2[k,h] (state h), vb = V1b[i1][(i3,h)][k]
            DTerm d = base(2, r3, d2, 1, -1.0, 0, 0, 0.0, 1.0, -sign);
            d.VA = O2; d.va_cplx = opc; d.va_hstate = 1; d.ah = 1; d.ak = d3;
            d.VB = pool + w.V1b; d.vb_cplx = 1; d.b1 = N3 * r3 * d2; d.b3 = (long)r3 * d2; d.bh = d2; d.bk = 1;
            dt.push_back(d);
            // T3b: va = Pc[i1][h][k], vb = rho[(i3,h)][k]
            DTerm e = base(2, r3, d1, 0, -1.0, 2, 1, 0.0, 1.0, sign);
            e.VA = pool + w.Pc; e.va_cplx = 1; e.a1 = (long)d1 * r3; e.ak = 1; e.ah = d1;
            e.VB = pool + w.Rho; e.vb_cplx = 1; e.b3 = (long)r3 * d1; e.bh = d1; e.bk = 1;
            dt.push_back(e);
        }
        if (r1) {  // T2a: va = X4[k,h] (state h), vb = V2a[i3][(i1,h)][k]
            DTerm d = base(0, r1, d4, 3, +1.0, 1, 0, 0.0, 1.0, sign);
            d.VA = X4; d.va_cplx = opc; d.va_hstate = 1; d.ah = 1; d.ak = d1;
            d.VB = pool + w.V2a; d.vb_cplx = 1; d.b3 = N1 * r1 * d4; d.b1 = (long)r1 * d4; d.bh = d4; d.bk = 1;
            dt.push_back(d);
            // T3a: va = PrAll[(i1,h)][k], vb = Qc[i3][h][k]
            DTerm e = base(0, r1, d3, 2, +1.0, 2, 1, 1.0, -1.0, sign);
            e.VA = pool + w.Pr; e.va_cplx = 1; e.a1 = (long)r1 * d3; e.ah = d3; e.ak = 1;
            e.VB = pool + w.Qc; e.vb_cplx = 1; e.b3 = (long)d3 * r1; e.bk = 1; e.bh = d3;
            dt.push_back(e);
        }
        if (r4) {  // T2b: va = X4[h,k] (state h), vb = V2b[i1][(i3,h)][k]
            DTerm d = base(3, r4, d1, 0, -1.0, 1, 0, 0.0, 1.0, sign);
            d.VA = X4; d.va_cplx = opc; d.va_hstate = 1; d.ah = d1; d.ak = 1;
            d.VB = pool + w.V2b; d.vb_cplx = 1; d.b1 = (long)d1 * N3 * r4; d.bk = 1; d.b3 = (long)r4 * d1; d.bh = d1;
            dt.push_back(d);
            // T4b: va = Rc[(i3,h)][k], vb = Lr[i1][h][k]
            DTerm e = base(3, r4, d2, 1, -1.0, 3, 1, 0.0, -1.0, sign);
            e.VA = pool + w.Rc; e.va_cplx = 1; e.ak = 1; e.a3 = (long)r4 * d2; e.ah = d2;
            e.VB = pool + w.Lr; e.vb_cplx = 1; e.b1 = (long)r4 * d2; e.bh = d2; e.bk = 1;
            dt.push_back(e);
        }
    }
    if (!dt.empty()) {
        // classes of every sub-term, grouped by tile shape (BM 32 or 64 rows,
        // BN 8 / 16 / 24 / 32 columns); a work item is one row tile of a class
        // over a range of anchors, about 2^22 complex multiply-adds
        std::vector<CClass> cls[CG_NBM][CG_NBN];
        std::vector<CItem> its[CG_NBM][CG_NBN];
        double macs[CG_NBM][CG_NBN] = {};
        for (size_t q = 0; q < dt.size(); ++q) {
            const DTerm& d = dt[q];
            APlan& pl = plans[d.plan];
            build_classes(pl, d.sidx, st);
            for (const CClass& c0 : pl.cls[d.sidx]) {
                int bm = 0, bn = 0;
                while (bm < CG_NBM - 1 && CG_BMS[bm] < c0.nrows) ++bm;
                while (CG_BNS[bn] < c0.ncols) ++bn;
                const int BM = CG_BMS[bm], BN = CG_BNS[bn];
                CClass c = c0;
                c.term = (int)q;
                const int ci = (int)cls[bm][bn].size();
                cls[bm][bn].push_back(c);
                const int hc = (int)std::max<long>(1, (1L << 22) / ((long)BM * BN * std::max(d.nk, 1)));
                for (int r0 = 0; r0 < c.nrows; r0 += BM)
                    for (int h0 = 0; h0 < d.nh; h0 += hc) its[bm][bn].push_back(CItem{ci, r0, h0, std::min(d.nh, h0 + hc)});
                macs[bm][bn] += (double)c.nrows * c.ncols * d.nh * d.nk;
            }
        }
        size_t bytes = ((dt.size() * sizeof(DTerm) + 255) & ~size_t(255));
        for (int a = 0; a < CG_NBM; ++a)
            for (int b = 0; b < CG_NBN; ++b)
                bytes += ((cls[a][b].size() * sizeof(CClass) + 255) & ~size_t(255)) +
                         ((its[a][b].size() * sizeof(CItem) + 255) & ~size_t(255));
        DevBuf& bd = c->scratch[3];
        bd.reserve(bytes);
        char* base_p = bd.as<char>();
        size_t o = 0;
        auto put = [&](const void* h, size_t n) {
            char* d = base_p + o;
            if (n) h2d(d, h, n, st);
            o += (n + 255) & ~size_t(255);
            return d;
        };
        const DTerm* d_terms = reinterpret_cast<const DTerm*>(put(dt.data(), dt.size() * sizeof(DTerm)));
        // profiler ranges per tile shape; 8 FP64 operations per complex
        // multiply-add of (h, k, triple)
        static const char* const kName[CG_NBM][CG_NBN] = {
            {"contract_gemm_kernel<8,8>", "contract_gemm_kernel<8,16>", "contract_gemm_kernel<8,24>",
             "contract_gemm_kernel<8,32>"},
            {"contract_gemm_kernel<16,8>", "contract_gemm_kernel<16,16>", "contract_gemm_kernel<16,24>",
             "contract_gemm_kernel<16,32>"},
            {"contract_gemm_kernel<24,8>", "contract_gemm_kernel<24,16>", "contract_gemm_kernel<24,24>",
             "contract_gemm_kernel<24,32>"},
            {"contract_gemm_kernel<32,8>", "contract_gemm_kernel<32,16>", "contract_gemm_kernel<32,24>",
             "contract_gemm_kernel<32,32>"},
            {"contract_gemm_kernel<64,8>", "contract_gemm_kernel<64,16>", "contract_gemm_kernel<64,24>",
             "contract_gemm_kernel<64,32>"}};
        const double tol2 = pole_res * pole_res;
        for (int a = 0; a < CG_NBM; ++a)
            for (int b = 0; b < CG_NBN; ++b) {
                if (its[a][b].empty()) continue;
                ProfRange pr(kName[a][b], st, 8.0 * macs[a][b], 0.0);
                PGX_CHECK(its[a][b].size() < (1u << 31), PGX_ERR_ARG, "G2 contraction: too many work items");
                const CClass* dc = reinterpret_cast<const CClass*>(put(cls[a][b].data(), cls[a][b].size() * sizeof(CClass)));
                const CItem* di = reinterpret_cast<const CItem*>(put(its[a][b].data(), its[a][b].size() * sizeof(CItem)));
                const unsigned n = (unsigned)its[a][b].size();
                launch_contract(CG_BMS[a], CG_BNS[b], n, st, d_terms, dc, di, P.beta, tol2, d_out);
            }
        check_launch("contract_gemm_kernel");
    }
    // the next batch reuses the device descriptor buffers in stream order
}

void run_g2_anchored(pgx_ctx* c, int nparts, const pgx_g2_part* parts, int nfreq, const double* z, double pole_res,
                     double anchor_tol, int split, double* out) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    // anchor states per block (weights above the threshold)
    const std::vector<double>& w = P.w_host;  // copied when the weights were computed
    PGX_CHECK((long)w.size() == P.esize, PGX_ERR_STATE, "pgx_weights first");
    std::vector<int> hot;
    std::vector<long> hot_off(P.nblocks + 1, 0);
    std::vector<int> nhot(P.nblocks, 0);
    for (int b = 0; b < P.nblocks; ++b) {
        hot_off[b] = (long)hot.size();
        for (int i = 0; i < P.dims[b]; ++i)
            if (w[P.eoff[b] + i] > anchor_tol) hot.push_back(i);
        nhot[b] = (int)(hot.size() - hot_off[b]);
    }
    hot_off[P.nblocks] = (long)hot.size();
    // Digits of the split products per anchor block.  A product's error
    // reaches G2 multiplied by the Boltzmann weights of its anchor states, so a
    // block whose largest weight is a factor 254^k below the overall largest
    // (with the budget F of pgx_set_g2_split_weight_budget as allowance) drops
    // k digits, each of which multiplies the product's error by about 254: no
    // product then carries more than F times the error of a product of the
    // dominant block at the full digit count.  At least 3 digits are kept.
    std::vector<int> bdig;
    if (split > 0 && c->g2_split_weight_budget > 0.0) {
        double wall = 0.0;
        std::vector<double> wb(P.nblocks, 0.0);
        for (int b = 0; b < P.nblocks; ++b)
            for (int i = 0; i < P.dims[b]; ++i) wb[b] = std::max(wb[b], w[P.eoff[b] + i]);
        for (double x : wb) wall = std::max(wall, x);
        bdig.assign(P.nblocks, split);
        for (int b = 0; b < P.nblocks; ++b) {
            if (!(wb[b] > 0.0) || !(wall > 0.0)) continue;
            const int k = (int)std::floor(std::log(c->g2_split_weight_budget * wall / wb[b]) / std::log(254.0));
            bdig[b] = std::max(std::min(3, split), split - std::max(0, k));
        }
    }
    DevBuf& bh = c->scratch[11];
    bh.reserve(std::max<size_t>(hot.size(), 1) * sizeof(int));
    if (!hot.empty()) h2d(bh.p, hot.data(), hot.size() * sizeof(int), st);
    // permutations of the parts, and the frequency sums of each
    std::map<std::tuple<int, int, int>, int> perm_id;
    std::vector<std::array<int, 3>> perms;
    std::vector<int> part_perm(nparts);
    for (int q = 0; q < nparts; ++q) {
        auto key = std::make_tuple(parts[q].perm[0], parts[q].perm[1], parts[q].perm[2]);
        auto it = perm_id.find(key);
        if (it == perm_id.end()) {
            it = perm_id.emplace(key, (int)perms.size()).first;
            perms.push_back({parts[q].perm[0], parts[q].perm[1], parts[q].perm[2]});
        }
        part_perm[q] = it->second;
    }
    std::vector<PermSums> sums(perms.size());
    for (size_t p = 0; p < perms.size(); ++p) build_sums(sums[p], perms[p].data(), nfreq, z, st);
    // anchor counts per part, and the workspace of one chain for N1 x N3 frequencies
    std::vector<std::array<int, 4>> rs(nparts);
    for (int q = 0; q < nparts; ++q)
        for (int k = 0; k < 4; ++k) rs[q][k] = nhot[parts[q].block[k]];
    auto chain_ws = [&](int q, long N1, long N3) {
        int d[4];
        for (int k = 0; k < 4; ++k) d[k] = P.dims[parts[q].block[k]];
        const auto& r = rs[q];
        ChainWs x{};
        long o = 0;
        auto take = [&](long n) {
            long r0 = o;
            o += (n + 1) & ~1L;  // keep 32-byte alignment of complex doubles
            return r0;
        };
        x.Lc = take((long)d[3] * N1 * r[1]);
        x.Lr = take(N1 * r[3] * d[1]);
        x.Pr = take(N1 * r[0] * d[2]);
        x.Pc = take(N1 * d[0] * r[2]);
        x.Rho = take(N3 * r[2] * d[0]);
        x.Qc = take(N3 * d[2] * r[0]);
        x.Rr = take(N3 * r[1] * d[3]);
        x.Rc = take((long)d[1] * N3 * r[3]);
        x.V1a = take(N3 * d[2] * N1 * r[1]);
        x.V1b = take(N1 * N3 * r[2] * d[1]);
        x.V2a = take(N3 * N1 * r[0] * d[3]);
        x.V2b = take(N1 * d[0] * N3 * r[3]);
        x.end = o;
        return x;
    };
    auto active = [&](int q) { return rs[q][0] + rs[q][1] + rs[q][2] + rs[q][3] > 0; };
    // Parts are batched up to `budget` of workspace.  One chain may take up to
    // `tile_budget` (by default half the free device memory, at most 48 GiB); beyond it
    // the permutation's (z1', z3') plane is cut into tiles, each with all of
    // its triples' z2'.  The stacked products are per (z1', z3') pair, so
    // tiling does not repeat them; the per-z1' and per-z3' anchored products
    // are repeated once per tile row or column.
    const long budget = (long)((c->g2_batch_bytes > 0 ? c->g2_batch_bytes : (3LL << 30)) / (long long)sizeof(cd));
    long tile_budget = -1;  // resolved when a chain exceeds the batch budget
    auto chain_limit = [&]() {
        if (tile_budget >= 0) return tile_budget;
        if (c->g2_chain_bytes > 0) {
            tile_budget = (long)(c->g2_chain_bytes / (long long)sizeof(cd));
        } else {
            size_t free_b = 0, total_b = 0;
            PGX_CUDA(cudaMemGetInfo(&free_b, &total_b));
            tile_budget = std::max(budget, (long)(std::min<size_t>(free_b / 2, size_t(48) << 30) / sizeof(cd)));
        }
        return tile_budget;
    };
    std::vector<APlan> plans;
    std::vector<std::vector<int>> perm_plans(perms.size());
    for (size_t p = 0; p < perms.size(); ++p) {
        PermIndex ix;
        index_perm(ix, perms[p].data(), nfreq, z);
        const long N1 = (long)ix.Z1.size(), N3 = (long)ix.Z3.size();
        auto fits = [&](long b) {
            for (int q = 0; q < nparts; ++q) {
                if (part_perm[q] != (int)p || !active(q)) continue;
                const long e = chain_ws(q, std::min(N1, b), std::min(N3, b)).end;
                if (e > budget && e > chain_limit()) return false;
            }
            return true;
        };
        long B = std::max<long>(1, std::max(N1, N3));
        while (B > 1 && !fits(B)) B = std::max<long>(1, std::min(B - 1, B * 3 / 4));
        const long T1 = ceil_div(std::max<long>(N1, 1), std::min(std::max<long>(N1, 1), B));
        const long T3 = ceil_div(std::max<long>(N3, 1), std::min(std::max<long>(N3, 1), B));
        const long b1 = ceil_div(std::max<long>(N1, 1), T1), b3 = ceil_div(std::max<long>(N3, 1), T3);
        std::vector<std::vector<int>> tiles((size_t)(T1 * T3));
        if (T1 * T3 == 1) {
            tiles[0].resize(nfreq);
            for (int t = 0; t < nfreq; ++t) tiles[0][t] = t;
        } else {
            for (int t = 0; t < nfreq; ++t) tiles[(size_t)((ix.j1[t] / b1) * T3 + ix.j3[t] / b3)].push_back(t);
        }
        for (long u = 0; u < T1; ++u)
            for (long v = 0; v < T3; ++v) {
                const auto& tl = tiles[(size_t)(u * T3 + v)];
                if (tl.empty()) continue;
                const int o1 = (int)(u * b1), o3 = (int)(v * b3);
                const int n1 = (int)std::min(b1, N1 - o1), n3 = (int)std::min(b3, N3 - o3);
                perm_plans[p].push_back((int)plans.size());
                plans.emplace_back();
                build_aplan(plans.back(), tl, ix, o1, n1, o3, n3, sums[p], st);
            }
    }
    DevBuf& pool_b = c->scratch[6];
    DevBuf& out_b = c->scratch[9];
    out_b.reserve(std::max(nfreq, 1) * sizeof(cd));
    PGX_CUDA(cudaMemsetAsync(out_b.p, 0, std::max(nfreq, 1) * sizeof(cd), st));
    std::vector<int> batch, bplan;
    std::vector<ChainWs> bws;
    long used = 0;
    auto flush = [&]() {
        if (batch.empty()) return;
        pool_b.reserve(std::max<long>(used, 1) * sizeof(cd));
        if (P.is_complex)
            run_batch<cd>(c, batch, bplan, bws, parts, plans, rs, pool_b.as<cd>(), bh.as<int>(), hot_off, pole_res,
                          split, bdig, out_b.as<cd>());
        else
            run_batch<double>(c, batch, bplan, bws, parts, plans, rs, pool_b.as<cd>(), bh.as<int>(), hot_off, pole_res,
                              split, bdig, out_b.as<cd>());
        batch.clear();
        bplan.clear();
        bws.clear();
        used = 0;
    };
    for (size_t p = 0; p < perms.size(); ++p)
        for (int pid : perm_plans[p])
            for (int q = 0; q < nparts; ++q) {
                if (part_perm[q] != (int)p || !active(q)) continue;
                ChainWs x = chain_ws(q, (long)plans[pid].Z1.size(), (long)plans[pid].Z3.size());
                if (used > 0 && used + x.end > budget) flush();
                for (long* f : {&x.Lc, &x.Lr, &x.Pr, &x.Pc, &x.Rho, &x.Qc, &x.Rr, &x.Rc, &x.V1a, &x.V1b, &x.V2a,
                                &x.V2b, &x.end})
                    *f += used;
                used = x.end;
                batch.push_back(q);
                bplan.push_back(pid);
                bws.push_back(x);
            }
    flush();
    PGX_CUDA(cudaMemcpyAsync(out, out_b.p, nfreq * sizeof(cd), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
}

}  // namespace pgx
