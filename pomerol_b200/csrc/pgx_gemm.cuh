// Batched FP64 (real / complex) GEMM over a flat tile list.
//
// One launch covers many independent products of uneven shapes (symmetry
// blocks of different sizes, frequency batches): the host builds a list of
// (problem, tile_m, tile_n) entries and the grid walks it, so no CTA idles
// on an empty tile of a small block.  Operands are addressed through
// arbitrary (row, column) strides, so transposes cost nothing, and the
// reduction index k may be gathered through index arrays with a per-k scale
// (the signed row gather of a fermionic operator).
#pragma once

#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "pgx_common.cuh"
#include "pgx_internal.h"

namespace pgx {

// An operand declared Dressed<T> is stored as the operator block X (type T,
// rows a, columns b in the block's own orientation) and enters the product as
// the complex matrix X[a][b] / (z - (Eb[b] - Ea[a])): the frequency dressing of
// a Lehmann factor, computed as the tile is loaded instead of materialised.
template <typename T> struct Dressed {};
template <typename T> struct is_dressed : std::false_type {};
template <typename T> struct is_dressed<Dressed<T>> : std::true_type {};
template <typename T> struct src_t { using type = T; };
template <typename T> struct src_t<Dressed<T>> { using type = T; };
template <typename T> struct val_t { using type = T; };
template <typename T> struct val_t<Dressed<T>> { using type = cd; };

template <typename TA, typename TB, typename TC> struct GemmProblem {
    const typename src_t<TA>::type* A;
    const typename src_t<TB>::type* B;
    TC* C;
    int M, N, K;
    long sa_i, sa_k;   // A(i,k) = A[i*sa_i + k'*sa_k], k' = a_kidx ? a_kidx[k] : k
    long sb_k, sb_j;   // B(k,j) = B[k''*sb_k + j*sb_j], k'' = b_kidx ? b_kidx[k] : k
    long sc_i, sc_j;
    const int* a_kidx;
    const int* b_kidx;
    const double* kscale;  // multiplies B(k, :) when non-null
    int accumulate;        // C += A B instead of C = A B
    int conj_a;            // use conj(A) (complex A only)
    const int* a_iidx;     // row gather of A: A(i,k) uses row a_iidx[i] (nullable)
    const int* b_jidx;     // column gather of B: B(k,j) uses column b_jidx[j] (nullable)
    const double* dEa;     // dressing of the Dressed<T> operand: energies of its rows,
    const double* dEb;     // of its columns (after the gathers),
    cd dz;                 // and the frequency (or dzs[b] for batch item b when dzs is set)
    // batch of nb products with the same shapes (nb <= 0 counts as 1): item b
    // uses A + b*ba, B + b*bb, C + b*bc
    int nb;
    long ba, bb, bc;
    const cd* dzs;
};

// Bytes of the per-class tile index a launch_gemm_batch of nprobs problems needs.
inline size_t gemm_index_bytes(size_t nprobs) { return (nprobs + 16) * sizeof(int); }

__device__ __forceinline__ void mac(double& c, double a, double b) { c = fma(a, b, c); }
__device__ __forceinline__ void mac(cd& c, cd a, double b) {
    c.x = fma(a.x, b, c.x);
    c.y = fma(a.y, b, c.y);
}
__device__ __forceinline__ void mac(cd& c, double a, cd b) {
    c.x = fma(a, b.x, c.x);
    c.y = fma(a, b.y, c.y);
}
__device__ __forceinline__ void mac(cd& c, cd a, cd b) {
    c.x = fma(a.x, b.x, c.x);
    c.x = fma(-a.y, b.y, c.x);
    c.y = fma(a.x, b.y, c.y);
    c.y = fma(a.y, b.x, c.y);
}
template <typename T> __device__ __forceinline__ cd dress(T x, double ea, double eb, cd z) {
    return tocd(x) * inv_fast(cd{z.x - (eb - ea), z.y});
}
__device__ __forceinline__ double scale_by(double a, double s) { return a * s; }
__device__ __forceinline__ cd scale_by(cd a, double s) { return cd{a.x * s, a.y * s}; }
__device__ __forceinline__ double maybe_conj(double a, int) { return a; }
__device__ __forceinline__ cd maybe_conj(cd a, int c) { return c ? cd{a.x, -a.y} : a; }
__device__ __forceinline__ void store_c(double& dst, double v, int acc) { dst = acc ? dst + v : v; }
__device__ __forceinline__ void store_c(cd& dst, double v, int acc) {
    dst = acc ? cd{dst.x + v, dst.y} : cd{v, 0.0};
}
__device__ __forceinline__ void store_c(cd& dst, cd v, int acc) { dst = acc ? dst + v : v; }
template <typename T> __device__ __forceinline__ T zero_of();
template <> __device__ __forceinline__ double zero_of<double>() { return 0.0; }
template <> __device__ __forceinline__ cd zero_of<cd>() { return cd{0.0, 0.0}; }

constexpr int GEMM_BM = 64, GEMM_BN = 64, GEMM_THREADS = 256;

// Tile shapes (BM x BN, outputs per thread): 64x64 (4x4); 16x128, 128x16
// (1x8, 8x1); 64x32, 64x48, 32x64, 48x64 (4x2, 4x3, 2x4, 3x4); 4x128, 128x4
// (1x2, 2x1) for products with at most 4 rows or columns, so the skinny
// products of the anchored G2 do not run in a wide tile.
// Shared memory is double-buffered: the next k-tile's global loads are issued
// into registers before the current tile's products, so their latency
// overlaps the arithmetic, and one barrier per k-tile suffices.
template <typename TA, typename TB, typename TC, int BM, int BN>
__global__ void __launch_bounds__(GEMM_THREADS, 2)
    gemm_tiles_kernel(const GemmProblem<TA, TB, TC>* __restrict__ probs, const int* __restrict__ tile0, int nprobs) {
    using VA = typename val_t<TA>::type;  // operand values as they enter the product
    using VB = typename val_t<TB>::type;
    using TAcc = typename std::conditional<is_cd<VA>::value || is_cd<VB>::value, cd, double>::type;
    constexpr int BK = (is_cd<VA>::value || is_cd<VB>::value) ? 8 : 16;
    // thread grid NY x NX (256 threads), each thread an TM x TN sub-tile
    constexpr int NX = (BM == 4) ? 64 : (BN == 4) ? 4 : 16;
    constexpr int NY = GEMM_THREADS / NX;
    constexpr int TM = BM / NY, TN = BN / NX;
    static_assert(TM * NY == BM && TN * NX == BN, "tile shape does not fit the thread grid");
    constexpr int LA = (BM * BK + GEMM_THREADS - 1) / GEMM_THREADS;
    constexpr int LB = (BN * BK + GEMM_THREADS - 1) / GEMM_THREADS;
    __shared__ VA As[2][BK][BM + 1];
    __shared__ VB Bs[2][BK][BN + 1];

    // tile0[q] = first tile of problem q (prefix sum); find this CTA's problem
    const int tile = blockIdx.x;
    int lo = 0, hi = nprobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile0[mid] <= tile) lo = mid;
        else hi = mid - 1;
    }
    GemmProblem<TA, TB, TC> p = probs[lo];
    const int tn_count = (p.N + BN - 1) / BN, per_item = ((p.M + BM - 1) / BM) * tn_count;
    const int local = tile - tile0[lo];
    const int item = local / per_item, rem = local % per_item;
    const int i0 = (rem / tn_count) * BM, j0 = (rem % tn_count) * BN;
    if (item > 0) {
        p.A += item * p.ba;
        p.B += item * p.bb;
        p.C += item * p.bc;
    }
    if (p.dzs) p.dz = p.dzs[item];
    const int tid = threadIdx.x, tx = tid % NX, ty = tid / NX;

    TAcc acc[TM][TN];
#pragma unroll
    for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) acc[a][b] = zero_of<TAcc>();

    const bool a_i_fast = (p.sa_i == 1);
    const bool b_j_fast = (p.sb_j == 1);
    VA ra[LA];
    VB rb[LB];
    // position (row or column, k) inside the tile of element l of a k-tile
    auto a_pos = [&](int l, int& ii, int& kk) {
        if (a_i_fast) {
            ii = l % BM;
            kk = l / BM;
        } else {
            ii = l / BK;
            kk = l % BK;
        }
    };
    auto b_pos = [&](int l, int& jj, int& kk) {
        if (b_j_fast) {
            jj = l % BN;
            kk = l / BN;
        } else {
            jj = l / BK;
            kk = l % BK;
        }
    };
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            const int l = tid + q * GEMM_THREADS;
            VA v = zero_of<VA>();
            if (l < BM * BK) {
                int ii, kk;
                a_pos(l, ii, kk);
                const int gi = i0 + ii, gk = k0 + kk;
                if (gi < p.M && gk < p.K) {
                    const long kq = p.a_kidx ? p.a_kidx[gk] : gk;
                    const long iq = p.a_iidx ? p.a_iidx[gi] : gi;
                    if constexpr (is_dressed<TA>::value)
                        v = dress(p.A[iq * p.sa_i + kq * p.sa_k], p.dEa[iq], p.dEb[kq], p.dz);
                    else
                        v = maybe_conj(p.A[iq * p.sa_i + kq * p.sa_k], p.conj_a);
                }
            }
            ra[q] = v;
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int l = tid + q * GEMM_THREADS;
            VB v = zero_of<VB>();
            if (l < BN * BK) {
                int jj, kk;
                b_pos(l, jj, kk);
                const int gj = j0 + jj, gk = k0 + kk;
                if (gj < p.N && gk < p.K) {
                    const long kq = p.b_kidx ? p.b_kidx[gk] : gk;
                    const long jq = p.b_jidx ? p.b_jidx[gj] : gj;
                    if constexpr (is_dressed<TB>::value) {
                        v = dress(p.B[kq * p.sb_k + jq * p.sb_j], p.dEa[kq], p.dEb[jq], p.dz);
                    } else {
                        v = p.B[kq * p.sb_k + jq * p.sb_j];
                        if (p.kscale) v = scale_by(v, p.kscale[gk]);
                    }
                }
            }
            rb[q] = v;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            const int l = tid + q * GEMM_THREADS;
            if (l < BM * BK) {
                int ii, kk;
                a_pos(l, ii, kk);
                As[buf][kk][ii] = ra[q];
            }
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int l = tid + q * GEMM_THREADS;
            if (l < BN * BK) {
                int jj, kk;
                b_pos(l, jj, kk);
                Bs[buf][kk][jj] = rb[q];
            }
        }
    };

    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < p.K; k0 += BK) {
        const bool more = k0 + BK < p.K;
        if (more) load(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            VA a[TM];
            VB b[TN];
#pragma unroll
            for (int q = 0; q < TM; ++q) a[q] = As[buf][kk][ty + NY * q];
#pragma unroll
            for (int q = 0; q < TN; ++q) b[q] = Bs[buf][kk][tx + NX * q];
#pragma unroll
            for (int qa = 0; qa < TM; ++qa)
#pragma unroll
                for (int qb = 0; qb < TN; ++qb) mac(acc[qa][qb], a[qa], b[qb]);
        }
        if (more) store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int qa = 0; qa < TM; ++qa) {
        const int gi = i0 + ty + NY * qa;
        if (gi >= p.M) continue;
#pragma unroll
        for (int qb = 0; qb < TN; ++qb) {
            const int gj = j0 + tx + NX * qb;
            if (gj >= p.N) continue;
            store_c(p.C[gi * p.sc_i + gj * p.sc_j], acc[qa][qb], p.accumulate);
        }
    }
}

template <typename T> struct type_tag_s {
    static const char* get() { return is_cd<T>::value ? "cd" : "double"; }
};
template <typename T> struct type_tag_s<Dressed<T>> {
    static const char* get() { return is_cd<T>::value ? "dressed<cd>" : "dressed<double>"; }
};
template <typename T> const char* type_tag() { return type_tag_s<T>::get(); }
template <typename TA, typename TB, typename TC> const char* gemm_name() {
    static const std::string n =
        std::string("gemm_tiles_kernel<") + type_tag<TA>() + ", " + type_tag<TB>() + ", " + type_tag<TC>() + ">";
    return n.c_str();
}

// Tile classes (BM x BN).  A problem takes the class that pads it least
// (ties: the larger tile); the classes other than 64x64 are used only when
// their short side covers the problem's M or N in one tile.
constexpr int GEMM_NCLS = 9;
constexpr int GEMM_CLS_M[GEMM_NCLS] = {64, 16, 128, 64, 64, 32, 48, 4, 128};
constexpr int GEMM_CLS_N[GEMM_NCLS] = {64, 128, 16, 32, 48, 64, 64, 128, 4};

template <typename P> inline int gemm_class(const P& p) {
    int best = 0;
    long best_area = (long)ceil_div(p.M, 64) * 64 * ((long)ceil_div(p.N, 64) * 64);
    for (int c = 1; c < GEMM_NCLS; ++c) {
        const int bm = GEMM_CLS_M[c], bn = GEMM_CLS_N[c];
        if (bm < 64 && p.M > bm) continue;
        if (bn < 64 && p.N > bn) continue;
        const long area = (long)ceil_div(p.M, bm) * bm * ((long)ceil_div(p.N, bn) * bn);
        if (area < best_area) {
            best = c;
            best_area = area;
        }
    }
    return best;
}

// ------------------------------------------------------------ tuned class choice
// A context's table of measured-fastest tile classes (pgx_autotune), keyed by
// the operand types and the (M, N) size buckets; -1 keeps the padding rule.
// The bucket bounds are the narrow classes' limits (4, 16, 32, 48), so a class
// measured at a bucket's upper bound is valid for every size in the bucket.
constexpr int GEMM_BUCKET_REP[GEMM_NBUCKET] = {4, 16, 32, 48, 64, 128, 256};
inline int gemm_bucket(int x) {
    return x <= 4 ? 0 : x <= 16 ? 1 : x <= 32 ? 2 : x <= 48 ? 3 : x <= 64 ? 4 : x <= 128 ? 5 : 6;
}
template <typename T> struct type_code { static constexpr int v = is_cd<T>::value ? 1 : 0; };
template <typename T> struct type_code<Dressed<T>> { static constexpr int v = 2 + (is_cd<T>::value ? 1 : 0); };
template <typename TA, typename TB, typename TC> constexpr int gemm_key() {
    return type_code<TA>::v * 8 + type_code<TB>::v * 2 + type_code<TC>::v;
}

inline bool gemm_class_valid(int c, int M, int N) {
    return (GEMM_CLS_M[c] >= 64 || M <= GEMM_CLS_M[c]) && (GEMM_CLS_N[c] >= 64 || N <= GEMM_CLS_N[c]);
}

template <typename TA, typename TB, typename TC> int gemm_class_for(const GemmProblem<TA, TB, TC>& p) {
    const int f = forced_gemm_class();
    if (f >= 0 && gemm_class_valid(f, p.M, p.N)) return f;
    const GemmTune* t = active_tune();
    if (t) {
        const int c = t->cls[gemm_key<TA, TB, TC>()][gemm_bucket(p.M)][gemm_bucket(p.N)];
        if (c >= 0 && gemm_class_valid(c, p.M, p.N)) return c;
    }
    return gemm_class(p);
}

template <typename TA, typename TB, typename TC, int BM, int BN>
void launch_gemm_class(const GemmProblem<TA, TB, TC>* dp, const int* d_index, size_t pb, size_t pe, int ntiles,
                       cudaStream_t st) {
    if (pe <= pb || ntiles <= 0) return;
    gemm_tiles_kernel<TA, TB, TC, BM, BN><<<(unsigned)ntiles, GEMM_THREADS, 0, st>>>(dp + pb, d_index, (int)(pe - pb));
    check_launch("gemm_tiles_kernel");
}

// Host helper: upload the problems (grouped by tile class) and, per class, the
// prefix sums of their tile counts into scratch buffers, and launch one kernel
// per tile class.  The index needs gemm_index_bytes(probs.size()) bytes.
template <typename TA, typename TB, typename TC>
void launch_gemm_batch(const std::vector<GemmProblem<TA, TB, TC>>& probs, void* d_probs, size_t probs_cap,
                       void* d_index, size_t index_cap, cudaStream_t st);

// Measures a batch for the tuner ahead of its real launch: per (M, N) bucket,
// the bucket's products run in every candidate class with each output
// redirected to its own stretch of scratch.  The inputs are read where they
// are, with the contents the real launch reads.
template <typename TA, typename TB, typename TC>
void record_gemm_batch(const std::vector<GemmProblem<TA, TB, TC>>& probs, cudaStream_t st) {
    TuneRecorder* rec = active_recorder();
    for (int mb = 0; mb < GEMM_NBUCKET; ++mb)
        for (int nb = 0; nb < GEMM_NBUCKET; ++nb) {
            std::vector<GemmProblem<TA, TB, TC>> grp;
            size_t bytes = 0;
            bool redirectable = true;
            for (const auto& g : probs) {
                if (g.M <= 0 || g.N <= 0 || gemm_bucket(g.M) != mb || gemm_bucket(g.N) != nb) continue;
                if (g.sc_i < 0 || g.sc_j < 0 || g.bc < 0) redirectable = false;  // not laid out in scratch
                // the output's extent: last item's last element
                const long items = std::max(g.nb, 1);
                const long last = (items - 1) * g.bc + (long)(g.M - 1) * g.sc_i + (long)(g.N - 1) * g.sc_j;
                grp.push_back(g);
                grp.back().C = reinterpret_cast<TC*>(bytes);  // offset into the scratch, made a pointer below
                bytes += ((size_t)(last + 1) * sizeof(TC) + 255) & ~size_t(255);
            }
            if (grp.empty() || !redirectable) continue;
            tune_measure(*rec, gemm_key<TA, TB, TC>(), mb, nb, bytes,
                         [&grp](int cls, void* scratch, DevBuf& pb, DevBuf& ib, cudaStream_t s2) {
                             std::vector<GemmProblem<TA, TB, TC>> q = grp;
                             for (auto& g : q)
                                 g.C = reinterpret_cast<TC*>(static_cast<char*>(scratch) +
                                                             reinterpret_cast<size_t>(g.C));
                             pb.reserve(q.size() * sizeof(q[0]));
                             ib.reserve(gemm_index_bytes(q.size()));
                             forced_gemm_class() = cls;
                             launch_gemm_batch(q, pb.p, pb.bytes, ib.p, ib.bytes, s2);
                             forced_gemm_class() = -1;
                         },
                         st);
        }
}

template <typename TA, typename TB, typename TC>
void launch_gemm_batch(const std::vector<GemmProblem<TA, TB, TC>>& probs, void* d_probs, size_t probs_cap,
                       void* d_index, size_t index_cap, cudaStream_t st) {
    if (probs.empty()) return;
    if (active_recorder()) record_gemm_batch(probs, st);
    std::vector<GemmProblem<TA, TB, TC>> sorted;
    sorted.reserve(probs.size());
    std::vector<int> index;  // per class: prefix over its problems, then the total
    index.reserve(probs.size() + 2 * GEMM_NCLS);
    size_t pstart[GEMM_NCLS + 1] = {}, istart[GEMM_NCLS] = {};
    int ntiles[GEMM_NCLS] = {};
    std::vector<int> cls(probs.size());
    for (size_t q = 0; q < probs.size(); ++q) cls[q] = gemm_class_for(probs[q]);
    for (int c = 0; c < GEMM_NCLS; ++c) {
        pstart[c] = sorted.size();
        istart[c] = index.size();
        long t = 0;
        for (size_t q = 0; q < probs.size(); ++q) {
            const auto& g = probs[q];
            if (g.M <= 0 || g.N <= 0 || cls[q] != c) continue;
            sorted.push_back(g);
            index.push_back((int)t);
            t += (long)std::max(g.nb, 1) * ceil_div(g.M, GEMM_CLS_M[c]) * ceil_div(g.N, GEMM_CLS_N[c]);
        }
        PGX_CHECK(t < (1L << 31), PGX_ERR_ARG, "gemm batch too large");
        index.push_back((int)t);
        ntiles[c] = (int)t;
    }
    pstart[GEMM_NCLS] = sorted.size();
    if (sorted.empty()) return;
    PGX_CHECK(sorted.size() * sizeof(sorted[0]) <= probs_cap, PGX_ERR_ARG, "gemm problem list overflow");
    PGX_CHECK(index.size() * sizeof(int) <= index_cap, PGX_ERR_ARG, "gemm tile index overflow");
    h2d(d_probs, sorted.data(), sorted.size() * sizeof(sorted[0]), st);
    h2d(d_index, index.data(), index.size() * sizeof(int), st);
    const auto* dp = static_cast<const GemmProblem<TA, TB, TC>*>(d_probs);
    const int* di = static_cast<const int*>(d_index);
    // real x real 2, real x complex 4, complex x complex 8 operations per product term;
    // minimum traffic: A, B and C once (C twice when accumulating)
    using VA = typename val_t<TA>::type;
    using VB = typename val_t<TB>::type;
    constexpr double mac = (is_cd<VA>::value && is_cd<VB>::value) ? 8.0
                           : (is_cd<VA>::value || is_cd<VB>::value) ? 4.0 : 2.0;
    double fl = 0.0, by = 0.0;
    for (const auto& q : sorted) {
        const double nb = std::max(q.nb, 1);
        fl += nb * mac * q.M * (double)q.N * q.K;
        by += nb * ((double)q.M * q.K * sizeof(typename src_t<TA>::type) +
                    (double)q.K * q.N * sizeof(typename src_t<TB>::type) +
                    (q.accumulate ? 2.0 : 1.0) * q.M * (double)q.N * sizeof(TC));
    }
    ProfRange pr(gemm_name<TA, TB, TC>(), st, fl, by);
    launch_gemm_class<TA, TB, TC, 64, 64>(dp, di + istart[0], pstart[0], pstart[1], ntiles[0], st);
    launch_gemm_class<TA, TB, TC, 16, 128>(dp, di + istart[1], pstart[1], pstart[2], ntiles[1], st);
    launch_gemm_class<TA, TB, TC, 128, 16>(dp, di + istart[2], pstart[2], pstart[3], ntiles[2], st);
    launch_gemm_class<TA, TB, TC, 64, 32>(dp, di + istart[3], pstart[3], pstart[4], ntiles[3], st);
    launch_gemm_class<TA, TB, TC, 64, 48>(dp, di + istart[4], pstart[4], pstart[5], ntiles[4], st);
    launch_gemm_class<TA, TB, TC, 32, 64>(dp, di + istart[5], pstart[5], pstart[6], ntiles[5], st);
    launch_gemm_class<TA, TB, TC, 48, 64>(dp, di + istart[6], pstart[6], pstart[7], ntiles[6], st);
    launch_gemm_class<TA, TB, TC, 4, 128>(dp, di + istart[7], pstart[7], pstart[8], ntiles[7], st);
    launch_gemm_class<TA, TB, TC, 128, 4>(dp, di + istart[8], pstart[8], pstart[9], ntiles[8], st);
}

// C = A B through the int8 split scheme (pgx_ozaki.cu): S slices, plain
// strided operands (one of them may be dressed), items as in launch_gemm_batch.
struct OzWork;
template <typename TA, typename TB>
void oz_zgemm(const GemmProblem<TA, TB, cd>& g, int S, OzWork& w, cudaStream_t st);

}  // namespace pgx
