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
    cd dz;                 // and the frequency
};

struct GemmTile {
    int prob, tm, tn, pad;
};

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

// Tile shapes: 64x64 (4x4 outputs per thread), 16x128 for problems with at
// most 16 rows and 128x16 for at most 16 columns (1x8 / 8x1 per thread), so
// the skinny products of the anchored G2 do not waste a 64-wide tile.
// Shared memory is double-buffered: the next k-tile's global loads are issued
// into registers before the current tile's products, so their latency
// overlaps the arithmetic, and one barrier per k-tile suffices.
template <typename TA, typename TB, typename TC, int BM, int BN>
__global__ void __launch_bounds__(GEMM_THREADS, 2)
    gemm_tiles_kernel(const GemmProblem<TA, TB, TC>* __restrict__ probs, const GemmTile* __restrict__ tiles) {
    using VA = typename val_t<TA>::type;  // operand values as they enter the product
    using VB = typename val_t<TB>::type;
    using TAcc = typename std::conditional<is_cd<VA>::value || is_cd<VB>::value, cd, double>::type;
    constexpr int BK = (is_cd<VA>::value || is_cd<VB>::value) ? 8 : 16;
    constexpr int TM = BM / 16, TN = BN / 16;
    constexpr int LA = (BM * BK + GEMM_THREADS - 1) / GEMM_THREADS;
    constexpr int LB = (BN * BK + GEMM_THREADS - 1) / GEMM_THREADS;
    __shared__ VA As[2][BK][BM + 1];
    __shared__ VB Bs[2][BK][BN + 1];

    const GemmTile t = tiles[blockIdx.x];
    const GemmProblem<TA, TB, TC> p = probs[t.prob];
    const int i0 = t.tm * BM, j0 = t.tn * BN;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

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
            for (int q = 0; q < TM; ++q) a[q] = As[buf][kk][ty + 16 * q];
#pragma unroll
            for (int q = 0; q < TN; ++q) b[q] = Bs[buf][kk][tx + 16 * q];
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
        const int gi = i0 + ty + 16 * qa;
        if (gi >= p.M) continue;
#pragma unroll
        for (int qb = 0; qb < TN; ++qb) {
            const int gj = j0 + tx + 16 * qb;
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
// their short side covers the problem's M or N in one tile, so the tile count
// never exceeds that of 64x64 tiles.
constexpr int GEMM_NCLS = 7;
constexpr int GEMM_CLS_M[GEMM_NCLS] = {64, 16, 128, 64, 64, 32, 48};
constexpr int GEMM_CLS_N[GEMM_NCLS] = {64, 128, 16, 32, 48, 64, 64};

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

template <typename TA, typename TB, typename TC, int BM, int BN>
void launch_gemm_class(const GemmProblem<TA, TB, TC>* dp, const GemmTile* dt, size_t b, size_t e, cudaStream_t st) {
    if (e <= b) return;
    gemm_tiles_kernel<TA, TB, TC, BM, BN><<<(unsigned)(e - b), GEMM_THREADS, 0, st>>>(dp, dt + b);
    check_launch("gemm_tiles_kernel");
}

// Host helper: upload problems + tile lists into scratch buffers and launch
// one kernel per tile class.  Tile capacity computed for 64x64 tiles is an
// upper bound for every class.
template <typename TA, typename TB, typename TC>
void launch_gemm_batch(const std::vector<GemmProblem<TA, TB, TC>>& probs, void* d_probs, size_t probs_cap,
                       void* d_tiles, size_t tiles_cap, cudaStream_t st) {
    if (probs.empty()) return;
    std::vector<GemmTile> tiles;
    size_t start[GEMM_NCLS + 1] = {};
    std::vector<int> cls(probs.size());
    for (size_t q = 0; q < probs.size(); ++q) cls[q] = gemm_class(probs[q]);
    for (int c = 0; c < GEMM_NCLS; ++c) {
        start[c] = tiles.size();
        for (size_t q = 0; q < probs.size(); ++q) {
            if (probs[q].M <= 0 || probs[q].N <= 0 || cls[q] != c) continue;
            const int tm = ceil_div(probs[q].M, GEMM_CLS_M[c]), tn = ceil_div(probs[q].N, GEMM_CLS_N[c]);
            for (int a = 0; a < tm; ++a)
                for (int b = 0; b < tn; ++b) tiles.push_back(GemmTile{(int)q, a, b, 0});
        }
    }
    start[GEMM_NCLS] = tiles.size();
    if (tiles.empty()) return;
    PGX_CHECK(probs.size() * sizeof(probs[0]) <= probs_cap, PGX_ERR_ARG, "gemm problem list overflow");
    PGX_CHECK(tiles.size() * sizeof(GemmTile) <= tiles_cap, PGX_ERR_ARG, "gemm tile list overflow");
    PGX_CUDA(cudaMemcpyAsync(d_probs, probs.data(), probs.size() * sizeof(probs[0]), cudaMemcpyHostToDevice, st));
    PGX_CUDA(cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(GemmTile), cudaMemcpyHostToDevice, st));
    const auto* dp = static_cast<const GemmProblem<TA, TB, TC>*>(d_probs);
    const auto* dt = static_cast<const GemmTile*>(d_tiles);
    // real x real 2, real x complex 4, complex x complex 8 operations per product term;
    // minimum traffic: A, B and C once (C twice when accumulating)
    using VA = typename val_t<TA>::type;
    using VB = typename val_t<TB>::type;
    constexpr double mac = (is_cd<VA>::value && is_cd<VB>::value) ? 8.0
                           : (is_cd<VA>::value || is_cd<VB>::value) ? 4.0 : 2.0;
    double fl = 0.0, by = 0.0;
    for (const auto& q : probs) {
        fl += mac * q.M * (double)q.N * q.K;
        by += (double)q.M * q.K * sizeof(typename src_t<TA>::type) + (double)q.K * q.N * sizeof(typename src_t<TB>::type) +
              (q.accumulate ? 2.0 : 1.0) * q.M * (double)q.N * sizeof(TC);
    }
    ProfRange pr(gemm_name<TA, TB, TC>(), st, fl, by);
    launch_gemm_class<TA, TB, TC, 64, 64>(dp, dt, start[0], start[1], st);
    launch_gemm_class<TA, TB, TC, 16, 128>(dp, dt, start[1], start[2], st);
    launch_gemm_class<TA, TB, TC, 128, 16>(dp, dt, start[2], start[3], st);
    launch_gemm_class<TA, TB, TC, 64, 32>(dp, dt, start[3], start[4], st);
    launch_gemm_class<TA, TB, TC, 64, 48>(dp, dt, start[4], start[5], st);
    launch_gemm_class<TA, TB, TC, 32, 64>(dp, dt, start[5], start[6], st);
    launch_gemm_class<TA, TB, TC, 48, 64>(dp, dt, start[6], start[7], st);
}

}  // namespace pgx
