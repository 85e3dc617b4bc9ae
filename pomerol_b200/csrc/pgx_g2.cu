// K4: two-particle Green's function, factorised Lehmann sum on the GPU.
//
// Reference: TwoParticleGFPart::computeImpl / addMultiterm (TwoParticleGFPart.cpp:189-298)
// enumerate every state quadruple (1,2,3,4) of a block chain with
// M = sign * O1_12 O2_23 O3_34 CX4_41 and four sub-terms; TwoParticleGFPart::operator()
// (TwoParticleGFPart.cpp:309-322, .hpp:475-495) sums them at a frequency triple.
//
// With A(z1)_12 = O1_12 / (z1 - (E2 - E1)) and C(z3)_34 = O3_34 / (z3 - (E4 - E3))
// the four sub-terms of the Lehmann sum become
//   T1 = -sign sum_23 X_32 O2_23 (w2 + w3) / (z2 - (E3 - E2)),    X = C(z3) CX4 A(z1)
//   T2 =  sign sum_14 Y_14 CX4_41 (w1 + w4) / (z1+z2+z3 - (E4 - E1)), Y = A(z1) O2 C(z3)
//   T3 =  sign sum_13 P_13 Q_31 F13(z1 + z2),   P = A(z1) O2, Q = C(z3) CX4
//   T4 =  sign sum_24 R_24 L_42 F24(z2 + z3),   R = O2 C(z3), L = CX4 A(z1)
// with the resonant rule of ResonantTerm::operator():
//   F13(s) = |s - (E3 - E1)| <= tol ? beta w1 : (w3 - w1) / (s - (E3 - E1))
//   F24(s) = |s - (E4 - E2)| <= tol ? -beta w2 : (w2 - w4) / (s - (E4 - E2)).
// Per chain: dressed operators per distinct z1 / z3, four batched GEMMs per
// distinct frequency, two batched GEMMs per distinct (z1, z3) pair (the
// dominant FP64 work), and four contractions over the triples of each pair.
// Everything stays FP64; the delta test is made per element in FP64.

#include <chrono>
#include <cstring>
#include <map>
#include <tuple>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

// out[iz][a][b] = O[a][b] / (z[iz] - (Eb[b] - Ea[a]))
template <typename T>
__global__ void dress_kernel(const T* O, int da, int db, const double* Ea, const double* Eb, const cd* z, int nz,
                             cd* out) {
    const long n = (long)da * db;
    const int iz = blockIdx.y;
    if (iz >= nz) return;
    const cd zz = z[iz];
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int a = (int)(e / db), b = (int)(e % db);
        const cd den{zz.x - (Eb[b] - Ea[a]), zz.y};
        out[(long)iz * n + e] = tocd(O[e]) * inv(den);
    }
}

struct ContractArgs {
    const cd* Lm;
    long L_stride;
    const int* L_idx;
    long L_sa, L_sb;
    const void* Rm;
    long R_stride;
    const int* R_idx;
    long R_sa, R_sb;
    const double *Ea, *Eb, *wa, *wb;
    int da, db;
    const int* pair_ptr;
    const int* slot_out;
    const cd* s;
    double beta, tol, coef;
    cd* out;
    int pair0;  // pairs of this launch start here; unindexed matrices are chunk-local
};

constexpr int CT_THREADS = 256, CT_CHUNK = 4096, CT_GROUP = 16;

__device__ __forceinline__ double wsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// MODE 1/2: K = (wa + wb) / (s - (Eb - Ea))
// MODE 3:   K = delta ? beta wa : (wb - wa) / (s - (Eb - Ea))
// MODE 4:   K = delta ? -beta wa : (wa - wb) / (s - (Eb - Ea))
template <typename TR, int MODE>
__global__ void __launch_bounds__(CT_THREADS) contract_kernel(ContractArgs g) {
    __shared__ cd s_s[CT_GROUP];
    __shared__ double s_acc[CT_GROUP][2];
    const int pl = blockIdx.y, p = g.pair0 + pl;
    const int t0 = g.pair_ptr[p], t1 = g.pair_ptr[p + 1];
    const long n = (long)g.da * g.db;
    const long e0 = (long)blockIdx.x * CT_CHUNK;
    const cd* L = g.Lm + (long)(g.L_idx ? g.L_idx[p] : pl) * g.L_stride;
    const TR* R = static_cast<const TR*>(g.Rm) + (long)(g.R_idx ? g.R_idx[p] : pl) * g.R_stride;
    for (int tg = t0; tg < t1; tg += CT_GROUP) {
        const int nt = min(CT_GROUP, t1 - tg);
        __syncthreads();
        if (threadIdx.x < nt) {
            s_s[threadIdx.x] = g.s[tg + threadIdx.x];
            s_acc[threadIdx.x][0] = 0.0;
            s_acc[threadIdx.x][1] = 0.0;
        }
        __syncthreads();
        cd acc[CT_GROUP];
#pragma unroll
        for (int j = 0; j < CT_GROUP; ++j) acc[j] = cd{0.0, 0.0};
        for (long e = e0 + threadIdx.x; e < min(n, e0 + CT_CHUNK); e += CT_THREADS) {
            const int a = (int)(e / g.db), b = (int)(e % g.db);
            const cd lr = L[a * g.L_sa + b * g.L_sb] * tocd(R[a * g.R_sa + b * g.R_sb]);
            if (lr.x == 0.0 && lr.y == 0.0) continue;
            const double dE = g.Eb[b] - g.Ea[a];
            const double wa = g.wa[a], wb = g.wb[b];
            double num;
            if (MODE <= 2) num = wa + wb;
            else if (MODE == 3) num = wb - wa;
            else num = wa - wb;
#pragma unroll
            for (int j = 0; j < CT_GROUP; ++j) {
                if (j < nt) {
                    const cd d{s_s[j].x - dE, s_s[j].y};
                    cd K;
                    if (MODE >= 3 && sqrt(abs2(d)) <= g.tol) {
                        K = cd{(MODE == 3 ? 1.0 : -1.0) * g.beta * wa, 0.0};
                    } else {
                        const double r = num / abs2(d);
                        K = cd{d.x * r, -d.y * r};
                    }
                    const cd v = lr * K;
                    acc[j].x += v.x;
                    acc[j].y += v.y;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < CT_GROUP; ++j) {
            if (j < nt) {
                const double x = wsum(acc[j].x), y = wsum(acc[j].y);
                if ((threadIdx.x & 31) == 0 && (x != 0.0 || y != 0.0)) {
                    atomicAdd(&s_acc[j][0], x);
                    atomicAdd(&s_acc[j][1], y);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x < nt) {
            const double x = s_acc[threadIdx.x][0], y = s_acc[threadIdx.x][1];
            if (x != 0.0 || y != 0.0) {
                cd* o = g.out + g.slot_out[tg + threadIdx.x];
                atomicAdd(&o->x, g.coef * x);
                atomicAdd(&o->y, g.coef * y);
            }
        }
    }
}

// Zero entries (|x| <= nz) of the four operator parts of a chain, as sorted
// index lists: rows of O1 (over i2), columns of O2 (over i2), rows of O3 (over
// i4), columns of CX4 (over i4).  off[i] .. off[i+1] delimits list i.
struct ZeroLists {
    const int *r1off, *r1idx;  // O1 row i1 -> zero i2
    const int *c2off, *c2idx;  // O2 column i3 -> zero i2
    const int *r3off, *r3idx;  // O3 row i3 -> zero i4
    const int *c4off, *c4idx;  // CX4 column i1 -> zero i4
};

__device__ __forceinline__ bool in_sorted(const int* a, int n, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && a[lo] == x;
}

// Size of the union of two sorted index lists and its members with w <= tol.
__device__ __forceinline__ void union_count(const int* a, int na, const int* b, int nb, const double* w, double tol,
                                            long& n, long& ncold) {
    int i = 0, j = 0;
    n = 0;
    ncold = 0;
    while (i < na || j < nb) {
        int x;
        if (j >= nb || (i < na && a[i] < b[j])) x = a[i++];
        else if (i >= na || b[j] < a[i]) x = b[j++];
        else {
            x = a[i++];
            ++j;
        }
        ++n;
        ncold += !(w[x] > tol);
    }
}

// Number of state quadruples of one chain that the reference enumerates
// (TwoParticleGFPart.cpp:210-250): all four rotated elements non-zero
// (|x| > nz) and w1 + w2 + w3 + w4 > tol, summed in that order as the
// reference does (:241).  One thread per (i1, i3).  The zero elements are
// few (rotated operators are dense), so the lists L2 = {i2 : O1[i1,i2] and
// O2[i2,i3] non-zero} and L4 are handled through their complements Z2, Z4.
// When w1 + w3 > tol every (i2, i4) of L2 x L4 counts (a rounded sum of
// non-negative weights only grows as terms are added); otherwise only pairs
// of cold states (w <= tol) can fail: of the cold pairs, those that pass are
// found per cold i2 of the shell (sorted descending, c2 / c2i) by a binary
// search over the sorted cold weights c4 of S4, minus the zero i4 among them.
__global__ void count_kernel(ZeroLists z, int d1, int d2, int d3, int d4, const double* w1, const double* w2,
                             const double* w3, const double* w4, const double* c2, const int* c2i, int n2c_all,
                             const double* c4, int n4c_all, double tol, unsigned long long* out) {
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    unsigned long long cnt = 0;
    if (idx < (long)d1 * d3) {
        const int i1 = (int)(idx / d3), i3 = (int)(idx % d3);
        const int* za = z.r1idx + z.r1off[i1];
        const int nza = z.r1off[i1 + 1] - z.r1off[i1];
        const int* zb = z.c2idx + z.c2off[i3];
        const int nzb = z.c2off[i3 + 1] - z.c2off[i3];
        const int* zc = z.r3idx + z.r3off[i3];
        const int nzc = z.r3off[i3 + 1] - z.r3off[i3];
        const int* zd = z.c4idx + z.c4off[i1];
        const int nzd = z.c4off[i1 + 1] - z.c4off[i1];
        long z2, z2c, z4, z4c;
        union_count(za, nza, zb, nzb, w2, tol, z2, z2c);
        union_count(zc, nzc, zd, nzd, w4, tol, z4, z4c);
        const long n2 = d2 - z2, n4 = d4 - z4;
        const double x1 = w1[i1], x3 = w3[i3];
        if (x1 + x3 > tol) {
            cnt = (unsigned long long)(n2 * n4);
        } else {
            const long n2c = n2c_all - z2c, n4c = n4c_all - z4c;
            long pass = 0;
            for (int q = 0; q < n2c_all; ++q) {
                const double s = (x1 + c2[q]) + x3;
                if (n4c_all == 0 || !(s + c4[0] > tol)) break;
                const int i2 = c2i[q];
                if (in_sorted(za, nza, i2) || in_sorted(zb, nzb, i2)) continue;
                int lo = 1, hi = n4c_all;  // c4[0 .. lo) pass
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (s + c4[mid] > tol) lo = mid + 1;
                    else hi = mid;
                }
                long drop = 0;  // zero i4 among the passing cold states
                for (int t = 0; t < nzc; ++t) {
                    const double v = w4[zc[t]];
                    drop += !(v > tol) && (s + v > tol);
                }
                for (int t = 0; t < nzd; ++t) {
                    const double v = w4[zd[t]];
                    drop += !(v > tol) && (s + v > tol) && !in_sorted(zc, nzc, zd[t]);
                }
                pass += lo - drop;
            }
            cnt = (unsigned long long)(n2 * n4 - n2c * n4c + pass);
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

// (row, column) of every zero entry (|x| <= nz) of one operator part, in no
// particular order; at most cap of them are written.
template <typename T>
__global__ void zero_list_kernel(const T* a, int rows, int cols, double nz, int2* out, unsigned long long* counter,
                                 long cap) {
    const long n = (long)rows * cols;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (!(sqrt(abs2(tocd(a[i]))) > nz)) {
            const unsigned long long k = atomicAdd(counter, 1ull);
            if ((long)k < cap) out[k] = make_int2((int)(i / cols), (int)(i % cols));
        }
    }
}

// Entries of one rotated operator part with |x| <= nz (absent from the
// reference's sparse matrices after sparseView).
template <typename T>
__global__ void zero_count_kernel(const T* a, long n, double nz, unsigned long long* out) {
    unsigned long long cnt = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        cnt += !(sqrt(abs2(tocd(a[i]))) > nz);
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

// Quadruples of one chain whose four rotated elements are all non-zero but
// which fail the weight filter: ((w1 + w2) + w3) + w4 <= tol.  Only states
// with w <= tol can take part ("cold" states; c1 .. c4 their weights, c2 and
// c4 sorted descending).  One thread per cold (i1, i3): of the n2 x n4 cold
// (i2, i4) pairs it subtracts those that pass, found per i2 by a binary
// search over c4 (the rounded sum is monotone in each weight); i2 stops at
// the first that cannot pass with the largest w4.
__global__ void cold_fail_kernel(const double* c1, int n1, const double* c3, int n3, const double* c2, int n2,
                                 const double* c4, int n4, double tol, unsigned long long* out) {
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    unsigned long long fail = 0;
    if (idx < (long)n1 * n3 && n2 > 0 && n4 > 0) {
        const double x1 = c1[idx / n3], x3 = c3[idx % n3];
        if (!(x1 + x3 > tol)) {
            unsigned long long pass = 0;
            for (int q = 0; q < n2; ++q) {
                const double s = (x1 + c2[q]) + x3;
                if (!(s + c4[0] > tol)) break;
                int lo = 1, hi = n4;  // c4[0 .. lo) pass; find the first index that fails
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (s + c4[mid] > tol) lo = mid + 1;
                    else hi = mid;
                }
                pass += (unsigned long long)lo;
            }
            fail = (unsigned long long)n2 * (unsigned long long)n4 - pass;
        }
    }
    for (int o = 16; o > 0; o >>= 1) fail += __shfl_xor_sync(0xffffffffu, fail, o);
    if ((threadIdx.x & 31) == 0 && fail) atomicAdd(out, fail);
}

// Frequency plan of one permutation: distinct z1, z3, distinct (z1, z3)
// pairs, and the triples of each pair in CSR order with the four s values.
struct Plan {
    std::vector<cd> Z1, Z3;
    std::vector<int> pi1, pi3, ptr, slot;
    std::vector<cd> s1, s2, s3, s4;
    // device
    DevBuf buf;
    cd *dZ1, *dZ3, *ds1, *ds2, *ds3, *ds4;
    int *dpi1, *dpi3, *dptr, *dslot;
};

struct Key {
    double a, b;
    bool operator<(const Key& o) const { return std::tie(a, b) < std::tie(o.a, o.b); }
};

void build_plan(Plan& pl, const int perm[3], int nfreq, const double* z) {
    std::map<Key, int> m1, m3;
    std::map<std::pair<int, int>, int> mp;
    std::vector<int> tp(nfreq);
    std::vector<cd> zz1(nfreq), zz2(nfreq), zz3(nfreq);
    for (int t = 0; t < nfreq; ++t) {
        const cd F[3] = {cd{z[6 * t], z[6 * t + 1]}, cd{z[6 * t + 2], z[6 * t + 3]}, cd{-z[6 * t + 4], -z[6 * t + 5]}};
        const cd a = F[perm[0]], b = F[perm[1]], c3 = F[perm[2]];
        zz1[t] = a;
        zz2[t] = b;
        zz3[t] = c3;
        auto i1 = m1.emplace(Key{a.x, a.y}, (int)pl.Z1.size());
        if (i1.second) pl.Z1.push_back(a);
        auto i3 = m3.emplace(Key{c3.x, c3.y}, (int)pl.Z3.size());
        if (i3.second) pl.Z3.push_back(c3);
        auto ip = mp.emplace(std::make_pair(i1.first->second, i3.first->second), (int)pl.pi1.size());
        if (ip.second) {
            pl.pi1.push_back(i1.first->second);
            pl.pi3.push_back(i3.first->second);
        }
        tp[t] = ip.first->second;
    }
    const int np = (int)pl.pi1.size();
    pl.ptr.assign(np + 1, 0);
    for (int t = 0; t < nfreq; ++t) pl.ptr[tp[t] + 1]++;
    for (int q = 0; q < np; ++q) pl.ptr[q + 1] += pl.ptr[q];
    std::vector<int> fill(pl.ptr.begin(), pl.ptr.end() - 1);
    pl.slot.resize(nfreq);
    pl.s1.resize(nfreq);
    pl.s2.resize(nfreq);
    pl.s3.resize(nfreq);
    pl.s4.resize(nfreq);
    for (int t = 0; t < nfreq; ++t) {
        const int k = fill[tp[t]]++;
        pl.slot[k] = t;
        pl.s1[k] = zz2[t];
        pl.s2[k] = zz1[t] + zz2[t] + zz3[t];
        pl.s3[k] = zz1[t] + zz2[t];
        pl.s4[k] = zz2[t] + zz3[t];
    }
}

void upload_plan(Plan& pl, cudaStream_t st) {
    const size_t n1 = pl.Z1.size(), n3 = pl.Z3.size(), np = pl.pi1.size(), nf = pl.slot.size();
    const size_t bytes = (n1 + n3 + 4 * nf) * sizeof(cd) + (2 * np + np + 1 + nf) * sizeof(int) + 256;
    pl.buf.reserve(bytes);
    char* p = pl.buf.as<char>();
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 15) & ~size_t(15);
        return r;
    };
    pl.dZ1 = reinterpret_cast<cd*>(take(n1 * sizeof(cd)));
    pl.dZ3 = reinterpret_cast<cd*>(take(n3 * sizeof(cd)));
    pl.ds1 = reinterpret_cast<cd*>(take(nf * sizeof(cd)));
    pl.ds2 = reinterpret_cast<cd*>(take(nf * sizeof(cd)));
    pl.ds3 = reinterpret_cast<cd*>(take(nf * sizeof(cd)));
    pl.ds4 = reinterpret_cast<cd*>(take(nf * sizeof(cd)));
    pl.dpi1 = reinterpret_cast<int*>(take(np * sizeof(int)));
    pl.dpi3 = reinterpret_cast<int*>(take(np * sizeof(int)));
    pl.dptr = reinterpret_cast<int*>(take((np + 1) * sizeof(int)));
    pl.dslot = reinterpret_cast<int*>(take(nf * sizeof(int)));
    auto up = [&](void* d, const void* h, size_t b) {
        if (b) h2d(d, h, b, st);
    };
    up(pl.dZ1, pl.Z1.data(), n1 * sizeof(cd));
    up(pl.dZ3, pl.Z3.data(), n3 * sizeof(cd));
    up(pl.ds1, pl.s1.data(), nf * sizeof(cd));
    up(pl.ds2, pl.s2.data(), nf * sizeof(cd));
    up(pl.ds3, pl.s3.data(), nf * sizeof(cd));
    up(pl.ds4, pl.s4.data(), nf * sizeof(cd));
    up(pl.dpi1, pl.pi1.data(), np * sizeof(int));
    up(pl.dpi3, pl.pi3.data(), np * sizeof(int));
    up(pl.dptr, pl.ptr.data(), (np + 1) * sizeof(int));
    up(pl.dslot, pl.slot.data(), nf * sizeof(int));
}

template <typename TA, typename TB>
GemmProblem<TA, TB, cd> prob(const TA* A, const TB* B, cd* C, int M, int N, int K) {
    GemmProblem<TA, TB, cd> g{};
    g.A = A;
    g.B = B;
    g.C = C;
    g.M = M;
    g.N = N;
    g.K = K;
    g.sa_i = K;
    g.sa_k = 1;
    g.sb_k = N;
    g.sb_j = 1;
    g.sc_i = N;
    g.sc_j = 1;
    return g;
}

struct Workspace {
    cd *A1, *C3, *L, *Pm, *Q, *R, *X;
    long pair_cap;  // complex elements available at X for X and Y of one pair chunk
    void* probs;
    size_t probs_cap;
    void* tiles;
    size_t tiles_cap;
};

template <typename T>
void g2_part(pgx_ctx* c, const pgx_g2_part& gp, const Plan& pl, Workspace& ws, double pole_res, cd* d_out,
             cudaEvent_t ev0, cudaEvent_t ev1, double& gemm_ms, double& gemm_flops) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    const int S1 = gp.block[0], S2 = gp.block[1], S3 = gp.block[2], S4 = gp.block[3];
    const int d1 = P.dims[S1], d2 = P.dims[S2], d3 = P.dims[S3], d4 = P.dims[S4];
    const Operator &o1 = P.ops[gp.op[0]], &o2 = P.ops[gp.op[1]], &o3 = P.ops[gp.op[2]], &o4 = P.ops[gp.op[3]];
    const T* O1 = o1.mat.as<T>() + o1.parts[o1.by_left[S1]].off;
    const T* O2 = o2.mat.as<T>() + o2.parts[o2.by_left[S2]].off;
    const T* O3 = o3.mat.as<T>() + o3.parts[o3.by_left[S3]].off;
    const T* X4 = o4.mat.as<T>() + o4.parts[o4.by_left[S4]].off;
    const double *E1 = P.d_E + P.eoff[S1], *E2 = P.d_E + P.eoff[S2], *E3 = P.d_E + P.eoff[S3], *E4 = P.d_E + P.eoff[S4];
    const double *w1 = P.d_w + P.eoff[S1], *w2 = P.d_w + P.eoff[S2], *w3 = P.d_w + P.eoff[S3], *w4 = P.d_w + P.eoff[S4];
    const int N1 = (int)pl.Z1.size(), N3 = (int)pl.Z3.size(), NP = (int)pl.pi1.size();
    const double sign = gp.sign;

    // dressed operators
    {
        dim3 g1(std::min(ceil_div((long)d1 * d2, 256), 256), N1);
        dress_kernel<T><<<g1, 256, 0, st>>>(O1, d1, d2, E1, E2, pl.dZ1, N1, ws.A1);
        dim3 g3(std::min(ceil_div((long)d3 * d4, 256), 256), N3);
        dress_kernel<T><<<g3, 256, 0, st>>>(O3, d3, d4, E3, E4, pl.dZ3, N3, ws.C3);
        check_launch("dress_kernel");
    }
    const long s12 = (long)d1 * d2, s34 = (long)d3 * d4, s42 = (long)d4 * d2, s13 = (long)d1 * d3,
               s31 = (long)d3 * d1, s24 = (long)d2 * d4, s32 = (long)d3 * d2, s14 = (long)d1 * d4;
    // per-frequency GEMMs
    {
        std::vector<GemmProblem<T, cd, cd>> pa;   // T x cd
        std::vector<GemmProblem<cd, T, cd>> pb;   // cd x T
        for (int i = 0; i < N1; ++i) {
            pa.push_back(prob<T, cd>(X4, ws.A1 + i * s12, ws.L + i * s42, d4, d2, d1));      // L = CX4 A1
            pb.push_back(prob<cd, T>(ws.A1 + i * s12, O2, ws.Pm + i * s13, d1, d3, d2));     // P = A1 O2
        }
        for (int i = 0; i < N3; ++i) {
            pb.push_back(prob<cd, T>(ws.C3 + i * s34, X4, ws.Q + i * s31, d3, d1, d4));      // Q = C3 CX4
            pa.push_back(prob<T, cd>(O2, ws.C3 + i * s34, ws.R + i * s24, d2, d4, d3));      // R = O2 C3
        }
        launch_gemm_batch(pa, ws.probs, ws.probs_cap, ws.tiles, ws.tiles_cap, st);
        launch_gemm_batch(pb, ws.probs, ws.probs_cap, ws.tiles, ws.tiles_cap, st);
    }
    // contractions that need no per-pair product: T3 and T4 over all pairs
    ContractArgs a{};
    a.pair_ptr = pl.dptr;
    a.slot_out = pl.dslot;
    a.beta = P.beta;
    a.tol = pole_res;
    a.out = d_out;
    auto launch = [&](auto kern, int da, int db, int npairs) {
        if (npairs <= 0 || da <= 0 || db <= 0) return;
        dim3 grid(ceil_div((long)da * db, CT_CHUNK), npairs);
        kern<<<grid, CT_THREADS, 0, st>>>(a);
        check_launch("contract_kernel");
    };
    a.pair0 = 0;
    // T3: a in S1, b in S3, L = P[z1] (a,b), R = Q[z3] (b,a)
    a.Lm = ws.Pm; a.L_stride = s13; a.L_idx = pl.dpi1; a.L_sa = d3; a.L_sb = 1;
    a.Rm = ws.Q; a.R_stride = s31; a.R_idx = pl.dpi3; a.R_sa = 1; a.R_sb = d1;
    a.Ea = E1; a.Eb = E3; a.wa = w1; a.wb = w3; a.da = d1; a.db = d3; a.s = pl.ds3; a.coef = sign;
    launch(contract_kernel<cd, 3>, d1, d3, NP);
    // T4: a in S2, b in S4, L = R[z3] (a,b), R = L[z1] (b,a)
    a.Lm = ws.R; a.L_stride = s24; a.L_idx = pl.dpi3; a.L_sa = d4; a.L_sb = 1;
    a.Rm = ws.L; a.R_stride = s42; a.R_idx = pl.dpi1; a.R_sa = 1; a.R_sb = d2;
    a.Ea = E2; a.Eb = E4; a.wa = w2; a.wb = w4; a.da = d2; a.db = d4; a.s = pl.ds4; a.coef = sign;
    launch(contract_kernel<cd, 4>, d2, d4, NP);

    // per-pair GEMMs (dominant), in chunks of pairs that fit the workspace
    const long per_pair = s32 + s14;
    const int chunk = (int)std::max<long>(1, std::min<long>(NP, ws.pair_cap / std::max<long>(per_pair, 1)));
    for (int q0 = 0; q0 < NP; q0 += chunk) {
        const int nq = std::min(chunk, NP - q0);
        std::vector<GemmProblem<cd, cd, cd>> pc;
        cd* X = ws.X;
        cd* Y = ws.X + (long)nq * s32;
        for (int q = 0; q < nq; ++q) {
            const int i1 = pl.pi1[q0 + q], i3 = pl.pi3[q0 + q];
            pc.push_back(prob<cd, cd>(ws.C3 + i3 * s34, ws.L + i1 * s42, X + q * s32, d3, d2, d4));   // X
            pc.push_back(prob<cd, cd>(ws.Pm + i1 * s13, ws.C3 + i3 * s34, Y + q * s14, d1, d4, d3));  // Y
        }
        PGX_CUDA(cudaEventRecord(ev0, st));
        launch_gemm_batch(pc, ws.probs, ws.probs_cap, ws.tiles, ws.tiles_cap, st);
        PGX_CUDA(cudaEventRecord(ev1, st));
        PGX_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.f;
        PGX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        gemm_ms += ms;
        gemm_flops += 8.0 * nq * ((double)d3 * d2 * d4 + (double)d1 * d4 * d3);
        a.pair0 = q0;
        // T1: a in S2, b in S3, L = X[pair] (X_ba), R = O2 (a,b)
        a.Lm = X; a.L_stride = s32; a.L_idx = nullptr; a.L_sa = 1; a.L_sb = d2;
        a.Rm = O2; a.R_stride = 0; a.R_idx = nullptr; a.R_sa = d3; a.R_sb = 1;
        a.Ea = E2; a.Eb = E3; a.wa = w2; a.wb = w3; a.da = d2; a.db = d3; a.s = pl.ds1; a.coef = -sign;
        launch(contract_kernel<T, 1>, d2, d3, nq);
        // T2: a in S1, b in S4, L = Y[pair] (a,b), R = CX4 (b,a)
        a.Lm = Y; a.L_stride = s14; a.L_idx = nullptr; a.L_sa = d4; a.L_sb = 1;
        a.Rm = X4; a.R_stride = 0; a.R_idx = nullptr; a.R_sa = 1; a.R_sb = d1;
        a.Ea = E1; a.Eb = E4; a.wa = w1; a.wb = w4; a.da = d1; a.db = d4; a.s = pl.ds2; a.coef = sign;
        launch(contract_kernel<T, 2>, d1, d4, nq);
    }
}

}  // namespace


void run_g2(pgx_ctx* c, int nparts, const pgx_g2_part* parts, int nfreq, const double* z, double pole_res,
            double coef_tol, int flags, double* out) {
    (void)coef_tol;
    (void)flags;
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    PGX_CHECK(P.have_w, PGX_ERR_STATE, "weights must be computed before pgx_g2");
    PGX_CHECK(nfreq >= 0 && nparts >= 0, PGX_ERR_ARG, "negative size");
    for (int q = 0; q < nparts; ++q) {
        const pgx_g2_part& gp = parts[q];
        for (int k = 0; k < 4; ++k) {
            PGX_CHECK(gp.op[k] >= 0 && gp.op[k] < (int)P.ops.size(), PGX_ERR_ARG, "bad operator id in G2 part");
            PGX_CHECK(gp.block[k] >= 0 && gp.block[k] < P.nblocks, PGX_ERR_ARG, "bad block in G2 part");
            PGX_CHECK(P.ops[gp.op[k]].rotated, PGX_ERR_STATE, "G2 operator not rotated");
        }
        for (int k = 0; k < 4; ++k) {
            const Operator& o = P.ops[gp.op[k]];
            const int left = gp.block[k], right = gp.block[(k + 1) % 4];
            const int pi = o.by_left[left];
            PGX_CHECK(pi >= 0 && o.parts[pi].right == right, PGX_ERR_ARG, "G2 part is not a block chain");
        }
        bool okp = true;
        for (int k = 0; k < 3; ++k) okp = okp && gp.perm[k] >= 0 && gp.perm[k] < 3;
        PGX_CHECK(okp && gp.perm[0] != gp.perm[1] && gp.perm[1] != gp.perm[2] && gp.perm[0] != gp.perm[2],
                  PGX_ERR_ARG, "bad permutation");
        PGX_CHECK(gp.sign == 1 || gp.sign == -1, PGX_ERR_ARG, "bad permutation sign");
    }
    if (flags & PGX_G2_ANCHORED) {
        PGX_CHECK(coef_tol >= 0.0, PGX_ERR_ARG, "anchor threshold must be non-negative");
        ScopedEvents ev(2);
        const cudaEvent_t a0 = ev[0], a1 = ev[1];
        PGX_CUDA(cudaEventRecord(a0, st));
        const int split = (flags & PGX_G2_SPLIT_I8) ? c->g2_split_slices : 0;
        if (split && c->oz.err.p) PGX_CUDA(cudaMemsetAsync(c->oz.err.p, 0, sizeof(int), st));
        run_g2_anchored(c, nparts, parts, nfreq, z, pole_res, coef_tol, split, out);
        if (split && c->oz.err.p) {
            int e = 0;
            PGX_CUDA(cudaMemcpy(&e, c->oz.err.p, sizeof(int), cudaMemcpyDeviceToHost));
            PGX_CHECK(e == 0, PGX_ERR_TIMEOUT, "split product: a tensor-core wait expired");
        }
        PGX_CUDA(cudaEventRecord(a1, st));
        PGX_CUDA(cudaEventSynchronize(a1));
        float t = 0.f;
        PGX_CUDA(cudaEventElapsedTime(&t, a0, a1));
        c->g2t.total_ms = t;
        c->g2t.gemm_ms = 0.0;
        c->g2t.gemm_flops = 0.0;
        return;
    }
    ScopedEvents ev(4);
    const cudaEvent_t e0 = ev[0], e1 = ev[1], ea = ev[2], eb = ev[3];
    PGX_CUDA(cudaEventRecord(ea, st));
    // one frequency plan per distinct permutation
    std::map<std::tuple<int, int, int>, int> perm_id;
    std::vector<Plan> plans;
    plans.reserve(6);
    std::vector<int> part_plan(nparts);
    for (int q = 0; q < nparts; ++q) {
        auto key = std::make_tuple(parts[q].perm[0], parts[q].perm[1], parts[q].perm[2]);
        auto it = perm_id.find(key);
        if (it == perm_id.end()) {
            it = perm_id.emplace(key, (int)plans.size()).first;
            plans.emplace_back();
        }
        part_plan[q] = it->second;
    }
    for (auto& kv : perm_id) {
        const int perm[3] = {std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first)};
        build_plan(plans[kv.second], perm, nfreq, z);
        upload_plan(plans[kv.second], st);
    }
    // workspace: the largest part decides
    long nA1 = 1, nC3 = 1, nL = 1, nPm = 1, nQ = 1, nR = 1, max_pair = 1, nprob = 1, ntile = 1;
    for (int q = 0; q < nparts; ++q) {
        const Plan& pl = plans[part_plan[q]];
        const long d1 = P.dims[parts[q].block[0]], d2 = P.dims[parts[q].block[1]], d3 = P.dims[parts[q].block[2]],
                   d4 = P.dims[parts[q].block[3]];
        const long N1 = pl.Z1.size(), N3 = pl.Z3.size(), NP = pl.pi1.size();
        nA1 = std::max(nA1, N1 * d1 * d2);
        nC3 = std::max(nC3, N3 * d3 * d4);
        nL = std::max(nL, N1 * d4 * d2);
        nPm = std::max(nPm, N1 * d1 * d3);
        nQ = std::max(nQ, N3 * d3 * d1);
        nR = std::max(nR, N3 * d2 * d4);
        max_pair = std::max(max_pair, d3 * d2 + d1 * d4);
        nprob = std::max(nprob, std::max(2 * NP, 2 * (N1 + N3)));
        const long tz = (N1 + N3) * ((long)ceil_div(d4, GEMM_BM) * ceil_div(d2, GEMM_BN) +
                                     (long)ceil_div(d1, GEMM_BM) * ceil_div(d3, GEMM_BN) +
                                     (long)ceil_div(d3, GEMM_BM) * ceil_div(d1, GEMM_BN) +
                                     (long)ceil_div(d2, GEMM_BM) * ceil_div(d4, GEMM_BN));
        const long tp = NP * ((long)ceil_div(d3, GEMM_BM) * ceil_div(d2, GEMM_BN) +
                              (long)ceil_div(d1, GEMM_BM) * ceil_div(d4, GEMM_BN));
        ntile = std::max(ntile, std::max(tz, tp));
    }
    long np_max = 1;
    for (auto& pl : plans) np_max = std::max<long>(np_max, (long)pl.pi1.size());
    // pair workspace: at most 16 GiB of complex doubles, at least one pair
    const long pair_budget = std::max<long>(max_pair, std::min<long>(np_max * max_pair, (16L << 30) / (long)sizeof(cd)));
    Workspace ws{};
    DevBuf* S = c->scratch;
    S[0].reserve(nA1 * sizeof(cd));
    S[1].reserve(nC3 * sizeof(cd));
    S[2].reserve(nL * sizeof(cd));
    S[3].reserve(nPm * sizeof(cd));
    S[4].reserve(nQ * sizeof(cd));
    S[5].reserve(nR * sizeof(cd));
    S[6].reserve(pair_budget * sizeof(cd));
    S[7].reserve(nprob * sizeof(GemmProblem<cd, cd, cd>));
    S[8].reserve(gemm_index_bytes(nprob));
    S[9].reserve(std::max(nfreq, 1) * sizeof(cd));
    ws.A1 = S[0].as<cd>();
    ws.C3 = S[1].as<cd>();
    ws.L = S[2].as<cd>();
    ws.Pm = S[3].as<cd>();
    ws.Q = S[4].as<cd>();
    ws.R = S[5].as<cd>();
    ws.X = S[6].as<cd>();
    ws.pair_cap = pair_budget;
    ws.probs = S[7].p;
    ws.probs_cap = S[7].bytes;
    ws.tiles = S[8].p;
    ws.tiles_cap = S[8].bytes;
    cd* d_out = S[9].as<cd>();
    PGX_CUDA(cudaMemsetAsync(d_out, 0, std::max(nfreq, 1) * sizeof(cd), st));
    double gemm_ms = 0.0, gemm_flops = 0.0;
    if (nfreq > 0) {
        for (int q = 0; q < nparts; ++q) {
            if (P.is_complex)
                g2_part<cd>(c, parts[q], plans[part_plan[q]], ws, pole_res, d_out, e0, e1, gemm_ms, gemm_flops);
            else
                g2_part<double>(c, parts[q], plans[part_plan[q]], ws, pole_res, d_out, e0, e1, gemm_ms, gemm_flops);
        }
    }
    if (nfreq > 0) PGX_CUDA(cudaMemcpyAsync(out, d_out, nfreq * sizeof(cd), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaEventRecord(eb, st));
    PGX_CUDA(cudaEventSynchronize(eb));
    float tot = 0.f;
    PGX_CUDA(cudaEventElapsedTime(&tot, ea, eb));
    c->g2t.total_ms = tot;
    c->g2t.gemm_ms = gemm_ms;
    c->g2t.gemm_flops = gemm_flops;
}

}  // namespace pgx

namespace pgx {

void run_g2_count(pgx_ctx* c, int nparts, const pgx_g2_part* parts, double coef_tol, double nz_tol,
                  long long* count) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    PGX_CHECK(P.have_w, PGX_ERR_STATE, "weights must be computed before counting");
    for (int q = 0; q < nparts; ++q) {
        const pgx_g2_part& gp = parts[q];
        for (int k = 0; k < 4; ++k) {
            PGX_CHECK(gp.op[k] >= 0 && gp.op[k] < (int)P.ops.size() && gp.block[k] >= 0 && gp.block[k] < P.nblocks,
                      PGX_ERR_ARG, "bad G2 part");
            const Operator& o = P.ops[gp.op[k]];
            const int pi = o.by_left[gp.block[k]];
            PGX_CHECK(o.rotated && pi >= 0 && o.parts[pi].right == gp.block[(k + 1) % 4], PGX_ERR_ARG,
                      "G2 part is not a block chain of rotated operators");
        }
    }
    // zero entries (|x| <= nz) of every operator part the chains use: a chain
    // whose four parts have none is counted in closed form
    std::map<std::pair<int, int>, int> zslot;
    for (int q = 0; q < nparts; ++q)
        for (int k = 0; k < 4; ++k) {
            const int pi = P.ops[parts[q].op[k]].by_left[parts[q].block[k]];
            zslot.emplace(std::make_pair(parts[q].op[k], pi), (int)zslot.size());
        }
    DevBuf& b = c->scratch[10];
    // slot 0: quadruples counted by count_kernel; slot 1: quadruples of the dense
    // chains that fail the weight filter; then one zero count per operator part
    b.reserve((2 + zslot.size()) * sizeof(unsigned long long));
    PGX_CUDA(cudaMemsetAsync(b.p, 0, (2 + zslot.size()) * sizeof(unsigned long long), st));
    unsigned long long* d_cnt = b.as<unsigned long long>();
    for (const auto& kv : zslot) {
        const Operator& o = P.ops[kv.first.first];
        const OpPart& op = o.parts[kv.first.second];
        const long n = (long)op.dl * op.dr;
        const int blocks = (int)std::max<long>(1, std::min<long>(ceil_div(n, 256), 148L * 8));
        if (o.is_complex)
            zero_count_kernel<cd><<<blocks, 256, 0, st>>>(o.mat.as<cd>() + op.off, n, nz_tol, d_cnt + 2 + kv.second);
        else
            zero_count_kernel<double><<<blocks, 256, 0, st>>>(o.mat.as<double>() + op.off, n, nz_tol,
                                                              d_cnt + 2 + kv.second);
        check_launch("zero_count_kernel");
    }
    std::vector<unsigned long long> zeros(zslot.size());
    if (!zeros.empty())
        PGX_CUDA(cudaMemcpyAsync(zeros.data(), d_cnt + 2, zeros.size() * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, st));
    std::vector<double> w(P.esize);
    PGX_CUDA(cudaMemcpyAsync(w.data(), P.d_w, P.esize * sizeof(double), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    // cold weights (w <= tol) of every block, sorted descending
    std::vector<double> cold;
    std::vector<long> cold_off(P.nblocks + 1, 0);
    for (int bl = 0; bl < P.nblocks; ++bl) {
        cold_off[bl] = (long)cold.size();
        for (int i = 0; i < P.dims[bl]; ++i) {
            const double x = w[P.eoff[bl] + i];
            if (!(x > coef_tol)) cold.push_back(x);
        }
        std::sort(cold.begin() + cold_off[bl], cold.end(), [](double x, double y) { return x > y; });
    }
    cold_off[P.nblocks] = (long)cold.size();
    // the block-local index of every cold weight, in the same order
    std::vector<int> coldi(cold.size());
    for (int bl = 0; bl < P.nblocks; ++bl) {
        std::vector<int> ord;
        for (int i = 0; i < P.dims[bl]; ++i)
            if (!(w[P.eoff[bl] + i] > coef_tol)) ord.push_back(i);
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return w[P.eoff[bl] + x] > w[P.eoff[bl] + y]; });
        std::copy(ord.begin(), ord.end(), coldi.begin() + cold_off[bl]);
    }
    DevBuf& cb = c->scratch[11];
    const size_t cbytes = (std::max<size_t>(cold.size(), 1) * sizeof(double) + 255) & ~size_t(255);
    cb.reserve(cbytes + std::max<size_t>(coldi.size(), 1) * sizeof(int));
    if (!cold.empty()) {
        h2d(cb.p, cold.data(), cold.size() * sizeof(double), st);
        h2d(cb.as<char>() + cbytes, coldi.data(), coldi.size() * sizeof(int), st);
    }
    const double* d_cold = cb.as<double>();
    const int* d_coldi = reinterpret_cast<const int*>(cb.as<char>() + cbytes);
    // zero lists of the operator parts of chains that have zero elements,
    // built on first use: (row, column) pairs gathered on the device, sorted
    // on the host into row and column lists
    struct ZLists {
        DevBuf buf;
        const int *roff = nullptr, *ridx = nullptr, *coff = nullptr, *cidx = nullptr;
    };
    std::map<int, ZLists> zcache;
    DevBuf pairs_b, ctr_b;
    auto zl = [&](int opid, int left, int key) -> const ZLists& {
        auto it = zcache.find(key);
        if (it != zcache.end()) return it->second;
        const Operator& o = P.ops[opid];
        const OpPart& op = o.parts[o.by_left[left]];
        const long nzero = (long)zeros[key];
        ZLists& L = zcache[key];
        std::vector<int2> pr(nzero);
        if (nzero > 0) {
            pairs_b.reserve(nzero * sizeof(int2));
            ctr_b.reserve(sizeof(unsigned long long));
            PGX_CUDA(cudaMemsetAsync(ctr_b.p, 0, sizeof(unsigned long long), st));
            const long n = (long)op.dl * op.dr;
            const int blocks = (int)std::max<long>(1, std::min<long>(ceil_div(n, 256), 148L * 8));
            if (o.is_complex)
                zero_list_kernel<cd><<<blocks, 256, 0, st>>>(o.mat.as<cd>() + op.off, op.dl, op.dr, nz_tol,
                                                             pairs_b.as<int2>(), ctr_b.as<unsigned long long>(), nzero);
            else
                zero_list_kernel<double><<<blocks, 256, 0, st>>>(o.mat.as<double>() + op.off, op.dl, op.dr, nz_tol,
                                                                 pairs_b.as<int2>(), ctr_b.as<unsigned long long>(),
                                                                 nzero);
            check_launch("zero_list_kernel");
            PGX_CUDA(cudaMemcpyAsync(pr.data(), pairs_b.p, nzero * sizeof(int2), cudaMemcpyDeviceToHost, st));
            PGX_CUDA(cudaStreamSynchronize(st));
        }
        std::vector<int> roff(op.dl + 1, 0), coff(op.dr + 1, 0), ridx(nzero), cidx(nzero);
        std::sort(pr.begin(), pr.end(), [](int2 x, int2 y) { return x.x != y.x ? x.x < y.x : x.y < y.y; });
        for (long k = 0; k < nzero; ++k) {
            ++roff[pr[k].x + 1];
            ridx[k] = pr[k].y;
        }
        std::sort(pr.begin(), pr.end(), [](int2 x, int2 y) { return x.y != y.y ? x.y < y.y : x.x < y.x; });
        for (long k = 0; k < nzero; ++k) {
            ++coff[pr[k].y + 1];
            cidx[k] = pr[k].x;
        }
        for (int r = 0; r < op.dl; ++r) roff[r + 1] += roff[r];
        for (int cc = 0; cc < op.dr; ++cc) coff[cc + 1] += coff[cc];
        auto al = [](size_t x) { return (x * sizeof(int) + 255) & ~size_t(255); };
        const size_t o1 = 0, o2 = o1 + al(roff.size()), o3 = o2 + al(std::max<long>(nzero, 1)),
                     o4 = o3 + al(coff.size()), tot = o4 + al(std::max<long>(nzero, 1));
        L.buf.reserve(tot);
        char* base = L.buf.as<char>();
        h2d(base + o1, roff.data(), roff.size() * sizeof(int), st);
        if (nzero) h2d(base + o2, ridx.data(), nzero * sizeof(int), st);
        h2d(base + o3, coff.data(), coff.size() * sizeof(int), st);
        if (nzero) h2d(base + o4, cidx.data(), nzero * sizeof(int), st);
        L.roff = reinterpret_cast<const int*>(base + o1);
        L.ridx = reinterpret_cast<const int*>(base + o2);
        L.coff = reinterpret_cast<const int*>(base + o3);
        L.cidx = reinterpret_cast<const int*>(base + o4);
        return L;
    };
    unsigned long long dense_total = 0;  // closed-form chains: d1 d2 d3 d4 each
    for (int q = 0; q < nparts; ++q) {
        const pgx_g2_part& gp = parts[q];
        const int S1 = gp.block[0], S2 = gp.block[1], S3 = gp.block[2], S4 = gp.block[3];
        const int d1 = P.dims[S1], d2 = P.dims[S2], d3 = P.dims[S3], d4 = P.dims[S4];
        bool dense = true;
        for (int k = 0; k < 4; ++k)
            dense = dense && zeros[zslot.at({gp.op[k], P.ops[gp.op[k]].by_left[gp.block[k]]})] == 0;
        if (dense) {
            // every (i1, i2, i3, i4) is enumerated; subtract those failing the weight filter
            dense_total += (unsigned long long)d1 * d2 * d3 * d4;
            const int n1 = (int)(cold_off[S1 + 1] - cold_off[S1]), n3 = (int)(cold_off[S3 + 1] - cold_off[S3]);
            const int n2 = (int)(cold_off[S2 + 1] - cold_off[S2]), n4 = (int)(cold_off[S4 + 1] - cold_off[S4]);
            const long n = (long)n1 * n3;
            if (n > 0 && n2 > 0 && n4 > 0) {
                cold_fail_kernel<<<(int)ceil_div(n, 256), 256, 0, st>>>(
                    d_cold + cold_off[S1], n1, d_cold + cold_off[S3], n3, d_cold + cold_off[S2], n2,
                    d_cold + cold_off[S4], n4, coef_tol, d_cnt + 1);
                check_launch("cold_fail_kernel");
            }
            continue;
        }
        // chains with zero elements: zero lists of the four parts, then one
        // thread per (i1, i3)
        const int keys[4] = {zslot.at({gp.op[0], P.ops[gp.op[0]].by_left[S1]}),
                             zslot.at({gp.op[1], P.ops[gp.op[1]].by_left[S2]}),
                             zslot.at({gp.op[2], P.ops[gp.op[2]].by_left[S3]}),
                             zslot.at({gp.op[3], P.ops[gp.op[3]].by_left[S4]})};
        const ZLists& L1 = zl(gp.op[0], S1, keys[0]);
        const ZLists& L2 = zl(gp.op[1], S2, keys[1]);
        const ZLists& L3 = zl(gp.op[2], S3, keys[2]);
        const ZLists& L4 = zl(gp.op[3], S4, keys[3]);
        ZeroLists zd{L1.roff, L1.ridx, L2.coff, L2.cidx, L3.roff, L3.ridx, L4.coff, L4.cidx};
        const long n = (long)d1 * d3;
        const double *w1 = P.d_w + P.eoff[S1], *w2 = P.d_w + P.eoff[S2], *w3 = P.d_w + P.eoff[S3], *w4 = P.d_w + P.eoff[S4];
        const int n2c = (int)(cold_off[S2 + 1] - cold_off[S2]), n4c = (int)(cold_off[S4 + 1] - cold_off[S4]);
        count_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(zd, d1, d2, d3, d4, w1, w2, w3, w4,
                                                                 d_cold + cold_off[S2], d_coldi + cold_off[S2], n2c,
                                                                 d_cold + cold_off[S4], n4c, coef_tol, d_cnt);
        check_launch("count_kernel");
    }
    unsigned long long h[2] = {0, 0};
    PGX_CUDA(cudaMemcpyAsync(h, d_cnt, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    *count = (long long)(h[0] + dense_total - h[1]);
}

}  // namespace pgx
