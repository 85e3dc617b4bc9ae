// Complex FP64 products on the int8 tensor cores (tcgen05, kind::i8): the
// split ("Ozaki") scheme.  Used by the anchored G2 for its largest products
// (the stacked (z1, z3) products) when PGX_G2_SPLIT_I8 is set.
//
// Each row of A and each column of B is scaled by a power of two so that its
// largest |Re| or |Im| is below 1, and cut into S balanced digits of base 254:
//   127 x 2^-e = sum_s d_s 254^-s,  d_s integer in [-127, 127]
// (d_0 = rint(127 x 2^-e), then each remainder, in [-1/2, 1/2], times 254 and
// rounded to the nearest integer: every digit fits a signed byte and carries
// log2(254) = 7.99 bits; the remainder left after S digits is below
// 254^-(S-1) / 254 of the row's or column's largest element).  The product is
//   C = diag(2^e) [ sum_{a+b<S} 254^-(a+b) / 127^2 A_a B_b ] diag(2^f),
// each A_a B_b exact in int32, the diagonals a+b = s summed in FP64.  The
// dropped diagonals (a+b >= S) are bounded by (S-1) 254^-S K |A|max |B|max,
// the remainders by 2 254^-S K |A|max |B|max: in all about 2^-37.4 K of
// |A|max |B|max at S = 5 and 2^-45.1 K at S = 6.
// Complex operands become one real product of twice the depth:
//   A' = [Re A, Im A] (M x 2K) and, per complex column j of B, two columns
//   [Re B_j; -Im B_j] (the real part of C_j) and [Im B_j; Re B_j] (its imaginary
//   part), so C' = A' B' holds Re C and Im C in adjacent columns.
// Digits are stored K-contiguous per row (A) or per column (B):
//   A row i: [digits of slice 0 | slice 1 | ... | slice S-1], each K2 = 2K
//   rounded up to 128 bytes; B column j: [slice S-1 | ... | slice 0].
// Then diagonal s is one product of depth (s+1) K2 with A from offset 0 and
// B from offset (S-1-s) K2: both operands are plain strided views.  Odd
// diagonals sweep their depth from the end, so consecutive diagonals meet on
// the planes and k-blocks read last (the int32 sums do not depend on order).
//
// The GEMM kernel: one CTA per 128 x 256 tile of C' (128 complex columns) and
// batch item; tcgen05.mma with M = 128, N = 256 and K = 32 bytes per
// instruction, into one of two TMEM accumulators (diagonals alternate between
// them, 2 x 256 = all 512 columns), so one diagonal is added into C while the
// next runs.  Every mbarrier wait
// is bounded (about 2 s of %globaltimer); on expiry the CTA sets the error
// flag, stops issuing work, waits (bounded) for its copies and tensor-core
// work in flight, frees its TMEM and returns.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <vector>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

constexpr int OZ_BM = 128, OZ_BN = 256, OZ_BK = 128;  // tile rows, tile columns, k-block bytes
constexpr int OZ_STAGES = 4;
// tiles run in groups of 16 row tiles: a wave of 148 CTAs then holds about 16
// row tiles x 9 column tiles, near the minimum of the A and B panel bytes it
// reads per k-block (16 KiB per row tile, 32 KiB per column tile)
constexpr int OZ_GROUP_M = 16;
constexpr int OZ_STAGE_BYTES = (OZ_BM + OZ_BN) * OZ_BK;  // 48 KiB
constexpr int OZ_SMEM = OZ_STAGES * OZ_STAGE_BYTES + 1024 + 256;
constexpr int OZ_TMEM_COLS = 2 * OZ_BN;  // two accumulators: all 512 columns
constexpr unsigned long long OZ_WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for phase `parity` of an mbarrier by a full warp; false (for
// the whole warp) when any lane's wait expired.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = gtimer();
    bool done = false;
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) {
            done = true;
            break;
        }
        if (gtimer() - t0 > OZ_WAIT_NS) break;
    }
    return __all_sync(0xffffffffu, done);
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (the layout written by oz_load_stage).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
    d |= (uint64_t)1 << 16;                    // leading byte offset (unused with this swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;          // stride byte offset: 8 rows x 128 bytes
    d |= (uint64_t)1 << 46;                    // descriptor version
    d |= (uint64_t)2 << 61;                    // 128-byte swizzle
    return d;
}

// Instruction descriptor: s32 accumulator, signed 8-bit A and B, both
// K-major, N = 128, M = 128.
constexpr uint32_t OZ_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_BN >> 3) << 17) |
                              ((uint32_t)(OZ_BM >> 4) << 24);

// 2^e exactly: the bit pattern of a normal double, ldexp outside that range.
__device__ __forceinline__ double pow2i(int e) {
    return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

// Digit base of the split and the weight of diagonal s of the product:
// 254^-s / 127^2 (127 scales the leading digit of each operand).
constexpr double OZ_BASE = 254.0;
constexpr double OZ_ROUND = 6755399441055744.0;  // 1.5 2^52
__device__ __forceinline__ double diag_weight(int s) {
    double w = 1.0 / (127.0 * 127.0);
    for (int t = 0; t < s; ++t) w *= 1.0 / OZ_BASE;
    return w;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

// The product kernel, with specialised warps (384 threads): warp 8 lane 0
// loads each k-block of A' and B' with the tensor-memory accelerator (3-D
// tensor maps over [item][row][S*K2], 128-byte boxes of 128 (A) or 256 (B)
// rows, 128-byte swizzle; rows past the matrix read as zero) into a 4-stage
// ring; warp 9 lane 0
// issues the MMAs as soon as a stage is full and releases it with
// tcgen05.commit; warps 0-7 (TMEM lanes 32 (w % 4) ..., 128 columns per warp
// half) read each finished diagonal's accumulator with tcgen05.ld, add it,
// scaled by 2^(e_i + f_j) 254^-s / 127^2, into C (stored by the first diagonal,
// read and added by the others; the tile stays in L2) and release it.  Barriers: full and
// empty per stage; per accumulator "finished" (commit) and "drained" (one
// arrival per drain warp).
struct OzArgs2 {
    int tiles_m, tiles_n;  // tile counts of C' (blockIdx.x enumerates both, grouped by OZ_GROUP_M row tiles)
    int a_items, b_items;  // 0: the operand is shared by all items
    const int* ea;
    long ea_item;
    const int* fb;
    long fb_item;
    int M, N, K2, S;
    cd* C;
    long c_item, sc_i, sc_j;
    int* err;
};

__device__ __forceinline__ void tma_load3(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(384, 1) oz_gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA,
                                                             const __grid_constant__ CUtensorMap tmB, OzArgs2 p) {
    extern __shared__ char oz_raw[];
    char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(oz_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + OZ_STAGES * OZ_STAGE_BYTES);
    uint64_t* empty = full + OZ_STAGES;
    uint64_t* accf = empty + OZ_STAGES;  // [2]
    uint64_t* acce = accf + 2;           // [2]
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(acce + 2);
    volatile int* s_fail = reinterpret_cast<volatile int*>(s_tmem + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int item = blockIdx.z;
    // tiles in groups of OZ_GROUP_M row tiles, columns within a group: the
    // CTAs resident together share few A and B panels, which then stay in L2
    const int lin = blockIdx.x, per_group = OZ_GROUP_M * p.tiles_n;
    const int first_m = (lin / per_group) * OZ_GROUP_M, gsz = min(p.tiles_m - first_m, OZ_GROUP_M);
    const int tm = first_m + (lin % per_group) % gsz, tn = (lin % per_group) / gsz;
    const int i0 = tm * OZ_BM, j0 = tn * OZ_BN;

    if (tid == 0) {
        for (int q = 0; q < OZ_STAGES; ++q) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[q])) : "memory");
        }
        for (int q = 0; q < 2; ++q) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&accf[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 8;\n" ::"r"(smem_u32(&acce[q])) : "memory");
        }
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(s_tmem)),
                     "r"(OZ_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *s_tmem;
    const int kbd = p.K2 / OZ_BK;
    int total = 0;
    for (int s = 0; s < p.S; ++s) total += (s + 1) * kbd;

    // single-thread bounded wait (the roles below run on one lane)
    auto wait1 = [&](uint32_t bar, uint32_t parity) {
        const unsigned long long t0 = gtimer();
        while (true) {
            uint32_t ok;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(ok)
                : "r"(bar), "r"(parity)
                : "memory");
            if (ok) return true;
            if (*s_fail || gtimer() - t0 > OZ_WAIT_NS) {
                *s_fail = 1;
                return false;
            }
        }
    };

    int issued = 0;                // producer: k-blocks whose loads were issued
    if (warp == 8 && lane == 0) {  // producer
        int s = 0, kb = 0;
        for (int it = 0; it < total; ++it) {
            const int st = it % OZ_STAGES, use = it / OZ_STAGES;
            if (use >= 1 && !wait1(smem_u32(&empty[st]), (uint32_t)((use - 1) & 1))) break;
            const uint32_t fb = smem_u32(&full[st]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb), "r"(OZ_STAGE_BYTES)
                         : "memory");
            const uint32_t dst = smem_u32(smem + st * OZ_STAGE_BYTES);
            // odd diagonals run backwards, so each diagonal starts on the
            // digit planes and k-blocks the previous one read last (still in L2)
            const int kx = (s & 1) ? (s + 1) * kbd - 1 - kb : kb;
            tma_load3(dst, &tmA, kx * OZ_BK, i0, p.a_items ? item : 0, fb);
            tma_load3(dst + OZ_BM * OZ_BK, &tmB, (p.S - 1 - s) * p.K2 + kx * OZ_BK, j0, p.b_items ? item : 0, fb);
            issued = it + 1;
            if (++kb == (s + 1) * kbd) {
                kb = 0;
                ++s;
            }
        }
    } else if (warp == 9 && lane == 0) {  // MMA issuer
        int s = 0, kb = 0, last = -1;
        for (int it = 0; it < total; ++it) {
            const int st = it % OZ_STAGES, use = it / OZ_STAGES;
            if (kb == 0 && s >= 2 && !wait1(smem_u32(&acce[s & 1]), (uint32_t)(((s >> 1) - 1) & 1))) break;
            if (!wait1(smem_u32(&full[st]), (uint32_t)(use & 1))) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = smem_u32(smem + st * OZ_STAGE_BYTES), sb = sa + OZ_BM * OZ_BK;
            const uint32_t dt = tmem + (uint32_t)((s & 1) * OZ_BN);
#pragma unroll
            for (int k = 0; k < OZ_BK / 32; ++k) {
                const uint64_t da = sw128_desc(sa + 32 * k), db = sw128_desc(sb + 32 * k);
                const uint32_t accum = (kb == 0 && k == 0) ? 0u : 1u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(dt), "l"(da), "l"(db), "r"(OZ_IDESC), "r"(accum)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&empty[st]))
                         : "memory");
            last = it;
            if (++kb == (s + 1) * kbd) {
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 smem_u32(&accf[s & 1]))
                             : "memory");
                kb = 0;
                ++s;
            }
        }
        // the tensor core has finished every issued MMA before TMEM is freed
        if (last >= 0) {
            const unsigned long long t0 = gtimer();
            while (true) {
                uint32_t ok;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(ok)
                    : "r"(smem_u32(&empty[last % OZ_STAGES])), "r"((uint32_t)((last / OZ_STAGES) & 1))
                    : "memory");
                if (ok) break;
                if (gtimer() - t0 > OZ_WAIT_NS) {
                    *s_fail = 1;
                    break;
                }
            }
        }
    }
    // drain: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows) and the
    // 128 accumulator columns of half w / 4, and adds them, scaled, to C
    const int lane_base = 32 * (warp & 3), col_base = 128 * ((warp >> 2) & 1);
    if (warp < 8) {
        const int i = i0 + lane_base + lane;
        const bool row_ok = i < p.M;
        const int ei = row_ok ? p.ea[item * p.ea_item + i] : 0;
        cd* crow = p.C + item * p.c_item + (long)(row_ok ? i : 0) * p.sc_i;
        const int* fbi = p.fb + item * p.fb_item;
        for (int s = 0; s < p.S; ++s) {
            if (!mbar_wait(smem_u32(&accf[s & 1]), (uint32_t)((s >> 1) & 1))) {
                *s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const double dw = diag_weight(s);
            const uint32_t base = tmem + ((uint32_t)lane_base << 16) + (uint32_t)((s & 1) * OZ_BN + col_base);
#pragma unroll 1
            for (int q = 0; q < 8; ++q) {
                uint32_t v[16];
                tmem_ld16(base + 16 * q, v);
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (row_ok) {
                    // the eight earlier partial sums are read before any store, so
                    // their loads are in flight together
                    const int jc0 = (j0 + col_base) / 2 + 8 * q;
                    cd old[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        old[e] = (s > 0 && jc0 + e < p.N) ? crow[(long)(jc0 + e) * p.sc_j] : cd{0.0, 0.0};
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int jc = jc0 + e;
                        if (jc < p.N) {
                            const double sc = pow2i(ei + fbi[jc]) * dw;
                            const cd add{(double)(int)v[2 * e] * sc, (double)(int)v[2 * e + 1] * sc};
                            crow[(long)jc * p.sc_j] = s == 0 ? add : cd{old[e].x + add.x, old[e].y + add.y};
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&acce[s & 1])) : "memory");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    // after a failure, loads issued but never consumed land before the CTA
    // exits: the latest use of each stage completes its phase (bounded waits)
    if (warp == 8 && lane == 0 && *s_fail) {
        for (int it = max(0, issued - OZ_STAGES); it < issued; ++it) {
            const unsigned long long t0 = gtimer();
            while (true) {
                uint32_t ok;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(ok)
                    : "r"(smem_u32(&full[it % OZ_STAGES])), "r"((uint32_t)((it / OZ_STAGES) & 1))
                    : "memory");
                if (ok || gtimer() - t0 > OZ_WAIT_NS) break;
            }
        }
    }
    __syncthreads();
    const bool ok = !*s_fail;
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(OZ_TMEM_COLS)
                     : "memory");
    }
    if (!ok && tid == 0) atomicExch(p.err, 1);
}

// ---- the same product on CTA pairs (tcgen05 cta_group::2): one 256 x 256
// tile of C' per pair of CTAs in a cluster of two.  CTA r of the pair loads
// rows 128 r .. 128 r + 127 of the tile's A' rows and of its B' rows (real
// columns of C') into its own shared memory; the even CTA issues
// tcgen05.mma.cta_group::2 with M = 256, N = 256, which reads both CTAs'
// operands and writes rows 128 r .. of the accumulator into CTA r's tensor
// memory.  Per SM, a k-block moves 32 KiB of operands for 128 x 256 x 128
// multiply-adds instead of 48 KiB: the operand traffic from L2, which bounds
// the single-CTA kernel, drops by a third.  Loads are plain (no multicast).
// Barriers: both CTAs' loads complete on the even CTA's "full" barrier (its
// producer posts the expected bytes of both); the even CTA's MMA thread
// commits each stage to the "empty" barrier and each finished diagonal to the
// "finished" barrier of both CTAs (one commit per CTA); the drain warps of
// both CTAs arrive on the even CTA's "drained" barrier (16 arrivals).  Every
// wait is bounded as in oz_gemm_tma_kernel; both CTAs always reach the final
// cluster barrier, so neither leaves while its partner may touch its memory.
constexpr int OZ2_HALF = 128;                                  // rows of A' / B' per CTA
constexpr int OZ2_STAGES = 7;  // 7 x 32 KiB + barriers: the most that fits the 227 KiB opt-in limit
constexpr int OZ2_STAGE_BYTES = 2 * OZ2_HALF * OZ_BK;          // 32 KiB per CTA
constexpr int OZ2_SMEM = OZ2_STAGES * OZ2_STAGE_BYTES + 1024 + 256;
constexpr uint32_t OZ2_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) |
                               ((uint32_t)(256 >> 4) << 24);

__device__ __forceinline__ uint32_t cluster_addr(uint32_t local, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}

__device__ __forceinline__ void tma_load3_pair(uint32_t dst, const CUtensorMap* map, int x, int y, int z,
                                               uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void commit_pair(uint32_t bar_cluster) {
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_cluster)
                 : "memory");
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(384, 1)
    oz_gemm_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzArgs2 p) {
    extern __shared__ char oz_raw[];
    char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(oz_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + OZ2_STAGES * OZ2_STAGE_BYTES);
    uint64_t* empty = full + OZ2_STAGES;
    uint64_t* accf = empty + OZ2_STAGES;  // [2]
    uint64_t* acce = accf + 2;            // [2]
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(acce + 2);
    volatile int* s_fail = reinterpret_cast<volatile int*>(s_tmem + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(rank));
    const bool lead = rank == 0;
    const int item = blockIdx.z;
    // tiles of 256 x 256 in groups of OZ_GROUP_M row tiles, one per CTA pair
    const int pair = blockIdx.x >> 1, per_group = OZ_GROUP_M * p.tiles_n;
    const int first_m = (pair / per_group) * OZ_GROUP_M, gsz = min(p.tiles_m - first_m, OZ_GROUP_M);
    const int tm = first_m + (pair % per_group) % gsz, tn = (pair % per_group) / gsz;
    const int i0 = tm * 2 * OZ2_HALF + OZ2_HALF * (int)rank;  // this CTA's rows of A' and of the accumulator
    const int jb = tn * 2 * OZ2_HALF + OZ2_HALF * (int)rank;  // this CTA's rows of B'
    const int j0 = tn * 2 * OZ2_HALF;                         // the pair's first real column of C'

    if (tid == 0) {
        for (int q = 0; q < OZ2_STAGES; ++q) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[q])) : "memory");
        }
        for (int q = 0; q < 2; ++q) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&accf[q])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 16;\n" ::"r"(smem_u32(&acce[q])) : "memory");
        }
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(s_tmem)),
                     "r"(OZ_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    cluster_sync_all();  // both CTAs' barriers exist before either signals the other's
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *s_tmem;
    const int kbd = p.K2 / OZ_BK;
    int total = 0;
    for (int s = 0; s < p.S; ++s) total += (s + 1) * kbd;

    auto wait1 = [&](uint32_t bar, uint32_t parity) {
        const unsigned long long t0 = gtimer();
        while (true) {
            uint32_t ok;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(ok)
                : "r"(bar), "r"(parity)
                : "memory");
            if (ok) return true;
            if (*s_fail || gtimer() - t0 > OZ_WAIT_NS) {
                *s_fail = 1;
                return false;
            }
        }
    };

    int issued = 0;
    if (warp == 8 && lane == 0) {  // producer (both CTAs): loads complete on the even CTA's full barrier
        int s = 0, kb = 0;
        for (int it = 0; it < total; ++it) {
            const int st = it % OZ2_STAGES, use = it / OZ2_STAGES;
            if (use >= 1 && !wait1(smem_u32(&empty[st]), (uint32_t)((use - 1) & 1))) break;
            const uint32_t fb_local = smem_u32(&full[st]);
            if (lead)
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(fb_local),
                             "r"(2 * OZ2_STAGE_BYTES)
                             : "memory");
            const uint32_t fb = cluster_addr(fb_local, 0);
            const uint32_t dst = smem_u32(smem + st * OZ2_STAGE_BYTES);
            const int kx = (s & 1) ? (s + 1) * kbd - 1 - kb : kb;  // odd diagonals backwards, as above
            tma_load3_pair(dst, &tmA, kx * OZ_BK, i0, p.a_items ? item : 0, fb);
            tma_load3_pair(dst + OZ2_HALF * OZ_BK, &tmB, (p.S - 1 - s) * p.K2 + kx * OZ_BK, jb, p.b_items ? item : 0,
                           fb);
            issued = it + 1;
            if (++kb == (s + 1) * kbd) {
                kb = 0;
                ++s;
            }
        }
    } else if (warp == 9 && lane == 0 && lead) {  // MMA issuer (even CTA only)
        int s = 0, kb = 0, last = -1;
        for (int it = 0; it < total; ++it) {
            const int st = it % OZ2_STAGES, use = it / OZ2_STAGES;
            if (kb == 0 && s >= 2 && !wait1(smem_u32(&acce[s & 1]), (uint32_t)(((s >> 1) - 1) & 1))) break;
            if (!wait1(smem_u32(&full[st]), (uint32_t)(use & 1))) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = smem_u32(smem + st * OZ2_STAGE_BYTES), sb = sa + OZ2_HALF * OZ_BK;
            const uint32_t dt = tmem + (uint32_t)((s & 1) * OZ_BN);
#pragma unroll
            for (int k = 0; k < OZ_BK / 32; ++k) {
                const uint64_t da = sw128_desc(sa + 32 * k), db = sw128_desc(sb + 32 * k);
                const uint32_t accum = (kb == 0 && k == 0) ? 0u : 1u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(dt), "l"(da), "l"(db), "r"(OZ2_IDESC), "r"(accum)
                    : "memory");
            }
            const uint32_t eb = smem_u32(&empty[st]);
            commit_pair(cluster_addr(eb, 0));
            commit_pair(cluster_addr(eb, 1));
            last = it;
            if (++kb == (s + 1) * kbd) {
                const uint32_t ab = smem_u32(&accf[s & 1]);
                commit_pair(cluster_addr(ab, 0));
                commit_pair(cluster_addr(ab, 1));
                kb = 0;
                ++s;
            }
        }
        // the tensor cores have finished every issued MMA before TMEM is freed
        if (last >= 0 && !wait1(smem_u32(&empty[last % OZ2_STAGES]), (uint32_t)((last / OZ2_STAGES) & 1))) {
            *s_fail = 1;
        }
    }
    // drain (both CTAs): warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows) and
    // the 128 accumulator columns of half w / 4, and adds them, scaled, to C
    const int lane_base = 32 * (warp & 3), col_base = 128 * ((warp >> 2) & 1);
    if (warp < 8) {
        const int i = i0 + lane_base + lane;
        const bool row_ok = i < p.M;
        const int ei = row_ok ? p.ea[item * p.ea_item + i] : 0;
        cd* crow = p.C + item * p.c_item + (long)(row_ok ? i : 0) * p.sc_i;
        const int* fbi = p.fb + item * p.fb_item;
        for (int s = 0; s < p.S; ++s) {
            if (!mbar_wait(smem_u32(&accf[s & 1]), (uint32_t)((s >> 1) & 1))) {
                *s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const double dw = diag_weight(s);
            const uint32_t base = tmem + ((uint32_t)lane_base << 16) + (uint32_t)((s & 1) * OZ_BN + col_base);
#pragma unroll 1
            for (int q = 0; q < 8; ++q) {
                uint32_t v[16];
                tmem_ld16(base + 16 * q, v);
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (row_ok) {
                    // the eight earlier partial sums are read before any store, so
                    // their loads are in flight together
                    const int jc0 = (j0 + col_base) / 2 + 8 * q;
                    cd old[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        old[e] = (s > 0 && jc0 + e < p.N) ? crow[(long)(jc0 + e) * p.sc_j] : cd{0.0, 0.0};
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int jc = jc0 + e;
                        if (jc < p.N) {
                            const double sc = pow2i(ei + fbi[jc]) * dw;
                            const cd add{(double)(int)v[2 * e] * sc, (double)(int)v[2 * e + 1] * sc};
                            crow[(long)jc * p.sc_j] = s == 0 ? add : cd{old[e].x + add.x, old[e].y + add.y};
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(
                                 cluster_addr(smem_u32(&acce[s & 1]), 0))
                             : "memory");
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    // after a failure, the even CTA waits (bounded) for the loads it can see
    // complete; a short pause covers loads of its partner that were issued
    // for phases it never posted, so nothing lands in freed shared memory
    if (warp == 8 && lane == 0 && *s_fail) {
        if (lead) {
            for (int it = max(0, issued - OZ2_STAGES); it < issued; ++it) {
                const unsigned long long t0 = gtimer();
                while (true) {
                    uint32_t ok;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                        "selp.u32 %0, 1, 0, p;\n\t}"
                        : "=r"(ok)
                        : "r"(smem_u32(&full[it % OZ2_STAGES])), "r"((uint32_t)((it / OZ2_STAGES) & 1))
                        : "memory");
                    if (ok || gtimer() - t0 > OZ_WAIT_NS) break;
                }
            }
        }
        const unsigned long long t0 = gtimer();
        while (gtimer() - t0 < 2000000ull) {
        }
    }
    __syncthreads();
    cluster_sync_all();  // neither CTA leaves while its partner may still use its memory
    const bool ok = !*s_fail;
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(OZ_TMEM_COLS)
                     : "memory");
    }
    if (!ok && tid == 0) atomicExch(p.err, 1);
}

// Digits of an operand.  Output row r (a row of A', or a complex column of B
// giving rows 2r and 2r+1 of B'), reduction index k < K:
//   x(r, k) = X[r*s_r + k*s_k] (+ item*s_item), dressed when Er/Ek are set:
//   x / (z - (Er[r] - Ek[k])) if rk_order, else x / (z - (Ek[k] - Er[r])) -- the
//   dress() convention with (row energy, column energy) of the dressed matrix.
struct OzSrc {
    const void* X;
    int cplx;
    const int* ridx;  // output row r reads source row ridx[r] (nullable), energies included
    long s_r, s_k, s_item;
    const double *Er, *Ek;
    int rk_order;  // 1: dressed matrix has rows r, columns k; 0: rows k, columns r
    const cd* zs;
};

__device__ __forceinline__ cd oz_value(const OzSrc& q, int item, int r, int k) {
    if (q.ridx) r = q.ridx[r];
    const long off = item * q.s_item + (long)r * q.s_r + (long)k * q.s_k;
    const cd x = q.cplx ? static_cast<const cd*>(q.X)[off] : cd{static_cast<const double*>(q.X)[off], 0.0};
    if (!q.Er) return x;
    const cd z = q.zs[item];
    return q.rk_order ? dress(x, q.Er[r], q.Ek[k], z) : dress(x, q.Ek[k], q.Er[r], z);
}

// Digits of an operand in two kernels.  oz_rowmax_kernel: the largest |Re|
// or |Im| of each output row over a range of reduction indices, as the
// exponent e with max < 2^e, merged into ex[] with atomicMax (ex starts below
// every exponent; rows without a non-zero value keep the floor -1000).
// oz_prep_kernel: one CTA per OP_ROWS rows x OP_KC reduction indices: the
// values scaled by 127 2^-e go through a shared tile, then each thread turns
// four consecutive k of one row into digits and stores each digit plane's four
// bytes as one 32-bit word (a warp writes 64 contiguous bytes per row); is_b
// selects the B' layout (two rows per complex column, digits in reverse
// order).  Source reads are coalesced either way: lanes run along k when the
// source is k-contiguous (s_k == 1), along the rows otherwise.
constexpr int OP_ROWS = 32, OP_KC = 64, OP_THREADS = 256, OP_KSPAN = 512;
constexpr int OP_EXP_FLOOR = -1000;  // rows below 2^-1000 keep a representable scale

// Tile slot of (row r, chunk index k): rows 65 slots apart, the 16-byte slot
// index XOR-swizzled so that row-wise, column-wise and 4-strided accesses of
// eight lanes fall on distinct banks.
__device__ __forceinline__ int op_slot(int r, int k) { return r * (OP_KC + 1) + (k ^ ((k >> 3) & 7)); }

__global__ void __launch_bounds__(OP_THREADS) oz_rowmax_kernel(OzSrc q, int R, int K, int* ex, long ex_item) {
    __shared__ double s_part[OP_THREADS / 32][OP_ROWS];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int item = blockIdx.z, r0 = blockIdx.x * OP_ROWS;
    const int k0 = blockIdx.y * OP_KSPAN, k1 = min(K, k0 + OP_KSPAN);
    double mrow = 0.0;  // thread t < OP_ROWS: the maximum of row r0 + t
    if (q.s_k == 1) {   // warp w: rows w, w + 8, w + 16, w + 24; lanes along k
        for (int rr = warp; rr < OP_ROWS; rr += OP_THREADS / 32) {
            double m = 0.0;
            if (r0 + rr < R)
                for (int k = k0 + lane; k < k1; k += 32) {
                    const cd v = oz_value(q, item, r0 + rr, k);
                    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
                }
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) s_part[0][rr] = m;
        }
        __syncthreads();
        if (t < OP_ROWS) mrow = s_part[0][t];
    } else {  // lane = row, warps along k
        double m = 0.0;
        if (r0 + lane < R)
            for (int k = k0 + warp; k < k1; k += OP_THREADS / 32) {
                const cd v = oz_value(q, item, r0 + lane, k);
                m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
            }
        s_part[warp][lane] = m;
        __syncthreads();
        if (t < OP_ROWS) {
            mrow = s_part[0][t];
            for (int w = 1; w < OP_THREADS / 32; ++w) mrow = fmax(mrow, s_part[w][t]);
        }
    }
    if (t < OP_ROWS && r0 + t < R) {
        int e = OP_EXP_FLOOR;
        if (mrow > 0.0) {
            frexp(mrow, &e);  // max = f 2^e, f in [0.5, 1): every |x| 2^-e < 1
            e = max(e, OP_EXP_FLOOR);
        }
        atomicMax(ex + item * ex_item + r0 + t, e);
    }
}

__global__ void __launch_bounds__(OP_THREADS) oz_prep_kernel(OzSrc q, int R, int K, int K2, int S, int is_b,
                                                             int8_t* out, long out_item, const int* ex, long ex_item) {
    __shared__ cd tile[OP_ROWS * (OP_KC + 1)];
    __shared__ double s_scale[OP_ROWS];
    const int t = threadIdx.x;
    const int item = blockIdx.z, r0 = blockIdx.x * OP_ROWS, k0 = blockIdx.y * OP_KC;
    const bool kcontig = q.s_k == 1;
    // 127 2^-e exactly: |x| 127 2^-e < 127, so the leading digit fits a signed byte
    if (t < OP_ROWS) s_scale[t] = r0 + t < R ? ldexp(127.0, -ex[item * ex_item + r0 + t]) : 0.0;
    __syncthreads();
    // scaled values of the chunk into the tile (zero past K and past R)
#pragma unroll 4
    for (int j = 0; j < OP_ROWS * OP_KC / OP_THREADS; ++j) {
        const int idx = t + OP_THREADS * j;
        const int rr = kcontig ? idx / OP_KC : idx % OP_ROWS;
        const int kk = kcontig ? idx % OP_KC : idx / OP_ROWS;
        cd v{0.0, 0.0};
        if (r0 + rr < R && k0 + kk < K) {
            v = oz_value(q, item, r0 + rr, k0 + kk);
            v.x *= s_scale[rr];
            v.y *= s_scale[rr];
        }
        tile[op_slot(rr, kk)] = v;
    }
    __syncthreads();
    const long row_bytes = (long)S * K2;
    const int half = K2 / 2;  // multiple of 64: K2 is a multiple of 128
    // digits: thread -> (row, four consecutive k); 16 threads per row
#pragma unroll
    for (int j = 0; j < OP_ROWS * OP_KC / 4 / OP_THREADS; ++j) {
        const int task = t + OP_THREADS * j;
        const int rr = task / (OP_KC / 4), g = task % (OP_KC / 4);
        uint32_t wr[8], wi[8];
#pragma unroll
        for (int d = 0; d < 8; ++d) wr[d] = wi[d] = 0u;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const cd v = tile[op_slot(rr, 4 * g + c)];
            double vr = v.x, vi = v.y;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                if (d >= S) break;
                if (d > 0) {  // remainders in [-1/2, 1/2]: the next digit in [-127, 127]
                    vr *= OZ_BASE;
                    vi *= OZ_BASE;
                }
                // round to nearest (ties to even) by adding and removing
                // 1.5 2^52: for |v| <= 128 the sum is exact up to that rounding,
                // and its low word holds the digit in two's complement, so the
                // digit costs FP64 additions instead of conversions
                const double tr = __dadd_rn(vr, OZ_ROUND), ti = __dadd_rn(vi, OZ_ROUND);
                const double dr = __dsub_rn(tr, OZ_ROUND), di = __dsub_rn(ti, OZ_ROUND);
                vr = __dsub_rn(vr, dr);
                vi = __dsub_rn(vi, di);
                wr[d] |= ((uint32_t)__double2loint(tr) & 0xFFu) << (8 * c);
                wi[d] |= ((uint32_t)__double2loint(ti) & 0xFFu) << (8 * c);
            }
        }
        if (r0 + rr >= R) continue;
        const int r = r0 + rr, k = k0 + 4 * g;
        int8_t* o0 = out + item * out_item + (long)(is_b ? 2 * r : r) * row_bytes;
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            if (d >= S) break;
            const long base = (long)(is_b ? S - 1 - d : d) * K2;
            // the first K2/2 positions pair with Re of the other side, the rest with Im
            if (!is_b) {  // A' = [Re A, Im A]
                *reinterpret_cast<uint32_t*>(o0 + base + k) = wr[d];
                *reinterpret_cast<uint32_t*>(o0 + base + half + k) = wi[d];
            } else {
                // negated bytes: each byte is in [-127, 127], so per-byte negation never carries
                uint32_t nwi = 0u;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    nwi |= ((uint32_t)(-(int)(int8_t)((wi[d] >> (8 * c)) & 0xFFu)) & 0xFFu) << (8 * c);
                int8_t* o1 = o0 + row_bytes;  // the imaginary-part column
                *reinterpret_cast<uint32_t*>(o0 + base + k) = wr[d];  // [Re B; -Im B]
                *reinterpret_cast<uint32_t*>(o0 + base + half + k) = nwi;
                *reinterpret_cast<uint32_t*>(o1 + base + k) = wi[d];  // [Im B; Re B]
                *reinterpret_cast<uint32_t*>(o1 + base + half + k) = wr[d];
            }
        }
    }
}

// Digits of one operand (rows R, reduction length K) for `items` items:
// exponents into ex[item][R], digits into out[item].
void oz_prepare(const OzSrc& q, int R, int K, int K2, int S, int is_b, int items, int8_t* out, long out_item, int* ex,
                double min_bytes, cudaStream_t st) {
    ProfRange pr("oz_prep_kernel", st, 0.0, min_bytes);
    // below every exponent (0x80808080 = -2139062144): each row's first atomicMax sets it
    PGX_CUDA(cudaMemsetAsync(ex, 0x80, (size_t)items * R * sizeof(int), st));
    dim3 g1((unsigned)ceil_div((long)R, (long)OP_ROWS), (unsigned)ceil_div((long)K, (long)OP_KSPAN), (unsigned)items);
    oz_rowmax_kernel<<<g1, OP_THREADS, 0, st>>>(q, R, K, ex, R);
    check_launch("oz_rowmax_kernel");
    dim3 g2((unsigned)ceil_div((long)R, (long)OP_ROWS), (unsigned)(K2 / 2 / OP_KC), (unsigned)items);
    oz_prep_kernel<<<g2, OP_THREADS, 0, st>>>(q, R, K, K2, S, is_b, out, out_item, ex, R);
    check_launch("oz_prep_kernel");
}

// cuTensorMapEncodeTiled through the runtime's driver entry point.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 f = nullptr;
    if (!f) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        PGX_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        PGX_CHECK(fn && q == cudaDriverEntryPointSuccess, PGX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        f = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    return f;
}

// Tensor map over digits [items][rows][row_bytes] (bytes): 128-byte x box_rows
// boxes, 128-byte swizzle, zero fill past the rows.
CUtensorMap digit_map(const void* base, long row_bytes, long rows, long items, int box_rows) {
    PGX_CHECK(reinterpret_cast<uintptr_t>(base) % 16 == 0 && row_bytes % 16 == 0, PGX_ERR_ARG,
              "split product: unaligned digit buffer");
    CUtensorMap m;
    const cuuint64_t dims[3] = {(cuuint64_t)row_bytes, (cuuint64_t)rows, (cuuint64_t)items};
    const cuuint64_t strides[2] = {(cuuint64_t)row_bytes, (cuuint64_t)(row_bytes * rows)};
    const cuuint32_t box[3] = {(cuuint32_t)OZ_BK, (cuuint32_t)box_rows, 1u};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    const CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims,
                                            strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    PGX_CHECK(r == CUDA_SUCCESS, PGX_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

}  // namespace

bool oz_supported(int M, int N, int K) { return M > 0 && N > 0 && K > 0 && 2L * K <= (1L << 20); }

// C (+ item strides) = A B for the nb items of g, through the split scheme.
template <typename TA, typename TB>
void oz_zgemm(const GemmProblem<TA, TB, cd>& g, int S, OzWork& w, cudaStream_t st) {
    static_assert(!is_dressed<TA>::value || !is_dressed<TB>::value, "one dressed operand at most");
    const int M = g.M, N = g.N, K = g.K, nb = std::max(g.nb, 1);
    PGX_CHECK(!g.accumulate && !g.a_kidx && !g.b_kidx && !g.kscale && !g.conj_a, PGX_ERR_ARG,
              "split product: strided operands with row / column gathers only");
    PGX_CHECK(S >= 1 && S <= 8, PGX_ERR_ARG, "split product: 1..8 slices");
    const int K2 = (int)(ceil_div(2L * K, OZ_BK) * OZ_BK);
    const long row_bytes = (long)S * K2;
    // an operand changes per item when it is dressed (per-item frequency) or strided over items
    const bool a_item = is_dressed<TA>::value || g.ba != 0;
    const bool b_item = is_dressed<TB>::value || g.bb != 0;
    // int32 accumulation: depth (S) K2 with |digit| <= 127 stays below 2^31
    PGX_CHECK((double)S * K2 * 127.0 * 127.0 < 2147483647.0, PGX_ERR_ARG, "split product too deep for int32");
    const long a_bytes = (long)M * row_bytes, b_bytes = 2L * N * row_bytes;
    // items per chunk under about 4 GiB of digits
    const long per_item = (a_item ? a_bytes : 0) + (b_item ? b_bytes : 0);
    int chunk = nb;
    if (per_item > 0) chunk = (int)std::max<long>(1, std::min<long>(nb, (4L << 30) / per_item));
    const long ac = a_item ? chunk : 1, bc = b_item ? chunk : 1;
    w.A.reserve(ac * a_bytes);
    w.B.reserve(bc * b_bytes);
    w.ea.reserve(ac * M * sizeof(int));
    w.fb.reserve(bc * N * sizeof(int));
    if (!w.err.p) {
        w.err.reserve(sizeof(int));
        PGX_CUDA(cudaMemsetAsync(w.err.p, 0, sizeof(int), st));
    }
    // the shared-memory opt-in is a property of each device's context: set it
    // once per device (every time for device numbers beyond the table)
    static bool attr[64] = {};
    int dev = 0;
    PGX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !attr[dev]) {
        PGX_CUDA(cudaFuncSetAttribute(oz_gemm_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_SMEM));
        PGX_CUDA(cudaFuncSetAttribute(oz_gemm_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ2_SMEM));
        if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    using SA = typename src_t<TA>::type;
    using SB = typename src_t<TB>::type;
    for (int b0 = 0; b0 < nb; b0 += chunk) {
        const int cn = std::min(chunk, nb - b0);
        // A rows: A(i, k) = A[i sa_i + k sa_k]; dressed as dress(x, dEa[i], dEb[k], z)
        if (a_item || b0 == 0) {
            OzSrc q{};
            q.X = g.A + (a_item ? b0 * g.ba : 0);
            q.cplx = is_cd<SA>::value;
            q.ridx = g.a_iidx;
            q.s_r = g.sa_i;
            q.s_k = g.sa_k;
            q.s_item = g.ba;
            if (is_dressed<TA>::value) {
                q.Er = g.dEa;
                q.Ek = g.dEb;
                q.rk_order = 1;
                q.zs = g.dzs + b0;
            }
            const int items = a_item ? cn : 1;
            // minimum traffic: the source values twice (maxima, digits), the digits once
            oz_prepare(q, M, K, K2, S, 0, items, w.A.as<int8_t>(), a_bytes, w.ea.as<int>(),
                       2.0 * items * M * K * (is_cd<SA>::value ? 16.0 : 8.0) + (double)items * a_bytes, st);
        }
        // B columns: B(k, j) = B[k sb_k + j sb_j]; dressed as dress(x, dEa[k], dEb[j], z)
        if (b_item || b0 == 0) {
            OzSrc q{};
            q.X = g.B + (b_item ? b0 * g.bb : 0);
            q.cplx = is_cd<SB>::value;
            q.ridx = g.b_jidx;
            q.s_r = g.sb_j;
            q.s_k = g.sb_k;
            q.s_item = g.bb;
            if (is_dressed<TB>::value) {
                q.Er = g.dEb;
                q.Ek = g.dEa;
                q.rk_order = 0;
                q.zs = g.dzs + b0;
            }
            const int items = b_item ? cn : 1;
            oz_prepare(q, N, K, K2, S, 1, items, w.B.as<int8_t>(), b_bytes, w.fb.as<int>(),
                       2.0 * items * N * K * (is_cd<SB>::value ? 16.0 : 8.0) + (double)items * b_bytes, st);
        }
        const bool pair = w.cta_pair != 0;
        const CUtensorMap tmA = digit_map(w.A.p, row_bytes, M, a_item ? cn : 1, pair ? OZ2_HALF : OZ_BM);
        const CUtensorMap tmB = digit_map(w.B.p, row_bytes, 2L * N, b_item ? cn : 1, pair ? OZ2_HALF : OZ_BN);
        OzArgs2 a{};
        a.a_items = a_item;
        a.b_items = b_item;
        a.ea = w.ea.as<int>();
        a.ea_item = a_item ? M : 0;
        a.fb = w.fb.as<int>();
        a.fb_item = b_item ? N : 0;
        a.M = M;
        a.N = N;
        a.K2 = K2;
        a.S = S;
        a.C = g.C + (long)b0 * g.bc;
        a.c_item = g.bc;
        a.sc_i = g.sc_i;
        a.sc_j = g.sc_j;
        a.err = w.err.as<int>();
        // algorithmic work, as int8 operations (2 per multiply-add): per complex
        // multiply-add 4 real ones in each of the S(S+1)/2 digit products;
        // minimum traffic: the digits of both operands once and C written once
        const double fl = 2.0 * 4.0 * (S * (S + 1) / 2) * (double)M * N * K * cn;
        const double by = (double)(a_item ? cn : 1) * a_bytes + (double)(b_item ? cn : 1) * b_bytes +
                          16.0 * (double)M * N * cn;
        if (pair) {  // 256 x 256 tiles, one per CTA pair
            a.tiles_m = (int)ceil_div((long)M, 2L * OZ2_HALF);
            a.tiles_n = (int)ceil_div(2L * N, 2L * OZ2_HALF);
            PGX_CHECK((long)a.tiles_m * a.tiles_n < (1L << 30), PGX_ERR_ARG, "split product: too many tiles");
            dim3 grid((unsigned)(2L * a.tiles_m * a.tiles_n), 1u, (unsigned)cn);
            ProfRange pr("oz_gemm_pair_kernel", st, fl, by);
            oz_gemm_pair_kernel<<<grid, 384, OZ2_SMEM, st>>>(tmA, tmB, a);
            check_launch("oz_gemm_pair_kernel");
        } else {
            a.tiles_m = (int)ceil_div((long)M, OZ_BM);
            a.tiles_n = (int)ceil_div(2L * N, OZ_BN);
            PGX_CHECK((long)a.tiles_m * a.tiles_n < (1L << 31), PGX_ERR_ARG, "split product: too many tiles");
            dim3 grid((unsigned)((long)a.tiles_m * a.tiles_n), 1u, (unsigned)cn);
            ProfRange pr("oz_gemm_tma_kernel", st, fl, by);
            oz_gemm_tma_kernel<<<grid, 384, OZ_SMEM, st>>>(tmA, tmB, a);
            check_launch("oz_gemm_tma_kernel");
        }
    }
}

template void oz_zgemm<Dressed<double>, cd>(const GemmProblem<Dressed<double>, cd, cd>&, int, OzWork&, cudaStream_t);
template void oz_zgemm<Dressed<cd>, cd>(const GemmProblem<Dressed<cd>, cd, cd>&, int, OzWork&, cudaStream_t);
template void oz_zgemm<cd, Dressed<double>>(const GemmProblem<cd, Dressed<double>, cd>&, int, OzWork&, cudaStream_t);
template void oz_zgemm<cd, Dressed<cd>>(const GemmProblem<cd, Dressed<cd>, cd>&, int, OzWork&, cudaStream_t);
template void oz_zgemm<cd, cd>(const GemmProblem<cd, cd, cd>&, int, OzWork&, cudaStream_t);
template void oz_zgemm<double, Dressed<double>>(const GemmProblem<double, Dressed<double>, cd>&, int, OzWork&,
                                                cudaStream_t);
template void oz_zgemm<Dressed<double>, double>(const GemmProblem<Dressed<double>, double, cd>&, int, OzWork&,
                                                cudaStream_t);

}  // namespace pgx

namespace pgx {

namespace {
// Seeded uniform values in [-1, 1) times 2^-(h mod 4) (SplitMix64 hash of the index).
__global__ void oz_fill_kernel(cd* x, long n, unsigned long long seed) {
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long h = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
    auto mix = [](unsigned long long z) {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const unsigned long long a = mix(h), b = mix(h ^ 0x5555555555555555ull);
    const double sc = ldexp(1.0, -(int)(a & 3));
    x[i] = cd{(((a >> 11) * 0x1.0p-53) * 2.0 - 1.0) * sc, (((b >> 11) * 0x1.0p-53) * 2.0 - 1.0) * sc};
}
}  // namespace

void run_split_gemm_check(pgx_ctx* c, int M, int N, int K, int nb, int S, unsigned long long seed, double* err,
                          double* ms_split, double* ms_fp64) {
    PGX_CHECK(M > 0 && N > 0 && K > 0 && nb > 0 && (long)M * K * nb < (1L << 31) && (long)K * N < (1L << 31),
              PGX_ERR_ARG, "split check: sizes out of range");
    cudaStream_t st = c->stream;
    DevBuf A, B, C1, C2;
    const long na = (long)nb * M * K, nbb = (long)K * N, nc = (long)nb * M * N;
    A.reserve(na * sizeof(cd));
    B.reserve(nbb * sizeof(cd));
    C1.reserve(nc * sizeof(cd));
    C2.reserve(nc * sizeof(cd));
    oz_fill_kernel<<<(unsigned)ceil_div(na, 256L), 256, 0, st>>>(A.as<cd>(), na, seed);
    oz_fill_kernel<<<(unsigned)ceil_div(nbb, 256L), 256, 0, st>>>(B.as<cd>(), nbb, seed ^ 0xABCDEFull);
    check_launch("oz_fill_kernel");
    GemmProblem<cd, cd, cd> g{};
    g.A = A.as<cd>();
    g.B = B.as<cd>();
    g.M = M;
    g.N = N;
    g.K = K;
    g.sa_i = K;
    g.sa_k = 1;
    g.sb_k = N;
    g.sb_j = 1;
    g.sc_i = N;
    g.sc_j = 1;
    g.nb = nb;
    g.ba = (long)M * K;
    g.bb = 0;
    g.bc = (long)M * N;
    cudaEvent_t e0, e1, e2;
    PGX_CUDA(cudaEventCreate(&e0));
    PGX_CUDA(cudaEventCreate(&e1));
    PGX_CUDA(cudaEventCreate(&e2));
    if (c->oz.err.p) PGX_CUDA(cudaMemsetAsync(c->oz.err.p, 0, sizeof(int), st));
    g.C = C1.as<cd>();
    PGX_CUDA(cudaEventRecord(e0, st));
    oz_zgemm(g, S, c->oz, st);
    PGX_CUDA(cudaEventRecord(e1, st));
    g.C = C2.as<cd>();
    std::vector<GemmProblem<cd, cd, cd>> probs{g};
    DevBuf pb, ib;
    pb.reserve(sizeof(g));
    ib.reserve(gemm_index_bytes(1));
    launch_gemm_batch(probs, pb.p, pb.bytes, ib.p, ib.bytes, st);
    PGX_CUDA(cudaEventRecord(e2, st));
    PGX_CUDA(cudaEventSynchronize(e2));
    float t1 = 0.f, t2 = 0.f;
    PGX_CUDA(cudaEventElapsedTime(&t1, e0, e1));
    PGX_CUDA(cudaEventElapsedTime(&t2, e1, e2));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    int flag = 0;
    PGX_CUDA(cudaMemcpy(&flag, c->oz.err.p, sizeof(int), cudaMemcpyDeviceToHost));
    PGX_CHECK(flag == 0, PGX_ERR_TIMEOUT, "split product: a tensor-core wait expired");
    std::vector<cd> h1(nc), h2(nc);
    PGX_CUDA(cudaMemcpy(h1.data(), C1.p, nc * sizeof(cd), cudaMemcpyDeviceToHost));
    PGX_CUDA(cudaMemcpy(h2.data(), C2.p, nc * sizeof(cd), cudaMemcpyDeviceToHost));
    double dmax = 0.0, cmax = 0.0;
    for (long i = 0; i < nc; ++i) {
        dmax = std::max(dmax, std::hypot(h1[i].x - h2[i].x, h1[i].y - h2[i].y));
        cmax = std::max(cmax, std::hypot(h2[i].x, h2[i].y));
    }
    *err = cmax > 0.0 ? dmax / cmax : dmax;
    *ms_split = t1;
    *ms_fp64 = t2;
}

}  // namespace pgx
