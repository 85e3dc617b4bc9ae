// GEMM tile-class autotuner (pgx_autotune_begin / pgx_autotune_end).
//
// launch_gemm_batch puts every product in one of GEMM_NCLS tile classes.
// Without tuning the class is the one that pads the product least.  The tuner
// measures instead, on the workload's own products: between begin and end,
// every batch a call launches is first run, per (M, N) size bucket, under the
// padding rule and in every class valid for the bucket, with its outputs
// redirected to scratch, before its real launch (tune_measure).  The times add
// up per operand-type combination and bucket; at the end each bucket keeps the
// candidate with the least total (the rule wins ties, so tuning never moves a
// bucket off a choice that measured at least as fast).
//
// Measuring where the products are launched, rather than replaying them
// later, means each candidate reads exactly the addresses and index tables
// of the real launch while they hold the same contents.

#include <cfloat>

#include "pgx_common.cuh"
#include "pgx_gemm.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {
constexpr int TUNE_REPS = 2;
}  // namespace

TuneRecorder::~TuneRecorder() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
}

void tune_measure(TuneRecorder& rec, int key, int mb, int nb, size_t c_bytes, const TuneLaunch& launch,
                  cudaStream_t st) {
    // the candidates neither record themselves nor enter the profile
    TuneRecorder* const saved_r = active_recorder();
    Profiler* const saved_p = active_profiler();
    active_recorder() = nullptr;
    active_profiler() = nullptr;
    auto restore = [&] {
        forced_gemm_class() = -1;
        active_recorder() = saved_r;
        active_profiler() = saved_p;
    };
    try {
        rec.scratch.reserve(std::max<size_t>(c_bytes, 256));
        if (!rec.e0) PGX_CUDA(cudaEventCreate(&rec.e0));
        if (!rec.e1) PGX_CUDA(cudaEventCreate(&rec.e1));
        // the inputs are written by earlier work on this or other streams;
        // nothing else runs while the candidates are timed
        PGX_CUDA(cudaDeviceSynchronize());
        auto& tot = rec.total[std::make_tuple(key, mb, nb)];
        if (tot.empty()) tot.assign(GEMM_NCLS + 1, 0.0);
        const int M = GEMM_BUCKET_REP[mb], N = GEMM_BUCKET_REP[nb];
        for (int cand = -1; cand < GEMM_NCLS; ++cand) {
            if (cand >= 0 && !gemm_class_valid(cand, M, N)) {
                tot[cand + 1] = DBL_MAX;
                continue;
            }
            launch(cand, rec.scratch.p, rec.probs, rec.index, st);  // warm-up
            PGX_CUDA(cudaEventRecord(rec.e0, st));
            for (int r = 0; r < TUNE_REPS; ++r) launch(cand, rec.scratch.p, rec.probs, rec.index, st);
            PGX_CUDA(cudaEventRecord(rec.e1, st));
            PGX_CUDA(cudaEventSynchronize(rec.e1));
            float ms = 0.0f;
            PGX_CUDA(cudaEventElapsedTime(&ms, rec.e0, rec.e1));
            if (tot[cand + 1] < DBL_MAX) tot[cand + 1] += ms;
        }
    } catch (...) {
        restore();
        throw;
    }
    restore();
}

int install_tuning(pgx_ctx* c, const TuneRecorder& rec) {
    c->tune = GemmTune();
    int changed = 0;
    for (const auto& kv : rec.total) {
        const auto& tot = kv.second;
        int best = -1;
        double bt = tot[0];
        for (int cand = 0; cand < GEMM_NCLS; ++cand)
            if (tot[cand + 1] < bt) {
                bt = tot[cand + 1];
                best = cand;
            }
        c->tune.cls[std::get<0>(kv.first)][std::get<1>(kv.first)][std::get<2>(kv.first)] = (signed char)best;
        if (best >= 0) ++changed;
    }
    c->tuned = true;
    return changed;
}

}  // namespace pgx
