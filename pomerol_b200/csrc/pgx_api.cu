// extern "C" entry points of libpgx (declared in include/pgx.h).
// Every call translates pgx::Error into a status code and a message; no
// exception crosses the ABI.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <utility>

#include "pgx_common.cuh"
#include "pgx_internal.h"

namespace pgx {
void launch_retained(Problem& P, double tol, int* d_flags, cudaStream_t st);
long long& launch_counter() {
    static long long n = 0;
    return n;
}

Profiler*& active_profiler() {
    static thread_local Profiler* p = nullptr;
    return p;
}

cudaEvent_t Profiler::event() {
    if (!spare.empty()) {
        cudaEvent_t e = spare.back();
        spare.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    PGX_CUDA(cudaEventCreate(&e));
    return e;
}

void Profiler::clear() {
    for (auto& r : open) {
        spare.push_back(r.a);
        spare.push_back(r.b);
    }
    open.clear();
    stats.clear();
}

void Profiler::resolve() {
    for (auto& r : open) {
        PGX_CUDA(cudaEventSynchronize(r.b));
        float t = 0.f;
        PGX_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        auto it = std::find_if(stats.begin(), stats.end(), [&](const KernelStat& k) { return k.name == r.name; });
        if (it == stats.end()) {
            stats.push_back(KernelStat{r.name});
            it = stats.end() - 1;
        }
        it->launches += 1;
        it->ms += t;
        it->flops += r.flops;
        it->bytes += r.bytes;
        spare.push_back(r.a);
        spare.push_back(r.b);
    }
    open.clear();
    std::stable_sort(stats.begin(), stats.end(), [](const KernelStat& x, const KernelStat& y) { return x.ms > y.ms; });
}

Profiler::~Profiler() {
    for (auto& r : open) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : spare) cudaEventDestroy(e);
}

GemmTune*& active_tune() {
    static thread_local GemmTune* t = nullptr;
    return t;
}
int& forced_gemm_class() {
    static thread_local int f = -1;
    return f;
}
TuneRecorder*& active_recorder() {
    static thread_local TuneRecorder* r = nullptr;
    return r;
}

unsigned long long& alloc_epoch() {
    static unsigned long long e = 0;
    return e;
}

HostArena*& active_arena() {
    static thread_local HostArena* a = nullptr;
    return a;
}

void* HostArena::put(const void* src, size_t n) {
    const size_t need = (n + 15) & ~size_t(15);
    while (cur < blocks.size() && used + need > blocks[cur].second) {
        ++cur;
        used = 0;
    }
    if (cur == blocks.size()) {
        const size_t cap = std::max<size_t>(need, std::max<size_t>(size_t(1) << 20, blocks.empty() ? 0 : 2 * blocks.back().second));
        void* p = nullptr;
        if (cudaMallocHost(&p, cap) != cudaSuccess) {
            cudaGetLastError();
            throw Error{PGX_ERR_OOM, "cudaMallocHost(" + std::to_string(cap) + " bytes) failed"};
        }
        blocks.emplace_back(static_cast<char*>(p), cap);
        used = 0;
    }
    char* dst = blocks[cur].first + used;
    std::memcpy(dst, src, n);
    used += need;
    dirty = true;
    return dst;
}

void HostArena::recycle(cudaStream_t st) {
    if (!dirty) return;
    const cudaError_t q = cudaStreamQuery(st);
    if (q == cudaErrorNotReady) {
        cudaGetLastError();  // not an error: copies are still pending, keep appending
        return;
    }
    if (q != cudaSuccess) return;
    cur = 0;
    used = 0;
    dirty = false;
}

HostArena::~HostArena() {
    for (auto& b : blocks) cudaFreeHost(b.first);
}

void h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (!bytes) return;
    HostArena* a = active_arena();
    const void* s = a ? a->put(src, bytes) : src;
    PGX_CUDA(cudaMemcpyAsync(dst, s, bytes, cudaMemcpyHostToDevice, st));
}

ProfRange::ProfRange(const char* name, cudaStream_t st, double flops, double bytes) {
    Profiler* p = active_profiler();
    if (!p || !p->on) return;
    Profiler::Range r{name, p->event(), p->event(), flops, bytes};
    PGX_CUDA(cudaEventRecord(r.a, st));
    p->open.push_back(r);
    p_ = p;
    st_ = st;
    idx_ = p->open.size() - 1;
}

ProfRange::~ProfRange() {
    if (p_) cudaEventRecord(p_->open[idx_].b, st_);
}
}

using pgx::Error;

namespace {

__global__ void recip_check_kernel(const double* x, double* y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = pgx::recip_pos(x[i]);
}

// Runs an entry point: its context's profiler and upload arena (the graph's
// own arena while a capture is open) are visible to the launch sites, and
// exceptions become status codes.  While a capture is open only the entry
// points that may be captured (capture_ok) run.
template <typename F> int guarded_impl(pgx_ctx* c, bool capture_ok, F&& f) {
    if (!c) return PGX_ERR_ARG;
    if (c->capturing && !capture_ok) {
        c->last_error = "this entry point cannot run while a graph is being captured";
        return PGX_ERR_STATE;
    }
    struct Scope {
        pgx::Profiler* saved_p;
        pgx::HostArena* saved_a;
        pgx::GemmTune* saved_t;
        pgx::TuneRecorder* saved_r;
        explicit Scope(pgx_ctx* c)
            : saved_p(pgx::active_profiler()), saved_a(pgx::active_arena()), saved_t(pgx::active_tune()),
              saved_r(pgx::active_recorder()) {
            pgx::active_profiler() = &c->prof;
            pgx::active_arena() = c->capturing ? c->cap.arena.get() : &c->arena;
            pgx::active_tune() = c->tuned ? &c->tune : nullptr;
            pgx::active_recorder() = c->capturing ? nullptr : c->recorder.get();
        }
        ~Scope() {
            pgx::active_profiler() = saved_p;
            pgx::active_arena() = saved_a;
            pgx::active_tune() = saved_t;
            pgx::active_recorder() = saved_r;
        }
    } scope(c);
    try {
        PGX_CUDA(cudaSetDevice(c->device));
        f();
        if (!c->capturing) c->arena.recycle(c->stream);
        c->last_error.clear();
        return PGX_OK;
    } catch (const Error& e) {
        c->last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        c->last_error = "host allocation failed";
        return PGX_ERR_OOM;
    } catch (...) {
        c->last_error = "unexpected host exception";
        return PGX_ERR_ARG;
    }
}
template <typename F> int guarded(pgx_ctx* c, F&& f) { return guarded_impl(c, false, std::forward<F>(f)); }
template <typename F> int guarded_cap(pgx_ctx* c, F&& f) { return guarded_impl(c, true, std::forward<F>(f)); }

void drop_graph(pgx_ctx::Graph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g.exec = nullptr;
    g.graph = nullptr;
    g.arena.reset();
}

void reset_problem(pgx::Problem& P) {
    pgx::Problem fresh;
    pgx::DevBuf pgx::Problem::*bufs[] = {&pgx::Problem::H,       &pgx::Problem::work,      &pgx::Problem::work2,
                                         &pgx::Problem::U,       &pgx::Problem::E,         &pgx::Problem::w,
                                         &pgx::Problem::dims_d,  &pgx::Problem::moff_d,    &pgx::Problem::eoff_d,
                                         &pgx::Problem::order_d, &pgx::Problem::status,    &pgx::Problem::tri,
                                         &pgx::Problem::tri_items, &pgx::Problem::eigh_gemm, &pgx::Problem::eigh_scratch,
                                         &pgx::Problem::op_probs, &pgx::Problem::op_tiles, &pgx::Problem::op_meta,
                                         &pgx::Problem::asm_buf, &pgx::Problem::cx_meta, &pgx::Problem::cx_H,
                                         &pgx::Problem::cx_A,    &pgx::Problem::cx_Zc,   &pgx::Problem::cx_U,
                                         &pgx::Problem::cx_E,    &pgx::Problem::cx_tri,  &pgx::Problem::cx_S,
                                         &pgx::Problem::cx_items, &pgx::Problem::cx_gemm, &pgx::Problem::vjp_buf,
                                         &pgx::Problem::chi3_small, &pgx::Problem::chi3_big};
    for (auto m : bufs) fresh.*m = std::move(P.*m);
    fresh.spare_ops = std::move(P.spare_ops);
    for (auto& op : P.ops) fresh.spare_ops.push_back(std::move(op));
    P = std::move(fresh);
}

}  // namespace

extern "C" {

int pgx_version(void) { return 10000; }

int pgx_create(int device, pgx_ctx** out) {
    if (!out) return PGX_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return PGX_ERR_NODEV;
    }
    if (device < 0 || device >= n) return PGX_ERR_ARG;
    pgx_ctx* c = new (std::nothrow) pgx_ctx();
    if (!c) return PGX_ERR_OOM;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return PGX_ERR_CUDA;
    }
    *out = c;
    return PGX_OK;
}

int pgx_destroy(pgx_ctx* c) {
    if (!c) return PGX_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    if (c->capturing) {
        cudaGraph_t gr = nullptr;
        cudaStreamEndCapture(c->stream, &gr);
        if (gr) cudaGraphDestroy(gr);
        cudaGetLastError();
        c->capturing = false;
    }
    drop_graph(c->cap);
    for (auto& g : c->graphs) drop_graph(g);
    reset_problem(c->P);
    for (auto& b : c->scratch) b.release();
    if (c->ev_begin) cudaEventDestroy(c->ev_begin);
    if (c->ev_end) cudaEventDestroy(c->ev_end);
    for (int i = 0; i < 4; ++i) {
        if (c->aux[i]) cudaStreamDestroy(c->aux[i]);
        if (c->join[i]) cudaEventDestroy(c->join[i]);
    }
    if (c->fork) cudaEventDestroy(c->fork);
    cudaStreamDestroy(c->stream);
    delete c;
    return PGX_OK;
}

const char* pgx_last_error(const pgx_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

int pgx_set_blocks(pgx_ctx* c, int32_t nblocks, const int32_t* dims, int32_t is_complex) {
    return guarded(c, [&] {
        PGX_CHECK(nblocks > 0 && dims, PGX_ERR_ARG, "need at least one block");
        for (int b = 0; b < nblocks; ++b) PGX_CHECK(dims[b] > 0, PGX_ERR_ARG, "block sizes must be positive");
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        ++c->problem_gen;
        ++c->ops_gen;
        reset_problem(c->P);
        pgx::Problem& P = c->P;
        // a failed allocation below leaves no half-declared problem behind
        struct Undo {
            pgx::Problem& P;
            bool armed = true;
            ~Undo() {
                if (armed) reset_problem(P);
            }
        } undo{P};
        P.nblocks = nblocks;
        P.is_complex = is_complex != 0;
        P.dims.assign(dims, dims + nblocks);
        P.moff.resize(nblocks);
        P.eoff.resize(nblocks);
        long m = 0, e = 0;
        for (int b = 0; b < nblocks; ++b) {
            P.moff[b] = m;
            P.eoff[b] = e;
            m += (long)dims[b] * dims[b];
            e += dims[b];
            P.dmax = std::max(P.dmax, (int)dims[b]);
        }
        P.msize = m;
        P.esize = e;
        const size_t sc = P.is_complex ? 2 : 1;
        P.H.reserve(m * sc * sizeof(double));
        P.U.reserve(m * sc * sizeof(double));
        P.work.reserve(m * sc * sizeof(double));
        P.work2.reserve(m * sc * sizeof(double));
        P.E.reserve(e * sizeof(double));
        P.w.reserve(e * sizeof(double));
        P.dims_d.reserve(nblocks * sizeof(int));
        P.moff_d.reserve(nblocks * sizeof(long));
        P.eoff_d.reserve(nblocks * sizeof(long));
        P.order_d.reserve(nblocks * sizeof(int));
        P.status.reserve(64);
        P.d_H = P.H.as<double>();
        P.d_U = P.U.as<double>();
        P.d_work = P.work.as<double>();
        P.d_work2 = P.work2.as<double>();
        P.d_E = P.E.as<double>();
        P.d_w = P.w.as<double>();
        P.d_dims = P.dims_d.as<int>();
        P.d_moff = P.moff_d.as<long>();
        P.d_eoff = P.eoff_d.as<long>();
        P.d_order = P.order_d.as<int>();
        P.d_status = P.status.as<int>();
        std::vector<int> order(nblocks);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dims[a] > dims[b]; });
        PGX_CUDA(cudaMemcpy(P.d_dims, dims, nblocks * sizeof(int), cudaMemcpyHostToDevice));
        PGX_CUDA(cudaMemcpy(P.d_moff, P.moff.data(), nblocks * sizeof(long), cudaMemcpyHostToDevice));
        PGX_CUDA(cudaMemcpy(P.d_eoff, P.eoff.data(), nblocks * sizeof(long), cudaMemcpyHostToDevice));
        PGX_CUDA(cudaMemcpy(P.d_order, order.data(), nblocks * sizeof(int), cudaMemcpyHostToDevice));
        PGX_CUDA(cudaMemset(P.d_status, 0, 64));
        undo.armed = false;
    });
}

int pgx_set_hamiltonian(pgx_ctx* c, const double* H) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.nblocks > 0, PGX_ERR_STATE, "pgx_set_blocks first");
        PGX_CHECK(H, PGX_ERR_ARG, "null Hamiltonian");
        const size_t sc = P.is_complex ? 2 : 1;
        // a NaN or infinity would only surface after the eigensolve: refuse it here
        for (size_t i = 0; i < P.msize * sc; ++i)
            PGX_CHECK(std::isfinite(H[i]), PGX_ERR_NUMERIC, "non-finite Hamiltonian entry " + std::to_string(i));
        PGX_CUDA(cudaMemcpyAsync(P.d_H, H, P.msize * sc * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        P.have_H = true;
        P.have_asm = false;  // H no longer comes from an assembled term list
        P.have_eig = P.have_w = false;
        for (auto& op : P.ops) op.rotated = false;
    });
}

int pgx_assemble_hamiltonian(pgx_ctx* c, int32_t nterms, const int32_t* ops, const double* coef, int32_t nmodes,
                             const uint64_t* fock, const int32_t* state_block, const int32_t* state_inner) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.nblocks > 0, PGX_ERR_STATE, "pgx_set_blocks first");
        PGX_CHECK(nterms >= 0 && (nterms == 0 || (ops && coef)), PGX_ERR_ARG, "bad term list");
        PGX_CHECK(nmodes >= 0 && nmodes <= 30, PGX_ERR_ARG, "nmodes must be in [0, 30]");
        PGX_CHECK(fock && state_block && state_inner, PGX_ERR_ARG, "null state table");
        PGX_CHECK(P.esize <= (1L << nmodes), PGX_ERR_ARG, "more block states than Fock states");
        pgx::assemble_hamiltonian(c, nterms, ops, coef, nmodes, fock, state_block, state_inner);
        P.have_H = true;
        P.have_eig = P.have_w = false;
        for (auto& op : P.ops) op.rotated = false;
    });
}

int pgx_gf_vjp(pgx_ctx* c, int32_t op1, int32_t op2, int32_t nparts, const int32_t* outer, const int32_t* inner,
               int32_t nz, const double* z, const double* lambda, double* dterm, double* dE) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nz >= 0 && (nparts == 0 || (outer && inner)) && (nz == 0 || (z && lambda)) && dterm,
                  PGX_ERR_ARG, "bad arguments");
        PGX_CHECK(!c->P.w_models, PGX_ERR_STATE, "needs the weights of one model (pgx_weights)");
        pgx::run_gf_vjp(c, op1, op2, nparts, outer, inner, nz, z, lambda, dterm, dE);
    });
}

int pgx_chi3(pgx_ctx* c, int32_t channel, int32_t nparts, const pgx_chi3_part* parts, int32_t nfreq,
             const double* z, double pole_res, double* out) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nfreq >= 0 && (nparts == 0 || parts) && (nfreq == 0 || (z && out)), PGX_ERR_ARG,
                  "bad arguments");
        PGX_CHECK(!c->P.w_models, PGX_ERR_STATE, "needs the weights of one model (pgx_weights)");
        pgx::run_chi3(c, channel, nparts, parts, nfreq, z, pole_res, out);
    });
}

int pgx_set_models(pgx_ctx* c, int32_t nmodels, const int32_t* first_block, const double* beta) {
    return guarded(c, [&] { pgx::set_models(c->P, nmodels, first_block, beta); });
}

int pgx_weights_models(pgx_ctx* c, double* w, double* E0, double* Z) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.have_eig, PGX_ERR_STATE, "pgx_eigh first");
        pgx::launch_weights_models(P, c->stream);
        P.have_w = true;
        P.w_models = true;
        P.retained.assign(P.nblocks, 1);
        if (w) std::copy(P.w_host.begin(), P.w_host.end(), w);
        if (E0) std::copy(P.model_E0.begin(), P.model_E0.end(), E0);
        if (Z) std::copy(P.model_Z.begin(), P.model_Z.end(), Z);
    });
}

int pgx_gf_models(pgx_ctx* c, int32_t op1, int32_t op2, int32_t nparts, const int32_t* outer, const int32_t* inner,
                  int32_t nz, const double* z, double coef_tol, double* out) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nz >= 0 && (nz == 0 || (z && out)) && (nparts == 0 || (outer && inner)), PGX_ERR_ARG,
                  "bad arguments");
        pgx::run_gf_models(c, op1, op2, nparts, outer, inner, nz, z, coef_tol, out);
    });
}

int pgx_susc_models(pgx_ctx* c, int32_t opA, int32_t opB, int32_t nparts, const int32_t* outer,
                    const int32_t* inner, int32_t nz, const double* z, double pole_res, double coef_tol, double* out,
                    double* zero_pole) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nz >= 0 && (nz == 0 || (z && out)) && (nparts == 0 || (outer && inner)), PGX_ERR_ARG,
                  "bad arguments");
        pgx::run_susc_models(c, opA, opB, nparts, outer, inner, nz, z, pole_res, coef_tol, out, zero_pole);
    });
}

int pgx_susc_vjp(pgx_ctx* c, int32_t opA, int32_t opB, int32_t nparts, const int32_t* outer, const int32_t* inner,
                 int32_t nz, const double* z, double pole_res, const double* lambda, double* dterm, double* dE) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nz >= 0 && (nparts == 0 || (outer && inner)) && (nz == 0 || (z && lambda)) && dterm,
                  PGX_ERR_ARG, "bad arguments");
        PGX_CHECK(!c->P.w_models, PGX_ERR_STATE, "needs the weights of one model (pgx_weights)");
        pgx::run_susc_vjp(c, opA, opB, nparts, outer, inner, nz, z, pole_res, lambda, dterm, dE);
    });
}

int pgx_split_gemm_check(pgx_ctx* c, int32_t M, int32_t N, int32_t K, int32_t nb, int32_t slices, uint64_t seed,
                         double* max_rel_err, double* ms_split, double* ms_fp64) {
    return guarded(c, [&] {
        PGX_CHECK(max_rel_err && ms_split && ms_fp64, PGX_ERR_ARG, "null output");
        pgx::run_split_gemm_check(c, M, N, K, nb, slices, seed, max_rel_err, ms_split, ms_fp64);
    });
}

int pgx_set_g2_split_threshold(pgx_ctx* c, double min_macs) {
    return guarded(c, [&] {
        PGX_CHECK(min_macs >= 0.0, PGX_ERR_ARG, "threshold must be >= 0");
        c->g2_split_min_macs = min_macs;
    });
}

int pgx_set_g2_split_weight_budget(pgx_ctx* c, double budget) {
    return guarded(c, [&] {
        PGX_CHECK(std::isfinite(budget), PGX_ERR_ARG, "budget must be finite");
        c->g2_split_weight_budget = budget;
    });
}

int pgx_set_split_cta_pair(pgx_ctx* c, int32_t cta_pair) {
    return guarded(c, [&] {
        PGX_CHECK(cta_pair == 0 || cta_pair == 1, PGX_ERR_ARG, "cta_pair must be 0 or 1");
        c->oz.cta_pair = cta_pair;
    });
}

int pgx_set_g2_split_slices(pgx_ctx* c, int32_t slices) {
    return guarded(c, [&] {
        PGX_CHECK(slices >= 1 && slices <= 8, PGX_ERR_ARG, "split slices must be 1..8");
        c->g2_split_slices = slices;
    });
}

int pgx_set_g2_workspace(pgx_ctx* c, int64_t batch_bytes, int64_t chain_bytes) {
    return guarded(c, [&] {
        PGX_CHECK(batch_bytes >= 0 && chain_bytes >= 0, PGX_ERR_ARG, "workspace limits must be >= 0");
        c->g2_batch_bytes = batch_bytes;
        c->g2_chain_bytes = chain_bytes;
    });
}

int pgx_autotune_begin(pgx_ctx* c) {
    return guarded(c, [&] {
        c->recorder.reset(new pgx::TuneRecorder());
        c->tuned = false;  // the recorded run uses the padding rule
    });
}

int pgx_autotune_end(pgx_ctx* c, int32_t* changed) {
    return guarded(c, [&] {
        PGX_CHECK(c->recorder != nullptr, PGX_ERR_STATE, "pgx_autotune_begin first");
        std::unique_ptr<pgx::TuneRecorder> rec = std::move(c->recorder);
        pgx::active_recorder() = nullptr;
        const int n = pgx::install_tuning(c, *rec);
        if (changed) *changed = n;
    });
}

int pgx_graph_begin(pgx_ctx* c) {
    return guarded(c, [&] {
        PGX_CHECK(!c->prof.on, PGX_ERR_STATE, "stop profiling before capturing a graph");
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        drop_graph(c->cap);
        c->cap = pgx_ctx::Graph{};
        c->cap.arena.reset(new pgx::HostArena());
        PGX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
        c->capturing = true;
    });
}

int pgx_graph_end(pgx_ctx* c, int32_t* graph_id) {
    return guarded_cap(c, [&] {
        PGX_CHECK(c->capturing, PGX_ERR_STATE, "no graph is being captured");
        PGX_CHECK(graph_id, PGX_ERR_ARG, "null graph id");
        c->capturing = false;
        cudaGraph_t gr = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c->stream, &gr);
        if (e != cudaSuccess || !gr) {
            cudaGetLastError();
            if (gr) cudaGraphDestroy(gr);
            drop_graph(c->cap);
            PGX_CHECK(false, PGX_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
        }
        c->cap.graph = gr;
        if (cudaGraphInstantiate(&c->cap.exec, gr, 0) != cudaSuccess) {
            cudaGetLastError();
            drop_graph(c->cap);
            PGX_CHECK(false, PGX_ERR_CUDA, "graph instantiation failed");
        }
        c->cap.epoch = pgx::alloc_epoch();
        c->cap.problem_gen = c->problem_gen;
        c->cap.ops_gen = c->ops_gen;
        size_t slot = 0;
        while (slot < c->graphs.size() && c->graphs[slot].exec) ++slot;
        if (slot == c->graphs.size()) c->graphs.emplace_back();
        c->graphs[slot] = std::move(c->cap);
        c->cap = pgx_ctx::Graph{};
        *graph_id = (int32_t)slot;
    });
}

int pgx_graph_replay(pgx_ctx* c, int32_t graph_id) {
    return guarded(c, [&] {
        PGX_CHECK(graph_id >= 0 && graph_id < (int)c->graphs.size() && c->graphs[graph_id].exec, PGX_ERR_ARG,
                  "bad graph id");
        pgx_ctx::Graph& g = c->graphs[graph_id];
        pgx::Problem& P = c->P;
        PGX_CHECK(g.epoch == pgx::alloc_epoch() && g.problem_gen == c->problem_gen && g.ops_gen == c->ops_gen,
                  PGX_ERR_STATE, "device buffers or operators changed since the capture; capture the graph again");
        PGX_CHECK(!g.eigh || P.have_H, PGX_ERR_STATE, "pgx_set_hamiltonian first");
        PGX_CHECK(g.eigh || P.have_eig, PGX_ERR_STATE, "pgx_eigh first");
        PGX_CUDA(cudaGraphLaunch(g.exec, c->stream));
        int st = 0;
        if (g.eigh) PGX_CUDA(cudaMemcpyAsync(&st, P.d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        if (g.eigh) {
            PGX_CHECK(st == 0, PGX_ERR_NUMERIC, "eigensolver did not converge");
            P.have_eig = true;
            P.have_w = false;
            for (auto& op : P.ops) op.rotated = false;
        }
        for (int op : g.rotated) P.ops[op].rotated = true;
    });
}

int pgx_graph_destroy(pgx_ctx* c, int32_t graph_id) {
    return guarded(c, [&] {
        PGX_CHECK(graph_id >= 0 && graph_id < (int)c->graphs.size() && c->graphs[graph_id].exec, PGX_ERR_ARG,
                  "bad graph id");
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        drop_graph(c->graphs[graph_id]);
    });
}

int pgx_get_hamiltonian(pgx_ctx* c, double* H) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.have_H && H, PGX_ERR_STATE, "no Hamiltonian on the device");
        const size_t sc = P.is_complex ? 2 : 1;
        PGX_CUDA(cudaMemcpyAsync(H, P.d_H, P.msize * sc * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int pgx_eigh(pgx_ctx* c) {
    return guarded_cap(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.have_H, PGX_ERR_STATE, "pgx_set_hamiltonian first");
        if (c->capturing) {  // device work only; the status is read when the graph is replayed
            PGX_CHECK(!P.is_complex, PGX_ERR_STATE, "complex blocks cannot be captured");
            PGX_CHECK(c->fork != nullptr, PGX_ERR_STATE, "run pgx_eigh once before capturing it");
            PGX_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int), c->stream));
            pgx::launch_eigh(c);
            c->cap.eigh = true;
            return;
        }
        PGX_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int), c->stream));
        pgx::launch_eigh(c);
        int st = 0;
        PGX_CUDA(cudaMemcpyAsync(&st, P.d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        PGX_CHECK(st == 0, PGX_ERR_NUMERIC, "eigensolver did not converge");
        P.have_eig = true;
        P.have_w = false;
        for (auto& op : P.ops) op.rotated = false;
    });
}

int pgx_get_eigensystem(pgx_ctx* c, double* E, double* U) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.have_eig, PGX_ERR_STATE, "pgx_eigh first");
        const size_t sc = P.is_complex ? 2 : 1;
        if (E) PGX_CUDA(cudaMemcpyAsync(E, P.d_E, P.esize * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (U) PGX_CUDA(cudaMemcpyAsync(U, P.d_U, P.msize * sc * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int pgx_set_eigensystem(pgx_ctx* c, const double* E, const double* U) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.nblocks > 0, PGX_ERR_STATE, "pgx_set_blocks first");
        PGX_CHECK(E && U, PGX_ERR_ARG, "null eigensystem");
        const size_t sc = P.is_complex ? 2 : 1;
        for (long i = 0; i < P.esize; ++i) PGX_CHECK(std::isfinite(E[i]), PGX_ERR_NUMERIC, "non-finite eigenvalue");
        for (long b = 0; b < P.nblocks; ++b)
            for (long i = P.eoff[b] + 1; i < P.eoff[b] + P.dims[b]; ++i)
                PGX_CHECK(E[i - 1] <= E[i], PGX_ERR_ARG, "eigenvalues must ascend inside every block");
        for (long i = 0; i < P.msize * (long)sc; ++i)
            PGX_CHECK(std::isfinite(U[i]), PGX_ERR_NUMERIC, "non-finite eigenvector entry");
        PGX_CUDA(cudaMemcpyAsync(P.d_E, E, P.esize * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PGX_CUDA(cudaMemcpyAsync(P.d_U, U, P.msize * sc * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        P.have_eig = true;
        P.have_w = false;
        for (auto& op : P.ops) op.rotated = false;
    });
}

int pgx_ground_energy(pgx_ctx* c, double* E0) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.have_eig && E0, PGX_ERR_STATE, "pgx_eigh first");
        std::vector<double> e(P.esize);
        PGX_CUDA(cudaMemcpyAsync(e.data(), P.d_E, P.esize * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        *E0 = *std::min_element(e.begin(), e.end());
    });
}

int pgx_weights(pgx_ctx* c, double beta, double* w, double* Z) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.have_eig, PGX_ERR_STATE, "pgx_eigh first");
        PGX_CHECK(beta > 0, PGX_ERR_ARG, "beta must be positive");
        pgx::launch_weights(P, beta, c->stream);
        P.beta = beta;
        P.have_w = true;
        P.w_models = false;
        P.retained.assign(P.nblocks, 1);
        if (w) {
            PGX_CUDA(cudaMemcpyAsync(w, P.d_w, P.esize * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            PGX_CUDA(cudaStreamSynchronize(c->stream));
        }
        if (Z) *Z = P.Z;
    });
}

int pgx_truncate_blocks(pgx_ctx* c, double tol, int32_t* retained) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(P.have_w, PGX_ERR_STATE, "pgx_weights first");
        pgx::DevBuf flags;
        flags.reserve(P.nblocks * sizeof(int));
        pgx::launch_retained(P, tol, flags.as<int>(), c->stream);
        P.retained.resize(P.nblocks);
        PGX_CUDA(cudaMemcpyAsync(P.retained.data(), flags.p, P.nblocks * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
        flags.release();
        if (retained) std::copy(P.retained.begin(), P.retained.end(), retained);
    });
}

int pgx_op_define(pgx_ctx* c, int32_t nparts, const int32_t* right_block, const int32_t* left_block,
                  const int32_t* target, const double* coef, int32_t* op_id) {
    return guarded(c, [&] {
        ++c->ops_gen;
        pgx::Problem& P = c->P;
        PGX_CHECK(P.nblocks > 0, PGX_ERR_STATE, "pgx_set_blocks first");
        PGX_CHECK(nparts >= 0 && op_id && (nparts == 0 || (right_block && left_block && target && coef)),
                  PGX_ERR_ARG, "bad operator description");
        pgx::Operator op = pgx::take_operator(P);
        op.by_left.assign(P.nblocks, -1);
        op.by_right.assign(P.nblocks, -1);
        std::vector<int> kA, kB;
        std::vector<double> ks;
        op.act_off.push_back(0);
        long in = 0, off = 0;
        for (int q = 0; q < nparts; ++q) {
            const int R = right_block[q], L = left_block[q];
            PGX_CHECK(R >= 0 && R < P.nblocks && L >= 0 && L < P.nblocks, PGX_ERR_ARG, "bad block in operator");
            PGX_CHECK(op.by_right[R] < 0 && op.by_left[L] < 0, PGX_ERR_ARG,
                      "an operator may connect a block to at most one block");
            const int dr = P.dims[R], dl = P.dims[L];
            for (int k = 0; k < dr; ++k) {
                const int t = target[in + k];
                PGX_CHECK(t >= -1 && t < dl, PGX_ERR_ARG, "operator target out of range");
                if (t >= 0 && coef[in + k] != 0.0) {
                    kA.push_back(t);
                    kB.push_back(k);
                    ks.push_back(coef[in + k]);
                }
            }
            in += dr;
            op.act_off.push_back((long)kA.size());
            op.by_right[R] = q;
            op.by_left[L] = q;
            op.parts.push_back(pgx::OpPart{R, L, dl, dr, off});
            off += (long)dl * dr;
        }
        op.total = off;
        const long K = (long)kA.size();
        op.target.reserve(std::max<long>(2 * K, 1) * sizeof(int));
        op.coef.reserve(std::max<long>(K, 1) * sizeof(double));
        if (K > 0) {
            PGX_CUDA(cudaMemcpy(op.target.as<int>(), kA.data(), K * sizeof(int), cudaMemcpyHostToDevice));
            PGX_CUDA(cudaMemcpy(op.target.as<int>() + K, kB.data(), K * sizeof(int), cudaMemcpyHostToDevice));
            PGX_CUDA(cudaMemcpy(op.coef.as<double>(), ks.data(), K * sizeof(double), cudaMemcpyHostToDevice));
        }
        P.ops.push_back(std::move(op));
        *op_id = (int32_t)P.ops.size() - 1;
    });
}

int pgx_op_rotate(pgx_ctx* c, int32_t op_id) {
    return guarded_cap(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(op_id >= 0 && op_id < (int)P.ops.size(), PGX_ERR_ARG, "bad operator id");
        PGX_CHECK(P.have_eig || (c->capturing && c->cap.eigh), PGX_ERR_STATE, "pgx_eigh first");
        PGX_CHECK(!P.ops[op_id].act_off.empty(), PGX_ERR_ARG, "operator has no Fock action (adjoint?)");
        if (c->capturing) {  // the rotation happens when the graph is replayed
            const bool was = P.ops[op_id].rotated;
            PGX_CHECK(!P.is_complex, PGX_ERR_STATE, "complex operators cannot be captured");
            pgx::rotate_operator(P, P.ops[op_id], c->stream);
            P.ops[op_id].rotated = was;
            c->cap.rotated.push_back(op_id);
            return;
        }
        pgx::rotate_operator(P, P.ops[op_id], c->stream);
    });
}

int pgx_op_adjoint(pgx_ctx* c, int32_t src, int32_t* op_id) {
    return guarded(c, [&] {
        ++c->ops_gen;
        pgx::Problem& P = c->P;
        PGX_CHECK(src >= 0 && src < (int)P.ops.size() && op_id, PGX_ERR_ARG, "bad operator id");
        PGX_CHECK(P.ops[src].rotated, PGX_ERR_STATE, "rotate the source operator first");
        pgx::Operator dst = pgx::take_operator(P);
        pgx::adjoint_operator(P, P.ops[src], dst, c->stream);
        dst.adj_src = src;
        P.ops.push_back(std::move(dst));
        *op_id = (int32_t)P.ops.size() - 1;
    });
}

int pgx_op_release(pgx_ctx* c, int32_t op_id) {
    return guarded(c, [&] {
        ++c->ops_gen;
        pgx::Problem& P = c->P;
        PGX_CHECK(op_id >= 0 && op_id < (int)P.ops.size(), PGX_ERR_ARG, "bad operator id");
        // work already queued on the context's stream that reads the operator
        // runs before anything that reuses its buffers (same stream)
        P.spare_ops.push_back(std::move(P.ops[op_id]));
        P.ops[op_id] = pgx::Operator();  // no parts, not rotated: every later use is rejected
    });
}

int pgx_op_info(pgx_ctx* c, int32_t op_id, int32_t* nparts, int32_t* right_block, int32_t* left_block) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(op_id >= 0 && op_id < (int)P.ops.size(), PGX_ERR_ARG, "bad operator id");
        const auto& op = P.ops[op_id];
        if (nparts) *nparts = (int32_t)op.parts.size();
        for (size_t q = 0; q < op.parts.size(); ++q) {
            if (right_block) right_block[q] = op.parts[q].right;
            if (left_block) left_block[q] = op.parts[q].left;
        }
    });
}

int pgx_op_read(pgx_ctx* c, int32_t op_id, int32_t part, double* out) {
    return guarded(c, [&] {
        pgx::Problem& P = c->P;
        PGX_CHECK(op_id >= 0 && op_id < (int)P.ops.size() && out, PGX_ERR_ARG, "bad operator id");
        const auto& op = P.ops[op_id];
        PGX_CHECK(op.rotated, PGX_ERR_STATE, "operator not rotated");
        PGX_CHECK(part >= 0 && part < (int)op.parts.size(), PGX_ERR_ARG, "bad part index");
        const auto& pt = op.parts[part];
        const size_t sc = P.is_complex ? 2 : 1;
        PGX_CUDA(cudaMemcpyAsync(out, op.mat.as<double>() + pt.off * sc, (size_t)pt.dl * pt.dr * sc * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream));
        PGX_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int pgx_gf(pgx_ctx* c, int32_t op1, int32_t op2, int32_t nparts, const int32_t* outer, const int32_t* inner,
           int32_t nz, const double* z, double coef_tol, double* out) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nz >= 0 && (nz == 0 || (z && out)) && (nparts == 0 || (outer && inner)), PGX_ERR_ARG,
                  "bad arguments");
        pgx::run_gf(c, op1, op2, nparts, outer, inner, nz, z, coef_tol, out);
    });
}

int pgx_susc(pgx_ctx* c, int32_t opA, int32_t opB, int32_t nparts, const int32_t* outer, const int32_t* inner,
             int32_t nz, const double* z, double pole_res, double coef_tol, double beta, double* out,
             double* zero_pole) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nz >= 0 && (nz == 0 || (z && out)) && (nparts == 0 || (outer && inner)), PGX_ERR_ARG,
                  "bad arguments");
        pgx::run_susc(c, opA, opB, nparts, outer, inner, nz, z, pole_res, coef_tol, beta, out, zero_pole);
    });
}

int pgx_ensemble_average(pgx_ctx* c, int32_t op, double* out) {
    return guarded(c, [&] {
        PGX_CHECK(out, PGX_ERR_ARG, "null output");
        pgx::run_ensemble_average(c, op, out);
    });
}

int pgx_g2(pgx_ctx* c, int32_t nparts, const pgx_g2_part* parts, int32_t nfreq, const double* z, double pole_res,
           double coef_tol, int32_t flags, double* out) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && nfreq >= 0 && (nparts == 0 || parts) && (nfreq == 0 || (z && out)), PGX_ERR_ARG,
                  "bad arguments");
        PGX_CHECK(!c->P.w_models, PGX_ERR_STATE, "needs the weights of one model (pgx_weights)");
        pgx::run_g2(c, nparts, parts, nfreq, z, pole_res, coef_tol, flags, out);
    });
}

int pgx_g2_count(pgx_ctx* c, int32_t nparts, const pgx_g2_part* parts, double coef_tol, double nz_tol,
                 long long* count) {
    return guarded(c, [&] {
        PGX_CHECK(nparts >= 0 && (nparts == 0 || parts) && count, PGX_ERR_ARG, "bad arguments");
        pgx::run_g2_count(c, nparts, parts, coef_tol, nz_tol, count);
    });
}

int pgx_timer_begin(pgx_ctx* c) {
    return guarded(c, [&] {
        if (!c->ev_begin) PGX_CUDA(cudaEventCreate(&c->ev_begin));
        if (!c->ev_end) PGX_CUDA(cudaEventCreate(&c->ev_end));
        PGX_CUDA(cudaEventRecord(c->ev_begin, c->stream));
    });
}

int pgx_timer_end(pgx_ctx* c, double* ms) {
    return guarded(c, [&] {
        PGX_CHECK(c->ev_begin && ms, PGX_ERR_STATE, "pgx_timer_begin first");
        PGX_CUDA(cudaEventRecord(c->ev_end, c->stream));
        PGX_CUDA(cudaEventSynchronize(c->ev_end));
        float t = 0.f;
        PGX_CUDA(cudaEventElapsedTime(&t, c->ev_begin, c->ev_end));
        *ms = t;
    });
}

long long pgx_launch_count(void) { return pgx::launch_counter(); }

int pgx_recip_check(const double* x, int32_t n, double* out) {
    if (!x || !out || n < 1) return PGX_ERR_ARG;
    double *dx = nullptr, *dy = nullptr;
    int rc = PGX_OK;
    if (cudaMalloc(&dx, n * sizeof(double)) != cudaSuccess || cudaMalloc(&dy, n * sizeof(double)) != cudaSuccess) {
        rc = PGX_ERR_OOM;
    } else if (cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        rc = PGX_ERR_CUDA;
    } else {
        recip_check_kernel<<<(n + 255) / 256, 256>>>(dx, dy, n);
        ++pgx::launch_counter();
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(out, dy, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = PGX_ERR_CUDA;
    }
    cudaGetLastError();
    if (dx) cudaFree(dx);
    if (dy) cudaFree(dy);
    return rc;
}

int pgx_profile_begin(pgx_ctx* c) {
    return guarded(c, [&] {
        c->prof.clear();
        c->prof.on = true;
    });
}

int pgx_profile_end(pgx_ctx* c, int32_t* nkernels) {
    return guarded(c, [&] {
        PGX_CHECK(c->prof.on, PGX_ERR_STATE, "pgx_profile_begin first");
        c->prof.on = false;
        c->prof.resolve();
        if (nkernels) *nkernels = (int32_t)c->prof.stats.size();
    });
}

int pgx_profile_kernel(pgx_ctx* c, int32_t i, char* name, int32_t name_cap, int32_t* launches, double* ms,
                       double* flops, double* bytes) {
    return guarded(c, [&] {
        PGX_CHECK(i >= 0 && i < (int32_t)c->prof.stats.size(), PGX_ERR_ARG, "kernel index out of range");
        const pgx::KernelStat& k = c->prof.stats[i];
        if (name && name_cap > 0) {
            const size_t n = std::min<size_t>(k.name.size(), (size_t)name_cap - 1);
            std::copy(k.name.begin(), k.name.begin() + n, name);
            name[n] = '\0';
        }
        if (launches) *launches = k.launches;
        if (ms) *ms = k.ms;
        if (flops) *flops = k.flops;
        if (bytes) *bytes = k.bytes;
    });
}

int pgx_g2_last_timing(pgx_ctx* c, double* total_ms, double* gemm_ms, double* gemm_flops) {
    return guarded(c, [&] {
        if (total_ms) *total_ms = c->g2t.total_ms;
        if (gemm_ms) *gemm_ms = c->g2t.gemm_ms;
        if (gemm_flops) *gemm_flops = c->g2t.gemm_flops;
    });
}

}  // extern "C"
