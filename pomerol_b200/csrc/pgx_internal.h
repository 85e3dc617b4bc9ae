// Internal state of a libpgx context (host side of the device runtime).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "pgx_common.cuh"

namespace pgx {

// A context's table of measured-fastest GEMM tile classes (pgx_autotune_end),
// indexed by operand-type key and the (M, N) size buckets; -1 keeps the
// padding rule (see gemm_class_for).
constexpr int GEMM_NKEY = 32, GEMM_NBUCKET = 7;
struct GemmTune {
    signed char cls[GEMM_NKEY][GEMM_NBUCKET][GEMM_NBUCKET];
    GemmTune() { std::memset(cls, -1, sizeof(cls)); }
};
GemmTune*& active_tune();   // the running context's table (null: untuned)
int& forced_gemm_class();   // a class imposed while the tuner measures it (-1: none)

// The tuner (pgx_autotune_begin .. end) measures products where they are
// launched: while a context records, launch_gemm_batch first runs each size
// bucket's products in every candidate (the padding rule and every valid
// class), outputs redirected to scratch, and adds the times to the context's
// TuneRecorder (defined below DevBuf).
struct TuneRecorder;
TuneRecorder*& active_recorder();  // non-null while a context records
struct DevBuf;
// launch(cls, scratch, probs, index, st): the bucket's products in class cls
// (-1: the padding rule), outputs in scratch, descriptors in probs and index.
using TuneLaunch = std::function<void(int cls, void* scratch, DevBuf& probs, DevBuf& index, cudaStream_t st)>;
void tune_measure(TuneRecorder& rec, int key, int mb, int nb, size_t c_bytes, const TuneLaunch& launch,
                  cudaStream_t st);

// Counts device allocations and frees in the process: a captured CUDA graph
// records it and refuses to replay once any buffer may have moved.
unsigned long long& alloc_epoch();

// Device allocation owned by a context.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void reserve(size_t n) {
        if (n <= bytes) return;
        release();
        if (n == 0) return;
        cudaError_t e = cudaMalloc(&p, n);
        ++alloc_epoch();
        if (e != cudaSuccess) {
            p = nullptr;
            bytes = 0;
            cudaGetLastError();
            throw Error{PGX_ERR_OOM, "cudaMalloc(" + std::to_string(n) + " bytes) failed"};
        }
        bytes = n;
    }
    void release() {
        if (p) {
            cudaFree(p);
            ++alloc_epoch();
        }
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Workspace of the int8 split products (digits, exponents, error flag).
struct OzWork {
    DevBuf A, B, ea, fb, err;
    int cta_pair = 0;  // 0: 128 x 256 tiles on single CTAs (measured faster); 1: 256 x 256 tiles on CTA pairs
};

// Times of the products measured since pgx_autotune_begin, per (operand-type
// key, M bucket, N bucket): index 0 the padding rule, c + 1 tile class c
// (DBL_MAX where c is not valid for the bucket).
struct TuneRecorder {
    std::map<std::tuple<int, int, int>, std::vector<double>> total;
    DevBuf scratch, probs, index;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TuneRecorder() = default;
    TuneRecorder(const TuneRecorder&) = delete;
    TuneRecorder& operator=(const TuneRecorder&) = delete;
    ~TuneRecorder();
};

// One rotated monomial operator.
struct OpPart {
    int right, left;     // blocks
    int dl, dr;          // sizes
    long off;            // element offset of the rotated matrix in Operator::mat
};

struct Operator {
    std::vector<OpPart> parts;
    std::vector<int> by_left, by_right;  // block -> part index or -1
    DevBuf mat;                           // rotated parts (double or cd), row-major dl x dr
    DevBuf target, coef;                  // Fock action (int per right state, double per right state)
    std::vector<long> act_off;            // offset into target/coef per part
    bool rotated = false;
    bool is_complex = false;
    long total = 0;                       // elements in mat
    int adj_src = -1;                     // for an adjoint: the operator it was formed from
};

// One exact-diagonalisation problem: blocks, eigensystem, weights, operators.
struct Problem {
    int nblocks = 0;
    int dmax = 0;
    bool is_complex = false;
    std::vector<int> dims;
    std::vector<long> moff, eoff;  // matrix / vector offsets
    long msize = 0, esize = 0;
    bool have_H = false, have_eig = false, have_w = false;
    double beta = 0.0, E0 = 0.0, Z = 0.0;
    std::vector<int> retained;

    DevBuf H, work, work2, U, E, w, dims_d, moff_d, eoff_d, order_d, status, tri, tri_items, eigh_gemm,
        eigh_scratch;
    DevBuf op_probs, op_tiles, op_meta;  // descriptor lists of operator rotation / adjoint
    DevBuf asm_buf;                      // term list and state tables of the Hamiltonian assembly
    // device copies of the last assembly's inputs (valid while have_asm)
    bool have_asm = false;
    int asm_nterms = 0;
    const int* d_asm_ops = nullptr;
    const uint64_t* d_asm_fock = nullptr;
    const int* d_asm_sb = nullptr;
    const int* d_asm_si = nullptr;
    DevBuf vjp_buf;                      // gradient workspace of pgx_gf_vjp
    DevBuf chi3_small, chi3_big;         // per-part constants / frequency-dependent matrices of pgx_chi3
    // complex blocks: real embedding of twice the size and its eigensolver workspace
    DevBuf cx_meta, cx_H, cx_A, cx_Zc, cx_U, cx_E, cx_tri, cx_S, cx_items, cx_gemm;
    std::vector<double> w_host;          // host copy of the weights (set with them)
    // independent models sharing the context (pgx_set_models): blocks
    // model_first[m] .. model_first[m+1]-1 form model m, at inverse temperature model_beta[m]
    int nmodels = 0;
    std::vector<int> model_first, block_model;
    std::vector<double> model_beta, model_E0, model_Z;
    bool w_models = false;               // the weights are per model (pgx_weights_models)
    DevBuf model_buf;                    // state ranges, inverse temperatures, E0 and Z per model
    int* d_dims = nullptr;
    long* d_moff = nullptr;
    long* d_eoff = nullptr;
    int* d_order = nullptr;
    int* d_status = nullptr;
    double* d_H = nullptr;
    double* d_work = nullptr;
    double* d_work2 = nullptr;
    double* d_U = nullptr;
    double* d_E = nullptr;
    double* d_w = nullptr;

    std::vector<Operator> ops;
    std::vector<Operator> spare_ops;  // released operators whose device buffers are reused
};

// An operator with the device buffers of a released one, if any.
inline Operator take_operator(Problem& P) {
    if (P.spare_ops.empty()) return Operator();
    Operator op = std::move(P.spare_ops.back());
    P.spare_ops.pop_back();
    op.parts.clear();
    op.by_left.clear();
    op.by_right.clear();
    op.act_off.clear();
    op.rotated = op.is_complex = false;
    op.total = 0;
    op.adj_src = -1;
    return op;
}

// Events owned by one call, destroyed on every exit from it (a throw included).
struct ScopedEvents {
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
    explicit ScopedEvents(int n) {
        for (int i = 0; i < n && i < 4; ++i) {
            const cudaError_t r = cudaEventCreate(&e[i]);
            if (r != cudaSuccess) {
                e[i] = nullptr;
                release();
                throw Error{PGX_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(r)};
            }
        }
    }
    ~ScopedEvents() { release(); }
    ScopedEvents(const ScopedEvents&) = delete;
    ScopedEvents& operator=(const ScopedEvents&) = delete;
    cudaEvent_t operator[](int i) const { return e[i]; }

  private:
    void release() {
        for (auto& x : e) {
            if (x) cudaEventDestroy(x);
            x = nullptr;
        }
    }
};

struct G2Timing {
    double total_ms = 0, gemm_ms = 0, gemm_flops = 0;
};

// Pinned host staging for descriptor uploads.  Append-only while copies from
// it may be pending, so the source of every asynchronous copy stays intact
// until the copy has run; recycled at the end of an entry-point call whose
// stream is idle (every call that returns results ends that way).  Blocks are
// kept across calls.
struct HostArena {
    std::vector<std::pair<char*, size_t>> blocks;  // (pinned pointer, capacity)
    size_t cur = 0, used = 0;                      // block in use, bytes used in it
    bool dirty = false;                            // copies may be pending
    void* put(const void* src, size_t n);
    void recycle(cudaStream_t st);
    HostArena() = default;
    HostArena(const HostArena&) = delete;
    HostArena& operator=(const HostArena&) = delete;
    ~HostArena();
};

// Arena of the context whose entry point runs on this thread (or null).
HostArena*& active_arena();

// Host-to-device copy of a descriptor list on stream st: staged through the
// active context's pinned arena (fully asynchronous), else a pageable copy.
void h2d(void* dst, const void* src, size_t bytes, cudaStream_t st);

// Per-kernel device times of a context, on request (pgx_profile_begin/end):
// each instrumented launch site brackets its kernel with an event pair on the
// launching stream and states the kernel's algorithmic FLOPs and DRAM bytes.
struct KernelStat {
    std::string name;
    int launches = 0;
    double ms = 0, flops = 0, bytes = 0;
};

struct Profiler {
    struct Range {
        std::string name;
        cudaEvent_t a, b;
        double flops, bytes;
    };
    bool on = false;
    std::vector<Range> open;
    std::vector<cudaEvent_t> spare;
    std::vector<KernelStat> stats;
    cudaEvent_t event();
    void clear();
    void resolve();  // waits for the recorded events and folds them into stats
    ~Profiler();
};

// Profiler of the context whose entry point runs on this thread (or null).
Profiler*& active_profiler();

// Brackets the launches of its scope on stream st when profiling is on.
class ProfRange {
  public:
    ProfRange(const char* name, cudaStream_t st, double flops, double bytes);
    ~ProfRange();
    ProfRange(const ProfRange&) = delete;
    ProfRange& operator=(const ProfRange&) = delete;

  private:
    Profiler* p_ = nullptr;
    cudaStream_t st_ = nullptr;
    size_t idx_ = 0;
};

}  // namespace pgx

struct pgx_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    pgx::Problem P;
    pgx::G2Timing g2t;
    pgx::Profiler prof;
    pgx::HostArena arena;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    // side streams (and their fork / join events) for independent launches
    cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};
    long long g2_batch_bytes = 0, g2_chain_bytes = 0;  // pgx_set_g2_workspace (0: defaults)
    double g2_split_min_macs = 1e9;                     // pgx_set_g2_split_threshold
    double g2_split_weight_budget = 4.0;                // pgx_set_g2_split_weight_budget (<= 0: every product at full digits)
    int g2_split_slices = 6;                            // pgx_set_g2_split_slices
    pgx::OzWork oz;                                     // int8 split products
    cudaEvent_t fork = nullptr, join[4] = {nullptr, nullptr, nullptr, nullptr};
    // scratch for G2 and Lehmann kernels
    pgx::DevBuf scratch[12];
    // CUDA graphs of captured entry-point sequences (pgx_graph_begin / end / replay)
    struct Graph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        std::unique_ptr<pgx::HostArena> arena;  // staging of the captured copies, kept with the graph
        unsigned long long epoch = 0;           // alloc_epoch() at the end of the capture
        unsigned long problem_gen = 0, ops_gen = 0;
        bool eigh = false;                      // the sequence contains pgx_eigh
        std::vector<int> rotated;               // operators the sequence rotates
    };
    std::vector<Graph> graphs;
    bool capturing = false;
    Graph cap;                                  // the graph being captured
    unsigned long problem_gen = 0;              // bumped by pgx_set_blocks
    unsigned long ops_gen = 0;                  // bumped when operators are defined, formed or released
    pgx::GemmTune tune;                         // pgx_autotune_end's measured tile classes
    bool tuned = false;
    std::unique_ptr<pgx::TuneRecorder> recorder;  // open between pgx_autotune_begin and end
};

namespace pgx {

void launch_eigh(pgx_ctx* c);
void ensure_side_streams(pgx_ctx* c);  // the context's four side streams and their events

// Makes stream st wait for the context's first n side streams when the scope
// ends, on a throw too: work issued there before the throw then completes
// before st's later work and before the host staging is recycled.
struct SideJoin {
    pgx_ctx* c;
    cudaStream_t st;
    int n;
    SideJoin(pgx_ctx* c_, cudaStream_t st_, int n_) : c(c_), st(st_), n(n_) {}
    ~SideJoin() {
        for (int k = 0; k < n; ++k) {
            cudaEventRecord(c->join[k], c->aux[k]);
            cudaStreamWaitEvent(st, c->join[k], 0);
        }
    }
    SideJoin(const SideJoin&) = delete;
    SideJoin& operator=(const SideJoin&) = delete;
};

// Device buffers of one eigensolve (any number of blocks), all caller-owned.
struct EighDev {
    const int* dims;
    const long* moff;
    const long* eoff;
    const double* H;     // packed blocks, row-major
    double* A;           // workspace, sum d^2 (later the eigenvectors of T)
    double* Zc;          // workspace, sum d^2
    double* tri;         // workspace, 2 sum d (diagonal, sub-diagonal)
    double* lam;         // workspace, sum d
    int* sb;             // workspace, 2 sum d
    int* rank;           // workspace, sum d
    double* S;           // workspace, eigh_vec_scratch_doubles(dims)
    void* items;         // workspace, eigh_item_bytes(dims)
    void* gemm_probs;    // workspace, eigh_gemm_bytes(dims, ...)
    void* gemm_tiles;    // workspace, tile bytes from eigh_gemm_bytes
    double* U;           // output, sum d^2
    double* E;           // output, sum d
    int* status;         // PGX_ERR_NUMERIC when a vector is not finite
    // optional: streams on which independent Householder launches run
    // concurrently with the main stream (all null: everything on one stream)
    cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[4] = {nullptr, nullptr, nullptr, nullptr};
};
size_t eigh_item_bytes(const std::vector<int>& dims);
size_t eigh_gemm_bytes(const std::vector<int>& dims, size_t* tiles_bytes);
size_t eigh_vec_scratch_doubles(const std::vector<int>& dims);
void launch_eigh_raw(const EighDev& d, const std::vector<int>& dims, const std::vector<long>& moff,
                     cudaStream_t st);
void launch_weights(Problem& P, double beta, cudaStream_t st);
void assemble_hamiltonian(pgx_ctx* c, int nterms, const int32_t* ops, const double* coef, int nmodes,
                          const uint64_t* fock, const int32_t* state_block, const int32_t* state_inner);
void run_gf_vjp(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                const double* z, const double* lambda, double* dterm, double* dE);
void run_susc_vjp(pgx_ctx* c, int opA, int opB, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                  const double* z, double pole_res, const double* lambda, double* dterm, double* dE);
void rotate_operator(Problem& P, Operator& op, cudaStream_t st);
void adjoint_operator(Problem& P, const Operator& src, Operator& dst, cudaStream_t st);
void run_gf(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner, int nz,
            const double* z, double coef_tol, double* out);
void run_susc(pgx_ctx* c, int opA, int opB, int nparts, const int32_t* outer, const int32_t* inner, int nz,
              const double* z, double pole_res, double coef_tol, double beta, double* out, double* zero_pole);
void run_ensemble_average(pgx_ctx* c, int op, double* out);
void run_g2(pgx_ctx* c, int nparts, const pgx_g2_part* parts, int nfreq, const double* z, double pole_res,
            double coef_tol, int flags, double* out);
void run_g2_anchored(pgx_ctx* c, int nparts, const pgx_g2_part* parts, int nfreq, const double* z, double pole_res,
                     double anchor_tol, int split_slices, double* out);
void run_split_gemm_check(pgx_ctx* c, int M, int N, int K, int nb, int S, unsigned long long seed, double* err,
                          double* ms_split, double* ms_fp64);
void run_chi3(pgx_ctx* c, int channel, int nparts, const pgx_chi3_part* parts, int nfreq, const double* z,
              double pole_res, double* out);
void set_models(Problem& P, int nmodels, const int32_t* first_block, const double* beta);
void launch_weights_models(Problem& P, cudaStream_t st);
void run_gf_models(pgx_ctx* c, int op1, int op2, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                   const double* z, double coef_tol, double* out);
void run_susc_models(pgx_ctx* c, int opA, int opB, int nparts, const int32_t* outer, const int32_t* inner, int nz,
                     const double* z, double pole_res, double coef_tol, double* out, double* zero_pole);
int install_tuning(pgx_ctx* c, const TuneRecorder& rec);
void run_g2_count(pgx_ctx* c, int nparts, const pgx_g2_part* parts, double coef_tol, double nz_tol, long long* count);

}  // namespace pgx
