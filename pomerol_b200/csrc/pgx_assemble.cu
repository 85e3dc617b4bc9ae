// Block Hamiltonians assembled on the device from the Fock action of their
// monomial terms.
//
// Replaces the dense assembly of HamiltonianPart::prepare
// (HamiltonianPart.cpp:56-76): for every Fock state |s> of a block (a column
// of the block matrix) and every term c_t O_t of H, O_t |s> = sign |o> adds
// sign * c_t to H[o][s].  One thread per column applies the terms in their
// given order, so each entry receives its contributions in the same order as
// a sequential host assembly (bitwise the same sums) and no two threads write
// the same entry.

#include "pgx_common.cuh"
#include "pgx_internal.h"

namespace pgx {

namespace {

struct AssembleArgs {
    const int* ops;            // nterms x PGX_TERM_OPS (2 mode + dagger, -1 padding)
    const double* coef;        // nterms x (re, im)
    int nterms;
    const uint64_t* fock;      // Fock state of every (block, inner) pair, blocks in order
    long nstates;
    const int* state_block;    // by Fock state
    const int* state_inner;    // by Fock state
    const int* dims;
    const long* moff;
    int is_complex;
    double* H;
    int* status;
};

__global__ void assemble_kernel(AssembleArgs g) {
    extern __shared__ int sops[];  // the term list, staged once per CTA
    const int nops = g.nterms * PGX_TERM_OPS;
    for (int i = threadIdx.x; i < nops; i += blockDim.x) sops[i] = g.ops[i];
    __syncthreads();
    const long col = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (col >= g.nstates) return;
    const uint64_t s0 = g.fock[col];
    const int b = g.state_block[s0], j = g.state_inner[s0];
    const long d = g.dims[b];
    double* Hb = g.H + (g.is_complex ? 2 : 1) * g.moff[b];
    for (int t = 0; t < g.nterms; ++t) {
        const int* op = sops + t * PGX_TERM_OPS;
        uint64_t s = s0;
        double sign = 1.0;
        bool ok = true;
        for (int k = PGX_TERM_OPS - 1; k >= 0 && ok; --k) {  // the rightmost operator acts first
            const int o = op[k];
            if (o < 0) continue;
            const uint64_t mask = 1ull << (o >> 1);
            const bool occ = (s & mask) != 0;
            if ((o & 1) == (int)occ) {  // c^+ on an occupied or c on an empty mode
                ok = false;
                break;
            }
            if (__popcll(s & (mask - 1)) & 1) sign = -sign;
            s ^= mask;
        }
        if (!ok) continue;
        if (g.state_block[s] != b) {
            atomicExch(g.status, PGX_ERR_ARG);
            continue;
        }
        const long idx = (long)g.state_inner[s] * d + j;
        if (g.is_complex) {
            Hb[2 * idx] += sign * g.coef[2 * t];
            Hb[2 * idx + 1] += sign * g.coef[2 * t + 1];
        } else {
            Hb[idx] += sign * g.coef[2 * t];
        }
    }
}

}  // namespace

void assemble_hamiltonian(pgx_ctx* c, int nterms, const int32_t* ops, const double* coef, int nmodes,
                          const uint64_t* fock, const int32_t* state_block, const int32_t* state_inner) {
    Problem& P = c->P;
    cudaStream_t st = c->stream;
    const long nfock = 1L << nmodes;
    // every index the kernel follows is checked here
    for (long q = 0; q < (long)nterms * PGX_TERM_OPS; ++q)
        PGX_CHECK(ops[q] < 2 * nmodes && ops[q] >= -1, PGX_ERR_ARG, "term operator out of range");
    for (long s = 0; s < nfock; ++s) {
        PGX_CHECK(state_block[s] >= 0 && state_block[s] < P.nblocks, PGX_ERR_ARG, "state block out of range");
        PGX_CHECK(state_inner[s] >= 0 && state_inner[s] < P.dims[state_block[s]], PGX_ERR_ARG,
                  "state position out of range");
    }
    for (int b = 0; b < P.nblocks; ++b)
        for (int i = 0; i < P.dims[b]; ++i) {
            const uint64_t s = fock[P.eoff[b] + i];
            PGX_CHECK(s < (uint64_t)nfock && state_block[s] == b && state_inner[s] == i, PGX_ERR_ARG,
                      "Fock state list disagrees with the state tables");
        }
    const size_t sc = P.is_complex ? 2 : 1;
    const size_t b_ops = (size_t)std::max(nterms, 1) * PGX_TERM_OPS * sizeof(int);
    const size_t b_coef = (size_t)std::max(nterms, 1) * 2 * sizeof(double);
    const size_t b_fock = (size_t)P.esize * sizeof(uint64_t);
    const size_t b_tab = (size_t)nfock * sizeof(int);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    P.asm_buf.reserve(al(b_ops) + al(b_coef) + al(b_fock) + 2 * al(b_tab));
    char* base = P.asm_buf.as<char>();
    int* d_ops = reinterpret_cast<int*>(base);
    double* d_coef = reinterpret_cast<double*>(base + al(b_ops));
    uint64_t* d_fock = reinterpret_cast<uint64_t*>(base + al(b_ops) + al(b_coef));
    int* d_sb = reinterpret_cast<int*>(base + al(b_ops) + al(b_coef) + al(b_fock));
    int* d_si = reinterpret_cast<int*>(base + al(b_ops) + al(b_coef) + al(b_fock) + al(b_tab));
    if (nterms > 0) {
        h2d(d_ops, ops, (size_t)nterms * PGX_TERM_OPS * sizeof(int), st);
        h2d(d_coef, coef, (size_t)nterms * 2 * sizeof(double), st);
    }
    h2d(d_fock, fock, b_fock, st);
    h2d(d_sb, state_block, b_tab, st);
    h2d(d_si, state_inner, b_tab, st);
    PGX_CUDA(cudaMemsetAsync(P.d_H, 0, P.msize * sc * sizeof(double), st));
    PGX_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int), st));
    AssembleArgs a{d_ops, d_coef, nterms, d_fock, P.esize, d_sb, d_si, P.d_dims, P.d_moff, P.is_complex ? 1 : 0,
                   P.d_H, P.d_status};
    const size_t smem = (size_t)nterms * PGX_TERM_OPS * sizeof(int);
    PGX_CHECK(smem <= 200 * 1024, PGX_ERR_ARG, "too many Hamiltonian terms for one launch");
    if (smem > 48 * 1024)
        PGX_CUDA(cudaFuncSetAttribute(assemble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {
        double nnz = (double)P.esize * nterms;  // one term application per (state, term)
        ProfRange pr("assemble_kernel", st, 0.0, 8.0 * sc * P.msize + 16.0 * nnz / std::max(nterms, 1));
        assemble_kernel<<<ceil_div(P.esize, 128), 128, smem, st>>>(a);
        check_launch("assemble_kernel");
    }
    int status = 0;
    PGX_CUDA(cudaMemcpyAsync(&status, P.d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    PGX_CUDA(cudaStreamSynchronize(st));
    PGX_CHECK(status == 0, PGX_ERR_ARG, "a Hamiltonian term connects different blocks");
    P.have_asm = true;
    P.asm_nterms = nterms;
    P.d_asm_ops = d_ops;
    P.d_asm_fock = d_fock;
    P.d_asm_sb = d_sb;
    P.d_asm_si = d_si;
}

}  // namespace pgx
