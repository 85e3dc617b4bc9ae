/*
 * libpgx: C ABI of the B200 (sm_100a) engine behind pomerol's G2 / G / chi path.
 *
 * One context = one GPU, one CUDA stream, and every device buffer of one
 * exact-diagonalisation problem (symmetry blocks, eigensystem, Boltzmann
 * weights, rotated monomial operators).  Callers pass host pointers with
 * explicit sizes; every entry point returns a PGX_* status and never throws.
 * Complex numbers are interleaved (re, im) doubles.  Matrices are row-major.
 *
 * Each entry point names the reference code it replaces (pomerol 2.3 paths,
 * relative to the reference project root).
 */
#ifndef PGX_H
#define PGX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PGX_OK 0
#define PGX_ERR_ARG 1       /* invalid argument or size */
#define PGX_ERR_OOM 2       /* device allocation failed */
#define PGX_ERR_CUDA 3      /* CUDA runtime error */
#define PGX_ERR_TIMEOUT 4   /* bounded device wait expired */
#define PGX_ERR_NUMERIC 5   /* eigensolver did not converge / non-finite input */
#define PGX_ERR_STATE 6     /* call order violated (e.g. rotate before eigh) */
#define PGX_ERR_NODEV 7     /* no CUDA device */

/* G2 evaluation flags */
#define PGX_G2_EXACT 0           /* no coefficient filters */
#define PGX_G2_REFERENCE_RULE 1  /* apply the reference's weight filter at block level */
#define PGX_G2_ANCHORED 2        /* weight-anchored sum: each sub-term is restricted to the
                                    states of its weighted index with w > coef_tol */
#define PGX_G2_SPLIT_I8 4        /* with PGX_G2_ANCHORED: the stacked (z1, z3) products run on
                                    the int8 tensor cores, operands split into balanced
                                    base-254 digits (six by default) with power-of-two
                                    row/column scales (Ozaki scheme), int32-exact partial
                                    products summed in FP64 */

typedef struct pgx_ctx pgx_ctx;

/* Library version (major*10000 + minor*100 + patch). */
int pgx_version(void);

/* Create a context on `device` (one CUDA stream, no device memory yet). */
int pgx_create(int device, pgx_ctx** out);
/* Destroy a context and free all of its device memory. */
int pgx_destroy(pgx_ctx* ctx);
/* Message of the last failed call on this context ("" if none). */
const char* pgx_last_error(const pgx_ctx* ctx);

/* ------------------------------------------------------------------------
 * Symmetry blocks and K1 eigensolve.
 * Replaces: StatesClassification block sizes (StatesClassification.hpp:59-70)
 * and HamiltonianPart::computeImpl / Hamiltonian::compute
 * (HamiltonianPart.cpp:90-102, Hamiltonian.cpp:69-113).
 * ------------------------------------------------------------------------ */

/* Declare nblocks blocks of sizes dims[b] (real symmetric: is_complex = 0;
 * complex Hermitian: 1).  Resets every per-problem device buffer. */
int pgx_set_blocks(pgx_ctx* ctx, int32_t nblocks, const int32_t* dims, int32_t is_complex);

/* Upload the block Hamiltonians: block b is dims[b]^2 consecutive (row-major)
 * elements, blocks in order.  Host -> device copy only. */
int pgx_set_hamiltonian(pgx_ctx* ctx, const double* H);

/* Assemble the block Hamiltonians on the device from their monomial terms
 * (in place of pgx_set_hamiltonian; replaces the dense assembly of
 * HamiltonianPart::prepare, HamiltonianPart.cpp:56-76).  Term t is the product
 * of the operators ops[t*PGX_TERM_OPS .. t*PGX_TERM_OPS+PGX_TERM_OPS-1] read
 * left to right (entry 2*mode + 1 for c^+_mode, 2*mode for c_mode, -1 to pad
 * the tail) times the complex coefficient (coef[2t], coef[2t+1]; real blocks
 * use the real part).  It acts on a Fock state from its rightmost operator,
 * with the Jordan-Wigner sign (-1)^(occupied modes below) for each operator.
 * fock lists the Fock state of every block position, blocks in the order of
 * pgx_set_blocks (sum of dims entries); state_block[s] and state_inner[s]
 * give, for every s < 2^nmodes, its block and position (nmodes <= 30).
 * Returns PGX_ERR_ARG if the tables disagree or a term maps a state out of
 * its block. */
#define PGX_TERM_OPS 8
int pgx_assemble_hamiltonian(pgx_ctx* ctx, int32_t nterms, const int32_t* ops, const double* coef, int32_t nmodes,
                             const uint64_t* fock, const int32_t* state_block, const int32_t* state_inner);

/* Copy the block Hamiltonians on the device (uploaded or assembled) to the
 * host, packed like pgx_set_hamiltonian's input. */
int pgx_get_hamiltonian(pgx_ctx* ctx, double* H);

/* Reverse-mode derivative of a Green's function through the whole chain
 * eigensolve -> weights -> operator rotation -> Lehmann sum (the reference
 * has no derivatives).  G(z_n) is the function pgx_gf evaluates for the same
 * (op1, op2, parts, z) without coefficient filtering; for a loss L with
 * dL = Re sum_n lambda[n] dG(z_n) (lambda: nz complex, e.g. 2 conj(G - G_target)
 * for sum |G - G_target|^2) it returns dterm[t] = dL/dc_t for every term of
 * the last pgx_assemble_hamiltonian call (real part of the coefficient;
 * a term and its Hermitian conjugate are separate terms, and the derivative
 * assumes the perturbation of H stays symmetric), and, when dE is non-NULL,
 * dL/dE_s for every state.  op1 and op2 are operators defined by their Fock
 * action or adjoints of such operators.  Real Hamiltonians only; derivative
 * terms between eigenvalues closer than 1e-10 max|E| are dropped (exact for
 * G, which does not depend on the basis of a degenerate subspace). */
int pgx_gf_vjp(pgx_ctx* ctx, int32_t op1, int32_t op2, int32_t nparts, const int32_t* outer, const int32_t* inner,
               int32_t nz, const double* z, const double* lambda, double* dterm, double* dE);

/* The same for a susceptibility: chi(z_n) as pgx_susc evaluates it for the
 * same (opA, opB, parts, z, pole_res) without coefficient filtering, with
 * beta the one of the last pgx_weights call (its zero-pole terms act at z = 0
 * and are differentiated as beta A B w; the disconnected part is not
 * included, as in pgx_susc).  Outputs as pgx_gf_vjp. */
int pgx_susc_vjp(pgx_ctx* ctx, int32_t opA, int32_t opB, int32_t nparts, const int32_t* outer, const int32_t* inner,
                 int32_t nz, const double* z, double pole_res, const double* lambda, double* dterm, double* dE);

/* Diagonalise every block in one launch (FP64).  Eigenvalues ascending per
 * block; eigenvectors are the columns of each block's U.  The uploaded
 * Hamiltonian is kept, so this can be re-run. */
int pgx_eigh(pgx_ctx* ctx);

/* Copy the eigensystem to the host: E (sum of dims), U (packed like H).
 * Either pointer may be NULL. */
int pgx_get_eigensystem(pgx_ctx* ctx, double* E, double* U);

/* Load an eigensystem saved from pgx_get_eigensystem (same layout: E sum of
 * dims, ascending inside every block; U packed like H, complex interleaved
 * for complex blocks) in place of pgx_eigh, so a restart skips the
 * eigensolve (checkpoint / reload of the eigendata; the reference recomputes
 * Hamiltonian::compute, Hamiltonian.cpp:69-113, every time).  Call after
 * pgx_set_blocks with the same blocks; operators must be rotated again. */
int pgx_set_eigensystem(pgx_ctx* ctx, const double* E, const double* U);

/* Ground energy min_b min E (Hamiltonian::computeGroundEnergy,
 * Hamiltonian.cpp:125-130). */
int pgx_ground_energy(pgx_ctx* ctx, double* E0);

/* ------------------------------------------------------------------------
 * K5 Boltzmann weights.
 * Replaces: DensityMatrixPart::computeUnnormalized/normalize/truncate and
 * DensityMatrix::compute/truncateBlocks (DensityMatrixPart.cpp:23-50,
 * DensityMatrix.cpp:38-92).
 * ------------------------------------------------------------------------ */

/* w_s = exp(-beta (E_s - E0)) / Z for every state; w (sum of dims) and Z are
 * copied out when non-NULL. */
int pgx_weights(pgx_ctx* ctx, double beta, double* w, double* Z);

/* Retained flag per block: any weight > tol (all blocks retained if never
 * called). */
int pgx_truncate_blocks(pgx_ctx* ctx, double tol, int32_t* retained);

/* ------------------------------------------------------------------------
 * K2 monomial-operator rotation.
 * Replaces: MonomialOperator::prepare/compute (MonomialOperator.hpp:160-195,
 * MonomialOperator.cpp:33-46), MonomialOperatorPart::computeImpl and
 * setFromAdjoint (MonomialOperatorPart.cpp:48-111), FieldOperatorContainer::
 * computeAll (FieldOperatorContainer.cpp:22-37).
 * ------------------------------------------------------------------------ */

/* Define a monomial operator by its Fock action.  Part p maps right block
 * right_block[p] into left block left_block[p]; for state k (inner index) of
 * the right block, target[k] is the inner index of O|k> in the left block (-1
 * if O|k> = 0) and coef[k] its coefficient (Jordan-Wigner sign times the
 * monomial's coefficient; real).  target/coef are concatenated over parts in
 * order, dims[right_block[p]] entries per part.  Returns an operator id. */
int pgx_op_define(pgx_ctx* ctx, int32_t nparts, const int32_t* right_block, const int32_t* left_block,
                  const int32_t* target, const double* coef, int32_t* op_id);

/* O'_p = U_L^dagger (O U_R) for every part of the operator, in one launch. */
int pgx_op_rotate(pgx_ctx* ctx, int32_t op_id);

/* New operator whose parts are the adjoints of `src`'s rotated parts
 * (c from c^+).  Returns its id. */
int pgx_op_adjoint(pgx_ctx* ctx, int32_t src, int32_t* op_id);

/* Release an operator: its device memory is kept by the context and reused
 * by the next pgx_op_define / pgx_op_adjoint (as when the reference destroys a
 * MonomialOperator).  The id stays invalid afterwards. */
int pgx_op_release(pgx_ctx* ctx, int32_t op_id);

/* Number of parts, and per part (right block, left block). */
int pgx_op_info(pgx_ctx* ctx, int32_t op_id, int32_t* nparts, int32_t* right_block, int32_t* left_block);

/* Copy part `part` of a rotated operator (d_left x d_right, row-major). */
int pgx_op_read(pgx_ctx* ctx, int32_t op_id, int32_t part, double* out);

/* ------------------------------------------------------------------------
 * K3 pair-Lehmann sums: G and chi, plus <A>.
 * Replaces: GreensFunction(Part) compute/operator() (GreensFunction.cpp:41-100,
 * GreensFunctionPart.cpp:24-110, GreensFunction.hpp:123-136) and
 * Susceptibility(Part) (Susceptibility.cpp:42-119, SusceptibilityPart.cpp:27-127,
 * SusceptibilityPart.hpp:212-220), EnsembleAverage (EnsembleAverage.cpp:27-67).
 * ------------------------------------------------------------------------ */

/* G(z_n) = sum over parts (outer block o, inner block i) of
 * sum_{a in o, b in i} F1_ab F2_ba (w_a + w_b) / (z_n - (E_b - E_a)),
 * dropping residues with |R| <= coef_tol.  F1 is the part of op1 whose left
 * block is o; F2 the part of op2 whose right block is o.  z: nz complex;
 * out: nz complex. */
int pgx_gf(pgx_ctx* ctx, int32_t op1, int32_t op2, int32_t nparts, const int32_t* outer, const int32_t* inner,
           int32_t nz, const double* z, double coef_tol, double* out);

/* chi(z_n) = -sum R/(z_n - P) + (|z_n| <= eps ? beta * W0 : 0), where pairs
 * with |P| < pole_res go to the zero-pole weight W0 = sum A_ab B_ba w_a and the
 * rest carry R = A_ab B_ba (w_a - w_b) (dropped if |R| <= coef_tol).  The
 * zero-pole weight is also returned (complex) when zero_pole is non-NULL. */
int pgx_susc(pgx_ctx* ctx, int32_t opA, int32_t opB, int32_t nparts, const int32_t* outer, const int32_t* inner,
             int32_t nz, const double* z, double pole_res, double coef_tol, double beta, double* out,
             double* zero_pole);

/* <A> = sum over diagonal, retained parts of sum_a A_aa w_a (complex out). */
int pgx_ensemble_average(pgx_ctx* ctx, int32_t op, double* out);

/* ------------------------------------------------------------------------
 * K4 two-particle Green's function.
 * Replaces: TwoParticleGFPart::computeImpl/addMultiterm/operator()
 * (TwoParticleGFPart.cpp:189-322, TwoParticleGFPart.hpp:475-495) and the
 * frequency loop of TwoParticleGF::compute (TwoParticleGF.cpp:123-204).
 * ------------------------------------------------------------------------ */

/* One block chain <S1|O1|S2><S2|O2|S3><S3|O3|S4><S4|CX4|S1>: the operator ids
 * in chain order (O1, O2, O3, CX4), the blocks S1..S4, the permutation of the
 * frequencies {z1, z2, -z3} that the chain uses and its sign. */
typedef struct pgx_g2_part {
    int32_t op[4];
    int32_t block[4];
    int32_t perm[3];
    int32_t sign;
} pgx_g2_part;

/* out[t] = sum over parts of the Lehmann sum at triple t = (z1, z2, z3)
 * (z: 3*nfreq complex; out: nfreq complex).  Resonant terms use the delta
 * rule |D| <= pole_res.  flags: PGX_G2_EXACT or PGX_G2_REFERENCE_RULE. */
int pgx_g2(pgx_ctx* ctx, int32_t nparts, const pgx_g2_part* parts, int32_t nfreq, const double* z,
           double pole_res, double coef_tol, int32_t flags, double* out);

/* Device workspace limits of pgx_g2's anchored form (0 keeps a default).
 * batch_bytes: parts are evaluated together while their workspaces fit in it
 * (default 3 GiB).  chain_bytes: the most one part may take (default half the
 * free device memory, at most 48 GiB); a part that needs more at the call's
 * frequency count is evaluated in tiles of the (z1, z3) plane, each with all
 * of its triples' z2.  Results do not depend on either limit beyond the
 * summation order. */
int pgx_set_g2_workspace(pgx_ctx* ctx, int64_t batch_bytes, int64_t chain_bytes);

/* With PGX_G2_SPLIT_I8: products of at least min_macs complex multiply-adds
 * run on the int8 tensor cores, smaller ones on the FP64 tiles (default 1e9;
 * 0 sends every stacked and anchored product to the tensor cores). */
int pgx_set_g2_split_threshold(pgx_ctx* ctx, double min_macs);

/* With PGX_G2_SPLIT_I8: digits per operand element, 1..8 (default 6), each a
 * signed byte of a balanced base-254 expansion (7.99 bits).  The products keep
 * the digit pairs a + b < slices; the error left is below about
 * (slices + 1) * 254^(-slices) * K of |A|max |B|max per element (2^-37.4 K at
 * 5 digits, 2^-45.1 K at 6), with no counterpart in the reference, which
 * computes in FP64 only. */
int pgx_set_g2_split_slices(pgx_ctx* ctx, int32_t slices);

/* With PGX_G2_SPLIT_I8: digits per product from its anchor states' weights
 * (no counterpart in the reference).  A product's error reaches G2 multiplied
 * by the Boltzmann weights of its anchor block, so a block whose largest
 * weight is below the overall largest by budget x 254^k or more runs its
 * products with k fewer digits (at least 3): none then carries more than
 * `budget` times the G2 error of a full-digit product of the dominant block.
 * Default 4; budget <= 0 gives every product `slices` digits. */
int pgx_set_g2_split_weight_budget(pgx_ctx* ctx, double budget);

/* Tile shape of the int8 split products (no counterpart in the reference):
 * 0 (default) runs 128 x 256 tiles on single CTAs, 1 runs 256 x 256 tiles on
 * pairs of CTAs (tcgen05 cta_group::2, each SM loading half of the tile's
 * operands).  Results are identical; on the 8-site ring's products the single
 * CTAs measured 4-7% faster. */
int pgx_set_split_cta_pair(pgx_ctx* ctx, int32_t cta_pair);

/* Self-check of the int8 split product (no counterpart in the reference):
 * C = A B for nb items of seeded random complex A (M x K) and B (K x N) with
 * entries spread over four binary orders of magnitude, once through the split
 * scheme with `slices` slices and once through the FP64 product.  Returns
 * max|C_split - C_fp64| / max|C_fp64| and the device time of each (ms). */
int pgx_split_gemm_check(pgx_ctx* ctx, int32_t M, int32_t N, int32_t K, int32_t nb, int32_t slices, uint64_t seed,
                         double* max_rel_err, double* ms_split, double* ms_fp64);

/* Number of state quadruples the reference enumerates for these parts
 * (TwoParticleGFPart.cpp:210-250): all four rotated elements |x| > nz_tol and
 * w1 + w2 + w3 + w4 > coef_tol.  The work unit of the G2 throughput metric. */
int pgx_g2_count(pgx_ctx* ctx, int32_t nparts, const pgx_g2_part* parts, double coef_tol, double nz_tol,
                 long long* count);

/* ------------------------------------------------------------------------
 * GEMM tile-class autotuning (no counterpart in the reference).  Every
 * batched product of the library runs in one of nine tile classes; by default
 * the class is the one that pads the product least.  Between
 * pgx_autotune_begin and pgx_autotune_end (run the workload once in between)
 * each batch of products a call launches is first timed under the padding
 * rule and in every class valid for its (M, N) size bucket, outputs
 * redirected to scratch, before its real launch; results are unchanged and
 * those calls are slower.  pgx_autotune_end installs per operand-type
 * combination and bucket the candidate with the least total time.  Later
 * calls on the context use it.  changed (may be NULL) receives the number of
 * buckets that left the padding rule.
 * ------------------------------------------------------------------------ */
int pgx_autotune_begin(pgx_ctx* ctx);
int pgx_autotune_end(pgx_ctx* ctx, int32_t* changed);

/* ------------------------------------------------------------------------
 * CUDA graphs of captured sequences (the reference has no device work to
 * capture).  Between pgx_graph_begin and pgx_graph_end the context's stream
 * is captured instead of run: pgx_eigh (real blocks; after one uncaptured
 * call, which sizes every buffer) and pgx_op_rotate record their device work
 * into the graph, and every other entry point returns PGX_ERR_STATE.  Host
 * data they upload is staged in memory the graph keeps.  pgx_graph_replay
 * runs the graph on the context's current inputs (e.g. new block
 * Hamiltonians from pgx_set_hamiltonian), waits for it, checks the
 * eigensolver status and marks the eigensystem and the rotated operators
 * valid, as the captured calls would.  A graph refuses to replay once any
 * device buffer of the process was allocated or freed, pgx_set_blocks ran,
 * or an operator was defined, formed or released after its capture.
 * ------------------------------------------------------------------------ */
int pgx_graph_begin(pgx_ctx* ctx);
int pgx_graph_end(pgx_ctx* ctx, int32_t* graph_id);
int pgx_graph_replay(pgx_ctx* ctx, int32_t graph_id);
int pgx_graph_destroy(pgx_ctx* ctx, int32_t graph_id);

/* ------------------------------------------------------------------------
 * Batches of independent models.
 * The reference holds one model per set of objects; for many impurity models
 * at once (the 64-model batch workload) a context may hold the blocks of
 * several models, diagonalised by one pgx_eigh, each model weighted at its
 * own inverse temperature and its pair sums evaluated at its own frequencies.
 * Per model this is DensityMatrix::compute (DensityMatrix.cpp:38-58) and
 * GreensFunctionPart / SusceptibilityPart (GreensFunctionPart.cpp:65-110,
 * SusceptibilityPart.cpp:76-127) as pgx_weights, pgx_gf and pgx_susc do.
 * ------------------------------------------------------------------------ */

/* Blocks first_block[m] .. first_block[m+1]-1 (first_block[0] = 0,
 * first_block[nmodels] = the number of blocks) form model m, at inverse
 * temperature beta[m].  Call after pgx_set_blocks (which forgets models). */
int pgx_set_models(pgx_ctx* ctx, int32_t nmodels, const int32_t* first_block, const double* beta);

/* Weights of every model on its own states: E0_m = min E, w = exp(-beta_m
 * (E - E0_m)) / Z_m.  w (sum of dims), E0 and Z (nmodels each) are copied out
 * when non-NULL.  pgx_g2, pgx_chi3 and pgx_gf_vjp need the weights of a
 * single model (pgx_weights) and refuse these. */
int pgx_weights_models(pgx_ctx* ctx, double* w, double* E0, double* Z);

/* pgx_gf / pgx_susc for every model at once: a part belongs to the model of
 * its blocks; z holds nz frequencies per model (nmodels x nz complex,
 * model-major) and out the values (same layout); zero_pole (nmodels complex,
 * or NULL) the zero-pole sums of each model.  The susceptibility's beta is
 * each model's own. */
int pgx_gf_models(pgx_ctx* ctx, int32_t op1, int32_t op2, int32_t nparts, const int32_t* outer, const int32_t* inner,
                  int32_t nz, const double* z, double coef_tol, double* out);
int pgx_susc_models(pgx_ctx* ctx, int32_t opA, int32_t opB, int32_t nparts, const int32_t* outer,
                    const int32_t* inner, int32_t nz, const double* z, double pole_res, double coef_tol, double* out,
                    double* zero_pole);

/* ------------------------------------------------------------------------
 * K6 Three-point fermion-boson susceptibility.
 * Replaces: ThreePointSusceptibility::compute / operator() and
 * ThreePointSusceptibilityPart::computeImpl, addMultiterm and the term
 * evaluation (ThreePointSusceptibility.cpp:144-230,
 * ThreePointSusceptibilityPart.cpp:243-357, ThreePointSusceptibilityPart.hpp:516-538).
 * ------------------------------------------------------------------------ */

#define PGX_PP 0  /* channels, as the reference's Channel enum (Misc.hpp:160-164) */
#define PGX_PH 1
#define PGX_XPH 2

/* One part <i|F1|j><j|F2|k><k|B1|m><m|B2|i> of ThreePointSusceptibility::prepare
 * (ThreePointSusceptibility.cpp:77-134): f1, f2 are the part's first and
 * second fermionic operators (already exchanged when swapped != 0), b1, b2
 * the factors of the quadratic operator; block = {i, j, k, m}. */
typedef struct pgx_chi3_part {
    int32_t f1, f2, b1, b2;
    int32_t block[4];
    int32_t swapped;
} pgx_chi3_part;

/* out[t] = sum over parts of the three-point susceptibility at the duplet
 * t = (z1, z2) (z: 2*nfreq complex; out: nfreq complex), summed over every
 * state triple without the reference's coefficient filter and pole merge.
 * The term type of a triple is chosen by |E_i - E_k| <= pole_res and the
 * resonant delta by |z1 - xi z2| <= pole_res (xi = -1 for PP, 1 otherwise),
 * as in the reference.  Needs pgx_weights (beta) first. */
int pgx_chi3(pgx_ctx* ctx, int32_t channel, int32_t nparts, const pgx_chi3_part* parts, int32_t nfreq,
             const double* z, double pole_res, double* out);

/* ------------------------------------------------------------------------
 * Allocation-free eigensolve (no counterpart in the reference).
 * For callers whose device memory belongs to an outer allocator (an
 * application's caching pool or a fixed arena) and which must not let a
 * library call cudaMalloc/cudaFree: diagonalises ONE real symmetric block of
 * size n <= PGX_NOALLOC_MAX_DIM on buffers the caller owns, keeping its
 * workspace in a static device array of the library (about 3 MiB per GPU,
 * held until the process exits).  H (n*n, row-major, read only), E (n) and U
 * (n*n, row-major, eigenvectors as columns, ascending eigenvalues) are DEVICE
 * pointers; stream is a cudaStream_t (NULL: default stream).  The call waits
 * for the stream before returning.  Larger n returns PGX_ERR_ARG.  All calls
 * on a device share the workspace: calls that overlap on the GPU race and
 * must be serialised by the caller.  The first call on a device looks up the
 * workspace's address and should come before any stream capture.
 * ------------------------------------------------------------------------ */
#define PGX_NOALLOC_MAX_DIM 256
int pgx_eigh_noalloc(const double* H, int32_t n, double* E, double* U, void* stream);

/* Device-side timing of everything the context issues between the two
 * calls (CUDA events on the context's stream). */
int pgx_timer_begin(pgx_ctx* ctx);
int pgx_timer_end(pgx_ctx* ctx, double* ms);

/* Number of kernels this library has launched in this process. */
long long pgx_launch_count(void);

/* Device time (ms) of the last pgx_g2 call and its dominant GEMM stage. */
int pgx_g2_last_timing(pgx_ctx* ctx, double* total_ms, double* gemm_ms, double* gemm_flops);

/* Numerics check of the device reciprocal used in the Lehmann kernels
 * (Newton-Raphson from a single-precision seed): out[i] = 1/x[i] for x[i] > 0,
 * host arrays, computed on the current device. */
int pgx_recip_check(const double* x, int32_t n, double* out);

/* Per-kernel profile of everything the context launches between the two
 * calls: CUDA event pairs on the launching stream around each instrumented
 * kernel, aggregated by kernel name and sorted by total time (largest first).
 * flops and bytes are the kernel's ALGORITHMIC floating-point operations and
 * DRAM bytes (minimum traffic) summed over its launches, 0 where not stated.
 * pgx_profile_end waits for the stream and returns the number of kernels. */
int pgx_profile_begin(pgx_ctx* ctx);
int pgx_profile_end(pgx_ctx* ctx, int32_t* nkernels);
int pgx_profile_kernel(pgx_ctx* ctx, int32_t i, char* name, int32_t name_cap, int32_t* launches, double* ms,
                       double* flops, double* bytes);

#ifdef __cplusplus
}
#endif

#endif /* PGX_H */
