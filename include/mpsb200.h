/*
 * mpsb200.h -- C ABI of the B200 (sm_100a) MPS two-site update library
 * (libmpsb200.so).
 *
 * Plain C: pointers, sizes, enums.  Every pointer marked "device" is CUDA
 * device memory owned by the caller; the library never allocates or frees
 * caller memory and keeps no per-call global state.  Every call is
 * stream-ordered and asynchronous on the given stream (no host sync inside)
 * unless its comment says otherwise.  Return value: MPSB_OK (0) or a negative
 * MPSB_E* code; mpsb_last_error() then holds a message for this host thread.
 * Numerical faults of individual pairs (no Jacobi convergence, non-finite
 * theta, bad bond dimensions) are reported per pair in `status`.
 *
 * Reference interfaces replaced (paths within nasir26/fpga-mps-simulator):
 *   mps_core.py:326-350   MPSState._apply_adjacent_2q  (contract -> gate -> SVD -> split)
 *   mps_core.py:277-300   MPSState._svd_truncate       (keep rule, renormalise, norm_log)
 *   fpga_mps_simulator.cpp:287-371 contract_and_apply_2q (the FPGA-offloaded contraction)
 *   fpga_mps_simulator.cpp:392-404 fpga_mps_simulator   (the FPGA kernel entry point)
 *   fpga_mps_simulator.py:566-635  2-qubit branch of _run_circuit_fpga (launch + host SVD)
 */
#ifndef MPSB200_H
#define MPSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MPSB_API __attribute__((visibility("default")))
#else
#define MPSB_API
#endif

struct CUstream_st;
typedef struct CUstream_st *mpsb_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* complex128, interleaved (re, im) -- the layout of numpy/torch complex128. */
typedef struct { double re, im; } mpsb_c128;

/* Largest bond dimension the kernels support (theta is at most 128 x 128). */
#define MPSB_CHI_LIMIT 64

/* One MPS chain resident in device memory (the state of mps_core.py:172-195).
 * Site k is stored C-order as (bonds[k], 2, bonds[k+1]) complex128 at the
 * start of its slot: sites + k * slot_elems.  bonds[0] = bonds[n] = 1.      */
typedef struct {
    mpsb_c128 *sites;      /* device: n * slot_elems complex128                  */
    int32_t   *bonds;      /* device: n + 1 bond dimensions                      */
    double    *norm_log;   /* device: one double, accumulated log-norm           */
    int32_t   *status_acc; /* device: OR of every pair status of this chain, or NULL */
    int64_t    slot_elems; /* complex elements per slot, >= 2 * chi_cap^2 of every
                              launch that touches the chain                        */
    int32_t    n;          /* number of sites                                    */
    int32_t    chi_max;    /* truncation cap (>= 1; mps_core's default is 256).  No
                              bond above MPSB_CHI_LIMIT is ever formed: a pair whose
                              rule would keep more keeps MPSB_CHI_LIMIT values and
                              reports MPSB_ST_CHI_LIMIT.  The launch's chi_cap must
                              cover min(chi_max, MPSB_CHI_LIMIT, 2^(n/2)).          */
    double     cutoff;     /* relative singular-value cutoff (svd_cutoff)       */
} mpsb_chain;

/* One two-site update: gate `gate` on sites (site, site + 1) of chain `chain`.
 * Pairs of one call must be disjoint, and all pairs of one chain must be
 * contiguous in the array (norm_log is folded per contiguous run, in order). */
typedef struct {
    int32_t chain;  /* index into the chain table                          */
    int32_t site;   /* left site i of the pair (i, i + 1)                   */
    int32_t gate;   /* index into the gate array (16 complex128, row-major) */
    int32_t out;    /* row of this pair in status / kept / trunc / spectra  */
} mpsb_pair;

/* One two-site update of a dependency-ordered work list (mpsb_update2q_flow):
 * the fields of mpsb_pair, then the list indices of the two items it must
 * wait for -- the last earlier items touching site `site` and site `site + 1`
 * of the same chain -- or -1 where there is none.  dep0, dep1 < own index. */
typedef struct {
    int32_t chain, site, gate, out;
    int32_t dep0, dep1;
} mpsb_flow_item;

/* One single-site gate: 2x2 gate `gate` on site `site` of chain `chain`. */
typedef struct {
    int32_t chain;
    int32_t site;
    int32_t gate;   /* index into the gate array (4 complex128, row-major) */
    int32_t pad;
} mpsb_site_op;

enum mpsb_precision {
    MPSB_FP64 = 0,        /* complex128 end to end (the drop-in form)                    */
    MPSB_MIXED_TF32X3 = 1 /* theta by 3xTF32 complex-3M tensor-core GEMMs (tcgen05), FP64
                             Jacobi SVD; singular values below 1e-6 S[0] (theta's rounding
                             floor) are never kept, whatever the cutoff.  At chi_cap <= 32
                             the contraction runs in FP64 (exact, no floor): the 128-row
                             tensor-core tile would be half padding or more, and the form
                             then differs from MPSB_FP64 only by its Jacobi tolerance
                             (1e-9 against 1e-14)                                        */,
    MPSB_TF32X3_ALL = 2   /* the 3xTF32 tensor-core theta at EVERY bond cap (M = 64 MMA
                             tiles at chi_cap <= 32, M = 128 above), FP64 Jacobi SVD, the
                             same 1e-6 S[0] floor and 1e-9 Jacobi tolerance as
                             MPSB_MIXED_TF32X3                                           */
};

enum mpsb_status_bits {
    MPSB_ST_OK = 0,
    MPSB_ST_NOCONV = 1,    /* Jacobi hit max_sweeps; result written anyway */
    MPSB_ST_NONFINITE = 2, /* theta held NaN or Inf                         */
    MPSB_ST_BADDIM = 4,    /* bond dimensions out of range; pair skipped    */
    MPSB_ST_TIMEOUT = 8,   /* a bounded wait gave up; result invalid             */
    MPSB_ST_CHI_LIMIT = 16 /* the keep rule asked for more than MPSB_CHI_LIMIT values
                              (chi_max above the limit): MPSB_CHI_LIMIT were kept, so
                              the state differs from mps_core's from here on        */
};

enum mpsb_error {
    MPSB_OK = 0,
    MPSB_EINVAL = -1,     /* bad argument (message in mpsb_last_error)  */
    MPSB_ELAUNCH = -2,    /* CUDA launch / runtime error                */
    MPSB_EWORKSPACE = -3, /* workspace too small                        */
    MPSB_ENODEV = -4      /* no sm_100 device current                   */
};

/* Library version string and the last error message of the calling thread. */
MPSB_API const char *mpsb_version(void);
MPSB_API const char *mpsb_last_error(void);

/* Bytes of device workspace mpsb_update2q_batch needs for `npairs` pairs
 * whose bond dimensions never exceed chi_cap. */
MPSB_API size_t mpsb_update2q_workspace_bytes(int npairs, int chi_cap);

/* Batched two-site update (mps_core.py:326-350 + :277-300 for every pair).
 * For each pair: theta = G . (A_i x A_{i+1}), M = theta as (2 chi_l) x (2 chi_r),
 * truncated SVD with keep = clip(#(S > cutoff*S[0]), 1, chi_max), norm_log
 * += 0.5 log(1 - dropped/total) when truncating, kept S renormalised to unit
 * 2-norm (norm_log += log norm when norm > 1e-15), sites i and i+1 replaced by
 * U sqrt(S) and sqrt(S) Vh in place, bonds[i+1] = keep.
 *   chains, pairs, gates: device.  chi_cap: largest bond of any chain touched.
 *   tol: Jacobi off-diagonal tolerance (<= 0 picks the form's default): a column
 *        pair rotates when |x^H y|^2 > tol^2 |x|^2 |y|^2; the sweeps end after a
 *        sweep in which no pair had |x^H y|^2 > 2 tol |x|^2 |y|^2 and no pair
 *        whose squared norms lie within 1 % of each other rotated at all.
 *   max_sweeps: Jacobi sweep bound (<= 0 picks 40).
 *   spectra (nullable): npairs_out x 128 doubles, full descending spectrum.
 *   kept, trunc (nullable): kept count and discarded weight dropped/total.
 *   status (required): per-pair MPSB_ST_* bits.
 * Replaces fpga_mps_simulator.py:566-635 (launch, read theta, host SVD, write back). */
MPSB_API int mpsb_update2q_batch(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs,
                        const mpsb_c128 *gates, int precision, int chi_cap,
                        double tol, int max_sweeps,
                        void *workspace, size_t workspace_bytes,
                        double *spectra, int32_t *kept, double *trunc, int32_t *status,
                        mpsb_stream_t stream);

/* Allocation-free form of mpsb_update2q_batch.  No counterpart in the
 * reference.  For callers that cannot allocate device memory -- a host that
 * hands the library only buffers registered up front, or a loop in which a
 * cudaMalloc would synchronise the device -- this entry takes the same inputs
 * and outputs but no workspace: its scratch is a fixed device array of
 * MPSB_NOALLOC_SCRATCH_BYTES (16 MiB: 63 pairs at chi_cap = 64, more at smaller
 * chi_cap) that every GPU loading the library holds until exit.  Batches that
 * need more scratch are rejected with MPSB_EWORKSPACE before any launch.  The
 * first call on a device looks up the array's device address (set-up), so
 * make that first call before any stream capture; the address is kept for the
 * life of the process, so do not use this entry across a cudaDeviceReset
 * of that device.  All calls share the
 * array: calls whose kernels overlap on the GPU race, serialise them on one
 * stream.  It allocates nothing (no cudaMalloc, no cudaFree). */
#define MPSB_NOALLOC_SCRATCH_BYTES (16u << 20)
MPSB_API int mpsb_update2q_batch_noalloc(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs,
                                         const mpsb_c128 *gates, int precision, int chi_cap,
                                         double tol, int max_sweeps,
                                         double *spectra, int32_t *kept, double *trunc, int32_t *status,
                                         mpsb_stream_t stream);

/* Persistent dataflow form of mpsb_update2q_batch: many layers of many
 * chains in ONE launch.  A grid of `nclusters` resident two-CTA clusters
 * claims the items in list order; an item starts as soon as its dep0 / dep1
 * items have finished (bounded waits: after poll_limit polls the item is
 * skipped, its sites unchanged, with MPSB_ST_TIMEOUT), so a pair of layer
 * L + 1 runs while unrelated pairs of layer L are still in flight.  Every
 * item computes exactly what mpsb_update2q_batch computes for it (same
 * per-pair code): sites, bonds, spectra, kept counts and statuses are
 * bit-identical to launching the layers one by one.
 *   items: device, nitems, in topological order (each dep < its own index).
 *   chain_order, chain_offsets: device; chain c's items, in the order they
 *     apply, are chain_order[chain_offsets[c] .. chain_offsets[c+1]); norm_log
 *     is folded per chain in that order (as per-layer launches fold it).
 *   threads: CTA size (0 = default; 64 or 128 at chi_cap <= 16, 128 or 256
 *     at chi_cap <= 32, 256 above) -- the shape the autotuner chooses.
 *   nclusters: grid size (<= 0 = every cluster that fits on the current device).
 *   poll_limit: polls per dependency wait before giving up (< 0 = 2^24).
 *   workspace: mpsb_update2q_flow_workspace_bytes(nitems, chi_cap, precision,
 *     threads, nclusters) bytes, 256-byte aligned.
 * Launches two memsets, the persistent kernel and a fold kernel.  No reference
 * counterpart: replaces the host loop over gates of fpga_mps_simulator.py:566-635
 * (one launch and one host round trip per gate). */
MPSB_API size_t mpsb_update2q_flow_workspace_bytes(int nitems, int chi_cap, int precision, int threads,
                                                   int nclusters);
MPSB_API int mpsb_update2q_flow_clusters(int chi_cap, int precision, int threads);
MPSB_API int mpsb_update2q_flow(const mpsb_chain *chains, int nchains, const mpsb_flow_item *items, int nitems,
                                const int32_t *chain_order, const int32_t *chain_offsets,
                                const mpsb_c128 *gates, int precision, int chi_cap, double tol, int max_sweeps,
                                int threads, int nclusters, int poll_limit,
                                void *workspace, size_t workspace_bytes,
                                double *spectra, int32_t *kept, double *trunc, int32_t *status,
                                mpsb_stream_t stream);

/* Contraction only: theta = G (A B) of each pair, without the SVD -- the work
 * of the reference's FPGA offload (contract_and_apply_2q,
 * fpga_mps_simulator.cpp:287-371, opcode 100 of its instruction stream) whose
 * result the host reads back as the (2 chi_l) x (2 chi_r) matrix
 * theta[a][s][d] for its own SVD (fpga_mps_simulator.py:597-600).
 *   theta:  device, complex128; pair k's matrix, row-major with leading
 *           dimension 2 * chi_r, starts at theta + pairs[k].out * (2 chi_cap)^2.
 *   status: device int32 per pairs[k].out: MPSB_ST_BADDIM, MPSB_ST_NONFINITE,
 *           MPSB_ST_TIMEOUT (cleared by the call).
 * precision: the contraction the update of that precision runs at this
 * chi_cap (FP64; 3xTF32 tensor cores for MPSB_MIXED_TF32X3 above chi_cap 32
 * and for MPSB_TF32X3_ALL), so an FP64 theta is bitwise the matrix
 * mpsb_update2q_batch factorises.  Gates are complex128 (the FPGA driver
 * rounds them to float32 first; mps_core does not).  Sites are only read, so
 * pairs may overlap; their `out` rows must be distinct.  Stream-ordered, no
 * host synchronisation. */
MPSB_API int mpsb_contract2q_batch(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs,
                                   const mpsb_c128 *gates, int precision, int chi_cap, mpsb_c128 *theta,
                                   int32_t *status, mpsb_stream_t stream);

/* Batched single-site gates, A'[l,s',r] = sum_s G[s',s] A[l,s,r], in place
 * (mps_core.py:267-273; fpga_mps_simulator.cpp:232-276 apply_1q_gate).
 * Ops of one call must touch distinct sites. */
MPSB_API int mpsb_apply1q_batch(const mpsb_chain *chains, const mpsb_site_op *ops, int nops,
                       const mpsb_c128 *gates, int chi_cap, mpsb_stream_t stream);

/* Dense statevector of one chain (n <= 24) in Qiskit order, including
 * exp(norm_log) (mps_core.py:433-461).  chain_dev: device pointer to the
 * chain.  out: device, 2^n complex128.  scratch: device, 2 * 2^n complex128.
 * Launches n + 1 kernels. */
MPSB_API int mpsb_statevector(const mpsb_chain *chain_dev, int n, int chi_cap, mpsb_c128 *out,
                     mpsb_c128 *scratch, size_t scratch_bytes, mpsb_stream_t stream);

/* Amplitudes <b|psi> of `nbits` basis states of chain `chain` (b given as
 * n bytes per state, byte k = value of qubit k), including exp(norm_log)
 * (the convention of mps_core.py:433-461).  out: device complex128 per state;
 * log_abs (nullable): log|amplitude| for chains where the value underflows. */
MPSB_API int mpsb_amplitude(const mpsb_chain *chains, int chain, int n, const uint8_t *bits, int nbits,
                   int chi_cap, mpsb_c128 *out, double *log_abs, mpsb_stream_t stream);

/* Bytes of device scratch mpsb_expect_local needs for chains of n sites. */
MPSB_API size_t mpsb_expect_workspace_bytes(int nchains, int n, int chi_cap);

/* Normalised local expectation values <psi|O|psi>/<psi|psi> for `nterms`
 * terms per chain, chains 0 .. nchains-1 of the table (all of length n).
 * Term t acts with ops[2*t] on site sites[t] and, if two_site[t] != 0, with
 * ops[2*t+1] on site sites[t]+1 (ops: device, 2x2 complex128 each).
 * out: device, nchains x nterms doubles.  No reference counterpart: the
 * semantics follow _pauli_expectation_sv (fpga_mps_simulator.py:1091-1108)
 * applied to the statevector of mps_core.py:433-461, normalised. */
MPSB_API int mpsb_expect_local(const mpsb_chain *chains, int nchains, int n, int chi_cap,
                      const int32_t *sites, const int32_t *two_site, const mpsb_c128 *ops,
                      int nterms, double *out, void *workspace, size_t workspace_bytes,
                      mpsb_stream_t stream);

/* Overlap <a|b> of two chains of n sites (both device pointers), returned
 * as out * exp(out_log) with the norm_log of both chains included, so that
 * <a|b> matches the inner product of the two get_statevector() vectors
 * (mps_core.py:433-461 convention).  workspace: 2 * chi_cap^2 complex128.
 * No reference counterpart: used to report the state infidelity of the
 * mixed-precision form against the FP64 form. */
MPSB_API int mpsb_overlap(const mpsb_chain *a, const mpsb_chain *b, int n, int chi_cap, mpsb_c128 *out,
                          double *out_log, void *workspace, size_t workspace_bytes, mpsb_stream_t stream);

/* ---------------------------------------------------------------- measurement */

/* Bytes of device workspace mpsb_sample needs (right environments). */
MPSB_API size_t mpsb_sample_workspace_bytes(int n, int chi_cap);

/* Conditional shot sampling of chain `chain` (n sites), replacing
 * MPSState.sample (mps_core.py:354-419): right environments, then per shot
 * a left-to-right sweep drawing each site's outcome.  uniforms: device,
 * shots x n doubles in [0, 1), one per (shot, site) in that order; site i of
 * shot k is 1 exactly when uniforms[k*n+i] >= p0 / (p0 + p1), the rule by
 * which numpy's Generator.choice(2, p) (the reference's draw) maps its one
 * uniform to an outcome, so the uniforms of the same seeded generator give
 * the reference's shots.  bits: device, shots x n bytes (byte i = site i). */
MPSB_API int mpsb_sample(const mpsb_chain *chains, int chain, int n, int chi_cap, const double *uniforms,
                         int shots, uint8_t *bits, void *workspace, size_t workspace_bytes,
                         mpsb_stream_t stream);

/* Site reset of _run_circuit_fpga (fpga_mps_simulator.py:530-552) for a batch
 * of distinct sites: zero the sigma = 1 half, divide by the remaining
 * Frobenius norm when it exceeds 1e-15, else set the tensor to zeros with a
 * 1 at [0, 0, 0].  ops: device (the gate field is ignored). */
MPSB_API int mpsb_reset_batch(const mpsb_chain *chains, const mpsb_site_op *ops, int nops, int chi_cap,
                              mpsb_stream_t stream);

/* Bytes of device workspace mpsb_canonicalize needs for nchains chains. */
MPSB_API size_t mpsb_canonicalize_workspace_bytes(int nchains, int chi_cap);

/* Canonical-form sweeps on chains chain_ids[0 .. nchains-1] (device array),
 * one CTA per chain.  direction 0: left_normalize_site(i) for i = lo .. hi
 * (mps_core.py:221-235: QR of site i as (2 chi_l) x chi_r, Q stays, R is
 * absorbed into site i+1); direction 1: right_normalize_site(i) for
 * i = hi .. lo (mps_core.py:237-252: LQ, L absorbed into site i-1).  The QR
 * follows LAPACK zgeqr2 / zung2r (the routines numpy.linalg.qr calls), so on
 * the same input the sites agree with the reference's to rounding.  Bonds are
 * updated on the device (k = min(rows, cols) of each QR). */
MPSB_API int mpsb_canonicalize(const mpsb_chain *chains, const int32_t *chain_ids, int nchains, int lo, int hi,
                               int direction, int chi_cap, void *workspace, size_t workspace_bytes,
                               mpsb_stream_t stream);

/* ---------------------------------------------------------------- adjoint
 * No reference counterpart: the reference engine has no gradients.  These
 * entries differentiate exactly what mpsb_update2q_batch and
 * mpsb_apply1q_batch compute, for a real loss L, with the cotangent of a
 * complex array z taken as z_bar = dL/dRe z + i dL/dIm z.  Cotangents live in
 * a second chain table `cot` whose sites array has the same slot layout as
 * the state's (only its sites and slot_elems fields are read); the shapes
 * come from the bonds of the `pre` table, the state before the op. */

/* Bytes of tape mpsb_update2q_batch_taped writes for npairs pairs (theta or
 * theta^H as factorised, one side's singular vectors times S -- the left
 * side, or the right side with a flag for pairs the QR preconditioner
 * handled -- and the spectrum). */
MPSB_API size_t mpsb_update2q_tape_bytes(int npairs, int chi_cap);

/* mpsb_update2q_batch that also records the tape of every pair (pair q at
 * q * mpsb_update2q_tape_bytes(1, chi_cap)).  The sites, bonds, norm_log and
 * outputs are bit-identical to mpsb_update2q_batch's. */
MPSB_API int mpsb_update2q_batch_taped(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs,
                                       const mpsb_c128 *gates, int precision, int chi_cap,
                                       double tol, int max_sweeps,
                                       void *workspace, size_t workspace_bytes,
                                       void *tape, size_t tape_bytes,
                                       double *spectra, int32_t *kept, double *trunc, int32_t *status,
                                       mpsb_stream_t stream);

/* Bytes of device workspace mpsb_update2q_backward_batch needs (256-byte
 * aligned; each pair's dead scratch is dropped from L2 unwritten): one scratch
 * region of 8 (2 chi_cap)^2 complex per CTA, min(npairs, CTAs resident on the
 * current device).  Call with the device of the launch current. */
MPSB_API size_t mpsb_update2q_backward_workspace_bytes(int npairs, int chi_cap);

/* Backward of one taped call: for every pair, the cotangents of the updated
 * sites (slots i and i+1 of `cot`, shapes (chi_l, 2, keep) and (keep, 2, chi_r))
 * are replaced in place by the cotangents of the sites before the update
 * (shapes (chi_l, 2, chi_m) and (chi_m, 2, chi_r)).  `pre` must hold the
 * sites and bonds the taped call started from.  The truncated-SVD backward
 * includes the kept/discarded coupling terms with Lorentzian-broadened
 * 1/(s_j^2 - s_i^2) (width 1e-12 s_0^2); discarded triplets below 1e-6 times
 * the smallest kept value are treated as an exact null space.
 * gate_grads (nullable): 16 complex128 per pair (row `out`), dL/dG.
 * status: per-pair bits (BADDIM: tape and bonds disagree). */
MPSB_API int mpsb_update2q_backward_batch(const mpsb_chain *pre, const mpsb_chain *cot, const mpsb_pair *pairs,
                                          int npairs, const mpsb_c128 *gates, int chi_cap,
                                          const void *tape, size_t tape_bytes, mpsb_c128 *gate_grads,
                                          void *workspace, size_t workspace_bytes, int32_t *status,
                                          mpsb_stream_t stream);

/* Backward of mpsb_apply1q_batch: cot site <- G^H cot site in place, and
 * (gate_grads nullable) 4 complex128 per op: dL/dG = sum cot' A^H. */
MPSB_API int mpsb_apply1q_backward_batch(const mpsb_chain *pre, const mpsb_chain *cot, const mpsb_site_op *ops,
                                         int nops, const mpsb_c128 *gates, int chi_cap, mpsb_c128 *gate_grads,
                                         mpsb_stream_t stream);

/* Bytes of device workspace mpsb_mpo_energy_grad needs. */
MPSB_API size_t mpsb_mpo_grad_workspace_bytes(int nchains, int n, int chi_cap, int mpo_bond);

/* Loss L_c = <psi_c|H|psi_c> / <psi_c|psi_c> of chains 0 .. nchains-1 (all of
 * n sites) for a matrix-product operator H, and the cotangent of every site,
 * weights[c] * 2 (H_eff A - L_c N_eff A) / <psi_c|psi_c>, written into `cot`.
 * mpo: device, n * D * D * 4 complex128, W[k][a][b] a 2x2 operator (row-major,
 * acting as |s><t| at [s][t]); state D-1 is the left boundary and state 0 the
 * right one, with W[k][D-1][D-1] = W[k][0][0] = identity and no transition
 * out of state 0 or into state D-1 (lower-triangular form).
 * weights (nullable = all ones), loss (nullable): device, nchains doubles. */
MPSB_API int mpsb_mpo_energy_grad(const mpsb_chain *chains, int nchains, int n, int chi_cap,
                                  const mpsb_c128 *mpo, int mpo_bond, const double *weights, double *loss,
                                  const mpsb_chain *cot, void *workspace, size_t workspace_bytes,
                                  mpsb_stream_t stream);

/* FP64 FMA throughput probe: `blocks` x `threads` threads each run eight
 * independent FMA chains of `iters` steps (16 * iters flops per thread).
 * The caller times the launch on `stream` to state the FP64 roofline.
 * sink: device, one double (written only to keep the chains live). */
MPSB_API int mpsb_fp64_probe(int64_t iters, int blocks, int threads, double *sink, mpsb_stream_t stream);

/* Dense TF32 tensor-core throughput probe (tcgen05.mma kind::tf32): `blocks`
 * CTAs, one per SM, each issue `iters` (1 .. 65536) M = 128, N = 256, K = 8
 * MMAs into one TMEM accumulator (2 * 128 * 256 * 8 * iters flops per CTA).
 * The caller times the launch on `stream` to state the tensor roofline of
 * the 3xTF32 contraction.  sink: device, `blocks` doubles (an accumulator
 * value, or -1 where the completion wait gave up). */
MPSB_API int mpsb_tf32_probe(int64_t iters, int blocks, double *sink, mpsb_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MPSB200_H */
