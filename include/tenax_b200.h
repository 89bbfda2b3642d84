/*
 * tenax_b200.h -- C ABI of the B200 block-sparse symmetric contraction library.
 *
 * The reference (tenax, pure Python/JAX) has no native boundary; these entry
 * points are the custom calls its Python layer binds (ctypes here, XLA FFI or
 * a torch extension elsewhere).  Each function names the reference function
 * whose behaviour it reproduces.  All entry points return an int status
 * (TNX_OK on success); no C++ exception crosses this boundary.  Device
 * pointers are caller-owned unless stated; `stream` is a cudaStream_t passed
 * as void*.  Block buffers hold one tensor's blocks contiguously, row-major,
 * in the order of the key list given to the planner (the Python layer uses
 * sorted-key order = tenax's pytree leaf order, core/tensor.py:572-578).
 */
#ifndef TENAX_B200_H
#define TENAX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; the Python layer maps them to the reference's exceptions */
enum {
  TNX_OK = 0,
  TNX_ERR_VALUE = 1,       /* ValueError   */
  TNX_ERR_TYPE = 2,        /* TypeError    */
  TNX_ERR_RUNTIME = 3,     /* RuntimeError */
  TNX_ERR_CUDA = 4,        /* CUDA API or launch failure */
  TNX_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  TNX_ERR_UNSUPPORTED = 6  /* valid input outside what this build implements */
};

/* arithmetic of the sector GEMMs */
enum {
  TNX_PREC_FP64 = 0,   /* DMMA f64 tensor-core GEMM, FP64 accumulate            */
  TNX_PREC_BF16X3 = 1, /* tcgen05 kind::f16: hi*hi + hi*lo + lo*hi, FP32 accum   */
  TNX_PREC_TF32 = 2    /* tcgen05 kind::tf32, FP32 accumulate                    */
};

/* block-matching semantics of a contraction plan */
enum {
  TNX_MATCH_FILTERED = 0,   /* _contract_symmetric: contraction/contractor.py:291-484 */
  TNX_MATCH_UNFILTERED = 1  /* _blockwise_contract: algorithms/dmrg.py:1048-1151      */
};

/* One operand's structure (no data).  charges: all legs' int32 charge
 * arrays concatenated (leg_dims[i] entries each); keys: n_blocks x n_legs. */
typedef struct tnx_tensor_desc {
  int32_t n_legs;
  const char* subs;       /* einsum chars, one per leg (may be NULL for H_eff) */
  const int32_t* flows;   /* +1 IN / -1 OUT                                  */
  const int32_t* charges;
  const int64_t* leg_dims;
  int64_t n_blocks;
  const int32_t* keys;
} tnx_tensor_desc;

typedef struct tnx_plan tnx_plan;
typedef struct tnx_heff tnx_heff;
typedef struct tnx_heff_batch tnx_heff_batch;

/* Text of the last error on the calling thread. */
const char* tnx_last_error(void);
int tnx_version(void);

/* Valid block keys, in the reference's order.  Replaces _compute_valid_blocks
 * (core/tensor.py:53-165).  modulus = 0 selects U(1), n >= 2 selects Z_n.
 * Call with keys_out == NULL to get the count in *n_keys. */
int tnx_valid_blocks(int32_t n_legs, const int32_t* charges, const int64_t* leg_dims, const int32_t* flows,
                     int32_t modulus, int32_t has_target, int64_t target, int64_t* n_keys, int32_t* keys_out,
                     int64_t keys_cap);

/* Device-side sector planning (no counterpart in the reference's API: the
 * same integer results as the host planner, computed by kernels on `stream`
 * from charge arrays and block keys in DEVICE memory; each call reads back
 * only the counts it returns and synchronises `stream`).  Limits: at most 12
 * legs, a charge range of at most 65536 per leg, at most 65536 valid output
 * keys per contraction.
 *   tnx_valid_blocks_dev: tnx_valid_blocks (_compute_valid_blocks,
 *     core/tensor.py:53-165) with charges_dev (all legs concatenated) and
 *     keys_dev (n_keys x n_legs) on the device; keys_dev may be NULL.
 *   tnx_contract_structure_dev: the output structure of a two-operand
 *     filtered contraction (_contract_symmetric, contraction/contractor.py:
 *     344-441): a->charges, a->keys, b->charges, b->keys are device
 *     pointers, subs are required.  Writes the output keys in sorted order
 *     (n_out_blocks x len(out_subs)), their block offsets (n_out_blocks + 1
 *     entries, the last one the total), and the matched block pairs (A block,
 *     B block, output block; int32 triples) ordered by A block then B block;
 *     any output pointer may be NULL (counts only).
 *   tnx_fused_charges_dev: _compute_fused_charges (algorithms/
 *     _tensor_utils.py:191-203): out[i*d_b + j] = fused_flow*(flow_a qa[i] +
 *     flow_b qb[j]) (mod n for Z_n, modulus > 0), device arrays. */
int tnx_valid_blocks_dev(int32_t n_legs, const int32_t* charges_dev, const int64_t* leg_dims, const int32_t* flows,
                         int32_t modulus, int32_t has_target, int64_t target, int64_t* n_keys, int32_t* keys_dev,
                         int64_t keys_cap, void* stream);
int tnx_contract_structure_dev(const tnx_tensor_desc* a, const tnx_tensor_desc* b, const char* out_subs,
                               int32_t modulus, int64_t* n_out_blocks, int32_t* out_keys_dev, int64_t* out_offsets_dev,
                               int64_t out_cap, int64_t* n_pairs, int32_t* pairs_dev, int64_t pairs_cap,
                               void* stream);
int tnx_fused_charges_dev(const int32_t* qa_dev, int64_t da, int32_t fa, const int32_t* qb_dev, int64_t db,
                          int32_t fb, int32_t fused_flow, int32_t modulus, int32_t* out_dev, void* stream);

/* Plan a block-sparse contraction of n_ops operands with subscripts
 * ops[i].subs -> out_subs.  mode TNX_MATCH_FILTERED reproduces
 * _contract_symmetric (contractor.py:291-484, output-target inference and
 * conservation filter; >= 3 operands with differing contracted sets give an
 * empty result as in the reference); TNX_MATCH_UNFILTERED reproduces
 * _blockwise_contract (dmrg.py:1048-1151, no output filter).  out_charges /
 * out_leg_dims / out_flows describe the output legs (used by the filter). */
int tnx_plan_create(const tnx_tensor_desc* ops, int32_t n_ops, const char* out_subs, int32_t mode,
                    int32_t modulus, const int32_t* out_charges, const int64_t* out_leg_dims,
                    const int32_t* out_flows, tnx_plan** plan);
/* tnx_plan_create for operands of a fermionic symmetry (FermionParity,
 * FermionicU1 with a built-in grading: parity = charge mod 2): every block
 * combination of a one- or two-operand contraction carries the reference's
 * exchange sign of the leg reordering (contraction/contractor.py:206-285,
 * :460-470); a one-operand plan is then the Koszul-signed transpose
 * (core/tensor.py:32-50).  fermionic = 0 is tnx_plan_create.  Three or more
 * operands: TNX_ERR_UNSUPPORTED (contract pairwise). */
int tnx_plan_create_graded(const tnx_tensor_desc* ops, int32_t n_ops, const char* out_subs, int32_t mode,
                           int32_t modulus, const int32_t* out_charges, const int64_t* out_leg_dims,
                           const int32_t* out_flows, int32_t fermionic, tnx_plan** plan);
/* Output structure: blocks in sorted-key order, contiguous. keys may be NULL. */
int tnx_plan_output(const tnx_plan* plan, int64_t* n_blocks, int32_t* keys, int64_t* total_elems,
                    int32_t* has_target, int64_t* target);
int tnx_plan_workspace(const tnx_plan* plan, int32_t precision, size_t* bytes);
double tnx_plan_flops(const tnx_plan* plan);
/* Execute on device FP64 data: inputs[i] are the operands' block buffers. */
int tnx_plan_execute(tnx_plan* plan, const double* const* inputs, double* out, int32_t precision, void* workspace,
                     size_t workspace_bytes, void* stream);
void tnx_plan_destroy(tnx_plan* plan);

/* tnx_plan_execute (FP64 sector GEMMs) for callers that cannot allocate
 * device memory.  No counterpart in the reference.  A caller embedded in a
 * framework that owns the GPU's memory -- an XLA custom call inside a JAX
 * process that has already reserved most of the device for its own pool, or
 * any host code that must not cudaMalloc behind its framework's allocator --
 * passes only its inputs and output; every scratch buffer (operand images,
 * sector result matrices, intermediates, device index tables) comes from one
 * file-scope 16 MiB device array that every GPU loading this library holds
 * until exit.  Plans that need more scratch fail with TNX_ERR_VALUE.  The
 * first call on a device looks up that array's device address (with that
 * device current).  Every call copies its tables, operand pointers and a
 * scalar from pageable host memory with cudaMemcpyAsync, so no call may be
 * made under stream capture (a CUDA graph or a command buffer): an XLA FFI
 * handler wrapping it must not declare itself command-buffer compatible.
 * All calls share the array: calls that overlap on the GPU race on it.
 * Allocates nothing: no cudaMalloc/cudaFree and no allocating library
 * routine. */
int tnx_plan_execute_static(const tnx_plan* plan, const double* const* inputs, double* out, void* stream);

/* Two-site effective Hamiltonian "abc,apqd,bpse,eqtf,dfg->cstg"
 * (dmrg.py:1282-1289) over the block structures of L, theta, W_l, W_r, R.
 * The output uses theta's block layout; tnx_heff_closed() reports whether
 * every output key is one of theta's keys (the caller extends theta's key
 * set until it is -- the key-union growth of the reference's Lanczos). */
int tnx_heff_create(const tnx_tensor_desc* L, const tnx_tensor_desc* theta, const tnx_tensor_desc* Wl,
                    const tnx_tensor_desc* Wr, const tnx_tensor_desc* R, tnx_heff** h);
/* The same, planned for the precision the operator will be packed in
 * (TNX_PREC_*): the mixed precisions lay the stage-1 result out for the fused
 * MPO kernel's aligned loads.  tnx_heff_set_operators with another
 * precision re-plans, so either create works with any precision. */
int tnx_heff_create_for(const tnx_tensor_desc* L, const tnx_tensor_desc* theta, const tnx_tensor_desc* Wl,
                        const tnx_tensor_desc* Wr, const tnx_tensor_desc* R, int32_t precision, tnx_heff** h);
/* Schedule of a mixed-precision operator's stages 1-3 (no counterpart in the
 * reference, which evaluates H_eff one block combination at a time).
 * fuse_mpo = 1: one tcgen05 kernel accumulates L.theta in tensor memory per
 * (q_c, q_d) sector pair and applies W_l W_r in its epilogue, writing the
 * stage-4 operand directly (no X1 in HBM), wherever the structure fits (at
 * most 48 input slots per sector pair, every pair's blocks side by side in
 * 256 accumulator columns); c_per_tile c values per tile, 0 = the largest
 * that fits.  fuse_mpo = 2 (routed): the stage-1 GEMM's epilogue writes
 * every W_l W_r output with a single term straight into the stage-4 operand
 * and keeps X1 only for the input slots that multi-term outputs read, which
 * the MPO kernel then forms; results equal the unfused schedule's bit for
 * bit.  fuse_mpo = 0: stage-1 GEMM, X1 in HBM, MPO kernel.  Other values:
 * TNX_ERR_VALUE.  fuse_mpo = -1 (automatic, also the schedule of an
 * operator given none): routed when its stage FLOPs (tnx_heff_flops) reach
 * 5e9, unfused below.  Takes effect at the
 * next tnx_heff_set_operators; FP64 operators always run unfused.  tnx_heff_get_schedule reports the schedule
 * in effect; before tnx_heff_set_operators, the one the precision given to
 * tnx_heff_create_for would get (host planning only). */
typedef struct tnx_heff_schedule {
  int32_t fuse_mpo;
  int32_t c_per_tile;
} tnx_heff_schedule;
int tnx_heff_set_schedule(tnx_heff* h, const tnx_heff_schedule* sched);
int tnx_heff_get_schedule(const tnx_heff* h, tnx_heff_schedule* sched);
int tnx_heff_closed(const tnx_heff* h, int32_t* closed);
/* Output keys of H_eff applied to theta's key set (structure only). */
int tnx_heff_out_keys(const tnx_heff* h, int64_t* n_keys, int32_t* keys);
/* Keys of theta that H_eff actually writes (others come out zero). */
double tnx_heff_flops(const tnx_heff* h);
/* Pack L, W_l, W_r, R (device FP64 block buffers) into GEMM operand images
 * for the given precision; done once per site, reused by every matvec. */
int tnx_heff_set_operators(tnx_heff* h, const double* L, const double* Wl, const double* Wr, const double* R,
                           int32_t precision, void* stream);
void tnx_heff_destroy(tnx_heff* h);

/* Many independent H_eff problems applied in one launch per stage
 * (persistent grouped GEMMs over all sectors of all problems).  The
 * operators of one batch must all run fused stages 1-3 or none of them
 * (tnx_heff_get_schedule); otherwise TNX_ERR_VALUE.  Routed and unfused
 * operators mix freely. */
int tnx_heff_batch_create(tnx_heff* const* hs, int32_t n, int32_t precision, tnx_heff_batch** b);
int tnx_heff_batch_apply(tnx_heff_batch* b, const double* const* thetas, double* const* outs, void* stream);
/* Host-resident streaming (no counterpart in the reference, which applies one
 * matvec at a time from device arrays): n_steps independent applications
 * whose inputs and outputs live in host memory (pinned for overlap).  host_in[s] / host_out[s]
 * hold all problems' theta buffers concatenated in batch order (offsets from
 * tnx_heff_batch_size).  Step s+1's copy in and step s-1's copy out run on
 * their own streams while step s computes; the call's work on `stream`
 * completes after the last copy out.  Device staging (two copies of inputs
 * and outputs) is allocated on the first call and kept with the batch. */
int tnx_heff_batch_apply_host(tnx_heff_batch* b, const double* const* host_in, double* const* host_out,
                              int32_t n_steps, void* stream);
/* Elements of the concatenated theta buffer and each problem's offset in it
 * (offsets: n doubles' worth of int64, or NULL). */
int tnx_heff_batch_size(const tnx_heff_batch* b, int64_t* total, int64_t* offsets);
/* Re-run one stage of the last apply (0 pack theta, 1 stage-1 GEMM, 2 fused
 * MPO, 3 stage-4 GEMM; with fused stages 1-3: 0 theta panels, 1 the fused
 * kernel, 2 nothing) with the same buffers -- per-kernel timing. */
int tnx_heff_batch_apply_stage(tnx_heff_batch* b, int32_t stage, void* stream);
/* Algorithmic flops of stage 1 (L.theta), stages 2+3 (MPO), stage 4 (.R). */
int tnx_heff_stage_flops(const tnx_heff* h, double* flops3);
/* Number of kernel launches one apply issues (launch accounting). */
int tnx_heff_batch_launches(const tnx_heff_batch* b, int32_t* n_launches);
/* Routed stage-1 tables (introspection, no reference counterpart): the number
 * of route records and the largest window of records one epilogue warp scans
 * for one 32-column chunk of a tile.  Both 0 when no operator is routed. */
int tnx_heff_batch_route_stats(const tnx_heff_batch* b, int64_t* n_routes, int32_t* max_window);
/* Device error flag of the tcgen05 GEMM (non-zero: a bounded wait gave up). */
int tnx_heff_batch_error(tnx_heff_batch* b, int32_t* err);
/* Optional device int32 flag: when non-zero, every kernel of an apply returns
 * immediately (Lanczos early exit inside a captured graph). */
int tnx_heff_batch_set_skip_flag(tnx_heff_batch* b, const int32_t* flag);
void tnx_heff_batch_destroy(tnx_heff_batch* b);

/* FP64 vector primitives on flat block buffers (inner/norm of the reference's
 * SymmetricTensor arithmetic, core/tensor.py:296-319, 863-868).  Reductions
 * are deterministic two-pass sums; `scratch` is a caller-owned device buffer
 * of tnx_reduce_scratch_len() doubles (calls sharing one scratch must be
 * stream-ordered).  Results are written to device memory. */
int64_t tnx_reduce_scratch_len(void);
int tnx_dot(const double* x, const double* y, int64_t n, double* result, double* scratch, void* stream);
int tnx_nrm2(const double* x, int64_t n, double* result, double* scratch, void* stream);

/* Bounded wait on a device flag (no counterpart in the reference): one
 * thread polls *flag until it equals `expected` or `timeout_ns` (at most
 * 10 s) has passed on the GPU timer, then writes *status (device memory):
 * 0, or TNX_ERR_TIMEOUT.  The kernel always returns, so the context stays
 * usable; it is the same deadline discipline as every wait inside the GEMM
 * kernels, exposed so callers (and tests) can exercise the timeout path. */
int tnx_wait_flag(const int32_t* flag, int32_t expected, int64_t timeout_ns, int32_t* status, void* stream);

/* Leg fusion of a block-sparse tensor (tenax algorithms/_tensor_utils.py:
 * 106-325, fuse_indices / _compute_fused_charges / _fuse_indices_symmetric).
 * Legs axis_a and axis_b become one leg at min(axis_a, axis_b) with flow
 * fused_flow (+1 IN, -1 OUT); position i*d_b + j of it carries charge
 * fused_flow*(flow_a q_a[i] + flow_b q_b[j]) (mod n for Z_n, modulus > 0).
 * Inside a fused sector, charge pairs (q_a, q_b) are stacked in sorted order
 * (q_a outer), each pair's rows row-major over the two legs' in-sector
 * positions; pairs without an input block are zero.  Tables are integer-exact
 * against the reference.  Output blocks are stored in sorted-key order.
 * `in` blocks must be laid out in the descriptor's key order; subs may be
 * NULL. tnx_fuse_plan_output: fused_charges holds d_a*d_b entries, keys
 * n_blocks*(n_legs-1); any pointer may be NULL. */
typedef struct tnx_fuse_plan tnx_fuse_plan;
int tnx_fuse_plan_create(const tnx_tensor_desc* in, int32_t modulus, int32_t axis_a, int32_t axis_b,
                         int32_t fused_flow, tnx_fuse_plan** out);
int tnx_fuse_plan_output(const tnx_fuse_plan* p, int32_t* fused_charges, int64_t* n_fused, int64_t* n_blocks,
                         int32_t* keys, int64_t* total);
int tnx_fuse_execute(tnx_fuse_plan* p, const double* in, double* out, void* stream);
void tnx_fuse_plan_destroy(tnx_fuse_plan* p);
/* The dense view of a fused leg (todense() of fuse_indices' result,
 * core/tensor.py:760-781): natural row i*d_b + j of the pair (leg a, leg b)
 * is placed at position map[i*d_b + j] of the fused leg.  Used by the
 * split-CTM moves, which fuse and densify grown corners
 * (algorithms/_split_ctm_tensor.py:522-541). */
int tnx_fuse_row_map(const int32_t* charges_a, int64_t d_a, int32_t flow_a, const int32_t* charges_b, int64_t d_b,
                     int32_t flow_b, int32_t fused_flow, int32_t modulus, int64_t* map);

/* Max-abs renormalisation of the CTM environment (tenax
 * algorithms/ipeps.py:1133-1149, _renormalize_env) for 1..8 tensors per call:
 *   y_t = x_t / (max|x_t| + eps),  stat[t] = max|x_t|  (device memory).
 * The adjoint maps gy_t = dL/dy_t to gx_t = dL/dx_t with the derivative of
 * the max split evenly among the entries attaining it (JAX's rule for
 * jnp.max): gx = gy/(m+eps) - <gy,x>/(m+eps)^2 * sign(x) [|x| == m] / count.
 * `stat` is the forward's.  x/y/gy/gx/n are HOST arrays of n_tensors device
 * pointers / sizes; `scratch` holds tnx_renorm_scratch_len() doubles.
 * y must not alias x; gx must not alias x or gy. */
int64_t tnx_renorm_scratch_len(void);
int tnx_renorm_maxabs(int n_tensors, const double* const* x, double* const* y, const int64_t* n, double eps,
                      double* stat, double* scratch, void* stream);
int tnx_renorm_maxabs_adjoint(int n_tensors, const double* const* x, const double* const* gy, double* const* gx,
                              const int64_t* n, double eps, const double* stat, double* scratch, void* stream);

/* Thin FP64 SVDs of independent sector matrices: the per-sector step of the
 * block-diagonal truncated SVD (tenax linalg.py:186-192, one
 * jnp.linalg.svd(matrix, full_matrices=False) per charge sector).
 * a[i] is m[i] x k[i], row-major, and is preserved; with r = min(m[i], k[i]),
 * u[i] receives m x r (row-major), s[i] the r singular values in descending
 * order and vh[i] r x k (row-major).  m, k, a, u, s, vh are HOST arrays of n
 * entries (extents and device pointers); sectors with m or k = 0 are skipped.
 * Sectors with min(m, k) >= polar_min run cuSOLVER's polar-decomposition SVD
 * (Xgesvdp), the others its Jacobi SVD (gesvdj): the polar driver is 2.5-3x
 * faster on large sectors and slower on small ones (128 is a good split).
 * They run on up to n_workers library-owned streams (1..32, one host thread
 * each), ordered after `stream`, which then waits for all of them; the call
 * returns once every decomposition has finished.  err_sigma (may be NULL)
 * receives the largest error estimate the polar driver reported.  Worker
 * scratch grows to the largest sector seen and is kept. */
int tnx_svd_batch(int32_t n, const int64_t* m, const int64_t* k, const double* const* a, double* const* u,
                  double* const* s, double* const* vh, int64_t polar_min, int32_t n_workers, double* err_sigma,
                  void* stream);

/* One Lanczos orthogonalisation step (dmrg.py:1005-1019) on device:
 *   alpha[k] = <v, w>;  w -= alpha[k] v  (- beta[k] v_prev if k > 0);
 *   beta[k+1] = ||w||;  if beta[k+1] < tol or beta[k+1] < tol_rel*|alpha[k]|: *done = 1
 *   else v_next = w / beta[k+1]
 * tol_rel = 0 is the reference's test; a mixed-precision matvec passes its
 * relative noise level so the recurrence stops instead of orthogonalising noise.
 * alpha/beta live in device memory; nothing is read back to the host.
 * Every kernel of the step returns immediately once *done is set. */
int tnx_lanczos_step(double* w, const double* v, const double* v_prev, double* v_next, int64_t n, double* alpha,
                     double* beta, int32_t k, double tol, double tol_rel, int32_t* done, double* scratch,
                     void* stream);
/* out = sum_k coefs[k] * basis[k], summed left to right as the reference's
 * eigenvector reconstruction (dmrg.py:1038-1040); device pointer table and
 * device coefficients. */
int tnx_combine(const double* const* basis_dev_table, const double* coefs_dev, int32_t n_vec, int64_t n, double* out,
                void* stream);
/* out = x * s (mode 0), x / s (mode 1), x / (s + 1e-15) (mode 2); s on device. */
int tnx_scale(const double* x, double* out, int64_t n, const double* scale_dev, int32_t mode, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TENAX_B200_H */
