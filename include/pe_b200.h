/*
 * pe_b200.h — C ABI of the B200 (sm_100a) Clifford & Clifford Fock sampler.
 *
 * Plain pointers and sizes only.  Every pointer named `d_*` is DEVICE memory owned by the caller;
 * every call is asynchronous on the caller's `stream` (cudaStream_t passed as void*) and returns a
 * status (0 = launched, < 0 = rejected before launch, see PE_ERR_*).  Errors found inside a kernel
 * (an out-of-range index that the host did not catch) are written to the device status word of the
 * workspace and read back with pe_read_status().  Nothing here allocates device memory: the caller
 * passes a workspace of pe_chain_workspace_bytes() bytes.
 *
 * Layout of the circuit data (one "instance" = the input columns of one circuit):
 *   d_acol      complex128 as interleaved float64 pairs, instance g occupies
 *               d_acol[2 * (inst_off[g] + j * inst_m[g] + rho)]  for input column j < inst_n[g] and
 *               output mode rho < inst_m[g]  (column-major: one input column = inst_m[g] contiguous
 *               complex values, so a marginal reads coalesced rows).
 *   d_inst_off  int64 [G] element offsets, d_inst_m / d_inst_n int32 [G].
 * Per stream s (a stream = one shot's chain):
 *   d_dp        int64 [S] instance of stream s
 *   d_nk        int32 [S] photons of stream s (<= n_stride), NULL = n_stride for every stream
 *   d_cols      int64 [S][n_stride] input columns in chain order (sigma applied; indices < inst_n)
 *   d_uniforms  float64 [S][n_stride] per-step uniforms in [0, 1), or NULL to draw them with
 *               Philox4x32-10 exactly as the reference's draw kernel does:
 *               u = (r0 + r1 2^-24) / (1 + 2^-24), r_i = tl.rand(seed, 2 off + i), with
 *               seed = d_seeds[seed_row[s] * n_stride + k] and off = d_rng_off[s]
 *   d_seed_row  int64 [S] (NULL = 0), d_rng_off int64 [S] (NULL = s)
 *   d_order     int64 [S] processing order of the streams (a permutation; NULL = 0..S-1): put the
 *               longest chains first for a short tail
 * Outputs:
 *   d_rows      int64 [S][n_stride] output modes in chain order (entries past nk[s] untouched)
 *   d_occ       int64 [S][occ_stride] occupations (row s fully written: zeros then counts), or NULL
 *   d_marg      float64 [S][n_stride][marg_stride] normalised weights w / sum(w) of every step, or NULL
 */
#ifndef PE_B200_H
#define PE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PE_OK 0
#define PE_ERR_ARG (-1)        /* a NULL pointer, a negative size, an unknown precision */
#define PE_ERR_SIZE (-2)       /* a size beyond the compiled limits (photons, modes, workspace) */
#define PE_ERR_CUDA (-3)       /* a CUDA runtime error at launch */
#define PE_ERR_DEVICE (-4)     /* an index error found on the device (see pe_read_status) */

#define PE_PRECISION_F64 0     /* complex FP64 throughout: the drop-in form */
#define PE_PRECISION_MIXED 1   /* FP32 Gray blocks, FP64 cross-block sum, FP64 marginal and CDF */
#define PE_PRECISION_COMPENSATED 2  /* FP32 Gray blocks in compensated double-float arithmetic (exact
                                       on-grid column sums, TwoProduct / TwoSum products and block sums),
                                       FP64 cross-block sum, marginal and CDF: FP64-level marginals */

#define PE_MAX_PHOTONS 64      /* photons per stream (cofactor tiers up to 64 columns) */
#define PE_MIXED_MAX_PHOTONS 32 /* the mixed forms (FP32 Gray blocks) up to 32; FP64 beyond */

/* Library version (major * 10000 + minor * 100 + patch). */
int pe_version(void);

/* Largest supported number of output modes for chains of up to 32 photons (shared-memory bound; the
 * wider tables of 33-64 photons leave fewer: pe_fock_chain answers PE_ERR_SIZE beyond them). */
int pe_max_modes(int block_threads);

/* Bytes of device workspace that pe_fock_chain needs (16-byte aligned pointer). */
size_t pe_chain_workspace_bytes(int64_t S);

/*
 * The whole Clifford & Clifford chain of S streams in ONE persistent kernel launch: per stream and
 * per step k = 1..nk[s], the Laplace cofactors of the chosen-rows block by the collapsed
 * (2020) Glynn Gray sum, the marginal over all output modes and the inverse-CDF pick.
 *
 * Replaces, for the lossless and the lossy/partially-distinguishable passes alike:
 *   photonic_engines/clifford/sampler.py:391-460          _sample_streams (the step loop)
 *   photonic_engines/clifford/cofactors_triton.py:413-485 multiplicity_tables, plan_multi,
 *                                                          cofactor_partials_multi
 *   photonic_engines/clifford/cuda_cofactors.py:278-299   cofactor_partials_cuda (cof_multi)
 *   photonic_engines/clifford/cofactors_triton.py:533-545 draw_step (_draw_kernel)
 *
 * precision: PE_PRECISION_F64, PE_PRECISION_MIXED or PE_PRECISION_COMPENSATED.  block_threads: 64, 128
 * or 256 (0 = default).  tpl: threads per Gray lane (1, 2 or 4; 0 = default).  grid_ctas: persistent
 * CTAs (0 = occupancy).
 */
int pe_fock_chain(int precision, const double* d_acol, const int64_t* d_inst_off, const int32_t* d_inst_m,
                  const int32_t* d_inst_n, int G, int m_max, int64_t S, const int64_t* d_dp,
                  const int32_t* d_nk, const int64_t* d_cols, int n_stride, const double* d_uniforms,
                  const int64_t* d_seeds, const int64_t* d_seed_row, const int64_t* d_rng_off,
                  const int64_t* d_order, int64_t* d_rows, int64_t* d_occ, int occ_stride, double* d_marg,
                  int marg_stride, void* d_workspace, size_t workspace_bytes, int block_threads, int tpl,
                  int grid_ctas, void* stream);

/*
 * The same chains with the heavy steps spread over several CTAs per stream, for batches with few
 * streams (down to one sample) where one CTA per stream leaves most SMs idle.  Steps 1..k_split-1 run
 * in the persistent kernel; every step k >= k_split runs as nch CTAs per stream, each summing its share
 * of the Gray lanes into a partial (workspace), then one CTA per stream sums the partials in a fixed
 * order and draws.  Same results as pe_fock_chain up to the rounding of the partial sums (FP64:
 * within 1e-12).  Workspace: pe_chain_split_workspace_bytes(S, nch).  k_split >= 2, nch >= 1.
 * Replaces, beside the step loop: photonic_engines/clifford/single.py:22-82 (fock_sample_single: one
 * sample over a fixed lane grid) and the lane planning of cofactors_triton.py:450-465.
 */
int pe_fock_chain_split(int precision, const double* d_acol, const int64_t* d_inst_off, const int32_t* d_inst_m,
                        const int32_t* d_inst_n, int G, int m_max, int64_t S, const int64_t* d_dp,
                        const int32_t* d_nk, const int64_t* d_cols, int n_stride, const double* d_uniforms,
                        const int64_t* d_seeds, const int64_t* d_seed_row, const int64_t* d_rng_off,
                        const int64_t* d_order, int64_t* d_rows, int64_t* d_occ, int occ_stride, double* d_marg,
                        int marg_stride, int k_split, int nch, void* d_workspace, size_t workspace_bytes,
                        int block_threads, int tpl, void* stream);

/*
 * The same chains in the warp-per-stream form, for short chains (n_stride <= 16): every warp of a CTA
 * runs its own stream (8 per CTA), so thousands of short chains progress at once without CTA-wide
 * barriers.  Same algorithm, draws and rules; workspace as pe_fock_chain; tpl 1 or 2 (0 = default).
 * Replaces, for small n, the launch-bound per-step loop of photonic_engines/clifford/sampler.py:420-456
 * (two or three launches per step, cofactors_triton.py:368-391 for K1 <= 10).
 */
int pe_fock_chain_warp(int precision, const double* d_acol, const int64_t* d_inst_off, const int32_t* d_inst_m,
                       const int32_t* d_inst_n, int G, int m_max, int64_t S, const int64_t* d_dp,
                       const int32_t* d_nk, const int64_t* d_cols, int n_stride, const double* d_uniforms,
                       const int64_t* d_seeds, const int64_t* d_seed_row, const int64_t* d_rng_off,
                       const int64_t* d_order, int64_t* d_rows, int64_t* d_occ, int occ_stride, double* d_marg,
                       int marg_stride, void* d_workspace, size_t workspace_bytes, int tpl, int grid_ctas,
                       void* stream);

/*
 * One tier of a length-sorted batch: as pe_fock_chain (warp = 0) or pe_fock_chain_warp (warp = 1; there
 * block_threads / 32 is the number of streams per CTA, 1 to 8, 0 = 8), but the
 * persistent queue runs only d_order[lo .. hi) with d_qrange = {lo, hi} read ON THE DEVICE (so a captured
 * CUDA graph replays it for every batch), and the kernel is chosen for chains of at most nk_max photons
 * (nk_max <= n_stride; a stream of the range with more is reported through the status word).  Launching
 * the tiers of one batch — e.g. nk > 20, 17..20 and <= 16 with the warp form — on separate streams, each
 * with its own workspace, runs every chain in the smallest kernel that holds it.  d_order and d_nk are
 * required.  No counterpart in the reference (its batched kernels take one lane plan per launch,
 * photonic_engines/clifford/cofactors_triton.py:450-465).
 */
int pe_fock_chain_range(int precision, const double* d_acol, const int64_t* d_inst_off, const int32_t* d_inst_m,
                        const int32_t* d_inst_n, int G, int m_max, int64_t S, const int64_t* d_dp,
                        const int32_t* d_nk, const int64_t* d_cols, int n_stride, const double* d_uniforms,
                        const int64_t* d_seeds, const int64_t* d_seed_row, const int64_t* d_rng_off,
                        const int64_t* d_order, int64_t* d_rows, int64_t* d_occ, int occ_stride, double* d_marg,
                        int marg_stride, void* d_workspace, size_t workspace_bytes, int block_threads, int tpl,
                        int grid_ctas, const int64_t* d_qrange, int nk_max, int warp, void* stream);

/*
 * One tier of a length-sorted batch, as pe_fock_chain_range (CTA form), with the heavy steps of its first
 * split_slots queue positions spread over nch CTAs per stream: the persistent kernel runs those positions'
 * steps 1..k_split-1 and every later position's whole chain; then every step k = k_split..nk_max runs the
 * split kernels over the slots (slot q = queue position q of the range, nothing past its end).  For the
 * longest chains of a ragged batch (a lossy batch's few 25-30-photon survivors), which would otherwise
 * each hold one CTA for the whole batch.  Workspace: pe_range_split_workspace_bytes(split_slots, nch).
 * No counterpart in the reference (its lossy passes run one launch grid per surviving count,
 * photonic_engines/clifford/sampler.py:188-215).
 */
int pe_fock_chain_range_split(int precision, const double* d_acol, const int64_t* d_inst_off,
                              const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max, int64_t S,
                              const int64_t* d_dp, const int32_t* d_nk, const int64_t* d_cols, int n_stride,
                              const double* d_uniforms, const int64_t* d_seeds, const int64_t* d_seed_row,
                              const int64_t* d_rng_off, const int64_t* d_order, int64_t* d_rows, int64_t* d_occ,
                              int occ_stride, double* d_marg, int marg_stride, void* d_workspace,
                              size_t workspace_bytes, int block_threads, int tpl, const int64_t* d_qrange,
                              int nk_max, int k_split, int nch, int64_t split_slots, void* stream);

/* Bytes of device workspace pe_fock_chain_range_split needs for split_slots slots of nch CTAs each. */
size_t pe_range_split_workspace_bytes(int64_t split_slots, int nch);

/* Bytes of device workspace pe_fock_chain_split needs for S streams and nch CTAs per stream. */
size_t pe_chain_split_workspace_bytes(int64_t S, int nch);

/* CTAs of the split-step kernel resident at once on the current device (SMs x CTAs per SM) for chains
 * of n_stride photons in the given precision, CTA size and lane width (0: the defaults of
 * pe_fock_chain_split); a negative status on bad arguments.  Callers size nch with it: S * nch a
 * little under a multiple of it, nch a power of two (the Gray lanes of a step come in powers of two).
 * Replaces the lane-grid sizing of photonic_engines/clifford/cofactors_triton.py:450-465. */
int pe_split_slots(int precision, int n_stride, int block_threads, int tpl);

/*
 * Adaptive chains: a forced prefix and an avoided set of output modes (photonic_engines/clifford/
 * sampler.py:391-460, `_sample_streams(..., prefix=, avoid=)`, reached from fock_sample(prefix=, avoid=),
 * sampler.py:57-182).  Every stream has n_stride photons (the reference allows prefix / avoid on lossless,
 * indistinguishable photons only).  d_rows [S][n_stride]: on entry its first n_prefix entries per stream
 * are the forced output modes; the chain runs steps n_prefix + 1 .. n_stride on the caller's column order
 * d_cols (whose first n_prefix columns are the set drawn for the prefix).
 * d_avoid (optional, uint8 [m_max], 1 = avoided mode): after every step past the first free one, a stream
 * whose last row is avoided is dropped, and the survivors of each pass chunk are renumbered before the
 * next step's draws exactly as the reference shrinks its batch (the Philox stream offset of a survivor is
 * its rank among the chunk's survivors; chunk start = s - d_rng_off[s]); the row of the last step is
 * checked too.  d_alive (uint8 [S], required with d_avoid): 1 for the streams that survived.  d_occ
 * (optional [S][occ_stride]): occupations including the prefix; rows of dropped streams are zeroed.
 * mode 0: one CTA per stream (k_split / nch as pe_fock_chain_split, or 0 / 0); mode 1: one warp per
 * stream (n_stride <= 16, no split).  Workspace: pe_adaptive_workspace_bytes(S, nch) (nch 0 without a
 * split).  With d_avoid the call is one launch per step plus a one-CTA survivor update between steps,
 * all on `stream` (no host synchronisation); without it, one launch.  Other arguments as pe_fock_chain.
 */
int pe_fock_chain_adaptive(int precision, const double* d_acol, const int64_t* d_inst_off, const int32_t* d_inst_m,
                           const int32_t* d_inst_n, int G, int m_max, int64_t S, const int64_t* d_dp,
                           const int64_t* d_cols, int n_stride, const double* d_uniforms, const int64_t* d_seeds,
                           const int64_t* d_seed_row, const int64_t* d_rng_off, int64_t* d_rows, int n_prefix,
                           const uint8_t* d_avoid, uint8_t* d_alive, int64_t* d_occ, int occ_stride, int k_split,
                           int nch, void* d_workspace, size_t workspace_bytes, int block_threads, int tpl, int mode,
                           void* stream);
size_t pe_adaptive_workspace_bytes(int64_t S, int nch);

/*
 * Emitter inputs (EmitterMPS with emitter dimension chi = 2, 1 or 2 labels per photon): one step of the
 * generalised chain rule, the matrix-cofactor sum of photonic_engines/clifford/emitter_reference.py:280-305
 * (matrix_cofactor_weights) as batched by emitter_sampler.py:150-175 (sample_torch) and by the reference's
 * CUDA kernel emit_multi (cuda_emitter.py:511).  A lane is one stream and one pure term of its reduced
 * state; lanes of a stream are contiguous (d_lstart / d_nlan per stream).
 *   d_ut        [M][m] complex: d_ut[mode * m + rho] = U[rho, mode]
 *   d_rows      [S][rows_stride] int64: the stream's k - 1 chosen output rows (chain order)
 *   d_colmode   [S][k][L] int32: input mode of label l of the stream's j-th placed photon (slots sorted)
 *   d_s0, d_f   [Tt][2] complex; d_mats [Tt][k][L][2][2] complex: the terms (s0_e, M~_e, f_e)
 *   d_lane_term, d_lane_stream [nl] int64; d_lstart, d_nlan [S] int64
 * Outputs: d_amp [nl][m] complex amplitudes, d_w [S][m] float64 weights (sum of |amp|^2 over the stream's
 * lanes, in lane order).  k <= 24.  Workspace: pe_emitter_workspace_bytes() (status word).
 */
int pe_emitter_weights(const double* d_ut, int m, int M, const int64_t* d_rows, int rows_stride,
                       const int32_t* d_colmode, int64_t S, int k, int L, int chi, const double* d_s0,
                       const double* d_f, const double* d_mats, int64_t Tt, const int64_t* d_lane_term,
                       const int64_t* d_lane_stream, const int64_t* d_lstart, const int64_t* d_nlan, int64_t nl,
                       double* d_amp, double* d_w, void* d_workspace, size_t workspace_bytes, void* stream);
size_t pe_emitter_workspace_bytes(void);

/*
 * The same emitter step with every term assembled on the device (no per-lane inputs): per-state tables
 *   d_gops [n][n][4][L][2][2]  K^(a,b)_r M_{a,l}: Kraus operator r of the run of photons between placed
 *                              slots a < b, times slot a's emission operator l;  d_rg [n][n] int32 ranks
 *   d_ops  [n][L][2][2]        emission operators (the last placed slot)
 *   d_pre  [n][2][2]           images of |s0> through the photons before slot a; d_r0 [n] int32 ranks
 *   d_suf  [nf][n][2][2]       images of <final| through the photons after slot b; d_rf [nf][n] ranks
 * (emitter_reference.py:190-277, gap_kraus_terms, split into its per-slot pieces), the streams' placed
 * slots d_T [S][k] (increasing) and final ids d_fid [S], d_modes [n][L].  pe_emitter_count writes the
 * number of terms of every stream (d_nlan [S]); the caller forms d_lstart = exclusive cumsum and nl, then
 * pe_emitter_step writes d_amp [nl][m] and d_w [S][m] as pe_emitter_weights.  Terms whose norm is below
 * 1e-14 of their scale add nothing (the reference drops them).  pe_emitter_count clears the workspace's
 * status word, pe_emitter_step keeps it.
 */
int pe_emitter_count(const int32_t* d_T, const int32_t* d_fid, int64_t S, int k, const int32_t* d_rg,
                     const int32_t* d_r0, const int32_t* d_rf, int n, int nf, int64_t* d_nlan, void* d_workspace,
                     size_t workspace_bytes, void* stream);
int pe_emitter_step(const double* d_ut, int m, int M, const int64_t* d_rows, int rows_stride, const int32_t* d_T,
                    const int32_t* d_fid, const int32_t* d_modes, int64_t S, int k, int L, int chi,
                    const double* d_gops, const int32_t* d_rg, const double* d_ops, const double* d_pre,
                    const int32_t* d_r0, const double* d_suf, const int32_t* d_rf, int n, int nf,
                    const int64_t* d_lstart, const int64_t* d_nlan, int64_t nl, double* d_amp, double* d_w,
                    void* d_workspace, size_t workspace_bytes, void* stream);

/*
 * pe_fock_chain without a workspace argument: the same chains and outputs, for callers that cannot
 * allocate device memory when they sample (a host callback or other context where CUDA allocation is not
 * allowed, a serving process whose device memory all belongs to its own arena, a foreign-language
 * binding that can pass buffers but cannot call cudaMalloc).  No counterpart in the reference.
 *
 * Its scratch (the work-queue counter and the status word) lives in a static device array of 4096
 * bytes that every GPU loading this library holds until exit; a requirement above that size is
 * rejected with PE_ERR_SIZE.  The first call on a device looks the array up with cudaGetSymbolAddress
 * (once per device): make that first call before any stream capture.  The call allocates nothing: no
 * cudaMalloc, no cudaFree.  All calls share the array and it keeps the last call's contents; each call
 * clears the queue counter and status word on its stream before its launch, and calls whose kernels
 * overlap on the GPU race on it.  d_status (optional, device int) receives the device status word
 * (0, or PE_ERR_DEVICE after an out-of-range index).  Other arguments as pe_fock_chain.
 */
int pe_fock_chain_noalloc(int precision, const double* d_acol, const int64_t* d_inst_off,
                          const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max, int64_t S,
                          const int64_t* d_dp, const int32_t* d_nk, const int64_t* d_cols, int n_stride,
                          const double* d_uniforms, const int64_t* d_seeds, const int64_t* d_seed_row,
                          const int64_t* d_rng_off, const int64_t* d_order, int64_t* d_rows, int64_t* d_occ,
                          int occ_stride, double* d_marg, int marg_stride, int* d_status, int block_threads,
                          int tpl, int grid_ctas, void* stream);

/*
 * Laplace cofactors P[s, c] = per(A_s[rows_s, all columns but c]) of S blocks, the reference's
 * 2020 kernel entry point:
 *   photonic_engines/clifford/cofactors_triton.py:509-530  laplace_cofactors_rows
 * d_a: complex128 [S][m][K] (interleaved), d_rows int64 [S][K - 1] (repeats allowed, < m),
 * d_p: complex128 [S][K] out.  K <= PE_MAX_PHOTONS.
 */
int pe_cofactors_rows(int precision, const double* d_a, const int64_t* d_rows, int64_t S, int m, int K,
                      double* d_p, void* d_workspace, size_t workspace_bytes, int block_threads, int tpl,
                      void* stream);

/*
 * Device-side partition of S shots into chains (batched form): per photon of shot s (instance dp[s],
 * inst_n[g] photons), lost with probability 1 - eta[g], else interfering with probability x[g] (x-model;
 * x >= 1: always), else alone.  Slot 0 of a shot holds its interfering photons in a uniformly random
 * order (d_nk = their count); with `singles` = 1, slots 1..n_stride hold one lone photon each (nk 0 or
 * 1).  Chain c = s * slots + q; d_cols [C][n_stride], d_nk [C], d_chain_dp [C] (instance), d_out_row [C]
 * (= s).  Draws: Philox4x32-10 keyed by the device int64 *d_key (graph-capturable).  The law of
 *   photonic_engines/imperfections.py:529-590   draw_roles / partition / route_classical
 *   photonic_engines/clifford/sampler.py:183-215 grouping by surviving columns, one pass per count
 * without host work; the draws differ from the reference's host draws (fock_sample keeps those).
 */
int pe_partition_shots(const int64_t* d_dp, const int32_t* d_inst_n, const double* d_eta, const double* d_x,
                       int64_t S, int n_stride, int singles, const int64_t* d_key, int64_t* d_cols, int32_t* d_nk,
                       int64_t* d_chain_dp, int64_t* d_out_row, int* d_status, void* stream);

/*
 * Occupations [S][occ_stride] from chains: zeroed, then occ[out_row[c]][rows[c][j]] += 1 for j < nk[c]
 * (photonic_engines/clifford/sampler.py:172, :214).  Index errors set *d_status to PE_ERR_DEVICE.
 */
int pe_scatter_occupations(const int64_t* d_rows, const int32_t* d_nk, const int64_t* d_out_row, int64_t C,
                           int n_stride, int64_t* d_occ, int occ_stride, int64_t S, int* d_status, void* stream);

/* Arithmetic-pipe probe (no counterpart in the reference: a measurement aid).  Launches 8 independent
 * FMA chains per thread, `iters` rounds, on (SMs x 8) CTAs of 256 threads, in FP64
 * (PE_PRECISION_F64) or FP32 (PE_PRECISION_MIXED); *flops receives the FLOPs the launch performs
 * (FMA = 2).  d_out needs SMs * 8 * 256 * sizeof(element) bytes.  The caller times it. */
int pe_pipe_probe(int precision, int iters, void* d_out, size_t out_bytes, double* flops, void* stream);

/* Copy the device status word of a workspace to *status (synchronises `stream`).
 * 0 = no device-side error; otherwise PE_ERR_DEVICE and the offending stream index in *detail. */
int pe_read_status(const void* d_workspace, int* status, int64_t* detail, void* stream);

/* Human-readable text of a status code. */
const char* pe_status_string(int status);

/* Text of the CUDA runtime error behind the calling thread's latest PE_ERR_CUDA return (no counterpart
 * in the reference, whose Python wrappers raise the runtime's own exceptions). */
const char* pe_last_cuda_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PE_B200_H */
