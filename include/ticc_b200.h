/*
 * ticc_b200 — C ABI of the B200 (sm_100a) coupled-channel scattering kernels.
 *
 * Every entry point is stream-ordered and non-blocking: it validates its
 * arguments on the host, enqueues kernels on `stream` (a cudaStream_t passed as
 * void*, NULL for the legacy default stream) and returns a status code.  All
 * buffers are caller-owned device pointers; no entry point allocates device
 * memory except the runtime's own one-time module state.  Scratch memory is a
 * caller-provided `workspace` whose size comes from the matching *_workspace_size
 * query.
 *
 * `device_status` (optional, may be NULL) points to int[4] of device memory that
 * the caller zeroes before the call and reads after synchronising the stream:
 * {code, batch item, detail, 0}.  Codes: 0 ok, 1 singular pivot block in a
 * symmetric sweep (detail = block index), 2 non-finite output, 3 Bessel continued
 * fraction did not converge (detail = channel), 4 energy exactly at a threshold,
 * 5 more open channels than the caller's max_open, 6 a step of a symmetric sweep
 * gave up waiting for a row-panel tile of its own launch (an internal error; the
 * wait is bounded, the results of that call are invalid).
 *
 * Matrices are row-major float64, or complex128 with interleaved (re, im) pairs
 * when `is_complex` is set.  Symmetric inputs are required where noted: their
 * antisymmetric part is ignored (the reference's callers only ever pass symmetric
 * matrices; see each entry).
 *
 * Each declaration names the reference (PyTICC, src/pyticc/...) function it
 * replaces; the Python host layer pyticc_b200 binds them through ctypes.
 */
#ifndef TICC_B200_H
#define TICC_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TICC_OK = 0,
  TICC_ERR_INVALID_ARGUMENT = 1,
  TICC_ERR_CUDA = 2,
  TICC_ERR_WORKSPACE = 3,
  TICC_ERR_UNSUPPORTED = 4
};

enum { TICC_PRECISION_FP64 = 0, TICC_PRECISION_MIXED = 1 };

/* Library ABI version (major * 10000 + minor * 100 + patch). */
int ticc_version(void);

/* Number of kernels this library has enqueued since the process loaded it (host-side
 * counter; a diagnostic for benchmarks, not a device query).  No reference counterpart. */
long long ticc_kernel_launches(void);

/* Copy the calling thread's most recent error message into buf (NUL-terminated).
 * Returns the message length. */
int ticc_last_error(char* buf, size_t len);

/* ---- symmetric inversion ---------------------------------------------------
 * Batched in-place inverse of symmetric (or complex symmetric) n x n matrices by
 * a blocked sweep with 128-wide pivot blocks and partial pivoting inside each
 * block.  Replaces the energy-shared jnp.linalg.solve(I - h^2 T_mid / 6, I) of
 * _correction_matrices (propagation/logd.py:162) and is the kernel behind every
 * inversion below.  M: batch x n x n at stride n*n (complex: interleaved). */
int ticc_sym_inverse_workspace_size(int n, int batch, int is_complex, size_t* bytes);
int ticc_sym_inverse(void* M, int n, int batch, int is_complex, void* workspace, size_t workspace_bytes, int* device_status, void* stream);

/* Allocation-free variant of ticc_sym_inverse, for callers that cannot allocate device
 * memory: plugin hosts that pass only buffers they own, runtimes that fix their device
 * memory budget at start-up, and C/Fortran drivers without a device allocator.  It has no counterpart in the reference.  Scratch comes from a fixed
 * 32 MiB device array inside the library (held by every GPU that loads it until the
 * process exits), so batch * (Np^2 + 128 Np + 32784) doubles must fit in 32 MiB, with
 * Np = n (2n when complex) rounded up to 128 — e.g. n <= 512 with batch <= 11; larger
 * requests are rejected with TICC_ERR_INVALID_ARGUMENT and a message.  The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  All calls on a device share
 * the one array: calls that overlap on the GPU (different streams, or threads) race and
 * must be serialised by the caller.  The caller clears nothing: each call zeroes the words
 * of the array that must start at zero (the sweep's work queues and tile flags) itself. */
int ticc_sym_inverse_noalloc(void* M, int n, int batch, int is_complex, int* device_status, void* stream);

/* Test hook with no counterpart in the reference: the number of polls a wait of the fused
 * sweep step (a tile waiting for the row-panel tiles it reads) may spend before it gives
 * up, raises the call's abort flag and reports device status 6 (the default, 2^22 polls,
 * is restored by passing 4194304).  0 makes every wait give up before its first poll, so a
 * test can check the bounded-wait path; the kernel then finishes without the skipped work
 * and the context stays usable.  Applies to the current device. */
int ticc_debug_set_step_poll_limit(long long polls);

/* Test hook with no counterpart in the reference: the tcgen05 TF32x3 trailing-update tile
 * run on its own.  For each listed tile t (tiles[3t .. 3t+2] = matrix b, row tile ta,
 * column tile tb, device ints) it computes, in the 128 x 128 block (ta, tb) of matrix b of
 * M (batch x np x np FP64, np a multiple of 128),
 *     M_tile <- M_tile - cold[b][:, ta block]^T U[b][:, tb block]
 * with cold and U given as batch x 128 x np FP64 panels (device), rounded to FP32 and split
 * into TF32 hi/lo words in shared memory, the three products hi*hi + hi*lo + lo*hi accumulated in FP32 in tensor memory.  A
 * diagonal tile (ta == tb) keeps its lower half and mirrors it into the upper half.
 * Listed tiles must be distinct. */
int ticc_debug_tc_update_workspace_size(int np, int batch, size_t* bytes);
int ticc_debug_tc_update(double* M, int np, int batch, const double* cold, const double* U, const int* tiles, int n_tiles, void* workspace,
                         size_t workspace_bytes, int* device_status, void* stream);

/* ---- LDMD propagation -------------------------------------------------------
 * Propagate n_energy log-derivative matrices Y through n_sector Manolopoulos LDMD
 * sectors.  Replaces propagate_logD (propagation/logd.py:340-398) with its
 * vmap/scan body _propagate_logD_jax (:288-330), _correction_matrices (:143-164),
 * _reference_values (:98-132) and _propagate_with_corrections (:168-194).
 *   Y          device, n_energy x n x n (complex interleaved if is_complex); read at
 *              the first sector start, overwritten with Y at the last sector end.
 *              Must be symmetric (the reference's initialisers are diagonal).
 *   energies   device, n_energy total energies (hartree).
 *   half_steps device, n_sector half-steps (bohr), all > 0.
 *   W_start/W_mid/W_end device, energy-independent W_base at the sector start,
 *              midpoint and end, each n x n and exactly symmetric (only W[i][j] is read
 *              for element (i, j); ticc_contract's W assembly produces such matrices), at
 *              the given element stride between consecutive sectors (e.g. 2*n*n for an
 *              interleaved point list).
 *   precision  TICC_PRECISION_FP64 (all-FP64) or TICC_PRECISION_MIXED: the sweep steps
 *              over the leading blocks whose channels are all closed with a local
 *              wavenumber above 30 bohr^-1 at the batch's highest energy take an
 *              FP32-accurate TF32x3 product for their row panel and trailing update;
 *              pivot inversions, the open blocks' steps, Q_mid and the Y recurrence stay
 *              FP64.  Order channels most-closed first to benefit. */
int ticc_ldmd_workspace_size(int n_channel, int n_energy, int n_sector, int is_complex, int precision, size_t* bytes);
int ticc_ldmd_propagate(void* Y, int is_complex, const double* energies, int n_energy, double reduced_mass, const double* half_steps,
                        const double* W_start, long long W_start_stride, const double* W_mid, long long W_mid_stride, const double* W_end,
                        long long W_end_stride, int n_sector, int n_channel, int precision, void* workspace, size_t workspace_bytes,
                        int* device_status, void* stream);

/* Diagnostic with no counterpart in the reference: after a mixed-precision
 * ticc_ldmd_propagate / ticc_ldmd_propagate_blocks call, the number of leading 128-wide
 * sweep blocks of each sector that took the TF32x3 product (both sweeps of a sector use
 * the same count), copied from the call's workspace into the HOST array counts[n_sector]
 * in stream order (enqueue it on the propagation's stream before the workspace is reused;
 * with pinned memory the copy is asynchronous: synchronise before reading counts).  Pass
 * the same sizes as the propagation call. */
int ticc_ldmd_reduced_blocks(const void* workspace, size_t workspace_bytes, int n_channel, int n_energy, int n_block, int n_sector, int is_complex,
                             int precision, int* counts, void* stream);

/* Several channel blocks through the same sectors in one call: the coupled-states and
 * NNCC K blocks of one (J, parity) system.  Replaces the per-block loop of
 * _propagate_blocks (propagation/runner.py:165-322), which calls propagate_logD once per
 * block and window.  Blocks share n_channel: pad a smaller block with decoupled closed
 * channels (zero off-diagonal W, a positive W_ii - 2 mu E and a diagonal Y), which leave
 * the real channels' arithmetic unchanged.
 *   Y          device, n_block x n_energy x n x n (block-major).
 *   W_*        block g reads W_*(sector s) at W_* + s * W_*_stride + g * W_block_stride.
 *   Other arguments as ticc_ldmd_propagate; n_block * n_energy and n_block * n_sector
 *   must not exceed 65535.  In mixed precision a sweep block is reduced only if it is
 *   strongly closed in every channel block. */
int ticc_ldmd_blocks_workspace_size(int n_channel, int n_energy, int n_block, int n_sector, int is_complex, int precision, size_t* bytes);
int ticc_ldmd_propagate_blocks(void* Y, int is_complex, const double* energies, int n_energy, double reduced_mass, const double* half_steps,
                               const double* W_start, long long W_start_stride, const double* W_mid, long long W_mid_stride, const double* W_end,
                               long long W_end_stride, long long W_block_stride, int n_sector, int n_channel, int n_block, int precision,
                               void* workspace, size_t workspace_bytes, int* device_status, void* stream);

/* One block of a state-resolved (diabatic) atom-diatom contraction, the weighted products of
 * src/pyticc/matrix/interaction/diabatic_atom_diatom.py:262-287 (_contract_weighted_basis):
 *     X(R)[i][j] = sum_q A[i][q] weights[R * w_stride + q] B[j][q]
 * written to out[R][pos_a[i]][pos_b[j]] (out: n_R x n x n, device) and, with `mirror`, also to
 * out[R][pos_b[j]][pos_a[i]] (the coupling blocks of two electronic states).  A `symmetric`
 * block (B == A, pos_b == pos_a: a diagonal block) is computed on its lower half and mirrored,
 * so it is exactly symmetric.  Entries outside the block are left as they are (the caller
 * zeroes out).  All arrays are device arrays; A and B have row stride n_grid. */
int ticc_contract_block(const double* A, int n_a, const double* B, int n_b, int n_grid, const double* weights, long long w_stride, int n_R, const int* pos_a,
                        const int* pos_b, int symmetric, int mirror, int n, double* out, void* stream);

/* Packed lower-triangle channel pairs of the fine-structure contractions into matrices (the
 * scatter of src/pyticc/matrix/interaction/fs_diatom_diatom.py:383-391 and
 * fs_diatom_diatom_spin.py:463-482): for pair p = (pair_rows[p], pair_cols[p]) (rows >= cols)
 * and every R, the value src[R * src_stride + p] (real) or the complex double at element p
 * (is_complex; conjugated where reversed[p] is non-zero) goes to out[R][i][j] and, mirrored
 * (conjugated when complex), to out[R][j][i]; a complex diagonal element keeps its real part.
 * out: n_R x n x n doubles or interleaved complex doubles.  Device arrays; reversed may be null. */
int ticc_pairs_to_matrix(const double* src, int is_complex, long long src_stride, int n_pairs, const int* pair_rows, const int* pair_cols,
                         const unsigned char* reversed, int n, int n_R, double* out, void* stream);

/* Analytic interaction PES on the atom-diatom tensor grid, in device memory (the host
 * evaluation it replaces: src/pyticc/pes/adiabatic.py:109-137, get_Vgrid_atom_diatom, R x r x
 * theta in meshgrid "ij" order).  For a PES in the Legendre-expansion form
 *     V(R, r, theta) = sum_t P_lam[t](cos theta) f_t(R) g_t(r - re),  g_t(d) = sum_q poly[t][q] d^q,
 *     f_t(R) = sum_p primitive(prim_kind[t][p], params[t][p][0..2], R),
 * writes V[a][i][k] = V(R[a], r[i], acos(x[k])) (device arrays R, r, x, V; V of n_R * n_r * n_x
 * doubles).  Primitive kinds: 0 a R^-b, 1 a exp(-b (R - c)), 2 a exp(-((R - c)/b)^2),
 * 3 a ((b/R)^12 - 2 (b/R)^6).  The term tables are host arrays laid out with 4 primitives
 * (3 parameters each) and 4 polynomial coefficients per term; at most 16 terms, lam <= 32. */
int ticc_pes_legendre_grid(const double* R, int n_R, const double* r, int n_r, const double* x, int n_x, int n_terms, const int* lam, const int* n_prim,
                           const int* prim_kind, const double* prim_params, const int* n_poly, const double* poly, double re, double* V, void* stream);

/* ---- PotentialGrid contraction and W assembly --------------------------------
 * V_K(R) = norm [(B_r v(R)) B_r^T + (B_i v(R)) B_i^T] per K group, scattered into the
 * (n_R, n_channel, n_channel) block-diagonal V.  Replaces contract_device /
 * _contract_block_device (matrix/interaction/common.py:153-211, :66-74).  With U
 * non-NULL the output is instead W_base(R) = U/R^2 + 2 mu [V(R) + diag(E_int)], the
 * device W assembly of propagation/runner.py:265-271.
 *   rows_real/rows_imag  device, n_rows x n_grid weighted basis rows, grouped by K:
 *                        group g owns rows [group_offsets[g], group_offsets[g+1]).
 *   group_offsets        HOST array of n_groups + 1 non-decreasing row offsets.
 *   row_out              device, output channel position of every row.
 *   potential            device, n_R rows of n_grid values at row stride pot_stride.
 *   radial_points        device, n_R values (used only when U != NULL).
 *   out                  device, n_R x n_channel x n_channel. */
int ticc_contract(const double* rows_real, const double* rows_imag, const int* group_offsets, int n_groups, const int* row_out, int n_grid,
                  double normalization, const double* potential, long long pot_stride, int n_R, int n_channel, const double* radial_points,
                  const double* U, const double* E_int, double reduced_mass, double* out, void* stream);

/* ---- BF -> SF transform --------------------------------------------------------
 * Y_SF = B^T Y_BF B for a batch.  Replaces transform_logD_BF_to_SF
 * (match/asymptotic.py:82-110).  Y, Y_out: batch x n x n (complex interleaved if
 * is_complex; in-place allowed); B: n x n real. */
int ticc_transform_workspace_size(int n, int batch, int is_complex, size_t* bytes);
int ticc_transform_bf_to_sf(const void* Y, void* Y_out, const double* B, int n, int batch, int is_complex, void* workspace, size_t workspace_bytes,
                            void* stream);

/* ---- Riccati-Bessel functions --------------------------------------------------
 * out[4*i .. 4*i+3] = (j, n, j', n') of order ell[i] at x[i] (nu = ell + 1/2).
 * Replaces riccati_bessel_jy (match/bessel.py:7-45). */
int ticc_riccati_bessel_jy(const double* ell, const double* x, int n, double* out, int* device_status, void* stream);

/* out[i] = K'_nu(x)/K_nu(x) = -K_{nu-1}(x)/K_nu(x) - nu/x.
 * Replaces modified_bessel_K_logD (match/bessel.py:90-122). */
int ticc_bessel_k_logd(const double* nu, const double* x, int n, double* out, int* device_status, void* stream);

/* ---- asymptotic matching --------------------------------------------------------
 * S matrices from SF log-derivatives.  Replaces get_Smat (match/smatrix.py:139-223)
 * with _reference_functions (:10-79) and _open_reaction_matrix (:86-132).
 *   Y       device, n_energy x n x n SF log-derivatives (complex if is_complex), symmetric.
 *   E_int, L, energies  device.
 *   S       device, n_energy x n x n complex128: S[e] holds the n_open[e] x n_open[e]
 *           S matrix in its top-left corner, rows/columns in the order of
 *           flatnonzero(E_int < energy); the rest is zero.
 *   n_open  device, n_energy ints.
 *   max_open host bound on the open-channel count at every energy (the caller knows
 *           E_int and the energies); a larger count sets device status 5. */
int ticc_match_workspace_size(int n_channel, int n_energy, int is_complex, int max_open, size_t* bytes);
int ticc_match_smatrix(const void* Y, int is_complex, double Rmatch, const double* energies, int n_energy, double reduced_mass, const double* E_int,
                       const double* L, int n_channel, int max_open, double* S, int* n_open, void* workspace, size_t workspace_bytes,
                       int* device_status, void* stream);

/* ---- learned sector widths ------------------------------------------------------
 * No counterpart in the reference, which propagates on the fixed grid of
 * build_radial_sectors (propagation/grid.py:193-239) only.  A small MLP proposes, per
 * fixed-step sector, log2 of how many aligned sectors may be merged into one; merged
 * sectors keep their start/mid/end points on the same grid, so the PotentialGrid is
 * unchanged.  Every learned schedule is checked against the fixed-step propagation.
 *
 * Network: n_feature -> n_hidden (tanh) -> n_hidden (tanh) -> 1, FP32 parameters packed as
 * W1[n_hidden][n_feature], b1, W2[n_hidden][n_hidden], b2, w3[n_hidden], b3. */
int ticc_mlp_shape(int* n_feature, int* n_hidden, int* n_param);

/* features[s][0..7] (FP32) of fixed-step sector s from its W_base start/mid/end matrices
 * (same layout and strides as ticc_ldmd_propagate); two_mu_emax / two_mu_emin are 2 mu E
 * at the highest and lowest energy of the batch.  All pointers device. */
int ticc_step_features(const double* W_start, long long W_start_stride, const double* W_mid, long long W_mid_stride, const double* W_end,
                       long long W_end_stride, const double* half_steps, int n_sector, int n_channel, double two_mu_emax, double two_mu_emin,
                       float* features, void* stream);

/* y[i] = MLP((x[i] - norm[0:8]) * norm[8:16]) for n samples.  All pointers device. */
int ticc_mlp_forward(const float* params, const float* norm, const float* x, int n, float* y, void* stream);

/* Gradient of the asymmetric weighted squared loss
 *   loss = inv_weight_sum * sum_i weight[i] c_i (y_i - target[i])^2,  c_i = over_weight if
 *   y_i > target[i] (a proposal wider than the label) else 1,
 * into grads[n_param] and loss[1] (device), summed in a fixed order. */
int ticc_mlp_workspace_size(int n, size_t* bytes);
int ticc_mlp_gradient(const float* params, const float* norm, const float* x, const float* target, const float* weight, int n, float over_weight,
                      float inv_weight_sum, float* grads, float* loss, void* workspace, size_t workspace_bytes, void* stream);

/* One Adam step (step counts from 1) on params with moments[2 * n_param] = (m, v). */
int ticc_mlp_adam(float* params, const float* grads, float* moments, int step, float lr, float beta1, float beta2, float eps, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TICC_B200_H */
