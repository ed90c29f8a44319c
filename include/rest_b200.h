/*
 * rest_b200.h -- C ABI of librest_b200.so, the B200 (sm_100a) RI Coulomb /
 * exchange Fock build of REST (jeanwsr/rest, src/scf_io).
 *
 * The entry points replace REST's Rust free functions one for one; each
 * declaration names the function it stands in for (file:line in REST).  All
 * matrices use REST's storage conventions:
 *
 *   MatrixFull[r, c]   column-major, element (i, j) at i + r*j
 *   MatrixUpper        packed upper triangle, column by column:
 *                      (i <= j) at j*(j+1)/2 + i          (npair = n(n+1)/2)
 *   RIFull[n, n, N]    (mu, nu, P) at mu + n*nu + n*n*P   ("ri3fn")
 *   rimatr             MatrixFull[npair, N]: column P is the packed upper
 *                      triangle of B_P                      ("rimatr")
 *
 * Spin-resolved arguments are stored spin after spin: dm is spin_channel
 * consecutive n*n matrices, eigv spin_channel consecutive n*num_state
 * matrices, occupation spin_channel consecutive num_state vectors, and every
 * output spin_channel consecutive results.  REST's second, one-element
 * placeholder slot for spin_channel == 1 is not written.
 *
 * Conventions: every call returns a status (RIJK_OK == 0).  Host pointers stay
 * owned by the caller; device memory is owned by the context.  Host-pointer
 * calls are synchronous; the *_dev calls take device pointers and enqueue on
 * the given stream (NULL = the context's stream) without synchronising.  A
 * context is not thread-safe: use one per host thread.  There is no CPU
 * fallback: without a usable sm_100 device rijk_ctx_create fails.
 */
#ifndef REST_B200_H
#define REST_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum rijk_status {
  RIJK_OK = 0,
  RIJK_ERR_ARG = 1,        /* invalid argument (sizes, null pointers, spin)        */
  RIJK_ERR_CUDA = 2,       /* CUDA runtime error; see rijk_ctx_last_error           */
  RIJK_ERR_NOT_SPD = 3,    /* metric not positive definite (failing pivot given)   */
  RIJK_ERR_NO_TENSOR = 4,  /* no fitted tensor loaded in the context               */
  RIJK_ERR_TIMEOUT = 5,    /* a device-side wait ran out of its time budget         */
  RIJK_ERR_NOMEM = 6,      /* device allocation failed                              */
  RIJK_ERR_NONFINITE = 7,  /* NaN/Inf in a density, orbital or occupation element a
                              build reads (checked on the device, reported by the
                              next synchronising call)                             */
  RIJK_ERR_TOO_LARGE = 8   /* size beyond a documented maximum                      */
};

typedef struct rijk_ctx rijk_ctx;

/* ---- context --------------------------------------------------------------- */
int rijk_ctx_create(int device, rijk_ctx** out);
int rijk_ctx_destroy(rijk_ctx* ctx);
const char* rijk_ctx_last_error(const rijk_ctx* ctx);
const char* rijk_status_string(int status);
/* Sizes of the loaded tensor (0 if none) and device bytes it occupies.  A
 * context keeps its tensor allocation when a smaller tensor replaces a larger
 * one (a set of molecules can reuse one context, largest first); tensor_bytes
 * is the loaded tensor's size, which may be less than the context holds. */
int rijk_ctx_info(const rijk_ctx* ctx, int64_t* num_basis, int64_t* num_auxbas, int64_t* tensor_bytes);
/* The context's CUDA stream (a cudaStream_t). */
void* rijk_ctx_stream(rijk_ctx* ctx);
/* Device pointer of the tile-packed tensor and its row stride in doubles. */
int rijk_ctx_tensor(rijk_ctx* ctx, const double** d_tensor, int64_t* row_stride);
/* Number of CUDA kernels this library has launched in this process (all
 * contexts); a caller can difference it around a region to count launches. */
int64_t rijk_kernel_launches(void);
/* Per-kernel-class CUDA-event timers (REST's TimeRecords, src/utilities/mod.rs:27-84,
 * for device work).  When enabled, every J/K launch is bracketed by events on
 * its own stream.  rijk_ctx_profile_read synchronises, writes the accumulated
 * milliseconds and launch counts of each class (arrays of RIJK_PROF_NCLASS)
 * and resets them. */
enum rijk_prof_class {
  RIJK_PROF_J_PASS1 = 0,    /* w_P = B . D                      */
  RIJK_PROF_J_PASS2 = 1,    /* J = B^T w                        */
  RIJK_PROF_J_OTHER = 2,    /* density folding, reduction       */
  RIJK_PROF_K_HALF = 3,     /* X_P = B_P C (or B_P D)           */
  RIJK_PROF_K_RANK = 4,     /* K += X_P X_P^T                   */
  RIJK_PROF_K_DM = 5,       /* K += (B_P D) B_P                 */
  RIJK_PROF_K_OTHER = 6,    /* operand preparation, reduction   */
  RIJK_PROF_NCLASS = 7
};
/* CTA shapes of the K kernels (results agree to rounding across them), for
 * both the half-transform and the updates; DMMA warps of 32x32 outputs unless noted:
 * 0: 64x64, 4 warps, cp.async staging, 3 stages (2 CTAs/SM); 1: 64x64,
 * cp.async, 2 stages (3 CTAs/SM, the default); 2: 64x64, cp.async, 4 stages
 * (1 CTA/SM); 3: 64x64, bulk copies issued by a producer warp, 3 stages;
 * 4: 128x64, 8 warps, cp.async, 2 stages (2 CTAs/SM); 5: 64x128, 4 warps of
 * 32x64 outputs, cp.async, 2 stages (2 CTAs/SM).  RIJK_HT_CFG / RIJK_RK_CFG
 * override the defaults at context creation. */
#define RIJK_TILE_CFGS 6
int rijk_ctx_set_tiles(rijk_ctx* ctx, int half_transform_cfg, int update_cfg);
int rijk_ctx_get_tiles(const rijk_ctx* ctx, int* half_transform_cfg, int* update_cfg);
/* Autotuner: times every CTA shape of the half-transform and of the rank
 * update on sample_rows aux rows (<= 0: 512) of the loaded tensor with ncols
 * occupied columns, keeps the fastest of each and returns them; ms (if
 * non-NULL, 2 * RIJK_TILE_CFGS doubles) receives {half, update} milliseconds
 * per shape. */
int rijk_ctx_autotune(rijk_ctx* ctx, int64_t ncols, int64_t sample_rows, int* best_half, int* best_update,
                      double* ms);
/* No counterpart in REST.  While pinned != 0 the context never allocates,
 * grows or frees device memory: a call that would need more scratch than it
 * holds fails with RIJK_ERR_TOO_LARGE, and loading a new tensor fails with
 * RIJK_ERR_ARG.  Pin after one warm-up call of each *_dev form and before
 * capturing those calls into a CUDA graph, so that the graph's pointers stay
 * valid for as long as it is replayed. */
int rijk_ctx_pin_buffers(rijk_ctx* ctx, int pinned);
/* No counterpart in REST (its CPU build has no device-side waits).  Every
 * device-side wait in this context's kernels gives up after `nanoseconds` of
 * the GPU's global timer (0 = the default of 2 s; otherwise 10 ms to 600 s);
 * the next synchronising call then returns RIJK_ERR_TIMEOUT and the context
 * stays usable. */
int rijk_ctx_set_wait_budget(rijk_ctx* ctx, int64_t nanoseconds);
/* Runs one bounded wait on a barrier that nothing completes (one CTA, no copy
 * in flight), so that a caller can check that a device-side wait that runs out
 * is reported as RIJK_ERR_TIMEOUT, without any fault, and that the context
 * stays usable.  Returns RIJK_ERR_TIMEOUT when the path works. */
int rijk_ctx_selftest_timeout(rijk_ctx* ctx);
int rijk_ctx_profile(rijk_ctx* ctx, int enable);
int rijk_ctx_profile_read(rijk_ctx* ctx, double* ms, int64_t* launches);
/* Wait for the work enqueued on `stream` (NULL = the context's stream) and
 * report a device-side timeout recorded since the last check. */
int rijk_ctx_synchronize(rijk_ctx* ctx, void* stream);

/* ---- fitted tensor producers ------------------------------------------------ */
/* Load a fitted tensor computed elsewhere.
 * Replaces the SCF::rimatr produced by prepare_rimatr_for_ri_v_rayon_v02
 * (src/molecule_io/mod.rs:1563-1721), consumed by the _rimatr_ functions. */
int rijk_set_rimatr(rijk_ctx* ctx, const double* rimatr, int64_t num_basis, int64_t num_auxbas);
/* Replaces the SCF::ri3fn produced by prepare_ri3fn_for_ri_v_full_rayon
 * (src/molecule_io/mod.rs:1275-1393).  The upper triangle of each B_P is used. */
int rijk_set_ri3fn(rijk_ctx* ctx, const double* ri3fn, int64_t num_basis, int64_t num_auxbas);
/* Download the context's tensor as rimatr (npair x num_auxbas). */
int rijk_get_rimatr(rijk_ctx* ctx, double* rimatr);
/* Tensors produced on the device (e.g. by a device integral engine): allocate a
 * zero tensor for (num_basis, num_auxbas), then load aux rows [p0, p0+np) from
 * device memory, rimatr rows (layout 0, npair doubles each) or ri3fn blocks
 * (layout 1, n*n doubles each).  Same roles as rijk_set_rimatr/_ri3fn. */
int rijk_tensor_alloc(rijk_ctx* ctx, int64_t num_basis, int64_t num_auxbas);
int rijk_tensor_load_rows_dev(rijk_ctx* ctx, const double* d_rows, int64_t p0, int64_t np, int layout,
                              void* stream);

/* Metric step on the device: V = (P|Q) (num_auxbas^2, column-major) is
 * Cholesky-factored, V = L L^T, and the three-centre integrals int3c
 * ((mu nu|P) in rimatr layout) are fitted as B = int3c L^-T.  This is the
 * Cholesky variant REST keeps beside its live V^-1/2 whitening
 * (src/molecule_io/mod.rs:1582-1583, :1672-1675).  On RIJK_ERR_NOT_SPD,
 * *failed_pivot (if non-NULL) holds the 1-based index of the first
 * non-positive pivot; otherwise 0. */
int rijk_build_rimatr_cholesky(rijk_ctx* ctx, const double* aux_v, const double* int3c, int64_t num_basis,
                               int64_t num_auxbas, int64_t* failed_pivot);
/* Fit with a caller-supplied metric factor M (num_auxbas^2, column-major):
 * B = int3c M, i.e. the _dgemm(tmp_ovlp_matr, aux_v) of
 * src/molecule_io/mod.rs:1672-1675 with aux_v = V^-1/2 from lapack_power. */
int rijk_fit_rimatr(rijk_ctx* ctx, const double* metric_factor, const double* int3c, int64_t num_basis,
                    int64_t num_auxbas);

/* ---- Coulomb (J) ------------------------------------------------------------ */
/* vj_upper_with_ri_v_sync (src/scf_io/mod.rs:2428-2488):
 * per P, w_P = sum_{mu,nu} B_P[mu,nu] D[mu,nu]; J = scaling_factor sum_P upper(B_P) w_P.
 * dm: spin_channel x (n x n); vj: spin_channel x npair. */
int rijk_vj_upper_with_ri_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor, double* vj);
/* vj_upper_with_rimatr_v_sync (src/scf_io/mod.rs:2490-2561):
 * w_P = 2 sum_{mu<=nu} B[P,mu nu] D_{mu nu} - sum_mu B[P,mu mu] D_{mu mu}. */
int rijk_vj_upper_with_rimatr_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                double* vj);
/* vj_full_with_ri_v (src/scf_io/mod.rs:2564-2602): full n x n J per spin. */
int rijk_vj_full_with_ri_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor, double* vj_full);

/* ---- exchange (K) ----------------------------------------------------------- */
/* vk_upper_with_ri_v_sync (src/scf_io/mod.rs:2758-2834), occupied-orbital form:
 * per P, X = B_P C[:, :homo+1], K += X diag(occ) X^T; vk = scaling_factor upper(K).
 * eigv: spin_channel x (n x num_state); homo[spin]; occupation: spin_channel x
 * num_state (entries >= 0). */
int rijk_vk_upper_with_ri_v(rijk_ctx* ctx, const double* eigv, int64_t num_state, const int64_t* homo,
                            const double* occupation, int spin_channel, double scaling_factor, double* vk);
/* vk_upper_with_ri_v_use_dm_only_sync (src/scf_io/mod.rs:2640-2701):
 * per P, K += B_P D B_P (both B_P symmetric from their upper triangle). */
int rijk_vk_upper_with_ri_v_use_dm_only(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                        double* vk);
/* vk_upper_with_rimatr_use_dm_only_sync (src/scf_io/mod.rs:2703-2756): the same
 * contraction for a tensor loaded as rimatr. */
int rijk_vk_upper_with_rimatr_use_dm_only(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                          double* vk);
/* vk_full_fromdm_with_ri_v (src/scf_io/mod.rs:2603-2638): K = sum_P B_P D B_P^T
 * for an arbitrary (possibly non-symmetric) D; full n x n output per spin. */
int rijk_vk_full_fromdm_with_ri_v(rijk_ctx* ctx, const double* dm, int spin_channel, double scaling_factor,
                                  double* vk_full);

/* ---- device-resident forms (same semantics, device pointers) ----------------- */
/* dm_mode 0 = rijk_vj_upper_with_ri_v, 1 = rijk_vj_upper_with_rimatr_v. */
int rijk_vj_upper_dev(rijk_ctx* ctx, const double* d_dm, int spin_channel, double scaling_factor, int dm_mode,
                      double* d_vj, void* stream);
/* d_homo is a host array; d_eigv / d_occupation / d_vk are device arrays. */
int rijk_vk_upper_occ_dev(rijk_ctx* ctx, const double* d_eigv, int64_t num_state, const int64_t* homo,
                          const double* d_occupation, int spin_channel, double scaling_factor, double* d_vk,
                          void* stream);
int rijk_vk_upper_dm_dev(rijk_ctx* ctx, const double* d_dm, int spin_channel, double scaling_factor, double* d_vk,
                         void* stream);
/* J and K together from the occupied orbitals, as REST's SCF asks for them
 * (generate_hf_hamiltonian_ri_v, src/scf_io/mod.rs:1339-1381, which calls
 * vj_upper_with_ri_v_sync on dm = C diag(occ) C^T and vk_upper_with_ri_v_sync on
 * C).  dm_s = C_s[:, :homo+1] diag(occ_s) C_s[:, :homo+1]^T (REST's density
 * matrix where the states above homo are empty); d_vj = j_scaling_factor
 * upper(J[dm_s]) per spin, equal to rijk_vj_upper_dev(dm_mode 0) on that dm;
 * d_vk as rijk_vk_upper_occ_dev (occupations >= 0).  J's
 * per-aux-row scalars B_P : dm_s come out of the K half-transform, so the build
 * reads the tensor once for K and once for J instead of once for K and twice
 * for J. */
int rijk_vjk_upper_occ_dev(rijk_ctx* ctx, const double* d_eigv, int64_t num_state, const int64_t* homo,
                           const double* d_occupation, int spin_channel, double j_scaling_factor,
                           double k_scaling_factor, double* d_vj, double* d_vk, void* stream);
/* Host-pointer form of rijk_vjk_upper_occ_dev (inputs as rijk_vk_upper_with_ri_v;
 * vj and vk: spin_channel x npair each). */
int rijk_vjk_upper_with_ri_v(rijk_ctx* ctx, const double* eigv, int64_t num_state, const int64_t* homo,
                             const double* occupation, int spin_channel, double j_scaling_factor,
                             double k_scaling_factor, double* vj, double* vk);

/* ---- split-precision exchange on the 5th-generation tensor cores -------------- */
/* Same contraction as rijk_vk_upper_occ_dev (REST vk_upper_with_ri_v_sync,
 * src/scf_io/mod.rs:2758-2834) with every FP64 operand split into two BF16
 * parts and three tcgen05 products per pair accumulated in FP32 (relative
 * error about 1e-5 of |K|).  The first call after a tensor change builds BF16
 * hi / lo copies of the tensor (4 bytes per element of the upper 128 x 128
 * squares of each B_P). */
int rijk_vk_upper_occ_split_dev(rijk_ctx* ctx, const double* d_eigv, int64_t num_state, const int64_t* homo,
                                const double* d_occupation, int spin_channel, double scaling_factor, double* d_vk,
                                void* stream);
/* Low-rank form: d_vk (+)= scaling_factor * sum_P (B_P V) S (B_P V)^T with
 * S = +1 on columns [0, npos) and -1 on [npos, ncols) of V (n x ncols,
 * column-major, leading dimension ld_v even, 16-byte aligned).  With V the
 * signed square-root factor of a density difference dD = V S V^T this is the
 * exchange matrix of dD, whose split-precision error shrinks with |dD|. */
int rijk_vk_upper_lowrank_split_dev(rijk_ctx* ctx, const double* d_V, int64_t ld_v, int64_t ncols, int64_t npos,
                                    double scaling_factor, int accumulate, double* d_vk, void* stream);
/* J and K of the same difference: as rijk_vk_upper_lowrank_split_dev for d_vk,
 * and d_vj = j_scaling_factor * upper(J[dD]) (always overwritten), whose per-aux-
 * row scalars B_P : dD = sum_c S_c <V_c, (B_P V)_c> come out of the split
 * half-transform's epilogue (FP32 accumulators against V in FP64), followed by
 * one FP64 pass over the tensor.  For incremental builds J_k = J_ref + J[dD]
 * in which, as for K, the split error shrinks with |dD|. */
int rijk_vjk_upper_lowrank_split_dev(rijk_ctx* ctx, const double* d_V, int64_t ld_v, int64_t ncols, int64_t npos,
                                     double j_scaling_factor, double k_scaling_factor, int accumulate, double* d_vj,
                                     double* d_vk, void* stream);

/* ---- grouped build over a molecule set ----------------------------------------- */
/* No single counterpart in REST: REST builds J and K one SCF at a time
 * (vj_upper_with_rimatr_v_sync + vk_upper_with_ri_v_sync, src/scf_io/mod.rs:
 * 2490-2561, 2758-2834); a group runs that build for many molecules (one
 * context each, tensors loaded) in six launches for all of them, the two
 * tensor-core phases as persistent kernels over work items (molecule, aux row,
 * tile); J's aux-row scalars come out of the half-transform phase, so J reads
 * each tensor once.  nocc[m]: doubly occupied orbitals of molecule m.  The CTA shapes are
 * 0, 1 or 4 of rijk_ctx_set_tiles (the caller's autotuner picks them).  The
 * group owns the scratch of all molecules (one allocation at creation); its
 * contexts must stay loaded and unchanged while it exists (a call after one of
 * them loaded another tensor returns RIJK_ERR_ARG). */
typedef struct rijk_group rijk_group;
int rijk_group_create(rijk_ctx* const* ctxs, int count, const int64_t* nocc, int half_transform_cfg, int update_cfg,
                      rijk_group** out);
int rijk_group_destroy(rijk_group* group);
/* For every molecule m with d_active[m] != 0 (device int array):
 *   out_m = J(D_m) + k_scale K(C_m),  D_m = 2 C_m C_m^T over the nocc[m] columns,
 * written full and symmetric (n_m x n_m) at d_out + m out_mol with row stride ldo;
 * C_m(mu, i) = d_C[m c_mol + mu c_row + i c_col].  J is REST's rimatr J (a2),
 * K the occupied-orbital K (a3, occupation 2; k_scale = -0.5 for RHF).
 * Enqueued on `stream` without synchronising: the pointers may be captured in a
 * CUDA graph and the active flags changed between replays. */
int rijk_group_jk_occ_dev(rijk_group* group, const double* d_C, int64_t c_mol, int64_t c_row, int64_t c_col,
                          double k_scale, const int* d_active, double* d_out, int64_t out_mol, int64_t ldo,
                          void* stream);
/* Wait for `stream` and report a device-side timeout of the group's kernels. */
int rijk_group_synchronize(rijk_group* group, void* stream);

/* ---- batched symmetric eigensolver (FP64) ------------------------------------- */
/* The Fock diagonalisation of REST's SCF (diagonalize_hamiltonian,
 * src/scf_io/mod.rs:1843-1873, LAPACK dspgvx) for a batch of matrices already in
 * standard form (the batched driver forms X^T F X on the device).  d_a: batch
 * row-major ld x ld symmetric matrices (overwritten); matrix b uses its leading
 * d_nvalid[b] rows and columns (device int32).  Outputs: d_w (batch x ld)
 * eigenvalues ascending, then pad_value for the padding; d_v (batch x ld x ld,
 * row-major) eigenvectors as columns, unit vectors for the padding; d_work:
 * batch x ld x ld doubles; d_info[b] = 1 where an eigenvalue did not converge in
 * 30 QL sweeps (0 otherwise).  ld <= 768, else RIJK_ERR_TOO_LARGE.  One CTA per
 * matrix: Householder tridiagonalisation, explicit Q, implicit-shift QL. */
int rijk_eigh_batched_dev(double* d_a, int64_t ld, const int32_t* d_nvalid, int64_t batch, double pad_value,
                          double* d_w, double* d_v, double* d_work, int32_t* d_info, void* stream);

/* ---- batched DIIS coefficients (FP64) ------------------------------------------- */
/* REST's diis_solver (src/scf_io/mod.rs:3138-3188) for a batch of molecules:
 * d_gram: batch row-major m x m Gram matrices <e_i, e_j> of the error vectors
 * (device); molecule b uses its leading k = min(d_count[b], m) rows and columns
 * (d_count device int32; k = 0 writes zero coefficients).  d_coef (batch x m):
 * c = x / sum(x) with B x = 1, i.e. REST's row sums of B^-1 over their total.
 * Where B is exactly singular (a zero pivot of LU with partial pivoting, REST's
 * _dinverse failure) or the result is not finite, d_status[b] = 1 and the
 * coefficients are (1, 0, ..., 0): the caller restarts that history from its
 * newest Fock matrix, stored in slot 0.  m <= 32, else RIJK_ERR_TOO_LARGE. */
int rijk_diis_coefficients_dev(const double* d_gram, int64_t m, const int32_t* d_count, int64_t batch,
                               double* d_coef, int32_t* d_status, void* stream);

/* ---- J without any device allocation ----------------------------------------- */
/* No counterpart in REST.  Same result as rijk_vj_upper_dev for callers that
 * cannot let a library call cudaMalloc (their device memory is owned by another
 * allocator or a fixed arena, or a cudaMalloc between builds would synchronise
 * their pipeline).  Inputs and outputs are the caller's device pointers:
 * d_tensor/row_stride as returned by rijk_ctx_tensor for a loaded tensor;
 * d_dm, d_vj as in rijk_vj_upper_dev; the work is enqueued on `stream`.
 * Scratch lives in one static device array of RIJK_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until exit; sizes needing more
 * (2 spin ldB + spin N doubles: n <= 2016 for spin 1 and n <= 1408 for
 * spin 2 at N = 4n) return RIJK_ERR_TOO_LARGE.  The first call on a device
 * looks the array's address up (cudaGetSymbolAddress) and caches it by device
 * ordinal; make that first call before any stream capture.  The current device
 * at the call must be the device the pointers and the stream belong to, and the
 * library must not be used across a cudaDeviceReset of that device.  All calls
 * share the array: calls that overlap on the GPU race and must be serialised
 * by the caller.  An error already pending in the CUDA runtime when the call
 * starts is returned as RIJK_ERR_CUDA and left pending. */
#define RIJK_NOALLOC_SCRATCH_BYTES (32ull << 20)
int rijk_vj_upper_noalloc(const double* d_tensor, int64_t row_stride, int64_t num_basis, int64_t num_auxbas,
                          const double* d_dm, int spin_channel, double scaling_factor, int dm_mode, double* d_vj,
                          void* stream);

/* ---- integrals (host, OpenMP) ----------------------------------------------- */
/* Contracted Gaussian shells in plain arrays.  Shell s has angular momentum
 * l[s] (<= 6), nprim[s] primitives at exps/coefs[prim_off[s] ...], and centre
 * centers[3s..3s+2] in bohr.  coefs multiply unnormalised Cartesian
 * primitives x^i y^j z^k exp(-a r^2) and carry the caller's normalisation.
 * Functions are real solid harmonics: c2s[l] is the (2l+1) x (l+1)(l+2)/2
 * row-major transform for each l (Cartesian components ordered by descending
 * x power, then descending y power). */
typedef struct rijk_shells {
  int64_t nshell;
  const int32_t* l;
  const int32_t* nprim;
  const int64_t* prim_off;
  const double* exps;
  const double* coefs;
  const double* centers;
} rijk_shells;
/* Replaces libcint's int1e_ovlp / int1e_kin / int1e_nuc (kind 0 / 1 / 2) as
 * called by Molecule::int_ij_matrixupper (src/molecule_io/mod.rs:700-812).
 * out: n x n column-major.  kind 2 sums -Z_A / |r - R_A| over natom atoms. */
int rijk_int1e(const rijk_shells* bas, const double* const* c2s, int kind, int natom, const double* charges,
               const double* coords, double* out);
/* Replaces the cint_2c2e loop of int_ij_aux_columb_rayon (src/molecule_io/mod.rs:1072-1103):
 * V = (P|Q), naux x naux column-major. */
int rijk_int2c2e(const rijk_shells* aux, const double* const* c2s, double* out);
/* Replaces the cint_3c2e loop of prepare_rimatr_for_ri_v_rayon_v02
 * (src/molecule_io/mod.rs:1611-1660): (mu nu|P) in rimatr layout [npair, naux]. */
int rijk_int3c2e(const rijk_shells* bas, const rijk_shells* aux, const double* const* c2s, double* out);

/* ---- integrals (device) -------------------------------------------------------- */
/* The same integrals computed on the current CUDA device into device memory,
 * for AO shells with l <= 2 and auxiliary shells with l <= 4
 * (RIJK_ERR_TOO_LARGE otherwise); c2s must hold the matrices for l = 0..4.
 * They replace the libcint loops of int_ij_aux_columb (src/molecule_io/mod.rs:1038)
 * and prepare_rimatr_for_ri_v_rayon_v02 (src/molecule_io/mod.rs:1604-1660).
 * Both return after the results are complete on `stream` (NULL: legacy default
 * stream).  Calls from several host threads at once must be serialised. */
int rijk_int2c2e_dev(const rijk_shells* aux, const double* const* c2s, double* d_out, void* stream);
int rijk_int3c2e_dev(const rijk_shells* bas, const rijk_shells* aux, const double* const* c2s, double* d_out,
                     void* stream);
/* prepare_rimatr_for_ri_v_rayon_v02 (src/molecule_io/mod.rs:1563-1721) with
 * every step on the device: (P|Q) and (mu nu|P) from the device integral
 * engine (limits above), then the metric step.  metric_factor NULL: Cholesky
 * fit as in rijk_build_rimatr_cholesky (failed_pivot as there); otherwise the
 * host num_auxbas^2 factor M is applied, B = (mu nu|P) M, as rijk_fit_rimatr
 * does with REST's V^-1/2.  The tensor is left loaded in the context. */
int rijk_build_rimatr_from_shells(rijk_ctx* ctx, const rijk_shells* bas, const rijk_shells* aux,
                                  const double* const* c2s, const double* metric_factor, int64_t* failed_pivot);

/* ---- learned initial guess: per-atom-pair MLP kernels ----------------------------
 * No counterpart in REST, whose guesses (src/initial_guess/mod.rs) remain the
 * fallback of the driver that uses them.  Device pointers; BF16 values are
 * passed as uint16_t bit patterns; matrices are row-major; act 0 = identity,
 * 1 = SiLU.  Launches are asynchronous on `stream`.
 * Forward of one layer: z = x w^T + bias (m x n, FP32 accumulation), y = act(z);
 * any of z (FP32), y_bf16, y_f32 may be NULL but not all. */
int rijk_mlp_linear_fwd(const uint16_t* x, const uint16_t* w, const float* bias, int64_t m, int64_t k, int64_t n,
                        int act, float* z, uint16_t* y_bf16, float* y_f32, void* stream);
/* Backward of one layer from dy = dL/dy (m x n, FP32) and the forward's z:
 * dz = dy * act'(z) (into dz_scratch, BF16, m x n), dw = dz^T x (n x k, FP32),
 * db = column sums of the FP32 dz (n, may be NULL), dx = dz w (m x k, FP32, may be NULL).
 * dw, db, dx are overwritten (the split-k sums use FP32 atomics). */
int rijk_mlp_linear_bwd(const uint16_t* x, const uint16_t* w, const float* z, const float* dy, int64_t m, int64_t k,
                        int64_t n, int act, uint16_t* dz_scratch, float* dw, float* db, float* dx, void* stream);
/* loss += sum_e (mask_e (y_e - t_e))^2 / norm; dy_e = 2 mask_e (y_e - t_e) / norm
 * (mask may be NULL = all ones; loss may be NULL). */
int rijk_mlp_masked_mse(const float* y, const float* t, const float* mask, int64_t count, double norm, float* dy,
                        float* loss, void* stream);
/* Adam step `step` (1-based) on FP32 master weights w with moments m, v; the
 * BF16 copy w_bf16 (may be NULL) is refreshed. */
int rijk_mlp_adam(float* w, uint16_t* w_bf16, const float* g, float* m, float* v, int64_t count, double lr,
                  double beta1, double beta2, double eps, int64_t step, void* stream);
int rijk_mlp_to_bf16(const float* src, uint16_t* dst, int64_t count, void* stream);
/* Density assembly of the learned guess (no counterpart in REST).  y: the
 * network output, npairs_ordered x 196 FP32 (standardised 14 x 14 local blocks,
 * row-major); t_mean, t_std: 4 x 196 (per element-pair kind = 2 type(A) +
 * type(B)); upairs: 4 int32 per unordered atom pair A <= B within the cutoff
 * (A, B, row of (A, B) in y, row of (B, A) in y); per atom its first AO, element
 * type (0, 1), AO count (<= 14) and water index; rot: per water and element the
 * 14 x 14 rotation G of that element's AO block into the water's frame.  Writes
 * dm (num_basis^2, device): D_AB = 1/2 (G_A P_AB G_B^T |frame of A's water +
 * G_A P_BA^T G_B^T |frame of B's water), D_BA = D_AB^T, zero beyond the cutoff.
 * A pair with an atom of more than 14 AOs or a type other than 0 / 1 is skipped. */
int rijk_guess_assemble(const float* y, const float* t_mean, const float* t_std, const int32_t* upairs,
                        int64_t npairs, const int32_t* atom_first, const int32_t* atom_type, const int32_t* atom_nfun,
                        const int32_t* atom_water, const double* rot, int64_t num_basis, double* dm, void* stream);
/* Geometry of the learned guess for a set of water clusters (no counterpart in
 * REST), all device pointers.  xyz: natom x 3 (A), molecule after molecule,
 * each molecule O, H, H per water; atom_info: 3 int32 per atom (global index of
 * its molecule's first atom, the molecule's atom count, element type 0 = O /
 * 1 = H); table: the 516 constants (40 sample points x 3; for l = 1 then 2 the
 * Cartesian exponents, the c2s expansion transposed (ncart x (2l+1)) and the
 * pseudo-inverse of the harmonics at the samples ((2l+1) x 40); cutoff, radial
 * width, 8 radial centres); elem_shells: per element type 16 int32 (shell
 * count, then each shell's l, l <= 2, at most 14 functions).  Writes per water
 * its frame (frames, 9: rows p, b, n) and per water and element the 14 x 14
 * block rotation (rot, as rijk_guess_assemble reads it); per atom the number of
 * atoms of its molecule within the cutoff (counts[2a], itself included) and of
 * those with index >= a (counts[2a+1]), and its 16 radial counts (env). */
int rijk_guess_geometry(const double* xyz, const int32_t* atom_info, int64_t natom, const double* table,
                        const int32_t* elem_shells, double* frames, double* rot, int64_t* counts, double* env,
                        void* stream);
/* The pair rows of the learned guess from rijk_guess_geometry's output:
 * pair_off / up_off are the exclusive scans of counts[2a] / counts[2a+1]
 * (natom each), npairs / nup their totals.  Writes feats (npairs x 53, FP32,
 * (feature - f_mean) / f_std) for the ordered pairs (A, B) within the cutoff,
 * atom by atom in ascending B, and upairs (nup x 4 int32: A, B, row of (A, B),
 * row of (B, A), all relative to the molecule's first atom and first pair row),
 * the input of rijk_guess_assemble for each molecule. */
int rijk_guess_pairs(const double* xyz, const int32_t* atom_info, int64_t natom, const double* table,
                     const double* frames, const double* env, const int64_t* pair_off, const int64_t* up_off,
                     int64_t npairs, int64_t nup, const double* f_mean, const double* f_std, float* feats,
                     int32_t* upairs, void* stream);

/* ---- MO-basis three-centre tensor -------------------------------------------- */
/* generate_ri3mo_rayon / ao2mo_rayon (src/scf_io/mod.rs:2331-2359, :3270-3307):
 * ri3mo[P, a, i] = sum_{mu,nu} C[mu, a] B_P[mu, nu] C[nu, i] for a in
 * [row_begin, row_end), i in [col_begin, col_end); output per spin is REST's
 * RIFull[num_auxbas, nrow, ncol] (P fastest), spin after spin.  eigv:
 * spin_channel x (n x num_state). */
int rijk_ao2mo(rijk_ctx* ctx, const double* eigv, int64_t num_state, int64_t row_begin, int64_t row_end,
               int64_t col_begin, int64_t col_end, int spin_channel, double* ri3mo);

/* ---- SCF pieces around the build ------------------------------------------- */
/* generate_density_matrix (src/scf_io/mod.rs:441-478): D = (C occ) C^T over the
 * first homo+1 columns, per spin; dm: spin_channel x (n x n). */
int rijk_density_matrix(rijk_ctx* ctx, const double* eigv, int64_t num_basis, int64_t num_state,
                        const int64_t* homo, const double* occupation, int spin_channel, double* dm);
/* SCF::par_energy_contraction (src/scf_io/mod.rs:1787-1802):
 * 1/2 sum_ij a_ij b_ij from two MatrixUpper of length npair. */
double rijk_energy_contraction(const double* a_upper, const double* b_upper, int64_t npair);

#ifdef __cplusplus
}
#endif

#endif /* REST_B200_H */
