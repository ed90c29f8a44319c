// Host-side launchers of the RI J/K kernels (internal to librest_b200.so).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rest_b200.h"

namespace rijk {

// Geometry of the tile-packed tensor held by a context.
struct Geom {
  int64_t n = 0;      // num_basis
  int64_t naux = 0;   // num_auxbas
  int64_t nt = 0;     // ceil(n / 32)
  int64_t ntp = 0;    // nt (nt + 1) / 2
  int64_t ldB = 0;    // ntp * 1024 doubles per aux row
  int64_t npair = 0;  // n (n + 1) / 2
  int ht_cfg = 1;     // CTA shape of the half-transform (0..3)
  int rk_cfg = 1;     // CTA shape of the rank / dm updates (0..3)
};
Geom make_geom(int64_t n, int64_t naux);

// Process-wide count of kernels this library has launched (every launch_*
// and run_* helper adds the launches it issues).
void count_launch(int64_t k = 1);
int64_t launch_count();

// --- layout conversion -------------------------------------------------------
// rimatr (REST MatrixFull[npair, N], column P = packed upper of B_P), rows
// [p0, p0 + np) -> tile-packed rows [p0, p0 + np) of dB.
void launch_pack_rimatr(const Geom& g, const double* src, int64_t np, double* dst, cudaStream_t st);
// ri3fn (REST RIFull[n,n,N]), aux rows [p0, p0+np): upper triangle is the source.
void launch_pack_ri3fn(const Geom& g, const double* src, int64_t np, double* dst, cudaStream_t st);
// tile-packed rows -> rimatr rows.
void launch_unpack_rimatr(const Geom& g, const double* src, int64_t np, double* dst, cudaStream_t st);

// --- J ------------------------------------------------------------------------
// mode 0: full n*n dot (vj_upper_with_ri_v); mode 1: packed-upper formula
// (vj_upper_with_rimatr_v).  dm: nspin matrices n*n column-major, stride n*n.
// One CTA waits (bounded by the context's budget) on an mbarrier that nothing
// completes, and records DEV_WAIT_TIMEOUT: the timeout path without a fault.
void launch_wait_selftest(int* err, cudaStream_t st);
void launch_j_weights(const Geom& g, const double* dm, int nspin, int mode, double* W, int* err, cudaStream_t st);
// w[s*naux + P] = sum_k B[P,k] W[s*ldB + k]
void launch_j_pass1(const Geom& g, const double* B, const double* W, int nspin, double* w, cudaStream_t st);
// number of P-splits pass 2 uses (scratch = splits * nspin * ldB doubles)
int j_pass2_splits(const Geom& g);
void launch_j_pass2(const Geom& g, const double* B, const double* w, int nspin, int splits, double* Jpart,
                    cudaStream_t st);
// out_kind 0: packed upper (nspin x npair); 1: full n x n (nspin x n*n)
void launch_j_finalize(const Geom& g, const double* Jpart, int nspin, int splits, double scale, int out_kind,
                       double* out, cudaStream_t st);

// --- K ------------------------------------------------------------------------
// Cw[s] (ldc x ocols, column-major, zero padded) = C_s[:, :nw_s] * sqrt(occ_s)
void launch_k_prepare_c(const Geom& g, const double* eigv, int64_t ld_eigv, int64_t stride_eigv,
                        const double* occ, int64_t stride_occ, const int64_t* nw, int nspin, int64_t ldc,
                        int64_t ocols, double* Cw, int* err, cudaStream_t st);
// dense n x n (ld = n) -> padded ldc x ldc copy (zero padding)
void launch_pad_square(const double* src, int64_t n, int64_t ldsrc, int64_t ldc, double* dst, int* err,
                       cudaStream_t st);

// Where the half-transform stores column c of X_p = B_p W (p counted from the
// chunk's first aux row): at column dst(p, c) of X (leading dimension ldx), or
// nowhere when dst is negative.  Columns [0, lim_a) go to block a with per-row
// stride pstride_a; columns [coff_b, coff_b + lim_b) to block b, which starts at
// column base_b, with stride pstride_b.
struct XMap {
  int64_t pstride_a;
  int lim_a;
  int coff_b, lim_b;
  int64_t base_b, pstride_b;
  // every W column of every aux row at stride ncol (X_p is an ldx x ncol block)
  static XMap dense(int64_t ncol) { return {ncol, (int)ncol, 0, 0, 0, 0}; }
  __host__ __device__ int64_t dst(int64_t p, int c) const {
    if (c < lim_a) return p * pstride_a + c;
    if (c >= coff_b && c < coff_b + lim_b) return base_b + p * pstride_b + (c - coff_b);
    return -1;
  }
};

// X_p = B_{p0+p} * W for p in [0, np): W is ldw x ncol (ncol a multiple of 64);
// ldx = round_up(n, 128); the columns land where xm says.  Columns at or beyond
// ncol_valid of W are zero and their fragments are skipped.
// With wpart (scratch of 2 doubles per consumer warp, half_transform_warps of
// them) the launch also writes J's scalars w[s][p0 + p] = B_p : D_s for the aux
// rows of the chunk (D_s = W_s W_s^T; spin 1 = the columns from coff1 on).
int64_t half_transform_warps(const Geom& g, int64_t np, int64_t ldx, int64_t ncol);
void launch_half_transform(const Geom& g, const double* B, int64_t p0, int64_t np, const double* W, int64_t ldw,
                           int64_t ncol, int64_t ncol_valid, double* X, int64_t ldx, const XMap& xm, int* err,
                           cudaStream_t st, double* wpart = nullptr, double* w = nullptr, int nspin = 1,
                           int coff1 = 1 << 30);
// Kpart[split][q] (128x128 blocks q over block pairs) = sum over the aux rows p
// of the split of X_p X_p^T, where X holds X_p's nw columns at columns
// [p nw, (p + 1) nw) (leading dimension ldx; the 32 columns after the last row
// must be readable).  full = 0: pairs Ib<=Jb; 1: all pairs.
int k_rank_splits(const Geom& g, int64_t np, int full);
void launch_k_rank_update(const Geom& g, const double* X, int64_t ldx, int64_t np, int64_t nw, int splits, int full,
                          double* Kpart, int* err, cudaStream_t st);
// Kpart[split][q] = sum_p T_p B_{p0+p}  (dm form: T_p = B_p D)
void launch_k_dm_update(const Geom& g, const double* T, int64_t ldt, int64_t stp, const double* B, int64_t p0,
                        int64_t np, int splits, int full, double* Kpart, int* err, cudaStream_t st);
int64_t k_block_pairs(const Geom& g, int full);
// out (+)= scale * sum_split Kpart; out_kind 0: packed upper, 1: full n x n.
void launch_k_finalize(const Geom& g, const double* Kpart, int splits, int full, double scale, int accumulate,
                       int out_kind, double* out, cudaStream_t st);

// --- split-precision exchange on tcgen05 (rijk_tc.cu) --------------------------
struct TcGeom {
  int nmb = 0;   // 128-row blocks of n
  int nkb = 0;   // 64-wide K blocks of n
  int npad = 0;  // column count padded to 64 / 128 / 256
  int nib = 0;   // npad / 64
  int64_t block_elems = 0;
  int pair = 0;       // half-transform on SM pairs (cta_group::2); V stored in column halves
  int pair_rank = 0;  // rank update on SM pairs (cta_group::2)
  int ncols = 0;      // V columns actually used
  int nv = 0;         // V rows per K block as laid out: the paired half-transform's MMA width
                      // (ncols rounded up to 16, in two halves), else npad
};
TcGeom make_tc_geom(const Geom& g, int ncols);
// BF16 elements of one plane (hi or lo) of the split tensor
int64_t tc_tensor_elems(const Geom& g);
void launch_split_tensor(const Geom& g, const double* B, int64_t p0, int64_t np, void* hi, void* lo, cudaStream_t st);
void launch_split_cols(const Geom& g, const TcGeom& t, const double* V, int64_t ldv, int ncols, void* hi, void* lo,
                       cudaStream_t st);
// X (np x nmb x nib blocks, hi/lo) = B_{p0..p0+np} V
// J's scalars from the split half-transform: w[p0 + p] += sgn <V, X_p> with V the
// FP64 columns (ldv x ncols, column c at Vd + c ldv) the launch multiplies by.
struct TcJ {
  const double* Vd;
  int64_t ldv;
  int ncols;
  double sgn;
  double* wpart;  // 4 nmb doubles per aux row of the chunk
  double* w;      // [naux]
};
void launch_half_tc(const Geom& g, const TcGeom& t, const void* Bhi, const void* Blo, int64_t p0, int64_t np,
                    const void* Vhi, const void* Vlo, void* Xhi, void* Xlo, int* err, cudaStream_t st,
                    const TcJ* jw = nullptr);
int tc_rank_splits(const TcGeom& t, int64_t np);
// part[split][pair][128x128] = sum_p X_p S X_p^T (S = -1 on blocks >= npos_blocks)
void launch_rank_tc(const Geom& g, const TcGeom& t, const void* Xhi, const void* Xlo, int64_t np, int npos_blocks,
                    int splits, float* part, int* err, cudaStream_t st);
void launch_rank_tc_finalize(const Geom& g, const TcGeom& t, const float* part, int splits, double scale,
                             int accumulate, double* out, cudaStream_t st);

// --- grouped build over a molecule set ---------------------------------------
// One molecule of a group (device-resident descriptor).
struct GroupMol {
  const double* B;  // tile-packed tensor of the molecule's context
  int64_t ldB;
  int n, nt, naux, nocc;
  double* Cw;       // sqrt(2) C, ldx x ocols, column-major
  int64_t ldx;
  int ocols;        // a multiple of the half-transform CTA width
  int ncb;          // column blocks launched (ocols / width, or the full blocks with remainder columns)
  int xcol0;        // > 0: columns [xcol0, nocc) are remainder columns of the last full block
  double* wpart;    // J scalars per half-transform warp: naux x (ldx / BM) x (ocols / BN) x warps
  int wper;         // wpart entries per aux row
  double* w;        // J scalars (naux)
  double* Jpart;    // jsplits x ldB
  int jsplits;
  double* X;        // ldx x (naux nocc + 32)
  double* Kpart;    // ksplits x pairs x 128 x 128
  int ksplits;
  int64_t nkb, pairs, npair;
};
// Work enumeration of the six phases: pre[phase] (device, count entries) are
// the prefix sums of each molecule's items, total[phase] their sum.
struct GroupPlan {
  GroupMol* mols;
  int count;
  int64_t* pre[6];
  int64_t total[6];
  int ht_cfg, rk_cfg;
  int remainder;  // some molecule has remainder columns (the half-transform variant that computes them)
};
int group_cta_rows(int cfg);
int group_cta_cols(int cfg);
int group_rank_subs(int cfg);
int group_cta_warps(int cfg);
int group_remainder_cols(int cfg);  // remainder columns the half-transform shape computes in its last full block
// out[m] (ldo-strided, full and symmetric) = J(2 C_m C_m^T) + k_scale K(C_m) for
// every molecule m with active[m] != 0; molecule m's orbitals C(mu, i) at
// C0[m c_mol + mu c_row + i c_col] (occupation 2 for i < nocc).
void launch_group(const GroupPlan& gp, const double* C0, int64_t c_mol, int64_t c_row, int64_t c_col, double k_scale,
                  double* out0, int64_t out_mol, int64_t ldo, const int* active, int* err, int sms, cudaStream_t st);

// --- ri3mo ---------------------------------------------------------------------
// out (ldo x ncp, zero padded) = C[:, c0 : c0 + nc]
void launch_gather_cols(const double* C, int64_t n, int64_t ldc_in, int64_t c0, int64_t nc, int64_t ldo, int64_t ncp,
                        double* out, cudaStream_t st);
// out[p + np (a + nrow i)] = Y[p * sy + a + ldy i]
void launch_ri3mo_permute(const double* Y, int64_t ldy, int64_t sy, int64_t np, int64_t nrow, int64_t ncol,
                          double* out, cudaStream_t st);

// --- dense FP64 GEMM on the DMMA mainloop (metric step) -----------------------
// C[MxN] = alpha op(A) op(B) + beta C, all column-major, M,N,K multiples of 32,
// pointers 16-byte aligned, leading dimensions even.  klim: bit 0 = op(A)
// lower (k <= m), bit 1 = op(B) upper (k <= n), bit 2 = op(A) upper (k >= m),
// bit 3 = op(B) lower (k >= n).  lower_only: skip C blocks above the diagonal.
// batch: gridDim.z copies with element offsets sa, sb, sc between them.
void launch_dgemm(int64_t M, int64_t N, int64_t K, double alpha, const double* A, int64_t lda, int ta,
                  const double* B, int64_t ldb, int tb, double beta, double* C, int64_t ldc, int klim, int lower_only,
                  int batch, int64_t sa, int64_t sb, int64_t sc, int* err, cudaStream_t st);

// --- metric -----------------------------------------------------------------
// In-place lower Cholesky of the np x np (np multiple of 32) matrix A (lda).
// Linvd receives the inverses of the 32x32 diagonal blocks.  *d_info = first
// failing pivot (1-based) or 0.
void run_potrf(double* A, int64_t np, int64_t lda, double* Linvd, int* d_info, int* err, cudaStream_t st);
// Linv (np x np, ld) = inverse of the lower-triangular L (ld); T is np x np scratch.
void run_trtri(const double* L, int64_t np, int64_t ld, const double* Linvd, double* Linv, double* T, int* err,
               cudaStream_t st);
// Copy a dense n x n (ld n) matrix into a zero-padded np x np (ld np) buffer.
void launch_pad_matrix(const double* src, int64_t n, int64_t np, double* dst, cudaStream_t st);

// --- device integral engine (rijk_ints_gpu.cu) ------------------------------------
// A plan holds the device copy of an AO shell set (may be null: metric only)
// and an auxiliary shell set, and loads the c2s table after `st` drains.
struct RiIntPlan;
int ri_plan_create(const rijk_shells* bas, const rijk_shells* aux, const double* const* c2s, cudaStream_t st,
                   RiIntPlan** out);
void ri_plan_destroy(RiIntPlan* p);
int64_t ri_plan_nbas(const RiIntPlan* p);
int64_t ri_plan_naux(const RiIntPlan* p);
int ri_plan_aux_shells(const RiIntPlan* p);
int64_t ri_plan_aux_offset(const RiIntPlan* p, int k);  // first function of auxiliary shell k (k <= nshell)
// (P|Q) into dV (naux x naux, column-major, leading dimension ldv)
void launch_int2c2e(const RiIntPlan* p, double* dV, int64_t ldv, cudaStream_t st);
// (mu nu|P) for the auxiliary shells [k0, k1): rimatr rows starting at the first function of k0
void launch_int3c2e(const RiIntPlan* p, int k0, int k1, double* out, cudaStream_t st);

}  // namespace rijk
