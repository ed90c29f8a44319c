// RI metric step in FP64 on the DMMA mainloop: the Cholesky factor of the
// auxiliary Coulomb metric V = (P|Q) = L L^T, its triangular inverse, and the
// fit B^T = L^-1 (Q|mu nu) that produces the tensor the J/K kernels read.
//
// REST whitens with V^-1/2 (lapack_power(-0.5, 1e-8), src/molecule_io/mod.rs:1582)
// and keeps the Cholesky form commented out beside it (:1583).  J and K depend on
// B only through B^T B = (mu nu|P) V^-1 (P|la si), so any factor M with M M^T = V^-1
// gives the same Fock matrix; the C ABI also accepts a caller-supplied factor
// (e.g. REST's V^-1/2) and applies it with the same GEMM.
#include <math.h>

#include <algorithm>

#include "rijk_dmma.cuh"
#include "rijk_internal.h"

namespace rijk {

static inline int64_t cdiv_m(int64_t a, int64_t b) { return (a + b - 1) / b; }

struct GemmSched {
  const double* A;
  int64_t lda;
  int ta;
  const double* B;
  int64_t ldb;
  int tb;
  int64_t m0, n0;
  int kt0;
  int64_t Mv, Nv;
  __device__ SlotSrc a(int kt, int mt) const {
    const int64_t m = m0 + mt * TS;
    if (m >= Mv) return {nullptr, TS, 0};
    const int64_t k0 = (int64_t)(kt0 + kt) * TS;
    if (ta == 0) return {A + m + k0 * lda, lda, 0};
    return {A + k0 + m * lda, lda, 1};
  }
  __device__ SlotSrc b(int kt, int ntl) const {
    const int64_t n = n0 + ntl * TS;
    if (n >= Nv) return {nullptr, TS, 0};
    const int64_t k0 = (int64_t)(kt0 + kt) * TS;
    if (tb == 0) return {B + k0 + n * ldb, ldb, 0};
    return {B + n + k0 * ldb, ldb, 1};
  }
};

template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS, 1) k_dgemm(int64_t M, int64_t N, int64_t K, double alpha,
                                                        const double* A, int64_t lda, int ta, const double* B,
                                                        int64_t ldb, int tb, double beta, double* C, int64_t ldc,
                                                        int klim, int lower_only, int64_t sa, int64_t sb, int64_t sc_,
                                                        int* err) {
  extern __shared__ __align__(128) double smem[];
  const int64_t m0 = (int64_t)blockIdx.x * Cfg::BM, n0 = (int64_t)blockIdx.y * Cfg::BN;
  if (lower_only && n0 >= m0 + Cfg::BM) return;
  A += blockIdx.z * sa;
  B += blockIdx.z * sb;
  C += blockIdx.z * sc_;
  const int KT = (int)(K / TS);
  int kb = 0, ke = KT;
  if (klim & 1) ke = std::min<int64_t>(ke, (m0 + Cfg::BM) / TS);
  if (klim & 2) ke = std::min<int64_t>(ke, (n0 + Cfg::BN) / TS);
  if (klim & 4) kb = std::max<int64_t>(kb, m0 / TS);
  if (klim & 8) kb = std::max<int64_t>(kb, n0 / TS);
  const int ktiles = ke > kb ? ke - kb : 0;
  GemmSched sc{A, lda, ta, B, ldb, tb, m0, n0, kb, M, N};
  double acc[Cfg::FM][Cfg::FN][2];
  if (!dmma_mainloop<Cfg>(sc, ktiles, smem, acc, err, (int)std::min<int64_t>(M - m0, 1 << 30),
                          (int)std::min<int64_t>(N - n0, 1 << 30)))
    return;
  dmma_for_each<Cfg>(acc, [&](int m, int n, double v0, double v1) {
    const int64_t gm = m0 + m, gn = n0 + n;
    if (gm >= M) return;
    if (gn < N) {
      double* c = C + gm + gn * ldc;
      *c = beta == 0.0 ? alpha * v0 : alpha * v0 + beta * *c;
    }
    if (gn + 1 < N) {
      double* c = C + gm + (gn + 1) * ldc;
      *c = beta == 0.0 ? alpha * v1 : alpha * v1 + beta * *c;
    }
  });
}

// 64 x 64 tiles of 4 DMMA warps with cp.async staging: 3 stages when the grid is
// small (latency), 2 stages / 3 CTAs per SM when it fills the GPU (throughput).
using GemmSmall = DmmaCfg<2, 2, 2, 2, 3, true>;
using GemmLarge = DmmaCfg<2, 2, 2, 2, 2, true>;

template <class Cfg>
static void launch_dgemm_cfg(int64_t M, int64_t N, int64_t K, double alpha, const double* A, int64_t lda, int ta,
                             const double* B, int64_t ldb, int tb, double beta, double* C, int64_t ldc, int klim,
                             int lower_only, int batch, int64_t sa, int64_t sb, int64_t sc, int* err,
                             cudaStream_t st) {
  cudaFuncSetAttribute(k_dgemm<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM_BYTES);
  dim3 grid((unsigned)cdiv_m(M, Cfg::BM), (unsigned)cdiv_m(N, Cfg::BN), (unsigned)batch);
  count_launch();
  k_dgemm<Cfg><<<grid, Cfg::THREADS, Cfg::SMEM_BYTES, st>>>(M, N, K, alpha, A, lda, ta, B, ldb, tb, beta, C, ldc,
                                                            klim, lower_only, sa, sb, sc, err);
}

void launch_dgemm(int64_t M, int64_t N, int64_t K, double alpha, const double* A, int64_t lda, int ta,
                  const double* B, int64_t ldb, int tb, double beta, double* C, int64_t ldc, int klim, int lower_only,
                  int batch, int64_t sa, int64_t sb, int64_t sc, int* err, cudaStream_t st) {
  if (M <= 0 || N <= 0 || batch <= 0) return;
  const int64_t ctas = cdiv_m(M, 64) * cdiv_m(N, 64) * batch;
  if (ctas >= 3 * 148)
    launch_dgemm_cfg<GemmLarge>(M, N, K, alpha, A, lda, ta, B, ldb, tb, beta, C, ldc, klim, lower_only, batch, sa, sb,
                                sc, err, st);
  else
    launch_dgemm_cfg<GemmSmall>(M, N, K, alpha, A, lda, ta, B, ldb, tb, beta, C, ldc, klim, lower_only, batch, sa, sb,
                                sc, err, st);
}

// ---------------------------------------------------------------------------
// Cholesky
// ---------------------------------------------------------------------------
// Factor the 32x32 diagonal block j (lower triangle of A is the input), write
// L_jj back with a zero upper triangle, and its inverse to Linvd[j].  A
// non-positive or non-finite pivot is recorded in *info (1-based global index,
// first failure wins) and replaced by 1 so that the factorisation finishes.
__global__ void __launch_bounds__(1024) k_potrf_diag(double* A, int64_t lda, int64_t j, double* Linvd, int* info) {
  __shared__ double a[TS][TS + 1];
  __shared__ double x[TS][TS + 1];
  const int tid = threadIdx.x, r = tid & 31, c = tid >> 5;
  double* blk = A + j * TS + lda * (j * TS);
  a[r][c] = blk[r + lda * c];
  __syncthreads();
  for (int k = 0; k < TS; ++k) {
    if (tid == 0) {
      double d = a[k][k];
      if (!(d > 0.0) || !isfinite(d)) {
        atomicCAS(info, 0, (int)(j * TS + k + 1));
        d = 1.0;
      }
      a[k][k] = sqrt(d);
    }
    __syncthreads();
    if (c == k && r > k) a[r][k] /= a[k][k];
    __syncthreads();
    if (c > k && r >= c) a[r][c] -= a[r][k] * a[c][k];
    __syncthreads();
  }
  blk[r + lda * c] = r >= c ? a[r][c] : 0.0;
  if (tid < TS) {
    const int col = tid;
    for (int i = 0; i < TS; ++i) {
      if (i < col) {
        x[i][col] = 0.0;
        continue;
      }
      double s = (i == col) ? 1.0 : 0.0;
      for (int k = col; k < i; ++k) s -= a[i][k] * x[k][col];
      x[i][col] = s / a[i][i];
    }
  }
  __syncthreads();
  Linvd[j * TILE_ELEMS + r + TS * c] = x[r][c];
}

void run_potrf(double* A, int64_t np, int64_t lda, double* Linvd, int* d_info, int* err, cudaStream_t st) {
  const int64_t nb = np / TS;
  for (int64_t j = 0; j < nb; ++j) {
    count_launch();
    k_potrf_diag<<<1, 1024, 0, st>>>(A, lda, j, Linvd, d_info);
    const int64_t rem = np - (j + 1) * TS;
    if (rem <= 0) break;
    double* panel = A + (j + 1) * TS + lda * (j * TS);
    // panel <- panel L_jj^-T
    launch_dgemm(rem, TS, TS, 1.0, panel, lda, 0, Linvd + j * TILE_ELEMS, TS, 1, 0.0, panel, lda, 0, 0, 1, 0, 0, 0,
                 err, st);
    // A22 <- A22 - panel panel^T (lower blocks only)
    double* a22 = A + (j + 1) * TS + lda * ((j + 1) * TS);
    launch_dgemm(rem, rem, TS, -1.0, panel, lda, 0, panel, lda, 1, 1.0, a22, lda, 0, 1, 1, 0, 0, 0, err, st);
  }
}

// Zero the strict upper triangle, then place the inverted diagonal blocks.
__global__ void __launch_bounds__(256) k_trtri_init(const double* Linvd, int64_t np, int64_t ld, double* Linv) {
  const int64_t total = np * np;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % np, c = e / np;
    double v = 0.0;
    if (r / TS == c / TS) v = Linvd[(r / TS) * TILE_ELEMS + (r % TS) + TS * (c % TS)];
    Linv[r + ld * c] = v;
  }
}

__global__ void __launch_bounds__(256) k_zero_upper(double* L, int64_t np, int64_t ld) {
  const int64_t total = np * np;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % np, c = e / np;
    if (r < c) L[r + ld * c] = 0.0;
  }
}

// Inverse of a lower-triangular matrix by block doubling:
// inv [[A, 0], [C, D]] = [[A^-1, 0], [-D^-1 C A^-1, D^-1]].
void run_trtri(const double* L, int64_t np, int64_t ld, const double* Linvd, double* Linv, double* T, int* err,
               cudaStream_t st) {
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_m(np * np, 256), 148 * 16));
  count_launch();
  k_trtri_init<<<blocks, 256, 0, st>>>(Linvd, np, ld, Linv);
  for (int64_t h = TS; h < np; h *= 2) {
    const int64_t full_pairs = np / (2 * h);
    const int64_t stride = 2 * h * (1 + ld);
    if (full_pairs > 0) {
      // T21 = L21 A^-1   (A^-1 lower: k >= n)
      launch_dgemm(h, h, h, 1.0, L + h, ld, 0, Linv, ld, 0, 0.0, T + h, ld, 8, 0, (int)full_pairs, stride, stride,
                   stride, err, st);
      // Linv21 = -D^-1 T21  (D^-1 lower: k <= m)
      launch_dgemm(h, h, h, -1.0, Linv + h + ld * h, ld, 0, T + h, ld, 0, 0.0, Linv + h, ld, 1, 0, (int)full_pairs,
                   stride, stride, stride, err, st);
    }
    const int64_t b = full_pairs * 2 * h;
    const int64_t h2 = np - b - h;
    if (h2 > 0) {
      const int64_t off = b + ld * b;
      launch_dgemm(h2, h, h, 1.0, L + off + h, ld, 0, Linv + off, ld, 0, 0.0, T + off + h, ld, 8, 0, 1, 0, 0, 0, err,
                   st);
      launch_dgemm(h2, h, h2, -1.0, Linv + off + h + ld * h, ld, 0, T + off + h, ld, 0, 0.0, Linv + off + h, ld, 1, 0,
                   1, 0, 0, 0, err, st);
    }
  }
  (void)k_zero_upper;
}

// dst (np x np, ld np) = src (n x n, ld n) padded with the identity.
__global__ void __launch_bounds__(256) k_pad_matrix(const double* __restrict__ src, int64_t n, int64_t np,
                                                    double* __restrict__ dst) {
  const int64_t total = np * np;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % np, c = e / np;
    dst[e] = (r < n && c < n) ? src[r + n * c] : (r == c ? 1.0 : 0.0);
  }
}

void launch_pad_matrix(const double* src, int64_t n, int64_t np, double* dst, cudaStream_t st) {
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_m(np * np, 256), 148 * 16));
  count_launch();
  k_pad_matrix<<<blocks, 256, 0, st>>>(src, n, np, dst);
}

// dB[P*ldB + k0 + r] = out[r + kc*P] for P < rows, r < kc.
__global__ void __launch_bounds__(256) k_fit_copy_back(const double* __restrict__ out, int64_t kc,
                                                       double* __restrict__ dB, int64_t ldB, int64_t k0,
                                                       int64_t rows) {
  const int64_t total = kc * rows;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % kc, p = e / kc;
    dB[p * ldB + k0 + r] = out[e];
  }
}

void launch_fit_copy_back(const double* out, int64_t kc, double* dB, int64_t ldB, int64_t k0, int64_t rows,
                          cudaStream_t st) {
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_m(kc * rows, 256), 148 * 32));
  count_launch();
  k_fit_copy_back<<<blocks, 256, 0, st>>>(out, kc, dB, ldB, k0, rows);
}

}  // namespace rijk
