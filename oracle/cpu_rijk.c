/*
 * CPU restatement of REST's RI J/K build -- test and benchmark infrastructure
 * only (the timed CPU baseline and a second CPU checker; never the product).
 *
 * REST itself (Rust) cannot be built here, so this file restates the
 * algorithm of its CPU path with the same per-aux-index BLAS structure:
 *
 *   vj_upper_with_rimatr_v_sync  (src/scf_io/mod.rs:2490-2561): a parallel
 *     loop over P computes w_P = 2 sum_{mu<=nu} B D - sum_diag and the scaled
 *     column B_P w_P; REST sends each column through a channel and adds them
 *     on one thread, which is restated as a serial accumulation.
 *   vk_upper_with_ri_v_sync      (src/scf_io/mod.rs:2758-2834): a parallel
 *     loop over P with single-threaded OpenBLAS inside (REST sets the OpenBLAS
 *     thread count to 1 around the rayon loop, :2765-2767): X = B_P C[:, :nw]
 *     (dgemm), Y = X diag(occ), K_P = Y X^T (dgemm), upper part accumulated.
 *
 * rayon is restated as OpenMP.  BLAS is the OpenBLAS shipped inside NumPy
 * (ILP64 symbols with the scipy_ prefix), loaded with dlopen by path.
 */
#include <dlfcn.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef void (*dgemm_t)(const char*, const char*, const int64_t*, const int64_t*, const int64_t*, const double*,
                        const double*, const int64_t*, const double*, const int64_t*, const double*, double*,
                        const int64_t*, size_t, size_t);
typedef void (*setthreads_t)(int);

static dgemm_t p_dgemm = 0;
static setthreads_t p_setthreads = 0;

/* Returns 0 on success. */
int cpu_rijk_init(const char* openblas_path) {
  void* h = dlopen(openblas_path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return 1;
  p_dgemm = (dgemm_t)dlsym(h, "scipy_dgemm_64_");
  p_setthreads = (setthreads_t)dlsym(h, "scipy_openblas_set_num_threads64_");
  return (p_dgemm && p_setthreads) ? 0 : 2;
}

static void dgemm(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha, const double* a, int64_t lda,
                  const double* b, int64_t ldb, double beta, double* c, int64_t ldc) {
  p_dgemm(&ta, &tb, &m, &n, &k, &alpha, a, &lda, b, &ldb, &beta, c, &ldc, 1, 1);
}

/* rimatr: npair x naux column-major (column P = packed upper of B_P);
 * dm: n x n column-major; vj: npair. */
int cpu_vj_upper_with_rimatr(const double* rimatr, int64_t n, int64_t naux, const double* dm, double scale,
                             int nthreads, double* vj) {
  const int64_t npair = n * (n + 1) / 2;
  double* w = (double*)malloc(sizeof(double) * naux);
  double* dup = (double*)malloc(sizeof(double) * npair);
  if (!w || !dup) return 1;
  for (int64_t j = 0, k = 0; j < n; ++j)
    for (int64_t i = 0; i <= j; ++i, ++k) dup[k] = dm[i + n * j];
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int64_t p = 0; p < naux; ++p) {
    const double* m = rimatr + p * npair;
    double t = 0.0, dg = 0.0;
    for (int64_t k = 0; k < npair; ++k) t += m[k] * dup[k];
    for (int64_t j = 0; j < n; ++j) dg += m[j * (j + 1) / 2 + j] * dm[j + n * j];
    w[p] = 2.0 * t - dg;
  }
  memset(vj, 0, sizeof(double) * npair);
  for (int64_t p = 0; p < naux; ++p) { /* REST's receive loop: one thread */
    const double* m = rimatr + p * npair;
    const double wp = w[p];
    for (int64_t k = 0; k < npair; ++k) vj[k] += m[k] * wp;
  }
  if (scale != 1.0)
    for (int64_t k = 0; k < npair; ++k) vj[k] *= scale;
  free(w);
  free(dup);
  return 0;
}

/* ri3fn: n x n x naux column-major; eigv: n x num_state; occ: num_state. */
int cpu_vk_upper_with_ri_v(const double* ri3fn, int64_t n, int64_t naux, const double* eigv, int64_t num_state,
                           int64_t homo, const double* occ, double scale, int nthreads, double* vk) {
  const int64_t npair = n * (n + 1) / 2;
  const int64_t nw = homo + 1;
  if (nw > num_state) return 2;
  p_setthreads(1);
  memset(vk, 0, sizeof(double) * npair);
  int err = 0;
#pragma omp parallel num_threads(nthreads)
  {
    double* x = (double*)malloc(sizeof(double) * n * nw);
    double* y = (double*)malloc(sizeof(double) * n * nw);
    double* kp = (double*)malloc(sizeof(double) * n * n);
    double* acc = (double*)calloc(npair, sizeof(double));
    if (!x || !y || !kp || !acc) {
#pragma omp atomic write
      err = 1;
    } else {
#pragma omp for schedule(dynamic, 1)
      for (int64_t p = 0; p < naux; ++p) {
        const double* bp = ri3fn + p * n * n;
        dgemm('N', 'N', n, nw, n, 1.0, bp, n, eigv, n, 0.0, x, n);
        for (int64_t i = 0; i < nw; ++i)
          for (int64_t r = 0; r < n; ++r) y[r + n * i] = x[r + n * i] * occ[i];
        dgemm('N', 'T', n, n, nw, 1.0, y, n, x, n, 0.0, kp, n);
        for (int64_t j = 0, k = 0; j < n; ++j)
          for (int64_t i = 0; i <= j; ++i, ++k) acc[k] += kp[i + n * j];
      }
#pragma omp critical
      for (int64_t k = 0; k < npair; ++k) vk[k] += acc[k];
    }
    free(x);
    free(y);
    free(kp);
    free(acc);
  }
  if (scale != 1.0)
    for (int64_t k = 0; k < npair; ++k) vk[k] *= scale;
  return err;
}

int cpu_max_threads(void) { return omp_get_max_threads(); }
