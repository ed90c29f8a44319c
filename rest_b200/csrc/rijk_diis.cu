// Batched DIIS coefficients (FP64) for the SCF's Fock extrapolation.
//
// REST's diis_solver (src/scf_io/mod.rs:3138-3188) takes the Gram matrix
// B_ij = <e_i, e_j> of the last k error vectors, inverts it (rest_tensors
// _dinverse: LU with partial pivoting, None when a pivot is exactly zero) and
// returns c_i = (sum_j Binv_ji) / (sum_jl Binv_jl).  Since B is symmetric,
// sum_j Binv_ji = x_i with B x = 1, so c = x / sum(x): one solve with a single
// right-hand side instead of the inverse.  A batched SCF needs these for every
// molecule of the set each iteration; one warp owns one molecule's k x k
// system (k <= 32): Gauss-Jordan elimination with partial pivoting, lane r
// holding row r.  A zero or non-finite pivot, or a non-finite or zero sum(x),
// is REST's failure case: the caller restarts that molecule's history from its
// newest Fock matrix, so the coefficients written are (1, 0, ..., 0) and
// status[b] = 1.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/rest_b200.h"
#include "rijk_internal.h"

namespace {

constexpr int MAXK = 32;
constexpr int WPB = 4;  // molecules (warps) per block

__global__ void __launch_bounds__(32 * WPB) k_diis_coef(const double* __restrict__ gram, int64_t m,
                                                        const int32_t* __restrict__ count, int64_t batch,
                                                        double* __restrict__ coef, int32_t* __restrict__ status) {
  __shared__ double a_s[WPB][MAXK][MAXK + 1];
  __shared__ double b_s[WPB][MAXK];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t mol = (int64_t)blockIdx.x * WPB + wib;
  if (mol >= batch) return;  // whole warp
  double(*a)[MAXK + 1] = a_s[wib];
  double* b = b_s[wib];
  const int64_t cnt = count[mol] > 0 ? (int64_t)count[mol] : 0;
  const int k = (int)(cnt < m ? cnt : m);
  const double* g = gram + mol * m * m;
  double* c = coef + mol * m;
  for (int j = lane; j < m; j += 32) c[j] = 0.0;
  if (k == 0) {
    if (lane == 0) status[mol] = 0;
    return;
  }
  if (lane < k) {
    for (int j = 0; j < k; ++j) a[lane][j] = g[(int64_t)lane * m + j];
    b[lane] = 1.0;
  }
  __syncwarp();
  bool fail = false;
  for (int p = 0; p < k; ++p) {
    // pivot: the largest |a[r][p]| over r >= p (lowest row on ties)
    double v = lane >= p && lane < k ? fabs(a[lane][p]) : -1.0;
    int r = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
      const int r2 = __shfl_xor_sync(0xffffffffu, r, o);
      if (v2 > v || (v2 == v && r2 < r)) {
        v = v2;
        r = r2;
      }
    }
    if (!(v > 0.0) || !isfinite(v)) {  // exactly singular (or NaN/Inf in B)
      fail = true;
      break;
    }
    if (r != p) {  // lanes swap the two rows column by column
      for (int j = lane; j < k; j += 32) {
        const double t = a[p][j];
        a[p][j] = a[r][j];
        a[r][j] = t;
      }
      if (lane == 0) {
        const double t = b[p];
        b[p] = b[r];
        b[r] = t;
      }
    }
    __syncwarp();
    // eliminate column p from every other row (lane i owns row i)
    if (lane < k && lane != p) {
      const double f = a[lane][p] / a[p][p];
      for (int j = p; j < k; ++j) a[lane][j] = fma(-f, a[p][j], a[lane][j]);
      b[lane] = fma(-f, b[p], b[lane]);
    }
    __syncwarp();
  }
  double x = 0.0;
  if (!fail && lane < k) x = b[lane] / a[lane][lane];
  double sum = x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  const bool ok = !fail && isfinite(sum) && sum != 0.0 && __all_sync(0xffffffffu, isfinite(x));
  if (ok) {
    if (lane < k) c[lane] = x / sum;
  } else if (lane == 0) {
    c[0] = 1.0;
  }
  if (lane == 0) status[mol] = ok ? 0 : 1;
}

}  // namespace

extern "C" int rijk_diis_coefficients_dev(const double* d_gram, int64_t m, const int32_t* d_count, int64_t batch,
                                          double* d_coef, int32_t* d_status, void* stream) {
  if (!d_gram || !d_count || !d_coef || !d_status || m <= 0 || batch < 0) return RIJK_ERR_ARG;
  if (m > MAXK) return RIJK_ERR_TOO_LARGE;
  if (batch == 0) return RIJK_OK;
  rijk::count_launch();
  k_diis_coef<<<(unsigned)((batch + WPB - 1) / WPB), 32 * WPB, 0, static_cast<cudaStream_t>(stream)>>>(
      d_gram, m, d_count, batch, d_coef, d_status);
  return cudaGetLastError() == cudaSuccess ? RIJK_OK : RIJK_ERR_CUDA;
}
