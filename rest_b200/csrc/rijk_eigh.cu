// Batched symmetric eigensolver (FP64) for the SCF's Fock matrices.
//
// REST diagonalises each Fock matrix with LAPACK's packed generalised solver
// (dspgvx, src/scf_io/mod.rs:1843-1873) after reducing it to the standard
// form; the batched driver forms X^T F X on the device and needs all
// eigenpairs of many small matrices (n <= a few hundred) at once.  One CTA
// owns one matrix:
//
//  1. Householder reduction to tridiagonal form.  For column k, the vector
//     v (unit, from A[k+1:, k]) defines H = I - 2 v v^T, and the trailing block
//     becomes A - v w^T - w v^T with p = A v, K = v^T p, w = 2 (p - K v).
//     A warp owns a row at a time, so every pass over the trailing block reads
//     and writes whole rows coalesced; the v's are kept in A's lower part.
//  2. Q = H_0 H_1 ... H_{n-3}, accumulated explicitly from the identity, held
//     transposed (Z = Q^T, each eigenvector-to-be a contiguous row).
//  3. Implicit QL with Wilkinson's shift on the tridiagonal (d, e): for each
//     eigenvalue l, sweeps over the unreduced block [l, m] until e[l] is
//     negligible.  One thread computes a sweep's chain of plane rotations into
//     shared memory; then every thread applies the whole chain to its own
//     element of the affected rows of Z, carrying one value in a register, so
//     no barrier runs between rotations.
//  4. Eigenvalues sorted ascending (the rows of Z with them), written out with
//     the eigenvectors as columns of a row-major matrix.
//
// Molecule b uses the leading nvalid[b] rows and columns of its ld x ld slot;
// the rest of its output is eigenvalue pad_value with unit vectors, so a
// padded batch keeps its padding last.  A sweep count beyond 30 per eigenvalue
// marks the matrix as failed (info[b] = 1) instead of looping.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/rest_b200.h"
#include "rijk_internal.h"

namespace {

constexpr int ET = 512;     // threads per matrix
constexpr int EW = ET / 32;  // warps
constexpr int MAX_N = 768;   // shared-memory vectors (d, e, v, w, rotations, ranks)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// CTA-wide sum of one value per thread (all threads call it).
__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < EW ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[0] = t;
  }
  __syncthreads();
  return red[0];
}

__global__ void __launch_bounds__(ET, 1) k_eigh(double* __restrict__ Aall, int64_t ld, const int32_t* __restrict__ nvalid,
                                             double pad_value, double* __restrict__ Wall, double* __restrict__ Vall,
                                             double* __restrict__ Zall, int32_t* __restrict__ info) {
  __shared__ double d[MAX_N], e[MAX_N], v[MAX_N], w[MAX_N], rc[MAX_N], rs[MAX_N];
  __shared__ int rank[MAX_N];
  __shared__ double red[32];
  __shared__ int sweep_info[2];
  const int64_t b = blockIdx.x;
  const int n = max(0, min(nvalid[b], (int)ld));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* A = Aall + b * ld * ld;   // row-major, overwritten
  double* Z = Zall + b * ld * ld;   // Z = Q^T (row i: vector i), then eigenvectors as rows
  double* W = Wall + b * ld;
  double* V = Vall + b * ld * ld;
  if (tid == 0) info[b] = 0;

  // ---- 1. tridiagonalisation ------------------------------------------------
  for (int k = 0; k + 2 < n; ++k) {
    // v from x = A[k+1:, k] (column k below the diagonal; A symmetric: row k)
    double part = 0.0;
    for (int j = k + 1 + tid; j < n; j += ET) {
      const double x = A[(int64_t)k * ld + j];
      v[j] = x;
      part += x * x;
    }
    const double xx = block_sum(part, red);
    const double x0 = v[k + 1];
    const double nx = sqrt(xx);
    const double alpha = x0 > 0.0 ? -nx : nx;
    // v = x - alpha e1, |v|^2 = xx - 2 alpha x0 + alpha^2
    const double vv = xx - 2.0 * alpha * x0 + alpha * alpha;
    const bool skip = !(vv > 1e-300 * (1.0 + xx));  // column already reduced
    __syncthreads();
    if (skip) {
      for (int j = k + 1 + tid; j < n; j += ET) v[j] = 0.0;
      if (tid == 0) {
        d[k] = A[(int64_t)k * ld + k];
        e[k] = x0;
      }
      __syncthreads();
      for (int j = k + 1 + tid; j < n; j += ET) A[(int64_t)j * ld + k] = 0.0;  // stored vector (none)
      continue;
    }
    const double inv = 1.0 / sqrt(vv);
    if (tid == 0) v[k + 1] = (x0 - alpha) * inv;
    for (int j = k + 2 + tid; j < n; j += ET) v[j] *= inv;
    __syncthreads();
    // p = A_t v (trailing rows and columns k+1 .. n-1), warp per row
    for (int r = k + 1 + warp; r < n; r += EW) {
      const double* row = A + (int64_t)r * ld;
      double s = 0.0;
      for (int j = k + 1 + lane; j < n; j += 32) s += row[j] * v[j];
      s = warp_sum(s);
      if (lane == 0) w[r] = s;
    }
    __syncthreads();
    double kp = 0.0;
    for (int j = k + 1 + tid; j < n; j += ET) kp += v[j] * w[j];
    const double K = block_sum(kp, red);
    for (int j = k + 1 + tid; j < n; j += ET) w[j] = 2.0 * (w[j] - K * v[j]);
    __syncthreads();
    // A_t -= v w^T + w v^T
    for (int r = k + 1 + warp; r < n; r += EW) {
      double* row = A + (int64_t)r * ld;
      const double vr = v[r], wr = w[r];
      for (int j = k + 1 + lane; j < n; j += 32) row[j] -= vr * w[j] + wr * v[j];
    }
    if (tid == 0) {
      d[k] = A[(int64_t)k * ld + k];
      e[k] = alpha;
    }
    __syncthreads();
    // keep v in column k below the diagonal (row k is no longer read)
    for (int j = k + 1 + tid; j < n; j += ET) A[(int64_t)j * ld + k] = v[j];
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = A[(int64_t)(n - 2) * ld + (n - 2)];
      e[n - 2] = A[(int64_t)(n - 1) * ld + (n - 2)];
      if (n >= 3) e[n - 2] = A[(int64_t)(n - 2) * ld + (n - 1)];
    }
    if (n >= 1) d[n - 1] = A[(int64_t)(n - 1) * ld + (n - 1)];
    e[n - 1] = 0.0;
  }
  __syncthreads();

  // ---- 2. Z = Q^T, Q = H_0 ... H_{n-3}: Z <- Z H_k for k = n-3 .. 0 ------------
  // (Z starts as the identity; Z H_k touches columns k+1 .. n-1 of every row.)
  for (int i = 0; i < n; ++i)
    for (int j = tid; j < n; j += ET) Z[(int64_t)i * ld + j] = i == j ? 1.0 : 0.0;
  __syncthreads();
  for (int k = n - 3; k >= 0; --k) {
    for (int j = k + 1 + tid; j < n; j += ET) v[j] = A[(int64_t)j * ld + k];
    __syncthreads();
    // row i of Z: z <- z - 2 (z . v) v over columns k+1 .. n-1; only rows whose
    // support reaches those columns change: rows k+1 .. n-1 (Z is the identity
    // elsewhere on them, as H_j for j > k only mixed columns > k)
    for (int r = k + 1 + warp; r < n; r += EW) {
      double* row = Z + (int64_t)r * ld;
      double s = 0.0;
      for (int j = k + 1 + lane; j < n; j += 32) s += row[j] * v[j];
      s = 2.0 * warp_sum(s);
      for (int j = k + 1 + lane; j < n; j += 32) row[j] -= s * v[j];
    }
    __syncthreads();
  }
  // Z = Q^T: row i holds the components of tridiagonal index i, so the QL
  // rotations below, which mix indices i and i+1, mix whole rows of Z.

  // ---- 3. implicit QL on (d, e) ------------------------------------------------
  // Each sweep: thread 0 finds the unreduced block [l, m], then computes the
  // chain of plane rotations i = m-1 .. lo one after another (a serial
  // recurrence) and publishes its progress in `prog`; warps 1.. apply each
  // rotation to their columns of Z as soon as it is published, so the rows of
  // Z stream through L2 while the chain is still being computed.  Waits are
  // bounded: a sweep whose chain is not published in time marks the matrix as
  // failed (info = 2) and the caller re-solves it with another solver.
  __shared__ volatile int prog, chain_done;
  for (int l = 0; l < n; ++l) {
    for (int iter = 0;; ++iter) {
      if (tid == 0) {
        int m = l;  // first index >= l with a negligible e[m]
        for (; m < n - 1; ++m) {
          const double dd = fabs(d[m]) + fabs(d[m + 1]);
          if (fabs(e[m]) + dd == dd) break;
        }
        if (m != l && iter >= 30) {
          info[b] = 1;  // no convergence: leave this eigenvalue as it stands
          m = l;
        }
        sweep_info[0] = m;
        sweep_info[1] = m;
        prog = m;
        chain_done = 0;
      }
      __syncthreads();
      const int m = sweep_info[0];
      if (m == l) break;
      if (tid == 0) {
        // Wilkinson's shift from the leading 2 x 2 of the block
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? fabs(r) : -fabs(r)));
        double s = 1.0, c = 1.0, p = 0.0;
        bool early = false;
        int i = m - 1;
        for (; i >= l; --i) {
          const double f = s * e[i];
          const double bb = c * e[i];
          // |f|, |g| are bounded by the matrix norm, far from FP64 overflow:
          // one reciprocal square root keeps the serial chain short
          const double r2 = fma(f, f, g * g);
          if (r2 == 0.0) {  // the sweep splits here: deflate and sweep again
            e[i + 1] = 0.0;
            d[i + 1] -= p;
            e[m] = 0.0;
            early = true;
            break;
          }
          const double ri = rsqrt(r2);
          r = r2 * ri;
          e[i + 1] = r;
          s = f * ri;
          c = g * ri;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * bb;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - bb;
          rc[i] = c;
          rs[i] = s;
          __threadfence_block();
          prog = i;  // rotations i .. m-1 are ready
        }
        if (!early) {
          d[l] -= p;
          e[l] = g;
          e[m] = 0.0;
        }
        sweep_info[1] = early ? i + 1 : l;
        __threadfence_block();
        chain_done = 1;
      } else if (warp > 0) {
        // the chain on rows i, i+1 of Z; each thread owns column t and carries
        // the partly rotated row i+1 in a register; rows are read up to eight
        // ahead of their rotations (each row before the rotation that
        // overwrites it)
        for (int t = tid - 32; t < n; t += ET - 32) {
          double zi1 = Z[(int64_t)m * ld + t];
          int i = m - 1;
          int lo = m;
          bool stalled = false;
          while (true) {
            int pr = prog, done = chain_done;
            for (int spin = 0; pr > i && !done; ++spin) {
              if (spin > (1 << 24)) {
                stalled = true;
                break;
              }
              pr = prog;
              done = chain_done;
            }
            if (stalled) break;
            __threadfence_block();
            if (done) lo = sweep_info[1];
            const int stop = done ? lo : pr;
            for (; i - 7 >= stop; i -= 8) {
              double zr[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) zr[u] = Z[(int64_t)(i - u) * ld + t];
#pragma unroll
              for (int u = 0; u < 8; ++u) {
                const double c = rc[i - u], s = rs[i - u];
                Z[(int64_t)(i - u + 1) * ld + t] = s * zr[u] + c * zi1;
                zi1 = c * zr[u] - s * zi1;
              }
            }
            for (; i >= stop; --i) {
              const double c = rc[i], s = rs[i];
              const double zi = Z[(int64_t)i * ld + t];
              Z[(int64_t)(i + 1) * ld + t] = s * zi + c * zi1;
              zi1 = c * zi - s * zi1;
            }
            if (done) break;
          }
          if (stalled) {
            info[b] = 2;
            break;
          }
          Z[(int64_t)lo * ld + t] = zi1;
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();

  // ---- 4. ascending order: each eigenvalue's rank (ties by index) -------------------
  for (int i = tid; i < n; i += ET) {
    const double di = d[i];
    int rk = 0;
    for (int j = 0; j < n; ++j) rk += (d[j] < di) || (d[j] == di && j < i);
    rank[i] = rk;
  }
  __syncthreads();
  for (int i = tid; i < n; i += ET) W[rank[i]] = d[i];
  for (int i = n + tid; i < ld; i += ET) W[i] = pad_value;
  // V[r][rank i] = component r of vector i = Z[i][r]; padding: unit vectors
  for (int64_t t = tid; t < ld * ld; t += ET) {
    const int i = (int)(t / ld), r = (int)(t % ld);
    if (i < n && r < n)
      V[(int64_t)r * ld + rank[i]] = Z[(int64_t)i * ld + r];
    else
      V[(int64_t)r * ld + i] = (r == i) ? 1.0 : 0.0;
  }
}

}  // namespace

extern "C" int rijk_eigh_batched_dev(double* d_a, int64_t ld, const int32_t* d_nvalid, int64_t batch,
                                     double pad_value, double* d_w, double* d_v, double* d_work, int32_t* d_info,
                                     void* stream) {
  if (!d_a || !d_nvalid || !d_w || !d_v || !d_work || !d_info || ld <= 0 || ld > MAX_N || batch < 0)
    return ld > MAX_N ? RIJK_ERR_TOO_LARGE : RIJK_ERR_ARG;
  if (batch == 0) return RIJK_OK;
  rijk::count_launch();
  k_eigh<<<(unsigned)batch, ET, 0, static_cast<cudaStream_t>(stream)>>>(d_a, ld, d_nvalid, pad_value, d_w, d_v,
                                                                        d_work, d_info);
  return cudaGetLastError() == cudaSuccess ? RIJK_OK : RIJK_ERR_CUDA;
}
