// Kernels of the learned initial guess: a per-atom-pair MLP with BF16 weights
// and activations and FP32 accumulation, trained and evaluated on the device.
// REST has no learned guess; its own guesses (src/initial_guess) stay the
// fallback of the driver that uses this network.
//
//   linear forward   Z = X W^T + b, Y = act(Z)      (X: m x k, W: n x k, row-major)
//   linear backward  dZ = dY * act'(Z), db = sum_m dZ (FP32), dW = dZ^T X, dX = dZ W (dZ as BF16)
//   masked MSE       loss += sum mask (Y - T)^2 / count, dY = 2 mask (Y - T) / count
//   Adam             FP32 master weights, BF16 copies written back
//
// The GEMMs are strided tiles (64 x 64, k-step 16, 4 x 4 outputs per thread)
// on the FP32 pipes: the network costs about 1.5 MFLOP per atom pair per
// training step, far from any bound that matters to the SCF.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/rest_b200.h"
#include "rijk_internal.h"

namespace {

constexpr int TM = 64, TN = 64, TK = 16, NT = 256;

__device__ __forceinline__ float bf(const uint16_t v) {
  return __bfloat162float(__ushort_as_bfloat16(v));
}
__device__ __forceinline__ uint16_t to_bf(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }

__device__ __forceinline__ float act_f(int act, float z) { return act == 1 ? z / (1.0f + expf(-z)) : z; }
__device__ __forceinline__ float act_d(int act, float z) {
  if (act != 1) return 1.0f;
  const float s = 1.0f / (1.0f + expf(-z));
  return s + z * s * (1.0f - s);
}

// C[i, j] = sum_l A(i, l) B(l, j) over l in this CTA's k-chunk, with
// A(i, l) = A[i*sai + l*sal] and B(l, j) = B[l*sbl + j*sbj] (BF16).
// epi 0: forward epilogue (bias, activation, Z / Ybf / Yf outputs, no split-k);
// epi 1: plain FP32 output, atomically added (split-k over blockIdx.z).
template <int EPI>
__global__ void __launch_bounds__(NT) k_gemm(int64_t M, int64_t N, int64_t K, int64_t kchunk,
                                             const uint16_t* __restrict__ A, int64_t sai, int64_t sal,
                                             const uint16_t* __restrict__ B, int64_t sbl, int64_t sbj,
                                             const float* __restrict__ bias, int act, float* __restrict__ Z,
                                             uint16_t* __restrict__ Ybf, float* __restrict__ Yf,
                                             float* __restrict__ C) {
  __shared__ float As[TK][TM + 4];
  __shared__ float Bs[TK][TN + 4];
  const int tid = threadIdx.x;
  const int ty = tid / 16, tx = tid % 16;
  const int64_t i0 = (int64_t)blockIdx.y * TM, j0 = (int64_t)blockIdx.x * TN;
  const int64_t l_begin = (int64_t)blockIdx.z * kchunk;
  const int64_t l_end = l_begin + kchunk < K ? l_begin + kchunk : K;
  float acc[4][4] = {};
  for (int64_t l0 = l_begin; l0 < l_end; l0 += TK) {
    for (int e = tid; e < TK * TM; e += NT) {
      const int r = e / TK, c = e % TK;  // row of the tile, k index
      const int64_t i = i0 + r, l = l0 + c;
      As[c][r] = (i < M && l < l_end) ? bf(A[i * sai + l * sal]) : 0.0f;
    }
    for (int e = tid; e < TK * TN; e += NT) {
      const int c = e / TN, r = e % TN;  // k index, column of the tile
      const int64_t j = j0 + r, l = l0 + c;
      Bs[c][r] = (j < N && l < l_end) ? bf(B[l * sbl + j * sbj]) : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < TK; ++c) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = As[c][ty + 16 * u];
#pragma unroll
      for (int u = 0; u < 4; ++u) b[u] = Bs[c][tx + 16 * u];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w) acc[u][w] = fmaf(a[u], b[w], acc[u][w]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int64_t i = i0 + ty + 16 * u;
    if (i >= M) continue;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const int64_t j = j0 + tx + 16 * w;
      if (j >= N) continue;
      if (EPI == 0) {
        const float z = acc[u][w] + (bias ? bias[j] : 0.0f);
        if (Z) Z[i * N + j] = z;
        const float y = act_f(act, z);
        if (Ybf) Ybf[i * N + j] = to_bf(y);
        if (Yf) Yf[i * N + j] = y;
      } else {
        atomicAdd(&C[i * N + j], acc[u][w]);
      }
    }
  }
}

// dZ = dY * act'(Z) as BF16, and db += column sums (rows split over blocks).
__global__ void __launch_bounds__(NT) k_act_bwd(int64_t M, int64_t N, const float* __restrict__ dY,
                                                const float* __restrict__ Z, int act, uint16_t* __restrict__ dZ,
                                                float* __restrict__ db, int64_t rows_per_block) {
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
  const int64_t r1 = r0 + rows_per_block < M ? r0 + rows_per_block : M;
  for (int64_t j = threadIdx.x; j < N; j += NT) {
    float s = 0.0f;
    for (int64_t i = r0; i < r1; ++i) {
      const float g = dY[i * N + j] * act_d(act, Z[i * N + j]);
      dZ[i * N + j] = to_bf(g);
      s += g;
    }
    if (db) atomicAdd(&db[j], s);
  }
}

__global__ void __launch_bounds__(NT) k_masked_mse(int64_t count, const float* __restrict__ Y,
                                                   const float* __restrict__ T, const float* __restrict__ mask,
                                                   float inv_n, float* __restrict__ dY, float* __restrict__ loss) {
  __shared__ float red[NT];
  float s = 0.0f;
  for (int64_t e = (int64_t)blockIdx.x * NT + threadIdx.x; e < count; e += (int64_t)gridDim.x * NT) {
    const float mk = mask ? mask[e] : 1.0f;
    const float d = (Y[e] - T[e]) * mk;
    dY[e] = 2.0f * d * inv_n;
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss) atomicAdd(loss, red[0] * inv_n);
}

__global__ void __launch_bounds__(NT) k_adam(int64_t count, float* __restrict__ w, uint16_t* __restrict__ wbf,
                                             const float* __restrict__ g, float* __restrict__ m,
                                             float* __restrict__ v, float lr, float b1, float b2, float eps,
                                             float bc1, float bc2) {
  for (int64_t e = (int64_t)blockIdx.x * NT + threadIdx.x; e < count; e += (int64_t)gridDim.x * NT) {
    const float ge = g[e];
    const float me = b1 * m[e] + (1.0f - b1) * ge;
    const float ve = b2 * v[e] + (1.0f - b2) * ge * ge;
    m[e] = me;
    v[e] = ve;
    const float we = w[e] - lr * (me / bc1) / (sqrtf(ve / bc2) + eps);
    w[e] = we;
    if (wbf) wbf[e] = to_bf(we);
  }
}

__global__ void __launch_bounds__(NT) k_to_bf16(int64_t count, const float* __restrict__ s, uint16_t* __restrict__ d) {
  for (int64_t e = (int64_t)blockIdx.x * NT + threadIdx.x; e < count; e += (int64_t)gridDim.x * NT)
    d[e] = to_bf(s[e]);
}

unsigned grid_for(int64_t count) {
  const int64_t b = (count + NT - 1) / NT;
  return (unsigned)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

int launch_status() { return cudaGetLastError() == cudaSuccess ? RIJK_OK : RIJK_ERR_CUDA; }

}  // namespace

extern "C" {

int rijk_mlp_linear_fwd(const uint16_t* x, const uint16_t* w, const float* bias, int64_t m, int64_t k, int64_t n,
                        int act, float* z, uint16_t* y_bf16, float* y_f32, void* stream) {
  if (!x || !w || m <= 0 || k <= 0 || n <= 0 || (act != 0 && act != 1) || (!z && !y_bf16 && !y_f32))
    return RIJK_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid((unsigned)((n + TN - 1) / TN), (unsigned)((m + TM - 1) / TM), 1);
  rijk::count_launch();
  k_gemm<0><<<grid, NT, 0, st>>>(m, n, k, k, x, k, 1, w, 1, k, bias, act, z, y_bf16, y_f32, nullptr);
  return launch_status();
}

int rijk_mlp_linear_bwd(const uint16_t* x, const uint16_t* w, const float* z, const float* dy, int64_t m, int64_t k,
                        int64_t n, int act, uint16_t* dz_scratch, float* dw, float* db, float* dx, void* stream) {
  if (!x || !w || !z || !dy || !dz_scratch || !dw || m <= 0 || k <= 0 || n <= 0 || (act != 0 && act != 1))
    return RIJK_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(dw, 0, (size_t)n * k * sizeof(float), st) != cudaSuccess) return RIJK_ERR_CUDA;
  if (db && cudaMemsetAsync(db, 0, (size_t)n * sizeof(float), st) != cudaSuccess) return RIJK_ERR_CUDA;
  const int64_t rpb = 64;
  rijk::count_launch();
  k_act_bwd<<<(unsigned)((m + rpb - 1) / rpb), NT, 0, st>>>(m, n, dy, z, act, dz_scratch, db, rpb);
  // dW[n x k] = dZ^T X: inner dimension m, split over blockIdx.z
  {
    const int64_t tiles = ((n + TM - 1) / TM) * ((k + TN - 1) / TN);
    int64_t splits = (4 * 148 + tiles - 1) / tiles;
    int64_t kchunk = (m + splits - 1) / splits;
    kchunk = (kchunk + TK - 1) / TK * TK;
    splits = (m + kchunk - 1) / kchunk;
    const dim3 grid((unsigned)((k + TN - 1) / TN), (unsigned)((n + TM - 1) / TM), (unsigned)splits);
    rijk::count_launch();
    k_gemm<1><<<grid, NT, 0, st>>>(n, k, m, kchunk, dz_scratch, 1, n, x, k, 1, nullptr, 0, nullptr, nullptr,
                                   nullptr, dw);
  }
  // dX[m x k] = dZ W: inner dimension n
  if (dx) {
    if (cudaMemsetAsync(dx, 0, (size_t)m * k * sizeof(float), st) != cudaSuccess) return RIJK_ERR_CUDA;
    const dim3 grid((unsigned)((k + TN - 1) / TN), (unsigned)((m + TM - 1) / TM), 1);
    rijk::count_launch();
    k_gemm<1><<<grid, NT, 0, st>>>(m, k, n, n, dz_scratch, n, 1, w, k, 1, nullptr, 0, nullptr, nullptr, nullptr,
                                   dx);
  }
  return launch_status();
}

int rijk_mlp_masked_mse(const float* y, const float* t, const float* mask, int64_t count, double norm, float* dy,
                        float* loss, void* stream) {
  if (!y || !t || !dy || count <= 0 || !(norm > 0.0)) return RIJK_ERR_ARG;
  rijk::count_launch();
  k_masked_mse<<<grid_for(count), NT, 0, static_cast<cudaStream_t>(stream)>>>(count, y, t, mask,
                                                                              (float)(1.0 / norm), dy, loss);
  return launch_status();
}

int rijk_mlp_adam(float* w, uint16_t* w_bf16, const float* g, float* m, float* v, int64_t count, double lr,
                  double beta1, double beta2, double eps, int64_t step, void* stream) {
  if (!w || !g || !m || !v || count <= 0 || step <= 0) return RIJK_ERR_ARG;
  const double bc1 = 1.0 - pow(beta1, (double)step), bc2 = 1.0 - pow(beta2, (double)step);
  rijk::count_launch();
  k_adam<<<grid_for(count), NT, 0, static_cast<cudaStream_t>(stream)>>>(
      count, w, w_bf16, g, m, v, (float)lr, (float)beta1, (float)beta2, (float)eps, (float)bc1, (float)bc2);
  return launch_status();
}

int rijk_mlp_to_bf16(const float* src, uint16_t* dst, int64_t count, void* stream) {
  if (!src || !dst || count <= 0) return RIJK_ERR_ARG;
  rijk::count_launch();
  k_to_bf16<<<grid_for(count), NT, 0, static_cast<cudaStream_t>(stream)>>>(count, src, dst);
  return launch_status();
}

}  // extern "C"
