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
// The GEMMs run on the tensor cores: BF16 operands staged in shared memory,
// mma.sync m16n8k16 with FP32 accumulation, 64 x 64 CTA tiles of four warps
// (32 x 32 each), k-step 32; operands of any stride (X W^T, dZ^T X, dZ W).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/rest_b200.h"
#include "rijk_internal.h"

namespace {

constexpr int NT = 256;                 // threads of the elementwise kernels
constexpr int TM = 64, TN = 64, TK = 32;  // GEMM CTA tile and k-step
constexpr int GT = 128;                 // GEMM threads: 4 warps of 32 x 32
constexpr int SK = TK + 8;              // smem row of a tile (BF16): 80 bytes, conflict-free fragment loads

__device__ __forceinline__ uint16_t to_bf(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }

__device__ __forceinline__ float act_f(int act, float z) { return act == 1 ? z / (1.0f + expf(-z)) : z; }
__device__ __forceinline__ float act_d(int act, float z) {
  if (act != 1) return 1.0f;
  const float s = 1.0f / (1.0f + expf(-z));
  return s + z * s * (1.0f - s);
}

// D(16x8) += A(16x16, row) B(16x8, col), BF16 in, FP32 accumulate.
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[i, j] = sum_l A(i, l) B(l, j) over l in this CTA's k-chunk, with
// A(i, l) = A[i*sai + l*sal] and B(l, j) = B[l*sbl + j*sbj] (BF16).  Tiles are
// staged as As[i][l] and Bs[j][l] (l contiguous), zero outside the matrices.
// epi 0: forward epilogue (bias, activation, Z / Ybf / Yf outputs, no split-k);
// epi 1: plain FP32 output, atomically added (split-k over blockIdx.z).
template <int EPI>
__global__ void __launch_bounds__(GT) k_gemm(int64_t M, int64_t N, int64_t K, int64_t kchunk,
                                             const uint16_t* __restrict__ A, int64_t sai, int64_t sal,
                                             const uint16_t* __restrict__ B, int64_t sbl, int64_t sbj,
                                             const float* __restrict__ bias, int act, float* __restrict__ Z,
                                             uint16_t* __restrict__ Ybf, float* __restrict__ Yf,
                                             float* __restrict__ C) {
  __shared__ __align__(16) uint16_t As[TM][SK];
  __shared__ __align__(16) uint16_t Bs[TN][SK];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;  // warp tile rows wm*32, cols wn*32
  const int64_t i0 = (int64_t)blockIdx.y * TM, j0 = (int64_t)blockIdx.x * TN;
  const int64_t l_begin = (int64_t)blockIdx.z * kchunk;
  const int64_t l_end = l_begin + kchunk < K ? l_begin + kchunk : K;
  float acc[2][4][4] = {};
  const int q = lane >> 2, r = lane & 3;
  for (int64_t l0 = l_begin; l0 < l_end; l0 += TK) {
    // consecutive threads take consecutive l when A (B) is contiguous in l,
    // else consecutive rows (columns)
    if (sal == 1) {
      for (int e = tid; e < TM * TK; e += GT) {
        const int rr = e / TK, c = e % TK;
        const int64_t i = i0 + rr, l = l0 + c;
        As[rr][c] = (i < M && l < l_end) ? A[i * sai + l] : (uint16_t)0;
      }
    } else {
      for (int e = tid; e < TM * TK; e += GT) {
        const int c = e / TM, rr = e % TM;
        const int64_t i = i0 + rr, l = l0 + c;
        As[rr][c] = (i < M && l < l_end) ? A[i * sai + l * sal] : (uint16_t)0;
      }
    }
    if (sbl == 1) {
      for (int e = tid; e < TN * TK; e += GT) {
        const int rr = e / TK, c = e % TK;
        const int64_t j = j0 + rr, l = l0 + c;
        Bs[rr][c] = (j < N && l < l_end) ? B[l + j * sbj] : (uint16_t)0;
      }
    } else {
      for (int e = tid; e < TN * TK; e += GT) {
        const int c = e / TN, rr = e % TN;
        const int64_t j = j0 + rr, l = l0 + c;
        Bs[rr][c] = (j < N && l < l_end) ? B[l * sbl + j * sbj] : (uint16_t)0;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k0 = 0; k0 < TK; k0 += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int rb = wm * 32 + mt * 16;
        af[mt][0] = *reinterpret_cast<const uint32_t*>(&As[rb + q][k0 + 2 * r]);
        af[mt][1] = *reinterpret_cast<const uint32_t*>(&As[rb + q + 8][k0 + 2 * r]);
        af[mt][2] = *reinterpret_cast<const uint32_t*>(&As[rb + q][k0 + 8 + 2 * r]);
        af[mt][3] = *reinterpret_cast<const uint32_t*>(&As[rb + q + 8][k0 + 8 + 2 * r]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int cb = wn * 32 + nt * 8;
        bfr[nt][0] = *reinterpret_cast<const uint32_t*>(&Bs[cb + q][k0 + 2 * r]);
        bfr[nt][1] = *reinterpret_cast<const uint32_t*>(&Bs[cb + q][k0 + 8 + 2 * r]);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16_16816(acc[mt][nt], af[mt], bfr[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t i = i0 + wm * 32 + mt * 16 + q + 8 * h;
      if (i >= M) continue;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int64_t j = j0 + wn * 32 + nt * 8 + 2 * r + e;
          if (j >= N) continue;
          const float v = acc[mt][nt][2 * h + e];
          if (EPI == 0) {
            const float z = v + (bias ? bias[j] : 0.0f);
            if (Z) Z[i * N + j] = z;
            const float y = act_f(act, z);
            if (Ybf) Ybf[i * N + j] = to_bf(y);
            if (Yf) Yf[i * N + j] = y;
          } else {
            atomicAdd(&C[i * N + j], v);
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

// Learned-guess density assembly (the inverse of the training targets' frame
// rotation).  Unordered atom pair u (A <= B, within the cutoff) is
// up[4u .. 4u+3] = (A, B, ordered pair index of (A, B), of (B, A)) into the
// network output y (standardised, 196 per pair: the 14 x 14 block, row-major).
// With P = y t_std[kind] + t_mean[kind] (kind = 2 type(A) + type(B)) and G_t(w)
// the rotation of element t's AO block into water w's frame (rot, 14 x 14 per
// water and element, row-major):
//   D_AB = 1/2 (G_tA(wA) P_AB G_tB(wA)^T + G_tA(wB) P_BA^T G_tB(wB)^T),
// the average of the (A, B) prediction and the transposed (B, A) one, each
// rotated back from its own water's frame.  D_AB and D_BA = D_AB^T are written
// once each (no atomics); one warp per pair.
constexpr int GB = 14, GB2 = GB * GB;

__global__ void __launch_bounds__(128) k_guess_assemble(const float* __restrict__ y, const float* __restrict__ t_mean,
                                                        const float* __restrict__ t_std, const int32_t* __restrict__ up,
                                                        int64_t nu, const int32_t* __restrict__ first,
                                                        const int32_t* __restrict__ type,
                                                        const int32_t* __restrict__ nfun,
                                                        const int32_t* __restrict__ water,
                                                        const double* __restrict__ rot, int64_t n,
                                                        double* __restrict__ D) {
  __shared__ double sm[4][4][GB2];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  double* P1 = sm[wl][0];   // P_AB            (na x nb)
  double* P2 = sm[wl][1];   // P_BA^T          (na x nb)
  double* T1 = sm[wl][2];   // P_AB G_tB(wA)^T (na x nb)
  double* T2 = sm[wl][3];   // P_BA^T G_tB(wB)^T
  for (int64_t u = (int64_t)blockIdx.x * 4 + wl; u < nu; u += (int64_t)gridDim.x * 4) {
    const int a = up[4 * u], b = up[4 * u + 1];
    const int64_t iab = up[4 * u + 2], iba = up[4 * u + 3];
    const int ta = type[a], tb = type[b], na = nfun[a], nb = nfun[b];
    if (na > GB || nb > GB || na < 0 || nb < 0 || (ta | tb) & ~1) continue;  // outside the 14 x 14 blocks: skipped
    const int kab = 2 * ta + tb, kba = 2 * tb + ta;
    const double* GAa = rot + ((int64_t)water[a] * 2 + ta) * GB2;
    const double* GBa = rot + ((int64_t)water[a] * 2 + tb) * GB2;
    const double* GAb = rot + ((int64_t)water[b] * 2 + ta) * GB2;
    const double* GBb = rot + ((int64_t)water[b] * 2 + tb) * GB2;
    for (int e = lane; e < GB2; e += 32) {
      const int r = e / GB, c = e % GB;
      double p1 = 0.0, p2 = 0.0;
      if (r < na && c < nb) {
        p1 = (double)(y[iab * GB2 + e] * t_std[kab * GB2 + e] + t_mean[kab * GB2 + e]);
        const int et = c * GB + r;  // (c, r) of the (B, A) block
        p2 = (double)(y[iba * GB2 + et] * t_std[kba * GB2 + et] + t_mean[kba * GB2 + et]);
      }
      P1[e] = p1;
      P2[e] = p2;
    }
    __syncwarp();
    for (int e = lane; e < GB2; e += 32) {
      const int r = e / GB, c = e % GB;
      double s1 = 0.0, s2 = 0.0;
      if (r < na && c < nb)
        for (int k = 0; k < nb; ++k) {
          s1 += P1[r * GB + k] * GBa[c * GB + k];
          s2 += P2[r * GB + k] * GBb[c * GB + k];
        }
      T1[e] = s1;
      T2[e] = s2;
    }
    __syncwarp();
    const int64_t fa = first[a], fb = first[b];
    for (int e = lane; e < GB2; e += 32) {
      const int r = e / GB, c = e % GB;
      // a diagonal block (A = B) is written from its upper triangle only, both
      // positions with one value, so the density is exactly symmetric
      if (r < na && c < nb && (a != b || r <= c)) {
        double s = 0.0;
        for (int k = 0; k < na; ++k) s += GAa[r * GB + k] * T1[k * GB + c] + GAb[r * GB + k] * T2[k * GB + c];
        if (a == b)  // average the two rounding-level different halves
          for (int k = 0; k < na; ++k) s += GAa[c * GB + k] * T1[k * GB + r] + GAb[c * GB + k] * T2[k * GB + r];
        s *= a == b ? 0.25 : 0.5;
        D[(fa + r) * n + fb + c] = s;
        D[(fb + c) * n + fa + r] = s;
      }
    }
    __syncwarp();
  }
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
  k_gemm<0><<<grid, GT, 0, st>>>(m, n, k, k, x, k, 1, w, 1, k, bias, act, z, y_bf16, y_f32, nullptr);
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
    k_gemm<1><<<grid, GT, 0, st>>>(n, k, m, kchunk, dz_scratch, 1, n, x, k, 1, nullptr, 0, nullptr, nullptr,
                                   nullptr, dw);
  }
  // dX[m x k] = dZ W: inner dimension n
  if (dx) {
    if (cudaMemsetAsync(dx, 0, (size_t)m * k * sizeof(float), st) != cudaSuccess) return RIJK_ERR_CUDA;
    const dim3 grid((unsigned)((k + TN - 1) / TN), (unsigned)((m + TM - 1) / TM), 1);
    rijk::count_launch();
    k_gemm<1><<<grid, GT, 0, st>>>(m, k, n, n, dz_scratch, n, 1, w, k, 1, nullptr, 0, nullptr, nullptr, nullptr,
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

int rijk_guess_assemble(const float* y, const float* t_mean, const float* t_std, const int32_t* upairs,
                        int64_t npairs, const int32_t* atom_first, const int32_t* atom_type, const int32_t* atom_nfun,
                        const int32_t* atom_water, const double* rot, int64_t num_basis, double* dm, void* stream) {
  if (!y || !t_mean || !t_std || !upairs || !atom_first || !atom_type || !atom_nfun || !atom_water || !rot || !dm ||
      npairs < 0 || num_basis <= 0)
    return RIJK_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(dm, 0, (size_t)num_basis * num_basis * sizeof(double), st) != cudaSuccess) return RIJK_ERR_CUDA;
  if (npairs == 0) return RIJK_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>((npairs + 3) / 4, 148 * 16);
  rijk::count_launch();
  k_guess_assemble<<<blocks, 128, 0, st>>>(y, t_mean, t_std, upairs, npairs, atom_first, atom_type, atom_nfun,
                                           atom_water, rot, num_basis, dm);
  return launch_status();
}

int rijk_mlp_to_bf16(const float* src, uint16_t* dst, int64_t count, void* stream) {
  if (!src || !dst || count <= 0) return RIJK_ERR_ARG;
  rijk::count_launch();
  k_to_bf16<<<grid_for(count), NT, 0, static_cast<cudaStream_t>(stream)>>>(count, src, dst);
  return launch_status();
}

}  // extern "C"
