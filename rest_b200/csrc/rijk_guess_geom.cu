// Geometry of the learned initial guess on the device: water frames, shell
// rotations, the atom pairs within the cutoff and their 53 standardised
// features, for a whole molecule set in three launches.  REST has no learned
// guess; these kernels feed the network whose density replaces REST's guess
// (src/initial_guess/mod.rs:15-80) when its electron count checks out.
//
//   frames     one thread per water (atoms 3w, 3w+1, 3w+2 = O, H1, H2): origin O,
//              axes p = unit(OH1 - OH2), b = unit(OH1 + OH2 - (.p) p), n = p x b;
//              the rotation G_l of the real solid harmonics l = 1, 2 under
//              r -> F^T r, G_l^T = pinv(Y_l(S)) Y_l(S F) over 40 fixed sample
//              points S (exact: both sides are degree-l polynomials), and per
//              element the block-diagonal rotation of its shells (14 x 14);
//   counts     one warp per atom A: neighbours B of A's molecule with |AB| <= cutoff
//              (all B, and B >= A), and the 8 + 8 Gaussian radial counts of O and
//              H neighbours (B != A, smooth cosine cutoff);
//   pairs      one warp per atom A: the ordered pairs (A, B) in ascending B, rows
//              at the exclusive scan of the counts, each row the pair's features
//              standardised by the network's feature mean and deviation; the
//              unordered pairs A <= B with the rows of (A, B) and (B, A), indices
//              local to the molecule, as the density assembly reads them.
//
// The constants (sample points, Cartesian exponents, harmonic expansions,
// pseudo-inverses, cutoff, radial centres and width) come from the caller in
// one table of GEO_TABLE doubles.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/rest_b200.h"
#include "rijk_internal.h"

namespace {

constexpr int NS = 40;   // sample points of the rotation fit
constexpr int GB = 14;   // AO block edge
constexpr int NF = 53;   // features per pair
constexpr int MAXSH = 15;
// table layout (doubles)
constexpr int T_SAMPLES = 0;                 // NS x 3
constexpr int T_L1 = T_SAMPLES + NS * 3;     // exps 3 x 3, c2s^T 3 x 3, pinv 3 x NS
constexpr int T_L2 = T_L1 + 9 + 9 + 3 * NS;  // exps 6 x 3, c2s^T 6 x 5, pinv 5 x NS
constexpr int T_PAR = T_L2 + 18 + 30 + 5 * NS;  // cutoff, sigma, mu[8]
constexpr int T_SIZE = T_PAR + 10;
static_assert(T_SIZE == 516, "table layout");

// |x_a - x_b| without contraction, so that every kernel (and both orders of a
// pair) takes the same decision at the cutoff
__device__ __forceinline__ double pair_dist(const double* __restrict__ xyz, int64_t a, int64_t b) {
  const double dx = __dsub_rn(xyz[3 * a], xyz[3 * b]);
  const double dy = __dsub_rn(xyz[3 * a + 1], xyz[3 * b + 1]);
  const double dz = __dsub_rn(xyz[3 * a + 2], xyz[3 * b + 2]);
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// G (NM x NM, row-major, G[i][j]) of the degree-L harmonics under the frame F
template <int L>
__device__ void shell_rotation(const double* __restrict__ tab, const double F[9], double* G) {
  constexpr int NC = (L + 1) * (L + 2) / 2, NM = 2 * L + 1;
  const double* ex = tab + (L == 1 ? T_L1 : T_L2);
  const double* c2s_t = ex + 3 * NC;  // NC x NM
  const double* pinv = c2s_t + NC * NM;  // NM x NS
  double acc[NM][NM];
#pragma unroll
  for (int j = 0; j < NM; ++j)
#pragma unroll
    for (int i = 0; i < NM; ++i) acc[j][i] = 0.0;
  for (int s = 0; s < NS; ++s) {
    const double* u = tab + T_SAMPLES + 3 * s;
    double pt[3];  // F^T u: pt[k] = sum_j u[j] F[j][k]
#pragma unroll
    for (int k = 0; k < 3; ++k) pt[k] = u[0] * F[k] + u[1] * F[3 + k] + u[2] * F[6 + k];
    double y[NM];
#pragma unroll
    for (int m = 0; m < NM; ++m) y[m] = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double mono = 1.0;
#pragma unroll
      for (int k = 0; k < 3; ++k)
        for (int e = 0; e < (int)ex[3 * c + k]; ++e) mono *= pt[k];
#pragma unroll
      for (int m = 0; m < NM; ++m) y[m] += mono * c2s_t[c * NM + m];
    }
#pragma unroll
    for (int j = 0; j < NM; ++j) {
      const double pj = pinv[j * NS + s];
#pragma unroll
      for (int i = 0; i < NM; ++i) acc[j][i] += pj * y[i];
    }
  }
#pragma unroll
  for (int i = 0; i < NM; ++i)
#pragma unroll
    for (int j = 0; j < NM; ++j) G[i * NM + j] = acc[j][i];
}

__global__ void __launch_bounds__(128) k_guess_frames(const double* __restrict__ xyz, int64_t nwater,
                                                      const double* __restrict__ tab,
                                                      const int32_t* __restrict__ elem_shells,
                                                      double* __restrict__ frames, double* __restrict__ rot) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwater) return;
  const double* o = xyz + 9 * w;
  double h1[3], h2[3], p[3], b[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    h1[k] = o[3 + k] - o[k];
    h2[k] = o[6 + k] - o[k];
    p[k] = h1[k] - h2[k];
    b[k] = h1[k] + h2[k];
  }
  const double np_ = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) p[k] /= np_;
  const double bp = b[0] * p[0] + b[1] * p[1] + b[2] * p[2];
#pragma unroll
  for (int k = 0; k < 3; ++k) b[k] -= bp * p[k];
  const double nb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) b[k] /= nb;
  const double F[9] = {p[0], p[1], p[2], b[0], b[1], b[2],
                       p[1] * b[2] - p[2] * b[1], p[2] * b[0] - p[0] * b[2], p[0] * b[1] - p[1] * b[0]};
#pragma unroll
  for (int k = 0; k < 9; ++k) frames[9 * w + k] = F[k];
  double G1[9], G2[25];
  shell_rotation<1>(tab, F, G1);
  shell_rotation<2>(tab, F, G2);
  for (int t = 0; t < 2; ++t) {
    double* R = rot + (w * 2 + t) * GB * GB;
    for (int e = 0; e < GB * GB; ++e) R[e] = 0.0;
    const int32_t* sl = elem_shells + t * (MAXSH + 1);
    const int ns = sl[0] < 0 ? 0 : (sl[0] > MAXSH ? MAXSH : sl[0]);
    int off = 0;
    for (int s = 0; s < ns; ++s) {
      const int l = sl[1 + s], d = 2 * l + 1;
      if (l < 0 || l > 2 || off + d > GB) break;  // the host refuses such element blocks
      for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j)
          R[(off + i) * GB + off + j] = l == 0 ? 1.0 : (l == 1 ? G1[i * 3 + j] : G2[i * 5 + j]);
      off += d;
    }
  }
}

// atom_info per atom: first atom of its molecule, atoms in the molecule, element type (0 O, 1 H)
__device__ __forceinline__ bool atom_span(const int32_t* __restrict__ info, int64_t a, int64_t natom, int64_t& m0,
                                          int64_t& m1) {
  m0 = info[3 * a];
  m1 = m0 + info[3 * a + 1];
  return m0 >= 0 && m0 <= a && m1 > a && m1 <= natom;
}

__global__ void __launch_bounds__(128) k_guess_counts(const double* __restrict__ xyz,
                                                      const int32_t* __restrict__ info, int64_t natom,
                                                      const double* __restrict__ tab, int64_t* __restrict__ counts,
                                                      double* __restrict__ env) {
  const int lane = threadIdx.x & 31;
  const int64_t a = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (a >= natom) return;
  int64_t m0, m1;
  const bool ok = atom_span(info, a, natom, m0, m1);
  const double cut = tab[T_PAR], sig2 = tab[T_PAR + 1] * tab[T_PAR + 1];
  int64_t cnt = 0, cup = 0;
  double e[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) e[k] = 0.0;
  if (ok)
    for (int64_t b = m0 + lane; b < m1; b += 32) {
      const double d = pair_dist(xyz, a, b);
      if (d <= cut) {
        ++cnt;
        if (b >= a) ++cup;
      }
      if (b != a && d < cut) {
        const double fc = 0.5 * (cos(M_PI * d / cut) + 1.0);
        const int tb = info[3 * b + 2] & 1;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const double x = d - tab[T_PAR + 2 + k];
          const double g = exp(-(x * x) / sig2) * fc;
          if (tb == 0)
            e[k] += g;
          else
            e[8 + k] += g;
        }
      }
    }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    cnt += __shfl_xor_sync(0xffffffffu, cnt, s);
    cup += __shfl_xor_sync(0xffffffffu, cup, s);
#pragma unroll
    for (int k = 0; k < 16; ++k) e[k] += __shfl_xor_sync(0xffffffffu, e[k], s);
  }
  if (lane == 0) {
    counts[2 * a] = cnt;
    counts[2 * a + 1] = cup;
  }
  if (lane < 16) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < 16; ++k) v = k == lane ? e[k] : v;
    env[16 * a + lane] = v;
  }
}

__global__ void __launch_bounds__(128) k_guess_pairs(
    const double* __restrict__ xyz, const int32_t* __restrict__ info, int64_t natom, const double* __restrict__ tab,
    const double* __restrict__ frames, const double* __restrict__ env, const int64_t* __restrict__ pair_off,
    const int64_t* __restrict__ up_off, int64_t npairs, int64_t nup, const double* __restrict__ f_mean,
    const double* __restrict__ f_std, float* __restrict__ feats, int32_t* __restrict__ up) {
  const int lane = threadIdx.x & 31;
  const int64_t a = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (a >= natom) return;
  int64_t m0, m1;
  if (!atom_span(info, a, natom, m0, m1)) return;
  const double cut = tab[T_PAR];
  const int64_t wa = a / 3;  // molecules start at a multiple of 3 atoms
  const double* F = frames + 9 * wa;
  const int ta = info[3 * a + 2] & 1;
  const unsigned lt = (1u << lane) - 1u;
  int64_t row = pair_off[a], urow = up_off[a];
  const int64_t prow0 = pair_off[m0];
  for (int64_t b0 = m0; b0 < m1; b0 += 32) {
    const int64_t b = b0 + lane;
    const bool in = b < m1 && pair_dist(xyz, a, b) <= cut;
    const unsigned mask = __ballot_sync(0xffffffffu, in);
    const unsigned umask = __ballot_sync(0xffffffffu, in && b >= a);
    if (in) {
      const int64_t r = row + __popc(mask & lt);
      if (r < npairs) {
        const int tb = info[3 * b + 2] & 1;
        const int64_t wb = b / 3;
        double f[NF];
        f[0] = ta == 0;
        f[1] = ta == 1;
        f[2] = tb == 0;
        f[3] = tb == 1;
        double dd = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const double v = F[3 * i] * (xyz[3 * b] - xyz[3 * a]) + F[3 * i + 1] * (xyz[3 * b + 1] - xyz[3 * a + 1]) +
                           F[3 * i + 2] * (xyz[3 * b + 2] - xyz[3 * a + 2]);
          f[4 + i] = v;
          dd += v * v;
        }
        f[7] = sqrt(dd);
        f[8] = wa == wb;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int64_t c = 3 * wb + k;
#pragma unroll
          for (int i = 0; i < 3; ++i)
            f[9 + 3 * k + i] = F[3 * i] * (xyz[3 * c] - xyz[3 * a]) + F[3 * i + 1] * (xyz[3 * c + 1] - xyz[3 * a + 1]) +
                               F[3 * i + 2] * (xyz[3 * c + 2] - xyz[3 * a + 2]);
        }
        const int64_t o = 3 * wa;
#pragma unroll
        for (int i = 0; i < 3; ++i)
          f[18 + i] = F[3 * i] * (xyz[3 * a] - xyz[3 * o]) + F[3 * i + 1] * (xyz[3 * a + 1] - xyz[3 * o + 1]) +
                      F[3 * i + 2] * (xyz[3 * a + 2] - xyz[3 * o + 2]);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          f[21 + k] = env[16 * a + k];
          f[37 + k] = env[16 * b + k];
        }
        float* out = feats + r * NF;
#pragma unroll
        for (int k = 0; k < NF; ++k) out[k] = (float)((f[k] - f_mean[k]) / f_std[k]);
        if (b >= a) {
          const int64_t u = urow + __popc(umask & lt);
          // row of (B, A): B's pairs run in ascending atom order, so A's place
          // among them is the number of B's neighbours before A
          int64_t rank = 0;
          for (int64_t c = m0; c < a; ++c) rank += pair_dist(xyz, b, c) <= cut;
          if (u < nup) {
            up[4 * u] = (int32_t)(a - m0);
            up[4 * u + 1] = (int32_t)(b - m0);
            up[4 * u + 2] = (int32_t)(r - prow0);
            up[4 * u + 3] = (int32_t)(pair_off[b] + rank - prow0);
          }
        }
      }
    }
    row += __popc(mask);
    urow += __popc(umask);
  }
}

unsigned warp_grid(int64_t natom) { return (unsigned)((natom * 32 + 127) / 128); }

}  // namespace

int rijk_guess_geometry(const double* xyz, const int32_t* atom_info, int64_t natom, const double* table,
                        const int32_t* elem_shells, double* frames, double* rot, int64_t* counts, double* env,
                        void* stream) {
  if (!xyz || !atom_info || !table || !elem_shells || !frames || !rot || !counts || !env || natom <= 0 ||
      natom % 3 != 0 || natom > ((int64_t)1 << 26))
    return RIJK_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t nw = natom / 3;
  rijk::count_launch(2);
  k_guess_frames<<<(unsigned)((nw + 127) / 128), 128, 0, st>>>(xyz, nw, table, elem_shells, frames, rot);
  k_guess_counts<<<warp_grid(natom), 128, 0, st>>>(xyz, atom_info, natom, table, counts, env);
  return cudaGetLastError() == cudaSuccess ? RIJK_OK : RIJK_ERR_CUDA;
}

int rijk_guess_pairs(const double* xyz, const int32_t* atom_info, int64_t natom, const double* table,
                     const double* frames, const double* env, const int64_t* pair_off, const int64_t* up_off,
                     int64_t npairs, int64_t nup, const double* f_mean, const double* f_std, float* feats,
                     int32_t* upairs, void* stream) {
  if (!xyz || !atom_info || !table || !frames || !env || !pair_off || !up_off || !f_mean || !f_std || !feats ||
      !upairs || natom <= 0 || natom % 3 != 0 || natom > ((int64_t)1 << 26) || npairs < 0 || nup < 0)
    return RIJK_ERR_ARG;
  if (npairs == 0) return RIJK_OK;
  rijk::count_launch();
  k_guess_pairs<<<warp_grid(natom), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      xyz, atom_info, natom, table, frames, env, pair_off, up_off, npairs, nup, f_mean, f_std, feats, upairs);
  return cudaGetLastError() == cudaSuccess ? RIJK_OK : RIJK_ERR_CUDA;
}
