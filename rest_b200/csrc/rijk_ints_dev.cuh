// Device code of the Coulomb integral engine shared by rijk_ints_gpu.cu (plan,
// two-centre kernel, launches) and rijk_ints_cls.cu (one three-centre class per
// translation unit, compiled in parallel).
// Classes up to 90 Cartesian component triples (and total l <= 6) are fully
// unrolled, so their Hermite tables live in registers; the larger ones keep
// their component loops rolled, which bounds code size and compile time.
// McMurchie-Davidson: Hermite expansion coefficients of the bra pair and of the
// single-centre ket, Hermite Coulomb integrals R_tuv from the Boys function, the
// Cartesian block, then real solid harmonics through the c2s matrices held in
// constant memory (one copy per translation unit, loaded by its own
// upload_tables).  Supported: AO shells l <= 2, auxiliary shells l <= 4.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace rijk {
namespace intsdev {

constexpr int GLA = 2;                                    // max AO l
constexpr int GLC = 4;                                    // max auxiliary l
constexpr int GL = 2 * GLA + GLC;                         // max total l of (ab|c) and (c|d)
constexpr int NTET = (GL + 1) * (GL + 2) * (GL + 3) / 6;  // R_tuv with t+u+v <= GL
constexpr double SCREEN_EXPONENT = 75.0;  // skip primitive pairs with mu |AB|^2 above this
// Boys function table: F_n(T) for n = 0..BOYS_NMAX at T = i * BOYS_STEP,
// i = 0..BOYS_NGRID-1 (T <= 40); orders above GL feed the Taylor expansion.
constexpr int BOYS_TAYLOR = 7;
constexpr int BOYS_NMAX = GL + BOYS_TAYLOR;
constexpr int BOYS_NGRID = 801;
constexpr double BOYS_STEP = 0.05;
constexpr double BOYS_TMAX = 40.0;
constexpr int C2S_TOTAL = 1 * 1 + 3 * 3 + 5 * 6 + 7 * 10 + 9 * 15;
struct DShells {
  int nshell;
  const int* l;
  const int* nprim;
  const int64_t* prim_off;
  const double* exps;
  const double* coefs;
  const double* centers;
  const int64_t* fun_off;
};

using Int3cKernel = void (*)(DShells, DShells, const int*, const int*, int, const int*, int, int64_t, int64_t,
                             double*);
// three-centre class kernels and table loaders, one pair per class
// (rijk_ints_cls.cu compiled with RIJK_LA, RIJK_LB, RIJK_LC)
#define RIJK_INT3C_CLASS(a, b, c)               \
  Int3cKernel int3c_kernel_##a##b##c();         \
  int int3c_tables_##a##b##c(const double* flat, const int* off, const double* boys);
#define RIJK_INT3C_LC(a, b) \
  RIJK_INT3C_CLASS(a, b, 0) RIJK_INT3C_CLASS(a, b, 1) RIJK_INT3C_CLASS(a, b, 2) RIJK_INT3C_CLASS(a, b, 3) \
  RIJK_INT3C_CLASS(a, b, 4)
RIJK_INT3C_LC(0, 0)
RIJK_INT3C_LC(0, 1)
RIJK_INT3C_LC(0, 2)
RIJK_INT3C_LC(1, 0)
RIJK_INT3C_LC(1, 1)
RIJK_INT3C_LC(1, 2)
RIJK_INT3C_LC(2, 0)
RIJK_INT3C_LC(2, 1)
RIJK_INT3C_LC(2, 2)
#undef RIJK_INT3C_LC
#undef RIJK_INT3C_CLASS

namespace {

__constant__ double c_c2s[C2S_TOTAL];
__constant__ int c_c2s_off[GLC + 1];
__device__ double g_boys[BOYS_NGRID * (BOYS_NMAX + 1)];

// loads this translation unit's copies of the c2s and Boys tables
int upload_tables(const double* flat, const int* off, const double* boys) {
  if (cudaMemcpyToSymbol(c_c2s, flat, C2S_TOTAL * sizeof(double)) != cudaSuccess) return 1;
  if (cudaMemcpyToSymbol(c_c2s_off, off, (GLC + 1) * sizeof(int)) != cudaSuccess) return 1;
  if (cudaMemcpyToSymbol(g_boys, boys, sizeof(double) * BOYS_NGRID * (BOYS_NMAX + 1)) != cudaSuccess) return 1;
  return 0;
}

__device__ __forceinline__ int ncart_d(int l) { return (l + 1) * (l + 2) / 2; }
__device__ __forceinline__ int tet(int t, int u, int v) {
  const int s = t + u + v, w = u + v;
  return s * (s + 1) * (s + 2) / 6 + w * (w + 1) / 2 + v;
}
// Cartesian component c of l, ordered by descending x power, then descending y:
// component c lies in row r (x power l - r) with r(r+1)/2 <= c < (r+1)(r+2)/2.
__device__ __forceinline__ void cart_ijk(int l, int c, int& i, int& j, int& k) {
  int r = 0;
  while ((r + 1) * (r + 2) / 2 <= c) ++r;
  i = l - r;
  j = r - (c - r * (r + 1) / 2);
  k = l - i - j;
}
__device__ __forceinline__ double c2s_at(int l, int m, int c) { return c_c2s[c_c2s_off[l] + m * ncart_d(l) + c]; }

// Boys function F_n(T), n = 0..nmax (nmax <= GL).  T <= 40: F_nmax from a
// Taylor expansion about the nearest tabulated point, dF_n/dT = -F_{n+1}, so
// F_nmax(T0 + d) = sum_k F_{nmax+k}(T0) (-d)^k / k! (|d| <= 0.025, seven terms:
// truncation below 2e-15 relative), then downward recursion
// F_{m-1} = (2T F_m + e^-T) / (2m-1).  T > 40: the asymptotic F_0 and upward
// recursion (stable there).  The table is filled on the host from the series.
__device__ void boys_d(int nmax, double T, double* F) {
  if (T > BOYS_TMAX) {
    F[0] = 0.5 * sqrt(3.14159265358979323846 / T);
    const double e = exp(-T);
    const double h = 0.5 / T;
    for (int n = 0; n < nmax; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) * h;
    return;
  }
  const int i = __double2int_rn(T * (1.0 / BOYS_STEP));
  const double d = T - i * BOYS_STEP;
  const double* row = g_boys + i * (BOYS_NMAX + 1) + nmax;
  // Horner form of sum_k row[k] (-d)^k / k!
  double f = row[BOYS_TAYLOR - 1];
#pragma unroll
  for (int k = BOYS_TAYLOR - 1; k >= 1; --k) f = row[k - 1] - d * f * (1.0 / k);
  F[nmax] = f;
  const double e = exp(-T);
  for (int m = nmax; m > 0; --m) F[m - 1] = (2 * T * F[m] + e) * (1.0 / (2 * m - 1));
}

// ---- three-centre integrals, one kernel per angular class (LA, LB, LC) -----------
// With the class fixed at compile time every angular loop has constant bounds,
// so the Hermite tables index with constants and live in registers for the
// small classes, and a warp runs one code path.

__host__ __device__ constexpr int ncart_c(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int cx_c(int l, int c) {
  int r = 0;
  while ((r + 1) * (r + 2) / 2 <= c) ++r;
  return l - r;
}
__host__ __device__ constexpr int cy_c(int l, int c) {
  int r = 0;
  while ((r + 1) * (r + 2) / 2 <= c) ++r;
  return r - (c - r * (r + 1) / 2);
}
__host__ __device__ constexpr int cz_c(int l, int c) { return l - cx_c(l, c) - cy_c(l, c); }

template <int LA, int LB>
__device__ __forceinline__ void herm_pair_t(double a, double b, double AB, double (&e)[LA + 1][LB + 1][LA + LB + 1]) {
  const double p = a + b, mu = a * b / p;
  const double XPA = -b / p * AB, XPB = a / p * AB, oo2p = 0.5 / p;
  e[0][0][0] = exp(-mu * AB * AB);
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j) {
      if (i == 0 && j == 0) continue;
      const int im = i > 0 ? i - 1 : i, jm = i > 0 ? j : j - 1;
      const double X = i > 0 ? XPA : XPB;
#pragma unroll
      for (int t = 0; t <= i + j; ++t) {
        double v = (t <= i + j - 1) ? X * e[im][jm][t] : 0.0;
        if (t > 0) v += oo2p * e[im][jm][t - 1];
        if (t + 1 <= i + j - 1) v += (t + 1) * e[im][jm][t + 1];
        e[i][j][t] = v;
      }
    }
}

template <int LC>
__device__ __forceinline__ void herm_single_t(double g, double (&f)[LC + 1][LC + 1]) {
  const double oo2g = 0.5 / g;
  f[0][0] = 1.0;
#pragma unroll
  for (int k = 1; k <= LC; ++k)
#pragma unroll
    for (int t = 0; t <= k; ++t) {
      double v = 0.0;
      if (t > 0) v += oo2g * f[k - 1][t - 1];
      if (t + 1 <= k - 1) v += (t + 1) * f[k - 1][t + 1];
      f[k][t] = v;
    }
}

// R^0_tuv (t+u+v <= L) in one buffer: level n is written over level n+1 in
// descending order of t+u+v, so each entry is replaced only after every entry
// that reads it (sums s-1 and s-2) has been updated.  UNR: loops unrolled so
// that the buffer indexes with constants.
template <int L, bool UNR>
__device__ __forceinline__ void herm_r_t(double alpha, const double* PC, double* r) {
  double F[L + 1];
  const double T = alpha * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
  boys_d(L, T, F);
  double f = 1.0;
#pragma unroll
  for (int n = 0; n < L; ++n) f *= -2.0 * alpha;
  r[0] = f * F[L];
  auto entry = [&](int t, int u, int v) {
    double val;
    if (t > 0) {
      val = PC[0] * r[tet(t - 1, u, v)];
      if (t > 1) val += (t - 1) * r[tet(t - 2, u, v)];
    } else if (u > 0) {
      val = PC[1] * r[tet(t, u - 1, v)];
      if (u > 1) val += (u - 1) * r[tet(t, u - 2, v)];
    } else {
      val = PC[2] * r[tet(t, u, v - 1)];
      if (v > 1) val += (v - 1) * r[tet(t, u, v - 2)];
    }
    r[tet(t, u, v)] = val;
  };
  if constexpr (UNR) {
#pragma unroll
    for (int n = L - 1; n >= 0; --n) {
      f /= -2.0 * alpha;
#pragma unroll
      for (int s = L - n; s >= 1; --s)
#pragma unroll
        for (int w = 0; w <= s; ++w)
#pragma unroll
          for (int v = 0; v <= w; ++v) entry(s - w, w - v, v);
      r[0] = f * F[n];
    }
  } else {
#pragma unroll 1
    for (int n = L - 1; n >= 0; --n) {
      f /= -2.0 * alpha;
#pragma unroll 1
      for (int s = L - n; s >= 1; --s)
        for (int w = 0; w <= s; ++w)
          for (int v = 0; v <= w; ++v) entry(s - w, w - v, v);
      r[0] = f * F[n];
    }
  }
}

// Cartesian (a u, b w | c qc) of one primitive triple, without the prefactor:
// sum over the bra Hermite indices of E^x E^y E^z times the signed ket sum of R.
template <int LA, int LB, int LC>
__device__ __forceinline__ double cart_value(int u, int w, int qc, const double (&ex)[LA + 1][LB + 1][LA + LB + 1],
                                             const double (&ey)[LA + 1][LB + 1][LA + LB + 1],
                                             const double (&ez)[LA + 1][LB + 1][LA + LB + 1],
                                             const double (&fk)[LC + 1][LC + 1], const double* r) {
  const int i1 = cx_c(LA, u), j1 = cy_c(LA, u), k1 = cz_c(LA, u);
  const int i2 = cx_c(LB, w), j2 = cy_c(LB, w), k2 = cz_c(LB, w);
  const int i3 = cx_c(LC, qc), j3 = cy_c(LC, qc), k3 = cz_c(LC, qc);
  double v = 0.0;
#pragma unroll
  for (int t = 0; t <= i1 + i2; ++t)
#pragma unroll
    for (int uu = 0; uu <= j1 + j2; ++uu)
#pragma unroll
      for (int vv = 0; vv <= k1 + k2; ++vv) {
        double inner = 0.0;
        // f[k][t] vanishes unless k - t is even
#pragma unroll
        for (int tt = i3 & 1; tt <= i3; tt += 2)
#pragma unroll
          for (int ww = j3 & 1; ww <= j3; ww += 2)
#pragma unroll
            for (int zz = k3 & 1; zz <= k3; zz += 2) {
              const double fv = fk[i3][tt] * fk[j3][ww] * fk[k3][zz];
              inner += (((tt + ww + zz) & 1) ? -fv : fv) * r[tet(t + tt, uu + ww, vv + zz)];
            }
        v += ex[i1][i2][t] * ey[j1][j2][uu] * ez[k1][k2][vv] * inner;
      }
  return v;
}

// acc[(u NB + w) SC + mc] += pref * sum_qc c2s[mc][qc] (a u, b w | c qc)
template <int LA, int LB, int LC>
__device__ __forceinline__ void accumulate_ab(int u, int w, double pref, double* acc,
                                              const double (&ex)[LA + 1][LB + 1][LA + LB + 1],
                                              const double (&ey)[LA + 1][LB + 1][LA + LB + 1],
                                              const double (&ez)[LA + 1][LB + 1][LA + LB + 1],
                                              const double (&fk)[LC + 1][LC + 1], const double* r) {
  constexpr int NB = ncart_c(LB), NC = ncart_c(LC), SC = 2 * LC + 1;
  double vq[NC];
#pragma unroll
  for (int qc = 0; qc < NC; ++qc) vq[qc] = cart_value<LA, LB, LC>(u, w, qc, ex, ey, ez, fk, r);
#pragma unroll
  for (int mc = 0; mc < SC; ++mc) {
    double s = 0.0;
#pragma unroll
    for (int qc = 0; qc < NC; ++qc) s += c2s_at(LC, mc, qc) * vq[qc];
    acc[(u * NB + w) * SC + mc] += pref * s;
  }
}

// task = kk * npc + q: shell pair q of class (LA, LB), auxiliary shell kc[kk]
// of angular momentum LC.  Rows are written relative to P0.  Small classes
// unroll every angular loop (tables in registers); large ones keep the
// component loops rolled, which bounds code size and compile time.
template <int LA, int LB, int LC>
__global__ void __launch_bounds__(128) k_int3c2e_cls(DShells A, DShells Cs, const int* __restrict__ pi,
                                                     const int* __restrict__ pj, int npc,
                                                     const int* __restrict__ kc, int nkc, int64_t npair_fun,
                                                     int64_t P0, double* __restrict__ out) {
  constexpr int NA = ncart_c(LA), NB = ncart_c(LB), NC = ncart_c(LC);
  constexpr int SA = 2 * LA + 1, SB = 2 * LB + 1, SC = 2 * LC + 1;
  constexpr int L = LA + LB + LC, NT = (L + 1) * (L + 2) * (L + 3) / 6;
  constexpr bool UNR = L <= 6 && NA * NB * NC <= 90;
  const int64_t task = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (task >= (int64_t)npc * nkc) return;
  const int q = (int)(task % npc), k = kc[task / npc];
  const int i = pi[q], j = pj[q];
  const double* Ra = A.centers + 3 * i;
  const double* Rb = A.centers + 3 * j;
  const double* Rc = Cs.centers + 3 * k;
  const double AB[3] = {Ra[0] - Rb[0], Ra[1] - Rb[1], Ra[2] - Rb[2]};
  const double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  double acc[NA * NB * SC];  // (Cartesian a, Cartesian b | spherical c)
#pragma unroll
  for (int x = 0; x < NA * NB * SC; ++x) acc[x] = 0.0;
  const int npa = A.nprim[i], npb = A.nprim[j], npk = Cs.nprim[k];
  const int64_t oa = A.prim_off[i], ob = A.prim_off[j], oc = Cs.prim_off[k];
  for (int pa = 0; pa < npa; ++pa)
    for (int pb = 0; pb < npb; ++pb) {
      const double a = A.exps[oa + pa], b = A.exps[ob + pb];
      const double p = a + b;
      // primitive-pair screening (libcint's exponent cutoff): the Gaussian
      // product carries exp(-mu |AB|^2); beyond mu |AB|^2 = 75 every term of the
      // pair is below 1e-28 of the largest integral
      if (a * b / p * AB2 > SCREEN_EXPONENT) continue;
      const double cab = A.coefs[oa + pa] * A.coefs[ob + pb];
      double ex[LA + 1][LB + 1][LA + LB + 1], ey[LA + 1][LB + 1][LA + LB + 1], ez[LA + 1][LB + 1][LA + LB + 1];
      herm_pair_t<LA, LB>(a, b, AB[0], ex);
      herm_pair_t<LA, LB>(a, b, AB[1], ey);
      herm_pair_t<LA, LB>(a, b, AB[2], ez);
      const double P[3] = {(a * Ra[0] + b * Rb[0]) / p, (a * Ra[1] + b * Rb[1]) / p, (a * Ra[2] + b * Rb[2]) / p};
      for (int pc = 0; pc < npk; ++pc) {
        const double g = Cs.exps[oc + pc];
        double fk[LC + 1][LC + 1];  // x, y and z share the single-centre coefficients
        herm_single_t<LC>(g, fk);
        const double alpha = p * g / (p + g);
        const double PC[3] = {P[0] - Rc[0], P[1] - Rc[1], P[2] - Rc[2]};
        double r[NT];
        herm_r_t<L, UNR>(alpha, PC, r);
        const double pref = 2.0 * 17.493418327624862 / (p * g * sqrt(p + g)) * cab * Cs.coefs[oc + pc];
        if constexpr (UNR) {
#pragma unroll
          for (int u = 0; u < NA; ++u)
#pragma unroll
            for (int w = 0; w < NB; ++w) accumulate_ab<LA, LB, LC>(u, w, pref, acc, ex, ey, ez, fk, r);
        } else {
#pragma unroll 1
          for (int u = 0; u < NA; ++u)
#pragma unroll 1
            for (int w = 0; w < NB; ++w) accumulate_ab<LA, LB, LC>(u, w, pref, acc, ex, ey, ez, fk, r);
        }
      }
    }
  // bra to spherical and store the packed upper triangle
  const int64_t fa = A.fun_off[i], fb = A.fun_off[j];
#pragma unroll
  for (int mc = 0; mc < SC; ++mc) {
    double* row = out + (Cs.fun_off[k] + mc - P0) * npair_fun;
#pragma unroll
    for (int ma = 0; ma < SA; ++ma) {
      double half[NB];
#pragma unroll
      for (int cb = 0; cb < NB; ++cb) {
        double v = 0.0;
#pragma unroll
        for (int ca = 0; ca < NA; ++ca) v += c2s_at(LA, ma, ca) * acc[(ca * NB + cb) * SC + mc];
        half[cb] = v;
      }
      const int64_t mu = fa + ma;
#pragma unroll
      for (int mb = 0; mb < SB; ++mb) {
        const int64_t nu = fb + mb;
        if (mu > nu) continue;
        double v = 0.0;
#pragma unroll
        for (int cb = 0; cb < NB; ++cb) v += c2s_at(LB, mb, cb) * half[cb];
        row[nu * (nu + 1) / 2 + mu] = v;
      }
    }
  }
}


}  // namespace
}  // namespace intsdev
}  // namespace rijk
