// Two- and three-centre Coulomb integrals on the GPU, the device counterpart of
// rijk_ints.cpp.  REST computes (P|Q) (int_ij_aux_columb,
// src/molecule_io/mod.rs:1038, called at :1577) and the (mu nu|P) blocks of
// prepare_rimatr_for_ri_v_rayon_v02 (:1604-1660) with libcint on the host
// before its metric step; here both are produced in HBM, so the fitted tensor
// is built without a host round trip.  Three-centre blocks: one thread per
// (AO shell pair, auxiliary shell), one kernel per angular class
// (rijk_ints_dev.cuh) over shell pairs sorted by class and primitive count, so
// that a warp runs one code path.  Two-centre blocks: one thread per auxiliary
// shell pair with run-time angular loops (a small share of the work).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../include/rest_b200.h"
#include "rijk_ints_dev.cuh"
#include "rijk_internal.h"

namespace rijk {

using namespace intsdev;

namespace {

// The 45 three-centre classes (rijk_ints_cls.cu), indexed (3 la + lb) 5 + lc.
using Int3cTables = int (*)(const double*, const int*, const double*);
using Int3cGetter = Int3cKernel (*)();
#define RIJK_CLS5(f, a, b) f##a##b##0, f##a##b##1, f##a##b##2, f##a##b##3, f##a##b##4
#define RIJK_CLS45(f)                                                                                   \
  RIJK_CLS5(f, 0, 0), RIJK_CLS5(f, 0, 1), RIJK_CLS5(f, 0, 2), RIJK_CLS5(f, 1, 0), RIJK_CLS5(f, 1, 1), \
      RIJK_CLS5(f, 1, 2), RIJK_CLS5(f, 2, 0), RIJK_CLS5(f, 2, 1), RIJK_CLS5(f, 2, 2)
const Int3cTables* int3c_class_tables() {
  static const Int3cTables t[45] = {RIJK_CLS45(int3c_tables_)};
  return t;
}
const Int3cGetter* int3c_class_kernels() {
  static const Int3cGetter k[45] = {RIJK_CLS45(int3c_kernel_)};
  return k;
}
#undef RIJK_CLS45
#undef RIJK_CLS5

// 1D Hermite coefficients e[i][j][t] (t <= i + j) of a Gaussian product with
// exponents a, b and AB = A - B.  i <= GLC covers a lone auxiliary bra shell (j = 0).
using HermE = double[GLC + 1][GLA + 1][GLC + 1];
__device__ void herm_pair(int la, int lb, double a, double b, double AB, HermE& e) {
  const double p = a + b, mu = a * b / p;
  const double XPA = -b / p * AB, XPB = a / p * AB, oo2p = 0.5 / p;
  e[0][0][0] = exp(-mu * AB * AB);
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      const int im = i > 0 ? i - 1 : i, jm = i > 0 ? j : j - 1;  // the predecessor (im, jm), im + jm = i + j - 1
      const double X = i > 0 ? XPA : XPB;
      for (int t = 0; t <= i + j; ++t) {
        double v = (t <= i + j - 1) ? X * e[im][jm][t] : 0.0;
        if (t > 0) v += oo2p * e[im][jm][t - 1];
        if (t + 1 <= i + j - 1) v += (t + 1) * e[im][jm][t + 1];
        e[i][j][t] = v;
      }
    }
}

// single-centre Hermite coefficients f[k][t] (t <= k) of x^k exp(-g x^2)
using HermF = double[GLC + 1][GLC + 1];
__device__ void herm_single(int lc, double g, HermF& f) {
  f[0][0] = 1.0;
  const double oo2g = 0.5 / g;
  for (int k = 1; k <= lc; ++k)
    for (int t = 0; t <= k; ++t) {
      double v = 0.0;
      if (t > 0) v += oo2g * f[k - 1][t - 1];
      if (t + 1 <= k - 1) v += (t + 1) * f[k - 1][t + 1];
      f[k][t] = v;
    }
}

// R^0_tuv for t+u+v <= L at (alpha, PC) into r0 (tetrahedral index); r1 is scratch.
// Level n holds R^n_tuv for t+u+v <= L - n and is built from level n+1.
__device__ void herm_r(int L, double alpha, const double* PC, double* r0, double* r1) {
  double F[GL + 1];
  const double T = alpha * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
  boys_d(L, T, F);
  double* cur = (L & 1) ? r1 : r0;  // after L swaps, level 0 lands in r0
  double f = 1.0;
  for (int n = 0; n < L; ++n) f *= -2.0 * alpha;
  cur[0] = f * F[L];
  for (int n = L - 1; n >= 0; --n) {
    double* nxt = (cur == r0) ? r1 : r0;
    f /= -2.0 * alpha;
    const int top = L - n;
    nxt[0] = f * F[n];
    for (int s = 1; s <= top; ++s)
      for (int w = 0; w <= s; ++w)
        for (int v = 0; v <= w; ++v) {
          const int u = w - v, t = s - w;
          double val;
          if (t > 0) {
            val = PC[0] * cur[tet(t - 1, u, v)];
            if (t > 1) val += (t - 1) * cur[tet(t - 2, u, v)];
          } else if (u > 0) {
            val = PC[1] * cur[tet(t, u - 1, v)];
            if (u > 1) val += (u - 1) * cur[tet(t, u - 2, v)];
          } else {
            val = PC[2] * cur[tet(t, u, v - 1)];
            if (v > 1) val += (v - 1) * cur[tet(t, u, v - 2)];
          }
          nxt[tet(t, u, v)] = val;
        }
    cur = nxt;
  }
}

// (ab|c) Cartesian block, out[(ca*nb + cb)*nc + cc].  pair = false: the bra is
// shell ia alone (lb = 0, b = 0), which gives (a|c) for the two-centre metric.
__device__ void triple_d(const DShells& A, int ia, int ib, bool pair, const DShells& Cs, int ic, double* out) {
  const int la = A.l[ia], lb = pair ? A.l[ib] : 0, lc = Cs.l[ic];
  const int na = ncart_d(la), nb = ncart_d(lb), nc = ncart_d(lc);
  const double* Ra = A.centers + 3 * ia;
  const double* Rb = pair ? A.centers + 3 * ib : Ra;
  const double* Rc = Cs.centers + 3 * ic;
  for (int k = 0; k < na * nb * nc; ++k) out[k] = 0.0;
  HermE ex, ey, ez;
  HermF fx, fy, fz;
  double r0[NTET], r1[NTET];
  const int npa = A.nprim[ia], npb = pair ? A.nprim[ib] : 1;
  for (int pa = 0; pa < npa; ++pa)
    for (int pb = 0; pb < npb; ++pb) {
      const double a = A.exps[A.prim_off[ia] + pa];
      const double b = pair ? A.exps[A.prim_off[ib] + pb] : 0.0;
      const double cab = A.coefs[A.prim_off[ia] + pa] * (pair ? A.coefs[A.prim_off[ib] + pb] : 1.0);
      const double p = a + b;
      herm_pair(la, lb, a, b, Ra[0] - Rb[0], ex);
      herm_pair(la, lb, a, b, Ra[1] - Rb[1], ey);
      herm_pair(la, lb, a, b, Ra[2] - Rb[2], ez);
      const double P[3] = {(a * Ra[0] + b * Rb[0]) / p, (a * Ra[1] + b * Rb[1]) / p, (a * Ra[2] + b * Rb[2]) / p};
      for (int pc = 0; pc < Cs.nprim[ic]; ++pc) {
        const double g = Cs.exps[Cs.prim_off[ic] + pc];
        const double cg = Cs.coefs[Cs.prim_off[ic] + pc];
        herm_single(lc, g, fx);
        herm_single(lc, g, fy);
        herm_single(lc, g, fz);
        const double alpha = p * g / (p + g);
        const double PC[3] = {P[0] - Rc[0], P[1] - Rc[1], P[2] - Rc[2]};
        herm_r(la + lb + lc, alpha, PC, r0, r1);
        const double pref = 2.0 * 17.493418327624862 / (p * g * sqrt(p + g)) * cab * cg;  // 2 pi^(5/2)
        for (int u = 0; u < na; ++u) {
          int i1, j1, k1;
          cart_ijk(la, u, i1, j1, k1);
          for (int w = 0; w < nb; ++w) {
            int i2, j2, k2;
            cart_ijk(lb, w, i2, j2, k2);
            for (int q = 0; q < nc; ++q) {
              int i3, j3, k3;
              cart_ijk(lc, q, i3, j3, k3);
              double v = 0.0;
              for (int t = 0; t <= i1 + i2; ++t) {
                const double et = ex[i1][i2][t];
                for (int uu = 0; uu <= j1 + j2; ++uu) {
                  const double eu = et * ey[j1][j2][uu];
                  for (int vv = 0; vv <= k1 + k2; ++vv) {
                    const double ev = eu * ez[k1][k2][vv];
                    if (ev == 0.0) continue;
                    double inner = 0.0;
                    for (int tt = 0; tt <= i3; ++tt) {
                      const double ft = fx[i3][tt];
                      if (ft == 0.0) continue;
                      for (int ww = 0; ww <= j3; ++ww) {
                        const double fu = ft * fy[j3][ww];
                        if (fu == 0.0) continue;
                        for (int zz = 0; zz <= k3; ++zz) {
                          const double fv = fu * fz[k3][zz];
                          if (fv == 0.0) continue;
                          const double sg = ((tt + ww + zz) & 1) ? -1.0 : 1.0;
                          inner += sg * fv * r0[tet(t + tt, uu + ww, vv + zz)];
                        }
                      }
                    }
                    v += ev * inner;
                  }
                }
              }
              out[(u * nb + w) * nc + q] += pref * v;
            }
          }
        }
      }
    }
}

// In place: cart[ab*nc + mc] <- sum_cc c2s_lc[mc][cc] cart[ab*nc + cc], mc < 2 lc + 1.
__device__ void ket_to_sph(int nab, int lc, double* cart) {
  const int nc = ncart_d(lc), sc = 2 * lc + 1;
  for (int ab = 0; ab < nab; ++ab) {
    double tmp[2 * GLC + 1];
    for (int mc = 0; mc < sc; ++mc) {
      double v = 0.0;
      for (int cc = 0; cc < nc; ++cc) v += c2s_at(lc, mc, cc) * cart[ab * nc + cc];
      tmp[mc] = v;
    }
    for (int mc = 0; mc < sc; ++mc) cart[ab * nc + mc] = tmp[mc];
  }
}

// 2c2e over auxiliary shell pairs k1 <= k2: V (naux x naux, column-major, leading dim ldv).
__global__ void __launch_bounds__(64) k_int2c2e(DShells Cs, int nshell, int64_t ldv, double* __restrict__ V) {
  const int64_t task = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (task >= (int64_t)nshell * nshell) return;
  const int k1 = (int)(task % nshell), k2 = (int)(task / nshell);
  if (k1 > k2) return;
  const int l1 = Cs.l[k1], l2 = Cs.l[k2];
  const int n1 = ncart_d(l1), n2 = ncart_d(l2);
  double cart[15 * 15];
  triple_d(Cs, k1, 0, false, Cs, k2, cart);
  ket_to_sph(n1, l2, cart);
  for (int m2 = 0; m2 < 2 * l2 + 1; ++m2)
    for (int m1 = 0; m1 < 2 * l1 + 1; ++m1) {
      double v = 0.0;
      for (int c1 = 0; c1 < n1; ++c1) v += c2s_at(l1, m1, c1) * cart[c1 * n2 + m2];
      const int64_t r = Cs.fun_off[k1] + m1, c = Cs.fun_off[k2] + m2;
      V[r + ldv * c] = v;
      V[c + ldv * r] = v;
    }
}

}  // namespace

// Device copy of an (AO, auxiliary) pair of shell sets.  AO shell pairs are
// ordered by (l_i, l_j) so that a warp mostly runs one angular class.
struct RiIntPlan {
  // Every device array of the plan lives in one allocation from the
  // stream-ordered pool, filled by one copy and released in stream order.
  std::vector<unsigned char> host;  // staging image of that allocation
  std::vector<std::pair<const void**, size_t>> fixups;  // pointer field -> byte offset
  void* base = nullptr;
  cudaStream_t stream = nullptr;
  DShells A{}, C{};
  std::vector<int64_t> offA, offC;
  int64_t nA = 0, nC = 0;
  const int* dpi = nullptr;  // shell pairs sorted by (l_i, l_j, primitive count, separation)
  const int* dpj = nullptr;
  int npairs = 0;
  int pair_cls[10] = {};  // pairs of class la * 3 + lb are [pair_cls[c], pair_cls[c + 1])
  std::vector<int> aux_sorted;  // auxiliary shells sorted by (l, index)
  int aux_l_begin[GLC + 2] = {};
  const int* daux = nullptr;
  ~RiIntPlan() {
    if (base) cudaFreeAsync(base, stream);
  }
  template <class T>
  void up(const T*& field, const T* h, size_t n) {
    const size_t off = (host.size() + 255) / 256 * 256;
    host.resize(off + std::max<size_t>(n, 1) * sizeof(T));
    if (n) std::memcpy(host.data() + off, h, n * sizeof(T));
    fixups.push_back({reinterpret_cast<const void**>(&field), off});
  }
  int finalize(cudaStream_t st) {
    stream = st;
    if (cudaMallocAsync(&base, host.size(), st) != cudaSuccess) {
      cudaGetLastError();
      base = nullptr;
      return RIJK_ERR_NOMEM;
    }
    if (cudaMemcpyAsync(base, host.data(), host.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
      return RIJK_ERR_CUDA;
    for (auto& f : fixups) *f.first = static_cast<unsigned char*>(base) + f.second;
    return RIJK_OK;
  }
  int load(const rijk_shells* s, int lmax, DShells& d, std::vector<int64_t>& off, int64_t& nfun) {
    if (!s || s->nshell <= 0 || !s->l || !s->nprim || !s->prim_off || !s->exps || !s->coefs || !s->centers)
      return RIJK_ERR_ARG;
    if (s->nshell > (1 << 24)) return RIJK_ERR_TOO_LARGE;
    int64_t nprim_tot = 0;
    off.assign(s->nshell + 1, 0);
    nfun = 0;
    for (int64_t i = 0; i < s->nshell; ++i) {
      if (s->l[i] < 0 || s->nprim[i] <= 0 || s->prim_off[i] < 0) return RIJK_ERR_ARG;
      if (s->l[i] > lmax) return RIJK_ERR_TOO_LARGE;
      off[i] = nfun;
      nfun += 2 * s->l[i] + 1;
      nprim_tot = std::max<int64_t>(nprim_tot, s->prim_off[i] + s->nprim[i]);
    }
    off[s->nshell] = nfun;
    d.nshell = (int)s->nshell;
    up(d.l, s->l, s->nshell);
    up(d.nprim, s->nprim, s->nshell);
    up(d.prim_off, s->prim_off, s->nshell);
    up(d.exps, s->exps, nprim_tot);
    up(d.coefs, s->coefs, nprim_tot);
    up(d.centers, s->centers, 3 * s->nshell);
    up(d.fun_off, (const int64_t*)off.data(), s->nshell + 1);
    return RIJK_OK;
  }
};

namespace {

// F_n(T_i) for the device table: the series sum_k (2T)^k / ((2n+1)(2n+3)...(2n+2k+1))
// times e^-T at the top order, in long double (all terms positive), then
// downward recursion; computed once per process.
const std::vector<double>& boys_table() {
  static const std::vector<double> tab = [] {
    std::vector<double> t((size_t)BOYS_NGRID * (BOYS_NMAX + 1));
    for (int i = 0; i < BOYS_NGRID; ++i) {
      const long double T = (long double)i * BOYS_STEP;
      long double F[BOYS_NMAX + 1];
      const long double e = expl(-T);
      long double term = 1.0L / (2 * BOYS_NMAX + 1), sum = term;
      for (int k = 1; k < 2000; ++k) {
        term *= 2 * T / (2 * BOYS_NMAX + 2 * k + 1);
        sum += term;
        if (term < 1e-22L * sum) break;
      }
      F[BOYS_NMAX] = e * sum;
      for (int m = BOYS_NMAX; m > 0; --m) F[m - 1] = (2 * T * F[m] + e) / (2 * m - 1);
      for (int n = 0; n <= BOYS_NMAX; ++n) t[(size_t)i * (BOYS_NMAX + 1) + n] = (double)F[n];
    }
    return t;
  }();
  return tab;
}

int upload_c2s(const double* const* c2s, cudaStream_t st) {
  for (int l = 0; l <= GLC; ++l)
    if (!c2s[l]) return RIJK_ERR_ARG;
  std::vector<double> flat;
  int off[GLC + 1];
  for (int l = 0; l <= GLC; ++l) {
    off[l] = (int)flat.size();
    const int n = (2 * l + 1) * (l + 1) * (l + 2) / 2;
    flat.insert(flat.end(), c2s[l], c2s[l] + n);
  }
  // the tables change only with the caller's c2s matrices: upload once per device
  static std::mutex mu;
  static std::map<int, std::vector<double>> uploaded;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RIJK_ERR_CUDA;
  std::lock_guard<std::mutex> lock(mu);
  auto it = uploaded.find(dev);
  if (it != uploaded.end() && it->second == flat) return RIJK_OK;
  // earlier launches on this stream may still read the table: order after them
  if (cudaStreamSynchronize(st) != cudaSuccess) return RIJK_ERR_CUDA;
  // every translation unit with integral kernels holds its own copy of the table
  const double* boys = boys_table().data();
  bool bad = upload_tables(flat.data(), off, boys) != 0;
  for (int c = 0; c < 45 && !bad; ++c) bad = int3c_class_tables()[c](flat.data(), off, boys) != 0;
  if (bad)
    return RIJK_ERR_CUDA;
  uploaded[dev] = flat;
  return RIJK_OK;
}

}  // namespace

int ri_plan_create(const rijk_shells* bas, const rijk_shells* aux, const double* const* c2s, cudaStream_t st,
                   RiIntPlan** out) {
  *out = nullptr;
  if (!aux || !c2s) return RIJK_ERR_ARG;
  RiIntPlan* p = new RiIntPlan();
  int rc = upload_c2s(c2s, st);
  if (rc == RIJK_OK) rc = p->load(aux, GLC, p->C, p->offC, p->nC);
  if (rc == RIJK_OK) {
    for (int k = 0; k < p->C.nshell; ++k) p->aux_sorted.push_back(k);
    std::stable_sort(p->aux_sorted.begin(), p->aux_sorted.end(), [&](int x, int y) { return aux->l[x] < aux->l[y]; });
    for (int l = 0, t = 0; l <= GLC + 1; ++l) {
      while (t < p->C.nshell && aux->l[p->aux_sorted[t]] < l) ++t;
      p->aux_l_begin[l] = t;
    }
    p->up(p->daux, (const int*)p->aux_sorted.data(), p->aux_sorted.size());
  }
  if (rc == RIJK_OK && bas) {
    rc = p->load(bas, GLA, p->A, p->offA, p->nA);
    if (rc == RIJK_OK && (int64_t)p->A.nshell * (p->A.nshell + 1) / 2 > (1ll << 30)) rc = RIJK_ERR_TOO_LARGE;
    if (rc == RIJK_OK) {
      std::vector<int> pi, pj;
      for (int j = 0; j < p->A.nshell; ++j)
        for (int i = 0; i <= j; ++i) {
          pi.push_back(i);
          pj.push_back(j);
        }
      // class, then primitive count, then separation: neighbouring lanes share
      // their loop trip counts and, mostly, their screening outcomes
      auto key = [&](int x) {
        return (int64_t)(bas->l[pi[x]] * 3 + bas->l[pj[x]]) * 4096 + bas->nprim[pi[x]] * bas->nprim[pj[x]];
      };
      auto dist2 = [&](int x) {
        const double* a = bas->centers + 3 * pi[x];
        const double* b = bas->centers + 3 * pj[x];
        return (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]);
      };
      std::vector<int> order(pi.size());
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const int64_t kx = key(x), ky = key(y);
        return kx != ky ? kx < ky : dist2(x) < dist2(y);
      });
      std::vector<int> si(pi.size()), sj(pi.size());
      for (size_t t = 0; t < order.size(); ++t) {
        si[t] = pi[order[t]];
        sj[t] = pj[order[t]];
      }
      p->npairs = (int)si.size();
      for (int c = 0, t = 0; c <= 9; ++c) {
        while (t < p->npairs && bas->l[si[t]] * 3 + bas->l[sj[t]] < c) ++t;
        p->pair_cls[c] = t;
      }
      p->up(p->dpi, (const int*)si.data(), si.size());
      p->up(p->dpj, (const int*)sj.data(), sj.size());
    }
  }
  if (rc == RIJK_OK) rc = p->finalize(st);
  if (rc != RIJK_OK) {
    delete p;
    return rc;
  }
  *out = p;
  return RIJK_OK;
}

void ri_plan_destroy(RiIntPlan* p) { delete p; }
int64_t ri_plan_nbas(const RiIntPlan* p) { return p->nA; }
int64_t ri_plan_naux(const RiIntPlan* p) { return p->nC; }
int ri_plan_aux_shells(const RiIntPlan* p) { return p->C.nshell; }
int64_t ri_plan_aux_offset(const RiIntPlan* p, int k) { return p->offC[k]; }

void launch_int2c2e(const RiIntPlan* p, double* dV, int64_t ldv, cudaStream_t st) {
  const int64_t tasks = (int64_t)p->C.nshell * p->C.nshell;
  count_launch();
  k_int2c2e<<<(unsigned)((tasks + 63) / 64), 64, 0, st>>>(p->C, p->C.nshell, ldv, dV);
}

void launch_int3c2e(const RiIntPlan* p, int k0, int k1, double* out, cudaStream_t st) {
  const int64_t npair_fun = p->nA * (p->nA + 1) / 2;
  const int64_t P0 = p->offC[k0];
  for (int lc = 0; lc <= GLC; ++lc) {
    // the shells of [k0, k1) with l = lc are contiguous in the sorted list
    const int* b = p->aux_sorted.data() + p->aux_l_begin[lc];
    const int* e = p->aux_sorted.data() + p->aux_l_begin[lc + 1];
    const int* lo = std::lower_bound(b, e, k0);
    const int* hi = std::lower_bound(lo, e, k1);
    const int nkc = (int)(hi - lo);
    if (nkc == 0) continue;
    const int* dkc = p->daux + (lo - p->aux_sorted.data());
    for (int c = 0; c < 9; ++c) {
      const int npc = p->pair_cls[c + 1] - p->pair_cls[c];
      if (npc == 0) continue;
      const int64_t tasks = (int64_t)npc * nkc;
      count_launch();
      const Int3cKernel kern = int3c_class_kernels()[c * 5 + lc]();
      kern<<<(unsigned)((tasks + 127) / 128), 128, 0, st>>>(
          p->A, p->C, p->dpi + p->pair_cls[c], p->dpj + p->pair_cls[c], npc, dkc, nkc, npair_fun, P0, out);
    }
  }
}

}  // namespace rijk
