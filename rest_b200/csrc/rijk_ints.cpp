// Gaussian integrals over real solid-harmonic contracted shells (host, OpenMP):
// overlap, kinetic, nuclear attraction, two-centre Coulomb (P|Q) and
// three-centre Coulomb (mu nu|P).  These are the inputs REST obtains from
// libcint (src/molecule_io/mod.rs:700-812 one-electron, :1072-1103 2c2e,
// :1563-1721 3c2e) before its RI metric step; they are evaluated here with the
// McMurchie-Davidson scheme (Hermite expansion coefficients E, Hermite Coulomb
// integrals R from the Boys function).
//
// Shell data are passed as plain arrays (rijk_shells in include/rest_b200.h).
// Contraction coefficients multiply unnormalised Cartesian primitives
// x^i y^j z^k exp(-a r^2); the caller's coefficients already carry the
// normalisation it wants.  Cartesian blocks are turned into real solid
// harmonics with the caller's c2s matrices (one (2l+1) x (l+1)(l+2)/2 matrix
// per l, Cartesian components ordered lexicographically by (i desc, j desc)).
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "../../include/rest_b200.h"

namespace {

constexpr int LMAX = 6;                  // per shell
constexpr int LTOT = 3 * LMAX + 2;       // Boys order bound
constexpr double PI = 3.14159265358979323846;

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Cartesian exponent triples for angular momentum l, lexicographic (i desc, j desc).
struct CartTable {
  int ix[LMAX + 1][32], iy[LMAX + 1][32], iz[LMAX + 1][32];
  CartTable() {
    for (int l = 0; l <= LMAX; ++l) {
      int c = 0;
      for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) {
          ix[l][c] = i;
          iy[l][c] = j;
          iz[l][c] = l - i - j;
          ++c;
        }
    }
  }
};
const CartTable CT;

// Boys function F_n(T) for n = 0..nmax.
void boys(int nmax, double T, double* F) {
  if (T < 1e-14) {
    for (int n = 0; n <= nmax; ++n) F[n] = 1.0 / (2 * n + 1);
    return;
  }
  if (T > 40.0) {
    // asymptotic F_0 and upward recursion (stable for large T)
    F[0] = 0.5 * sqrt(PI / T);
    const double e = exp(-T);
    for (int n = 0; n < nmax; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) / (2 * T);
    return;
  }
  // series for the highest order, then downward recursion
  const double e = exp(-T);
  const int n = nmax;
  double term = 1.0 / (2 * n + 1), sum = term;
  for (int k = 1; k < 400; ++k) {
    term *= 2 * T / (2 * n + 2 * k + 1);
    sum += term;
    if (term < 1e-17 * sum) break;
  }
  F[n] = e * sum;
  for (int m = n; m > 0; --m) F[m - 1] = (2 * T * F[m] + e) / (2 * m - 1);
}

// 1D Hermite expansion coefficients E[i][j][t] of x_A^i x_B^j exp(..) products.
struct Herm1D {
  // E(i, j, t): i <= la, j <= lb, t <= i + j
  double e[LMAX + 3][LMAX + 3][2 * LMAX + 6];
  void build(int la, int lb, double a, double b, double AB) {
    const double p = a + b, mu = a * b / p;
    const double XPA = -b / p * AB, XPB = a / p * AB;  // AB = A - B
    const double oo2p = 0.5 / p;
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb; ++j)
        for (int t = 0; t <= i + j + 1; ++t) e[i][j][t] = 0.0;
    e[0][0][0] = exp(-mu * AB * AB);
    for (int i = 0; i <= la; ++i)
      for (int j = 0; j <= lb; ++j) {
        if (i == 0 && j == 0) continue;
        if (i > 0) {
          for (int t = 0; t <= i + j; ++t) {
            double v = XPA * e[i - 1][j][t];
            if (t > 0) v += oo2p * e[i - 1][j][t - 1];
            if (t + 1 <= i - 1 + j) v += (t + 1) * e[i - 1][j][t + 1];
            e[i][j][t] = v;
          }
        } else {
          for (int t = 0; t <= i + j; ++t) {
            double v = XPB * e[i][j - 1][t];
            if (t > 0) v += oo2p * e[i][j - 1][t - 1];
            if (t + 1 <= i + j - 1) v += (t + 1) * e[i][j - 1][t + 1];
            e[i][j][t] = v;
          }
        }
      }
  }
};

// Hermite Coulomb integrals R_{tuv}^0 for t+u+v <= L at (alpha, PC).
struct HermR {
  int L;
  std::vector<double> r;   // [(L+1)^3] indexed (t, u, v)
  std::vector<double> Rn;  // [(L+1)^4] indexed (n, t, u, v), reused between builds
  int stride;
  double& at(int t, int u, int v) { return r[(t * stride + u) * stride + v]; }
  void build(int Lmax, double alpha, const double* PC) {
    L = Lmax;
    stride = L + 1;
    r.assign((size_t)stride * stride * stride, 0.0);
    const double T = alpha * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
    double F[LTOT + 2];
    boys(L, T, F);
    // R^n_{000} = (-2 alpha)^n F_n; build with the n index as a separate dim.
    Rn.assign((size_t)(L + 1) * stride * stride * stride, 0.0);
    auto idx = [&](int n, int t, int u, int v) { return (((size_t)n * stride + t) * stride + u) * stride + v; };
    double f = 1.0;
    for (int n = 0; n <= L; ++n) {
      Rn[idx(n, 0, 0, 0)] = f * F[n];
      f *= -2.0 * alpha;
    }
    for (int n = L - 1; n >= 0; --n) {
      const int top = L - n;  // t+u+v <= L - n at order n
      for (int t = 0; t <= top; ++t)
        for (int u = 0; u + t <= top; ++u)
          for (int v = 0; v + u + t <= top; ++v) {
            if (t + u + v == 0) continue;
            double val;
            if (t > 0) {
              val = PC[0] * Rn[idx(n + 1, t - 1, u, v)];
              if (t > 1) val += (t - 1) * Rn[idx(n + 1, t - 2, u, v)];
            } else if (u > 0) {
              val = PC[1] * Rn[idx(n + 1, t, u - 1, v)];
              if (u > 1) val += (u - 1) * Rn[idx(n + 1, t, u - 2, v)];
            } else {
              val = PC[2] * Rn[idx(n + 1, t, u, v - 1)];
              if (v > 1) val += (v - 1) * Rn[idx(n + 1, t, u, v - 2)];
            }
            Rn[idx(n, t, u, v)] = val;
          }
    }
    for (int t = 0; t <= L; ++t)
      for (int u = 0; u + t <= L; ++u)
        for (int v = 0; v + u + t <= L; ++v) at(t, u, v) = Rn[idx(0, t, u, v)];
  }
};

struct Shells {
  const rijk_shells* s;
  std::vector<int64_t> off;  // first spherical function of each shell
  int64_t nfun = 0;
  explicit Shells(const rijk_shells* s_) : s(s_) {
    off.resize(s->nshell + 1);
    for (int64_t i = 0; i < s->nshell; ++i) {
      off[i] = nfun;
      nfun += 2 * s->l[i] + 1;
    }
    off[s->nshell] = nfun;
  }
  int l(int64_t i) const { return s->l[i]; }
  const double* ctr(int64_t i) const { return s->centers + 3 * i; }
};

// Cartesian -> spherical for a block: out[sa][sb] = sum C_a[sa][ca] C_b[sb][cb] in[ca][cb].
void c2s_2(const double* const* c2s, int la, int lb, const double* cart, double* sph) {
  const int na = ncart(la), nb = ncart(lb), sa = 2 * la + 1, sb = 2 * lb + 1;
  std::vector<double> tmp((size_t)sa * nb, 0.0);
  for (int i = 0; i < sa; ++i)
    for (int ca = 0; ca < na; ++ca) {
      const double w = c2s[la][i * na + ca];
      if (w == 0.0) continue;
      for (int cb = 0; cb < nb; ++cb) tmp[i * nb + cb] += w * cart[ca * nb + cb];
    }
  for (int i = 0; i < sa; ++i)
    for (int j = 0; j < sb; ++j) {
      double v = 0.0;
      for (int cb = 0; cb < nb; ++cb) v += c2s[lb][j * nb + cb] * tmp[i * nb + cb];
      sph[i * sb + j] = v;
    }
}

bool valid(const rijk_shells* s) {
  if (!s || s->nshell < 0) return false;
  for (int64_t i = 0; i < s->nshell; ++i)
    if (s->l[i] < 0 || s->l[i] > LMAX || s->nprim[i] <= 0) return false;
  return true;
}

// ---- one-electron ----------------------------------------------------------
// kind 0 overlap, 1 kinetic, 2 nuclear attraction (sum over atoms of -Z_C/|r-C|)
void shell_pair_1e(const Shells& A, int64_t ia, const Shells& B, int64_t ib, int kind, int natom, const double* Z,
                   const double* C, double* cart) {
  const int la = A.l(ia), lb = B.l(ib), na = ncart(la), nb = ncart(lb);
  const double* Ra = A.ctr(ia);
  const double* Rb = B.ctr(ib);
  for (int k = 0; k < na * nb; ++k) cart[k] = 0.0;
  Herm1D Ex, Ey, Ez;
  HermR R;
  for (int pa = 0; pa < A.s->nprim[ia]; ++pa)
    for (int pb = 0; pb < B.s->nprim[ib]; ++pb) {
      const double a = A.s->exps[A.s->prim_off[ia] + pa], b = B.s->exps[B.s->prim_off[ib] + pb];
      const double ca = A.s->coefs[A.s->prim_off[ia] + pa], cb = B.s->coefs[B.s->prim_off[ib] + pb];
      const double p = a + b;
      const int ext = kind == 1 ? 2 : 0;
      Ex.build(la, lb + ext, a, b, Ra[0] - Rb[0]);
      Ey.build(la, lb + ext, a, b, Ra[1] - Rb[1]);
      Ez.build(la, lb + ext, a, b, Ra[2] - Rb[2]);
      const double s0 = sqrt(PI / p);
      const double cc = ca * cb;
      if (kind == 0 || kind == 1) {
        for (int u = 0; u < na; ++u) {
          const int i1 = CT.ix[la][u], j1 = CT.iy[la][u], k1 = CT.iz[la][u];
          for (int w = 0; w < nb; ++w) {
            const int i2 = CT.ix[lb][w], j2 = CT.iy[lb][w], k2 = CT.iz[lb][w];
            const double sx = Ex.e[i1][i2][0] * s0, sy = Ey.e[j1][j2][0] * s0, sz = Ez.e[k1][k2][0] * s0;
            if (kind == 0) {
              cart[u * nb + w] += cc * sx * sy * sz;
            } else {
              auto t1 = [&](const Herm1D& E, int i, int j) {
                double v = 4 * b * b * E.e[i][j + 2][0] - 2 * b * (2 * j + 1) * E.e[i][j][0];
                if (j >= 2) v += j * (j - 1) * E.e[i][j - 2][0];
                return -0.5 * v * s0;
              };
              const double tx = t1(Ex, i1, i2), ty = t1(Ey, j1, j2), tz = t1(Ez, k1, k2);
              cart[u * nb + w] += cc * (tx * sy * sz + sx * ty * sz + sx * sy * tz);
            }
          }
        }
      } else {
        const double P[3] = {(a * Ra[0] + b * Rb[0]) / p, (a * Ra[1] + b * Rb[1]) / p, (a * Ra[2] + b * Rb[2]) / p};
        for (int at = 0; at < natom; ++at) {
          const double PC[3] = {P[0] - C[3 * at], P[1] - C[3 * at + 1], P[2] - C[3 * at + 2]};
          R.build(la + lb, p, PC);
          const double pref = -Z[at] * 2 * PI / p * cc;
          for (int u = 0; u < na; ++u) {
            const int i1 = CT.ix[la][u], j1 = CT.iy[la][u], k1 = CT.iz[la][u];
            for (int w = 0; w < nb; ++w) {
              const int i2 = CT.ix[lb][w], j2 = CT.iy[lb][w], k2 = CT.iz[lb][w];
              double v = 0.0;
              for (int t = 0; t <= i1 + i2; ++t)
                for (int uu = 0; uu <= j1 + j2; ++uu)
                  for (int vv = 0; vv <= k1 + k2; ++vv)
                    v += Ex.e[i1][i2][t] * Ey.e[j1][j2][uu] * Ez.e[k1][k2][vv] * R.at(t, uu, vv);
              cart[u * nb + w] += pref * v;
            }
          }
        }
      }
    }
}

// ---- Coulomb, bra = product of two shells (or one, with lb = -1), ket = one shell
// (ab|c) for all Cartesian components: out[(ca*nb + cb)*nc + cc]
void shell_triple(const Shells& A, int64_t ia, const Shells* B, int64_t ib, const Shells& Cs, int64_t ic,
                  double* out) {
  const int la = A.l(ia), lb = B ? B->l(ib) : 0, lc = Cs.l(ic);
  const int na = ncart(la), nb = ncart(lb), nc = ncart(lc);
  const double* Ra = A.ctr(ia);
  const double* Rb = B ? B->ctr(ib) : Ra;
  const double* Rc = Cs.ctr(ic);
  for (int k = 0; k < na * nb * nc; ++k) out[k] = 0.0;
  Herm1D Ex, Ey, Ez, Cx, Cy, Cz;
  HermR R;
  const int npb = B ? B->s->nprim[ib] : 1;
  for (int pa = 0; pa < A.s->nprim[ia]; ++pa)
    for (int pb = 0; pb < npb; ++pb) {
      const double a = A.s->exps[A.s->prim_off[ia] + pa];
      const double b = B ? B->s->exps[B->s->prim_off[ib] + pb] : 0.0;
      const double cab = A.s->coefs[A.s->prim_off[ia] + pa] * (B ? B->s->coefs[B->s->prim_off[ib] + pb] : 1.0);
      const double p = a + b;
      Ex.build(la, lb, a, b, Ra[0] - Rb[0]);
      Ey.build(la, lb, a, b, Ra[1] - Rb[1]);
      Ez.build(la, lb, a, b, Ra[2] - Rb[2]);
      const double P[3] = {(a * Ra[0] + b * Rb[0]) / p, (a * Ra[1] + b * Rb[1]) / p, (a * Ra[2] + b * Rb[2]) / p};
      for (int pc = 0; pc < Cs.s->nprim[ic]; ++pc) {
        const double g = Cs.s->exps[Cs.s->prim_off[ic] + pc];
        const double cg = Cs.s->coefs[Cs.s->prim_off[ic] + pc];
        // single-centre Hermite expansion of the ket (b = 0 limit)
        Cx.build(lc, 0, g, 0.0, 0.0);
        Cy.build(lc, 0, g, 0.0, 0.0);
        Cz.build(lc, 0, g, 0.0, 0.0);
        const double alpha = p * g / (p + g);
        const double PC[3] = {P[0] - Rc[0], P[1] - Rc[1], P[2] - Rc[2]};
        R.build(la + lb + lc, alpha, PC);
        const double pref = 2.0 * pow(PI, 2.5) / (p * g * sqrt(p + g)) * cab * cg;
        for (int u = 0; u < na; ++u) {
          const int i1 = CT.ix[la][u], j1 = CT.iy[la][u], k1 = CT.iz[la][u];
          for (int w = 0; w < nb; ++w) {
            const int i2 = CT.ix[lb][w], j2 = CT.iy[lb][w], k2 = CT.iz[lb][w];
            for (int q = 0; q < nc; ++q) {
              const int i3 = CT.ix[lc][q], j3 = CT.iy[lc][q], k3 = CT.iz[lc][q];
              double v = 0.0;
              for (int t = 0; t <= i1 + i2; ++t) {
                const double et = Ex.e[i1][i2][t];
                if (et == 0.0) continue;
                for (int uu = 0; uu <= j1 + j2; ++uu) {
                  const double eu = et * Ey.e[j1][j2][uu];
                  if (eu == 0.0) continue;
                  for (int vv = 0; vv <= k1 + k2; ++vv) {
                    const double ev = eu * Ez.e[k1][k2][vv];
                    if (ev == 0.0) continue;
                    double inner = 0.0;
                    for (int tt = 0; tt <= i3; ++tt) {
                      const double ft = Cx.e[i3][0][tt];
                      if (ft == 0.0) continue;
                      for (int ww = 0; ww <= j3; ++ww) {
                        const double fu = ft * Cy.e[j3][0][ww];
                        if (fu == 0.0) continue;
                        for (int zz = 0; zz <= k3; ++zz) {
                          const double fv = fu * Cz.e[k3][0][zz];
                          if (fv == 0.0) continue;
                          const double sgn = ((tt + ww + zz) & 1) ? -1.0 : 1.0;
                          inner += sgn * fv * R.at(t + tt, uu + ww, vv + zz);
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

}  // namespace

extern "C" {

int rijk_int1e(const rijk_shells* bas, const double* const* c2s, int kind, int natom, const double* charges,
               const double* coords, double* out) {
  if (!valid(bas) || !c2s || !out || kind < 0 || kind > 2 || (kind == 2 && (!charges || !coords || natom <= 0)))
    return RIJK_ERR_ARG;
  Shells A(bas);
  const int64_t n = A.nfun;
#pragma omp parallel for schedule(dynamic)
  for (int64_t ij = 0; ij < bas->nshell * bas->nshell; ++ij) {
    const int64_t i = ij % bas->nshell, j = ij / bas->nshell;
    if (i > j) continue;
    const int li = A.l(i), lj = A.l(j);
    std::vector<double> cart(ncart(li) * ncart(lj)), sph((2 * li + 1) * (2 * lj + 1));
    shell_pair_1e(A, i, A, j, kind, natom, charges, coords, cart.data());
    c2s_2(c2s, li, lj, cart.data(), sph.data());
    const int si = 2 * li + 1, sj = 2 * lj + 1;
    for (int a = 0; a < si; ++a)
      for (int b = 0; b < sj; ++b) {
        const int64_t r = A.off[i] + a, c = A.off[j] + b;
        out[r + n * c] = sph[a * sj + b];
        out[c + n * r] = sph[a * sj + b];
      }
  }
  return RIJK_OK;
}

int rijk_int2c2e(const rijk_shells* aux, const double* const* c2s, double* out) {
  if (!valid(aux) || !c2s || !out) return RIJK_ERR_ARG;
  Shells A(aux);
  const int64_t n = A.nfun;
#pragma omp parallel for schedule(dynamic)
  for (int64_t ij = 0; ij < aux->nshell * aux->nshell; ++ij) {
    const int64_t i = ij % aux->nshell, j = ij / aux->nshell;
    if (i > j) continue;
    const int li = A.l(i), lj = A.l(j);
    std::vector<double> cart(ncart(li) * ncart(lj)), sph((2 * li + 1) * (2 * lj + 1));
    shell_triple(A, i, nullptr, 0, A, j, cart.data());
    c2s_2(c2s, li, lj, cart.data(), sph.data());
    const int si = 2 * li + 1, sj = 2 * lj + 1;
    for (int a = 0; a < si; ++a)
      for (int b = 0; b < sj; ++b) {
        const int64_t r = A.off[i] + a, c = A.off[j] + b;
        out[r + n * c] = sph[a * sj + b];
        out[c + n * r] = sph[a * sj + b];
      }
  }
  return RIJK_OK;
}

int rijk_int3c2e(const rijk_shells* bas, const rijk_shells* aux, const double* const* c2s, double* out) {
  if (!valid(bas) || !valid(aux) || !c2s || !out) return RIJK_ERR_ARG;
  Shells A(bas), C(aux);
  const int64_t n = A.nfun, naux = C.nfun, npair = n * (n + 1) / 2;
#pragma omp parallel
  {
    std::vector<double> cart, half, sph;
#pragma omp for schedule(dynamic)
    for (int64_t ij = 0; ij < bas->nshell * bas->nshell; ++ij) {
      const int64_t i = ij % bas->nshell, j = ij / bas->nshell;
      if (i > j) continue;
      const int li = A.l(i), lj = A.l(j), nai = ncart(li), naj = ncart(lj);
      const int si = 2 * li + 1, sj = 2 * lj + 1;
      for (int64_t k = 0; k < aux->nshell; ++k) {
        const int lk = C.l(k), nak = ncart(lk), sk = 2 * lk + 1;
        cart.assign((size_t)nai * naj * nak, 0.0);
        shell_triple(A, i, &A, j, C, k, cart.data());
        // c2s on the ket index first, then on the bra pair
        half.assign((size_t)nai * naj * sk, 0.0);
        for (int ab = 0; ab < nai * naj; ++ab)
          for (int q = 0; q < sk; ++q) {
            double v = 0.0;
            for (int c = 0; c < nak; ++c) v += c2s[lk][q * nak + c] * cart[(size_t)ab * nak + c];
            half[(size_t)ab * sk + q] = v;
          }
        sph.assign((size_t)si * sj * sk, 0.0);
        std::vector<double> blk(nai * naj), sb(si * sj);
        for (int q = 0; q < sk; ++q) {
          for (int ab = 0; ab < nai * naj; ++ab) blk[ab] = half[(size_t)ab * sk + q];
          c2s_2(c2s, li, lj, blk.data(), sb.data());
          for (int a = 0; a < si; ++a)
            for (int b = 0; b < sj; ++b) {
              const int64_t mu = A.off[i] + a, nu = A.off[j] + b;
              if (mu > nu) continue;  // packed upper triangle, mu <= nu
              const int64_t P = C.off[k] + q;
              out[P * npair + nu * (nu + 1) / 2 + mu] = sb[a * sj + b];
            }
        }
      }
    }
  }
  return RIJK_OK;
}

}  // extern "C"
