// gto_ints.cpp — McMurchie-Davidson Gaussian integrals for the RI-JK inputs.
//
// This is the host-side producer of the Fock build's inputs, standing in for the
// reference's libint2 calls (src/libint_link.cpp:2049-2107 for (P|Q),
// src/libint_link.cpp:2261-2350 for (mu nu|P), src/molecule.cpp:3757-3800 for S, T, V).
// The algorithm is the textbook McMurchie-Davidson scheme:
//   * a product of two Cartesian Gaussians is expanded in Hermite Gaussians with the
//     coefficients E^{ij}_t (one recurrence per Cartesian direction);
//   * Coulomb integrals over Hermite Gaussians are the R_{tuv} integrals, built from the
//     Boys function F_n(T) by the Hermite recurrence;
//   * spherical shells are real solid harmonics, obtained from their recurrence in
//     x, y, z and normalised against the Cartesian overlap.
// Normalisation follows libint: each primitive carries the x^l normalisation of its
// exponent and the contraction is rescaled to unit norm.
#include "gto_ints.h"
#include "gto_tables.h"

#include <omp.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

namespace {

using namespace gto_tab;

constexpr int RD = LTOT + 1;            // edge of the R_{tuv} cube

int g_threads = 0;

// ---------------------------------------------------------------- Boys function ----
// Evaluated by a 7-term Taylor expansion about the nearest grid point of the table
// (dF_m/dT = -F_{m+1}) followed by downward recursion F_{m-1} = (2T F_m + exp(-T)) / (2m-1).
// For T beyond the grid F_0 = sqrt(pi/T)/2 (exp(-T) < 1e-17 there) and upward recursion is stable.
std::vector<double> g_boys;  // [BOYS_NT][BOYS_MTAB]
std::once_flag g_boys_once;

void boys_table_init() { boys_table_fill(g_boys); }

inline void boys(int mmax, double T, double* F) {
  if (T < BOYS_TMAX - 0.5 / BOYS_NPER) {
    int i = static_cast<int>(T * BOYS_NPER + 0.5);
    double dt = static_cast<double>(i) / BOYS_NPER - T;  // expand about T_i: F(T) = sum F_{m+k}(T_i) dt^k / k!
    const double* row = &g_boys[static_cast<size_t>(i) * BOYS_MTAB];
    double f = row[mmax + 6];
    f = row[mmax + 5] + f * dt / 6.0;
    f = row[mmax + 4] + f * dt / 5.0;
    f = row[mmax + 3] + f * dt / 4.0;
    f = row[mmax + 2] + f * dt / 3.0;
    f = row[mmax + 1] + f * dt / 2.0;
    f = row[mmax] + f * dt;
    F[mmax] = f;
    double e = std::exp(-T);
    for (int m = mmax; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + e) / (2 * m - 1);
  } else {
    double e = std::exp(-T);
    F[0] = 0.5 * std::sqrt(PI / T);
    for (int m = 0; m < mmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
  }
}

struct CartList {
  int lx[NCART_MAX], ly[NCART_MAX], lz[NCART_MAX];
};
CartList cart_list(int l) {
  CartList c;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) {
      int i = cart_index(l, lx, ly);
      c.lx[i] = lx; c.ly[i] = ly; c.lz[i] = l - lx - ly;
    }
  return c;
}

}  // namespace

struct gto_shell {
  int l, pure, nprim, off, nfunc;
  double xyz[3];
  std::vector<double> exps, coefs;  // coefs normalised
};

struct gto_basis {
  std::vector<gto_shell> sh;
  int nbf = 0, lmax = 0;
};

namespace {

// Hermite expansion coefficients of a 1-D Gaussian product: E[i][j][t].
constexpr int EJ = LMAX + 3;  // j runs to lb+2 for the kinetic energy
struct Herm1D {
  double e[LMAX + 1][EJ][2 * LMAX + 4];
};
void hermite_1d(int la, int lb, double p, double xpa, double xpb, double k0, Herm1D& h) {
  const double o2p = 0.5 / p;
  const int tmax = la + lb;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t <= tmax + 1; ++t) h.e[i][j][t] = 0.0;
  h.e[0][0][0] = k0;
  for (int i = 0; i < la; ++i)
    for (int t = 0; t <= i + 1; ++t) {
      double v = xpa * h.e[i][0][t] + (t + 1) * h.e[i][0][t + 1];
      if (t > 0) v += o2p * h.e[i][0][t - 1];
      h.e[i + 1][0][t] = v;
    }
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j < lb; ++j)
      for (int t = 0; t <= i + j + 1; ++t) {
        double v = xpb * h.e[i][j][t] + (t + 1) * h.e[i][j][t + 1];
        if (t > 0) v += o2p * h.e[i][j][t - 1];
        h.e[i][j + 1][t] = v;
      }
}

// Hermite Coulomb integrals R_{tuv}(alpha, PC) for t+u+v <= L, written to r[t][u][v]
// (cube of edge RD).  Two layers of the n-recursion are kept.
struct RBuf {
  double a[RD * RD * RD];
  double b[RD * RD * RD];
};
inline int ri(int t, int u, int v) { return (t * RD + u) * RD + v; }

void hermite_R(int L, double alpha, double X, double Y, double Z, RBuf& buf, double*& out) {
  double F[LTOT + 2];
  double T = alpha * (X * X + Y * Y + Z * Z);
  boys(L, T, F);
  double* cur = buf.a;
  double* nxt = buf.b;  // holds layer n+1
  // n = L: only R^L_000
  double m2a = -2.0 * alpha, pw = 1.0;
  double pows[LTOT + 2] = {};
  for (int n = 0; n <= L; ++n) { pows[n] = pw; pw *= m2a; }
  nxt[0] = pows[L] * F[L];
  for (int n = L - 1; n >= 0; --n) {
    int lim = L - n;
    cur[0] = pows[n] * F[n];
    for (int t = 0; t <= lim; ++t)
      for (int u = 0; u <= lim - t; ++u)
        for (int v = 0; v <= lim - t - u; ++v) {
          if (t + u + v == 0) continue;
          double r;
          if (t > 0) {
            r = X * nxt[ri(t - 1, u, v)];
            if (t > 1) r += (t - 1) * nxt[ri(t - 2, u, v)];
          } else if (u > 0) {
            r = Y * nxt[ri(t, u - 1, v)];
            if (u > 1) r += (u - 1) * nxt[ri(t, u - 2, v)];
          } else {
            r = Z * nxt[ri(t, u, v - 1)];
            if (v > 1) r += (v - 1) * nxt[ri(t, u, v - 2)];
          }
          cur[ri(t, u, v)] = r;
        }
    double* tmp = cur; cur = nxt; nxt = tmp;
  }
  out = nxt;  // layer n = 0
}

// One-centre Hermite expansion of a spherical (or Cartesian) Gaussian shell primitive:
// list of (t,u,v,coef) terms per function m, coef including (-1)^{t+u+v} when `ket`.
struct HermTerm { int t, u, v; double c; };
struct OneCentre {
  int nfunc;
  std::vector<std::vector<HermTerm>> terms;  // [m]
};
OneCentre one_centre(int l, int pure, double gamma, double coef, bool ket) {
  Herm1D h;
  hermite_1d(l, 0, gamma, 0.0, 0.0, 1.0, h);
  CartList cl = cart_list(l);
  int nc = ncart(l);
  int nf = pure ? 2 * l + 1 : nc;
  OneCentre oc;
  oc.nfunc = nf;
  oc.terms.resize(nf);
  const std::vector<double>& T = sph().c[l];
  for (int m = 0; m < nf; ++m) {
    // accumulate dense cube then sparsify
    double cube[LMAX + 1][LMAX + 1][LMAX + 1];
    std::memset(cube, 0, sizeof(cube));
    for (int c = 0; c < nc; ++c) {
      double w = pure ? T[static_cast<size_t>(m) * nc + c] : (c == m ? 1.0 : 0.0);
      if (w == 0.0) continue;
      for (int t = 0; t <= cl.lx[c]; ++t)
        for (int u = 0; u <= cl.ly[c]; ++u)
          for (int v = 0; v <= cl.lz[c]; ++v)
            cube[t][u][v] += w * h.e[cl.lx[c]][0][t] * h.e[cl.ly[c]][0][u] * h.e[cl.lz[c]][0][v];
    }
    for (int t = 0; t <= l; ++t)
      for (int u = 0; u <= l - t; ++u)
        for (int v = 0; v <= l - t - u; ++v)
          if (cube[t][u][v] != 0.0) {
            double s = (ket && ((t + u + v) & 1)) ? -1.0 : 1.0;
            oc.terms[m].push_back({t, u, v, s * coef * cube[t][u][v]});
          }
  }
  return oc;
}

// Primitive-pair data of a shell pair.
struct PrimPair {
  double p, P[3], cc;  // cc = ca*cb (normalised contraction coefficients)
  Herm1D ex, ey, ez;
};
void make_pairs(const gto_shell& A, const gto_shell& B, int extra, std::vector<PrimPair>& out) {
  out.clear();
  double AB[3] = {A.xyz[0] - B.xyz[0], A.xyz[1] - B.xyz[1], A.xyz[2] - B.xyz[2]};
  double r2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  for (int i = 0; i < A.nprim; ++i)
    for (int j = 0; j < B.nprim; ++j) {
      double a = A.exps[i], b = B.exps[j], p = a + b, mu = a * b / p;
      double k = std::exp(-mu * r2);
      double cc = A.coefs[i] * B.coefs[j];
      if (std::fabs(cc * k) < 1e-22) continue;  // contributes below double precision
      PrimPair pp;
      pp.p = p;
      pp.cc = cc;
      for (int d = 0; d < 3; ++d) pp.P[d] = (a * A.xyz[d] + b * B.xyz[d]) / p;
      hermite_1d(A.l, B.l + extra, p, pp.P[0] - A.xyz[0], pp.P[0] - B.xyz[0], k, pp.ex);
      hermite_1d(A.l, B.l + extra, p, pp.P[1] - A.xyz[1], pp.P[1] - B.xyz[1], 1.0, pp.ey);
      hermite_1d(A.l, B.l + extra, p, pp.P[2] - A.xyz[2], pp.P[2] - B.xyz[2], 1.0, pp.ez);
      out.push_back(pp);
    }
}

// Cartesian -> spherical for a (na_c x nb_c x nc) block, in place into `out` (na x nb x nc).
void pair_to_sph(const gto_shell& A, const gto_shell& B, int nc, const double* cart, double* out,
                 std::vector<double>& tmp) {
  int nca = ncart(A.l), ncb = ncart(B.l);
  tmp.assign(static_cast<size_t>(A.nfunc) * ncb * nc, 0.0);
  if (A.pure) {
    const std::vector<double>& T = sph().c[A.l];
    for (int m = 0; m < A.nfunc; ++m)
      for (int a = 0; a < nca; ++a) {
        double w = T[static_cast<size_t>(m) * nca + a];
        if (w == 0.0) continue;
        const double* src = cart + static_cast<size_t>(a) * ncb * nc;
        double* dst = tmp.data() + static_cast<size_t>(m) * ncb * nc;
        for (int k = 0; k < ncb * nc; ++k) dst[k] += w * src[k];
      }
  } else {
    std::memcpy(tmp.data(), cart, sizeof(double) * nca * ncb * nc);
  }
  if (B.pure) {
    const std::vector<double>& T = sph().c[B.l];
    for (int a = 0; a < A.nfunc; ++a)
      for (int m = 0; m < B.nfunc; ++m) {
        double* dst = out + (static_cast<size_t>(a) * B.nfunc + m) * nc;
        for (int k = 0; k < nc; ++k) dst[k] = 0.0;
        for (int b = 0; b < ncb; ++b) {
          double w = T[static_cast<size_t>(m) * ncb + b];
          if (w == 0.0) continue;
          const double* src = tmp.data() + (static_cast<size_t>(a) * ncb + b) * nc;
          for (int k = 0; k < nc; ++k) dst[k] += w * src[k];
        }
      }
  } else {
    std::memcpy(out, tmp.data(), sizeof(double) * A.nfunc * ncb * nc);
  }
}

int nthreads() { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

}  // namespace

extern "C" {

int gto_basis_create(gto_basis** out, int nshell, const int* l, const int* pure, const int* nprim,
                     const double* xyz, const double* exps, const double* coefs) {
  if (!out || nshell < 0 || (nshell > 0 && (!l || !pure || !nprim || !xyz || !exps || !coefs)))
    return GTO_ERR_ARG;
  std::call_once(g_boys_once, boys_table_init);
  (void)sph();
  gto_basis* b = new (std::nothrow) gto_basis;
  if (!b) return GTO_ERR_ALLOC;
  int po = 0;
  for (int s = 0; s < nshell; ++s) {
    if (l[s] < 0 || l[s] > LMAX) { delete b; return GTO_ERR_LMAX; }
    if (nprim[s] < 1) { delete b; return GTO_ERR_ARG; }
    gto_shell sh;
    sh.l = l[s];
    sh.pure = pure[s] ? 1 : 0;
    sh.nprim = nprim[s];
    sh.nfunc = sh.pure ? 2 * sh.l + 1 : ncart(sh.l);
    for (int d = 0; d < 3; ++d) sh.xyz[d] = xyz[3 * s + d];
    sh.exps.assign(exps + po, exps + po + nprim[s]);
    sh.coefs.resize(nprim[s]);
    if (!normalise_shell(sh.l, sh.nprim, sh.exps.data(), coefs + po, sh.coefs.data())) { delete b; return GTO_ERR_ARG; }
    sh.off = b->nbf;
    b->nbf += sh.nfunc;
    if (sh.l > b->lmax) b->lmax = sh.l;
    b->sh.push_back(std::move(sh));
    po += nprim[s];
  }
  *out = b;
  return GTO_OK;
}

void gto_basis_destroy(gto_basis* b) { delete b; }
int gto_basis_nbf(const gto_basis* b) { return b ? b->nbf : GTO_ERR_ARG; }
int gto_basis_max_l(const gto_basis* b) { return b ? b->lmax : GTO_ERR_ARG; }
void gto_set_threads(int n) { g_threads = n; }

int gto_basis_norm_coefs(const gto_basis* b, double* out) {
  if (!b || !out) return GTO_ERR_ARG;
  size_t k = 0;
  for (const auto& s : b->sh)
    for (double c : s.coefs) out[k++] = c;
  return GTO_OK;
}

int gto_basis_shell_offsets(const gto_basis* b, int* out) {
  if (!b || !out) return GTO_ERR_ARG;
  for (size_t s = 0; s < b->sh.size(); ++s) out[s] = b->sh[s].off;
  return GTO_OK;
}

int gto_cart_to_sph(int l, double* out) {
  if (l < 0 || l > LMAX || !out) return GTO_ERR_ARG;
  const std::vector<double>& c = gto_tab::sph().c[l];
  std::copy(c.begin(), c.end(), out);
  return GTO_OK;
}

int gto_boys(int mmax, double T, double* F) {
  if (mmax < 0 || mmax > LTOT || T < 0.0 || !F) return GTO_ERR_ARG;
  std::call_once(g_boys_once, boys_table_init);
  boys(mmax, T, F);
  return GTO_OK;
}

// kind: 0 overlap, 1 kinetic, 2 nuclear attraction
static int one_electron(const gto_basis* b, int kind, int natom, const double* Z, const double* C, double* M) {
  if (!b || !M) return GTO_ERR_ARG;
  if (kind == 2 && natom > 0 && (!Z || !C)) return GTO_ERR_ARG;
  const int n = b->nbf;
  const int ns = static_cast<int>(b->sh.size());
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) pairs.emplace_back(i, j);
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<PrimPair> pp;
    RBuf* rb = new RBuf;
    std::vector<double> cart, sphb, tmpb;
#pragma omp for schedule(dynamic, 4)
    for (long q = 0; q < static_cast<long>(pairs.size()); ++q) {
      const gto_shell& A = b->sh[pairs[q].first];
      const gto_shell& B = b->sh[pairs[q].second];
      const int nca = ncart(A.l), ncb = ncart(B.l);
      CartList ca = cart_list(A.l), cb = cart_list(B.l);
      make_pairs(A, B, 0, pp);
      cart.assign(static_cast<size_t>(nca) * ncb, 0.0);
      if (kind == 0)
      for (const PrimPair& x : pp) {
        const double sp = std::pow(PI / x.p, 1.5);
        for (int ia = 0; ia < nca; ++ia)
          for (int ib = 0; ib < ncb; ++ib) {
            int ax = ca.lx[ia], ay = ca.ly[ia], az = ca.lz[ia];
            int bx = cb.lx[ib], by = cb.ly[ib], bz = cb.lz[ib];
            double v = x.ex.e[ax][bx][0] * x.ey.e[ay][by][0] * x.ez.e[az][bz][0] * sp;
            cart[static_cast<size_t>(ia) * ncb + ib] += x.cc * v;
          }
      }
      if (kind == 1) {
        // kinetic: the 1-D operator needs the ket exponent, so primitives are looped here
        double AB[3] = {A.xyz[0] - B.xyz[0], A.xyz[1] - B.xyz[1], A.xyz[2] - B.xyz[2]};
        double r2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
        for (int i = 0; i < A.nprim; ++i)
          for (int j = 0; j < B.nprim; ++j) {
            double a = A.exps[i], be = B.exps[j], p = a + be, mu = a * be / p;
            double k = std::exp(-mu * r2);
            double cc = A.coefs[i] * B.coefs[j];
            Herm1D ex, ey, ez;
            double P[3];
            for (int d = 0; d < 3; ++d) P[d] = (a * A.xyz[d] + be * B.xyz[d]) / p;
            hermite_1d(A.l, B.l + 2, p, P[0] - A.xyz[0], P[0] - B.xyz[0], 1.0, ex);
            hermite_1d(A.l, B.l + 2, p, P[1] - A.xyz[1], P[1] - B.xyz[1], 1.0, ey);
            hermite_1d(A.l, B.l + 2, p, P[2] - A.xyz[2], P[2] - B.xyz[2], 1.0, ez);
            const double s1 = std::sqrt(PI / p);
            auto S1 = [&](const Herm1D& e, int ii, int jj) { return jj < 0 ? 0.0 : e.e[ii][jj][0] * s1; };
            auto T1 = [&](const Herm1D& e, int ii, int jj) {
              double t = 4.0 * be * be * S1(e, ii, jj + 2) - 2.0 * be * (2 * jj + 1) * S1(e, ii, jj);
              if (jj >= 2) t += jj * (jj - 1) * S1(e, ii, jj - 2);
              return -0.5 * t;
            };
            for (int ia = 0; ia < nca; ++ia)
              for (int ib = 0; ib < ncb; ++ib) {
                int ax = ca.lx[ia], ay = ca.ly[ia], az = ca.lz[ia];
                int bx = cb.lx[ib], by = cb.ly[ib], bz = cb.lz[ib];
                double sx = S1(ex, ax, bx), sy = S1(ey, ay, by), sz = S1(ez, az, bz);
                double v = T1(ex, ax, bx) * sy * sz + sx * T1(ey, ay, by) * sz + sx * sy * T1(ez, az, bz);
                cart[static_cast<size_t>(ia) * ncb + ib] += cc * k * v;
              }
          }
      } else if (kind == 2) {
        const int L = A.l + B.l;
        for (const PrimPair& x : pp) {
          const double pref = 2.0 * PI / x.p;
          for (int c = 0; c < natom; ++c) {
            double* R;
            hermite_R(L, x.p, x.P[0] - C[3 * c], x.P[1] - C[3 * c + 1], x.P[2] - C[3 * c + 2], *rb, R);
            const double w = -Z[c] * pref * x.cc;
            for (int ia = 0; ia < nca; ++ia)
              for (int ib = 0; ib < ncb; ++ib) {
                int ax = ca.lx[ia], ay = ca.ly[ia], az = ca.lz[ia];
                int bx = cb.lx[ib], by = cb.ly[ib], bz = cb.lz[ib];
                double v = 0.0;
                for (int t = 0; t <= ax + bx; ++t) {
                  double et = x.ex.e[ax][bx][t];
                  if (et == 0.0) continue;
                  for (int u = 0; u <= ay + by; ++u) {
                    double eu = et * x.ey.e[ay][by][u];
                    if (eu == 0.0) continue;
                    for (int vv = 0; vv <= az + bz; ++vv) v += eu * x.ez.e[az][bz][vv] * R[ri(t, u, vv)];
                  }
                }
                cart[static_cast<size_t>(ia) * ncb + ib] += w * v;
              }
          }
        }
      }
      sphb.assign(static_cast<size_t>(A.nfunc) * B.nfunc, 0.0);
      pair_to_sph(A, B, 1, cart.data(), sphb.data(), tmpb);
      for (int fa = 0; fa < A.nfunc; ++fa)
        for (int fb = 0; fb < B.nfunc; ++fb) {
          double v = sphb[static_cast<size_t>(fa) * B.nfunc + fb];
          M[static_cast<size_t>(A.off + fa) * n + B.off + fb] = v;
          M[static_cast<size_t>(B.off + fb) * n + A.off + fa] = v;
        }
    }
    delete rb;
  }
  return GTO_OK;
}

int gto_overlap(const gto_basis* b, double* S) { return one_electron(b, 0, 0, nullptr, nullptr, S); }
int gto_kinetic(const gto_basis* b, double* T) { return one_electron(b, 1, 0, nullptr, nullptr, T); }
int gto_nuclear(const gto_basis* b, int natom, const double* Z, const double* xyz, double* V) {
  return one_electron(b, 2, natom, Z, xyz, V);
}

int gto_coulomb_2c(const gto_basis* aux, double* V) {
  if (!aux || !V) return GTO_ERR_ARG;
  const int n = aux->nbf;
  const int ns = static_cast<int>(aux->sh.size());
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) pairs.emplace_back(i, j);
#pragma omp parallel num_threads(nthreads())
  {
    RBuf* rb = new RBuf;
    std::vector<double> acc;
#pragma omp for schedule(dynamic, 4)
    for (long q = 0; q < static_cast<long>(pairs.size()); ++q) {
      const gto_shell& A = aux->sh[pairs[q].first];
      const gto_shell& B = aux->sh[pairs[q].second];
      acc.assign(static_cast<size_t>(A.nfunc) * B.nfunc, 0.0);
      const int L = A.l + B.l;
      for (int i = 0; i < A.nprim; ++i) {
        OneCentre oa = one_centre(A.l, A.pure, A.exps[i], A.coefs[i], false);
        for (int j = 0; j < B.nprim; ++j) {
          OneCentre ob = one_centre(B.l, B.pure, B.exps[j], B.coefs[j], true);
          double g1 = A.exps[i], g2 = B.exps[j];
          double al = g1 * g2 / (g1 + g2);
          double pref = 2.0 * std::pow(PI, 2.5) / (g1 * g2 * std::sqrt(g1 + g2));
          double* R;
          hermite_R(L, al, A.xyz[0] - B.xyz[0], A.xyz[1] - B.xyz[1], A.xyz[2] - B.xyz[2], *rb, R);
          for (int fa = 0; fa < A.nfunc; ++fa)
            for (int fb = 0; fb < B.nfunc; ++fb) {
              double v = 0.0;
              for (const HermTerm& x : oa.terms[fa])
                for (const HermTerm& y : ob.terms[fb]) v += x.c * y.c * R[ri(x.t + y.t, x.u + y.u, x.v + y.v)];
              acc[static_cast<size_t>(fa) * B.nfunc + fb] += pref * v;
            }
        }
      }
      for (int fa = 0; fa < A.nfunc; ++fa)
        for (int fb = 0; fb < B.nfunc; ++fb) {
          double v = acc[static_cast<size_t>(fa) * B.nfunc + fb];
          V[static_cast<size_t>(A.off + fa) * n + B.off + fb] = v;
          V[static_cast<size_t>(B.off + fb) * n + A.off + fa] = v;
        }
    }
    delete rb;
  }
  return GTO_OK;
}

int gto_coulomb_3c(const gto_basis* orb, const gto_basis* aux, int layout, double* out) {
  if (!orb || !aux || !out) return GTO_ERR_ARG;
  if (layout != GTO_3C_NOPT_FULL && layout != GTO_3C_PACKED) return GTO_ERR_ARG;
  const long n = orb->nbf, naux = aux->nbf;
  const int ns = static_cast<int>(orb->sh.size());
  const int nsa = static_cast<int>(aux->sh.size());
  // One-centre Hermite expansions of every aux primitive (ket side).
  std::vector<std::vector<OneCentre>> auxe(nsa);
  for (int c = 0; c < nsa; ++c)
    for (int k = 0; k < aux->sh[c].nprim; ++k)
      auxe[c].push_back(one_centre(aux->sh[c].l, aux->sh[c].pure, aux->sh[c].exps[k], aux->sh[c].coefs[k], true));
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) pairs.emplace_back(i, j);
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<PrimPair> pp;
    RBuf* rb = new RBuf;
    std::vector<double> cart, sphb, tmpb;
    std::vector<double> W;  // [m][t][u][v] over the pair's Hermite cube
#pragma omp for schedule(dynamic, 1)
    for (long q = 0; q < static_cast<long>(pairs.size()); ++q) {
      const gto_shell& A = orb->sh[pairs[q].first];
      const gto_shell& B = orb->sh[pairs[q].second];
      const int nca = ncart(A.l), ncb = ncart(B.l);
      const int Lab = A.l + B.l;
      const int HD = Lab + 1;
      CartList ca = cart_list(A.l), cb = cart_list(B.l);
      make_pairs(A, B, 0, pp);
      for (int c = 0; c < nsa; ++c) {
        const gto_shell& Cs = aux->sh[c];
        const int nfc = Cs.nfunc;
        cart.assign(static_cast<size_t>(nca) * ncb * nfc, 0.0);
        W.assign(static_cast<size_t>(nfc) * HD * HD * HD, 0.0);
        const int L = Lab + Cs.l;
        for (const PrimPair& x : pp) {
          for (int kc = 0; kc < Cs.nprim; ++kc) {
            const double g = Cs.exps[kc];
            const double al = x.p * g / (x.p + g);
            const double pref = 2.0 * std::pow(PI, 2.5) / (x.p * g * std::sqrt(x.p + g)) * x.cc;
            double* R;
            hermite_R(L, al, x.P[0] - Cs.xyz[0], x.P[1] - Cs.xyz[1], x.P[2] - Cs.xyz[2], *rb, R);
            const OneCentre& oc = auxe[c][kc];
            // W[m][t][u][v] = sum_terms c * R[t+tau][u+nu][v+phi]
            for (int m = 0; m < nfc; ++m) {
              double* w = &W[static_cast<size_t>(m) * HD * HD * HD];
              for (int t = 0; t <= Lab; ++t)
                for (int u = 0; u <= Lab - t; ++u)
                  for (int v = 0; v <= Lab - t - u; ++v) {
                    double s = 0.0;
                    for (const HermTerm& h : oc.terms[m]) s += h.c * R[ri(t + h.t, u + h.u, v + h.v)];
                    w[(t * HD + u) * HD + v] = s;
                  }
            }
            for (int ia = 0; ia < nca; ++ia)
              for (int ib = 0; ib < ncb; ++ib) {
                int ax = ca.lx[ia], ay = ca.ly[ia], az = ca.lz[ia];
                int bx = cb.lx[ib], by = cb.ly[ib], bz = cb.lz[ib];
                double* dst = &cart[(static_cast<size_t>(ia) * ncb + ib) * nfc];
                for (int t = 0; t <= ax + bx; ++t) {
                  double et = x.ex.e[ax][bx][t];
                  if (et == 0.0) continue;
                  for (int u = 0; u <= ay + by; ++u) {
                    double eu = et * x.ey.e[ay][by][u];
                    if (eu == 0.0) continue;
                    for (int v = 0; v <= az + bz; ++v) {
                      double e = pref * eu * x.ez.e[az][bz][v];
                      if (e == 0.0) continue;
                      const double* w = &W[(t * HD + u) * HD + v];
                      const size_t ms = static_cast<size_t>(HD) * HD * HD;
                      for (int m = 0; m < nfc; ++m) dst[m] += e * w[m * ms];
                    }
                  }
                }
              }
          }
        }
        sphb.assign(static_cast<size_t>(A.nfunc) * B.nfunc * nfc, 0.0);
        pair_to_sph(A, B, nfc, cart.data(), sphb.data(), tmpb);
        const long P0 = Cs.off;
        for (int fa = 0; fa < A.nfunc; ++fa)
          for (int fb = 0; fb < B.nfunc; ++fb) {
            const long mu = A.off + fa, nu = B.off + fb;
            const double* src = &sphb[(static_cast<size_t>(fa) * B.nfunc + fb) * nfc];
            if (layout == GTO_3C_NOPT_FULL) {
              double* d1 = out + (mu * n + nu) * naux + P0;
              double* d2 = out + (nu * n + mu) * naux + P0;
              for (int m = 0; m < nfc; ++m) { d1[m] = src[m]; d2[m] = src[m]; }
            } else {
              long hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
              double* d = out + (hi * (hi + 1) / 2 + lo) * naux + P0;
              for (int m = 0; m < nfc; ++m) d[m] = src[m];
            }
          }
      }
    }
    delete rb;
  }
  return GTO_OK;
}

}  // extern "C"
