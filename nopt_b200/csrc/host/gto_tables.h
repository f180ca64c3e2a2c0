// gto_tables.h — tables shared by the host integral engine (gto_ints.cpp) and the device
// integral kernels of librijk (k_eri.cu): the Boys-function grid, the real-solid-harmonic
// transformation matrices and the contraction normalisation.  Header-only so both libraries
// compile the same definitions.
//
// Conventions are libint's (the reference's integral library, called at
// src/libint_link.cpp:2080 and :2304): every primitive carries the x^l normalisation of its
// exponent, the contraction is rescaled to unit norm, and spherical shells are real solid
// harmonics normalised against the Cartesian overlap.
#pragma once

#include <cmath>
#include <vector>

namespace gto_tab {

constexpr int LMAX = 4;                 // highest shell angular momentum supported (g)
constexpr int NCART_MAX = (LMAX + 1) * (LMAX + 2) / 2;
constexpr int LTOT = 3 * LMAX;          // highest Boys order in a three-centre integral
constexpr double PI = 3.14159265358979323846;

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
inline int cart_index(int l, int lx, int ly) { return (l - lx) * (l - lx + 1) / 2 + (l - lx - ly); }

inline double dfact(int n) {  // (n)!! with (-1)!! = 0!! = 1
  double r = 1.0;
  for (int k = n; k > 1; k -= 2) r *= k;
  return r;
}

// ---------------------------------------------------------------- Boys function ----
// F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt on the grid T_i = i / BOYS_NPER, i < BOYS_NT, from the
// convergent series F_m(T) = exp(-T) sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)) in long double.
// Row i holds F_0 .. F_{BOYS_MTAB-1}; evaluation (Taylor about the nearest grid point, then
// downward recursion) needs orders up to m + 6.
constexpr double BOYS_TMAX = 40.0;
constexpr int BOYS_NPER = 16;
constexpr int BOYS_NT = static_cast<int>(BOYS_TMAX) * BOYS_NPER + 1;
constexpr int BOYS_MTAB = LTOT + 8;

inline void boys_table_fill(std::vector<double>& tab) {
  tab.assign(static_cast<size_t>(BOYS_NT) * BOYS_MTAB, 0.0);
  for (int i = 0; i < BOYS_NT; ++i) {
    long double T = static_cast<long double>(i) / BOYS_NPER;
    for (int m = 0; m < BOYS_MTAB; ++m) {
      long double term = 1.0L / (2 * m + 1), sum = term;
      for (int k = 1; k < 2000; ++k) {
        term *= 2.0L * T / (2 * m + 2 * k + 1);
        sum += term;
        if (term < sum * 1e-21L) break;
      }
      tab[static_cast<size_t>(i) * BOYS_MTAB + m] = static_cast<double>(expl(-T) * sum);
    }
  }
}

// ------------------------------------------------------- real solid harmonics ----
// c[l] is a (2l+1) x ncart(l) matrix C with Y_m = sum_c C[m][c] phi_c, where phi_c are the
// Cartesian functions normalised with the x^l convention, Cartesian order lx descending, then ly
// descending (cart_index).  Built from the solid-harmonic recurrence in x, y, z (Helgaker,
// Jorgensen, Olsen, Molecular Electronic-Structure Theory, eqs. 6.4.70-6.4.72) and normalised
// against the Cartesian overlap.
struct SphTables {
  std::vector<double> c[LMAX + 1];
  SphTables() {
    std::vector<std::vector<double>> S[LMAX + 1];  // S[l][m+l] polynomial over cart(l)
    S[0].assign(1, std::vector<double>(1, 1.0));
    auto mulx = [](const std::vector<double>& p, int l, int dir) {  // p of degree l times x/y/z
      std::vector<double> q(ncart(l + 1), 0.0);
      for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) {
          double v = p[cart_index(l, lx, ly)];
          if (v == 0.0) continue;
          int a = lx + (dir == 0), b = ly + (dir == 1);
          q[cart_index(l + 1, a, b)] += v;
        }
      return q;
    };
    auto mulr2 = [&](const std::vector<double>& p, int l) {
      std::vector<double> x = mulx(mulx(p, l, 0), l + 1, 0);
      std::vector<double> y = mulx(mulx(p, l, 1), l + 1, 1);
      std::vector<double> z = mulx(mulx(p, l, 2), l + 1, 2);
      for (size_t i = 0; i < x.size(); ++i) x[i] += y[i] + z[i];
      return x;
    };
    for (int l = 0; l < LMAX; ++l) {
      S[l + 1].assign(2 * l + 3, std::vector<double>());
      double f = std::sqrt((l == 0 ? 2.0 : 1.0) * (2 * l + 1) / (2.0 * l + 2));
      {
        std::vector<double> a = mulx(S[l][2 * l], l, 0);  // x S_{l,l}
        std::vector<double> b = mulx(S[l][2 * l], l, 1);  // y S_{l,l}
        if (l > 0) {
          std::vector<double> yb = mulx(S[l][0], l, 1);   // y S_{l,-l}
          std::vector<double> xb = mulx(S[l][0], l, 0);   // x S_{l,-l}
          for (size_t i = 0; i < a.size(); ++i) { a[i] -= yb[i]; b[i] += xb[i]; }
        }
        for (auto& v : a) v *= f;
        for (auto& v : b) v *= f;
        S[l + 1][2 * l + 2] = a;
        S[l + 1][0] = b;
      }
      for (int m = -l; m <= l; ++m) {
        std::vector<double> a = mulx(S[l][m + l], l, 2);
        for (auto& v : a) v *= (2 * l + 1);
        if (l >= 1 && std::abs(m) <= l - 1) {
          std::vector<double> r = mulr2(S[l - 1][m + l - 1], l - 1);
          double g = std::sqrt(static_cast<double>((l + m) * (l - m)));
          for (size_t i = 0; i < a.size(); ++i) a[i] -= g * r[i];
        }
        double h = 1.0 / std::sqrt(static_cast<double>((l + m + 1) * (l - m + 1)));
        for (auto& v : a) v *= h;
        S[l + 1][m + l + 1] = a;
      }
    }
    for (int l = 0; l <= LMAX; ++l) {
      int nc = ncart(l);
      c[l].assign(static_cast<size_t>(2 * l + 1) * nc, 0.0);
      std::vector<int> cx(nc), cy(nc), cz(nc);
      for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) {
          int i = cart_index(l, lx, ly);
          cx[i] = lx; cy[i] = ly; cz[i] = l - lx - ly;
        }
      for (int m = 0; m < 2 * l + 1; ++m) {
        const std::vector<double>& p = S[l][m];
        double n2 = 0.0;  // <Y|Y> relative to <x^l|x^l>
        for (int i = 0; i < nc; ++i)
          for (int j = 0; j < nc; ++j) {
            if (p[i] == 0.0 || p[j] == 0.0) continue;
            int sx = cx[i] + cx[j], sy = cy[i] + cy[j], sz = cz[i] + cz[j];
            if ((sx | sy | sz) & 1) continue;
            n2 += p[i] * p[j] * dfact(sx - 1) * dfact(sy - 1) * dfact(sz - 1);
          }
        n2 /= dfact(2 * l - 1);
        double s = 1.0 / std::sqrt(n2);
        for (int i = 0; i < nc; ++i) c[l][static_cast<size_t>(m) * nc + i] = p[i] * s;
      }
    }
  }
};

inline const SphTables& sph() {
  static SphTables t;
  return t;
}

// Normalised contraction coefficients of one shell: the x^l normalisation of each primitive,
// then the whole contraction scaled to unit norm.  Returns false for a non-positive exponent.
inline bool normalise_shell(int L, int nprim, const double* exps, const double* coefs, double* out) {
  for (int k = 0; k < nprim; ++k) {
    double a = exps[k];
    if (!(a > 0.0)) return false;
    double n2 = std::pow(4.0 * a, L) * std::pow(2.0 * a / PI, 1.5) / dfact(2 * L - 1);
    out[k] = coefs[k] * std::sqrt(n2);
  }
  double norm = 0.0;  // <x^l|x^l> of the contraction
  for (int i = 0; i < nprim; ++i)
    for (int j = 0; j < nprim; ++j) {
      double p = exps[i] + exps[j];
      norm += out[i] * out[j] * dfact(2 * L - 1) / std::pow(2.0 * p, L) * std::pow(PI / p, 1.5);
    }
  double sc = 1.0 / std::sqrt(norm);
  for (int k = 0; k < nprim; ++k) out[k] *= sc;
  return true;
}

}  // namespace gto_tab
