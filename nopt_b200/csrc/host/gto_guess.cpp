// gto_guess.cpp — superposition-of-atomic-densities (SAD) start for the RHF.
//
// The reference starts its RHF from Hueckel orbitals or from a SAD Fock matrix whose Fock
// build uses occupation-scaled atomic orbitals as MO rows (src/sad_guess.cpp:165-215, the
// call at :199-201).  Here one atom of each element runs a spherically averaged RHF with
// fractional occupations (degenerate levels share their electrons equally; occupations in the
// reference's normalisation, 1 = doubly occupied) in its own orbital and fitting basis, with
// RI-JK built from the engine's integrals and V^-1/2.  The molecular guess is the block-
// diagonal sum of the atomic densities; its factor rows sqrt(f_k) v_k (natural orbitals) feed
// the first Fock build in place of MO rows.
#include <cmath>
#include <vector>

#include "gto_ints.h"

namespace {

// Cyclic Jacobi eigensolver for a small symmetric matrix (row-major n x n, destroyed).
// w: eigenvalues ascending; V: eigenvectors as columns (row-major V[i*n+k] = component i of vector k).
void jacobi_eigh(std::vector<double>& A, int n, std::vector<double>& w, std::vector<double>& V) {
  V.assign(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[p * n + q] * A[p * n + q];
    if (off < 1e-30) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = A[i * n + i];
  // sort ascending
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (w[idx[j]] < w[idx[i]]) std::swap(idx[i], idx[j]);
  std::vector<double> w2(n), V2(static_cast<size_t>(n) * n);
  for (int k = 0; k < n; ++k) {
    w2[k] = w[idx[k]];
    for (int i = 0; i < n; ++i) V2[i * n + k] = V[i * n + idx[k]];
  }
  w = w2;
  V = V2;
}

// f(A) = V diag(g(w)) V^T for symmetric A
template <typename G>
std::vector<double> mat_func(const std::vector<double>& A, int n, G g) {
  std::vector<double> B = A, w, V;
  jacobi_eigh(B, n, w, V);
  std::vector<double> R(static_cast<size_t>(n) * n, 0.0);
  for (int k = 0; k < n; ++k) {
    double gk = g(w[k]);
    if (gk == 0.0) continue;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) R[i * n + j] += V[i * n + k] * gk * V[j * n + k];
  }
  return R;
}

}  // namespace

extern "C" int gto_atomic_density(const gto_basis* orb, const gto_basis* aux, double Z, const double* xyz,
                                  double* D, double* rows, int* nrows) {
  if (!orb || !aux || !xyz || !D || !rows || !nrows || Z <= 0) return GTO_ERR_ARG;
  const int n = gto_basis_nbf(orb), na = gto_basis_nbf(aux);
  std::vector<double> S(n * n), T(n * n), Vn(n * n), V2(na * na), I3(static_cast<size_t>(n) * n * na);
  int rc;
  if ((rc = gto_overlap(orb, S.data())) || (rc = gto_kinetic(orb, T.data())) ||
      (rc = gto_nuclear(orb, 1, &Z, xyz, Vn.data())) || (rc = gto_coulomb_2c(aux, V2.data())) ||
      (rc = gto_coulomb_3c(orb, aux, GTO_3C_NOPT_FULL, I3.data())))
    return rc;
  std::vector<double> H(n * n);
  for (int i = 0; i < n * n; ++i) H[i] = T[i] + Vn[i];
  // fitted tensor B[Q][m][n] = sum_P V^-1/2_QP (P|mn)
  std::vector<double> M = mat_func(V2, na, [](double l) { return l > 0.0 ? 1.0 / std::sqrt(l) : 0.0; });
  std::vector<double> B(static_cast<size_t>(na) * n * n, 0.0);
  for (int q = 0; q < na; ++q)
    for (int mn = 0; mn < n * n; ++mn) {
      double s = 0.0;
      for (int p = 0; p < na; ++p) s += M[q * na + p] * I3[static_cast<size_t>(mn) * na + p];
      B[static_cast<size_t>(q) * n * n + mn] = s;
    }
  std::vector<double> X = mat_func(S, n, [](double l) { return l > 1e-10 ? 1.0 / std::sqrt(l) : 0.0; });
  std::vector<double> F = H, Dm(n * n, 0.0), Fo(n * n), tmp(n * n), C(n * n), w, U;
  const double npair = Z / 2.0;
  for (int it = 0; it < 300; ++it) {
    // Fo = X^T F X
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += F[i * n + k] * X[k * n + j];
        tmp[i * n + j] = s;
      }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += X[k * n + i] * tmp[k * n + j];
        Fo[i * n + j] = s;
      }
    jacobi_eigh(Fo, n, w, U);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < n; ++k) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += X[i * n + j] * U[j * n + k];
        C[i * n + k] = s;
      }
    // fractional, spherically averaged occupations
    std::vector<double> f(n, 0.0);
    double rem = npair;
    for (int k = 0; k < n && rem > 1e-12;) {
      int g = k;
      while (g + 1 < n && std::fabs(w[g + 1] - w[k]) < 1e-6 * std::fmax(1.0, std::fabs(w[k]))) ++g;
      int size = g - k + 1;
      double take = std::fmin(1.0, rem / size);
      for (int j = k; j <= g; ++j) f[j] = take;
      rem -= take * size;
      k = g + 1;
    }
    double diff = 0.0;
    std::vector<double> Dn(n * n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += C[i * n + k] * f[k] * C[j * n + k];
        Dn[i * n + j] = s;
        diff = std::fmax(diff, std::fabs(s - Dm[i * n + j]));
      }
    Dm = Dn;
    if (diff < 1e-10 && it > 0) break;
    // F = 1/2 F + 1/2 (H + 2J - K)
    std::vector<double> wq(na, 0.0);
    for (int q = 0; q < na; ++q) {
      double s = 0.0;
      const double* Bq = &B[static_cast<size_t>(q) * n * n];
      for (int mn = 0; mn < n * n; ++mn) s += Bq[mn] * Dm[mn];
      wq[q] = s;
    }
    std::vector<double> J(n * n, 0.0), K(n * n, 0.0), BD(n * n);
    for (int q = 0; q < na; ++q) {
      const double* Bq = &B[static_cast<size_t>(q) * n * n];
      for (int mn = 0; mn < n * n; ++mn) J[mn] += wq[q] * Bq[mn];
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          double s = 0.0;
          for (int k = 0; k < n; ++k) s += Bq[i * n + k] * Dm[k * n + j];
          BD[i * n + j] = s;
        }
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          double s = 0.0;
          for (int k = 0; k < n; ++k) s += BD[i * n + k] * Bq[k * n + j];
          K[i * n + j] += s;
        }
    }
    for (int i = 0; i < n * n; ++i) F[i] = 0.5 * F[i] + 0.5 * (H[i] + 2.0 * J[i] - K[i]);
  }
  for (int i = 0; i < n * n; ++i) D[i] = Dm[i];
  // natural orbitals in the S metric: S^1/2 D S^1/2 = sum f w w^T, rows sqrt(f) S^-1/2 w
  std::vector<double> Sh = mat_func(S, n, [](double l) { return l > 0.0 ? std::sqrt(l) : 0.0; });
  std::vector<double> Shi = mat_func(S, n, [](double l) { return l > 1e-10 ? 1.0 / std::sqrt(l) : 0.0; });
  std::vector<double> A(n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += Sh[i * n + k] * Dm[k * n + j];
      tmp[i * n + j] = s;
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += tmp[i * n + k] * Sh[k * n + j];
      A[i * n + j] = s;
    }
  jacobi_eigh(A, n, w, U);
  int r = 0;
  for (int k = n - 1; k >= 0; --k) {
    if (w[k] <= 1e-10) continue;
    double sf = std::sqrt(w[k]);
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = 0; j < n; ++j) s += Shi[i * n + j] * U[j * n + k];
      rows[static_cast<size_t>(r) * n + i] = sf * s;
    }
    ++r;
  }
  *nrows = r;
  return GTO_OK;
}
