// k_eri.cu — the RI integrals on the GPU: (P|Q) and (mu nu|P) by the McMurchie-Davidson scheme,
// in FP64, written straight into the row blocks the metric contraction (K1) consumes.
//
// Replaces the reference's integral producers: RI_V_calc (src/libint_link.cpp:2049-2107, libint
// BraKet::xs_xs) and calc_2el_AO_INTS_RI (src/libint_link.cpp:2261-2350, BraKet::xs_xx), which
// gen_RI_AA (src/RI.cpp:34-79) calls once per geometry.  The arithmetic is the host engine's
// (gto_ints.cpp): bra primitive pairs expanded in Hermite Gaussians (E coefficients), Hermite
// Coulomb integrals R_tuv from the Boys function, aux functions as one-centre Hermite sums.
//
// Work decomposition.  One launch per angular class (l_A, l_B, l_C); a task is one shell triple
// (A B | C) and runs on a group of G lanes (G = 1 .. 32, chosen per class so that small classes
// keep the lanes busy).  Per bra primitive pair the group builds the three 1-D E tables, then per
// aux primitive the Boys values, the R_tuv layers (lanes over the entries of a layer), and
//     W[m][tuv] += pref * sum_terms d * (2 gamma)^-j * R[tuv + term]      (aux Hermite sum)
// and finally contracts acc[a][b][m] += sum_tuv E^ab_tuv W[m][tuv].  The bra's Cartesian block is
// transformed to spherical harmonics once per triple and stored.  Everything a group touches
// lives in its own slice of shared memory; lanes own disjoint outputs, so only group-wide
// __syncwarp separates the stages.
//
// The aux one-centre expansion is gamma-independent up to a power: the Hermite coefficient of
// x^i about its own centre is E^{i0}_t = a_{it} (2 gamma)^{-(i+t)/2}, so each aux function m
// is a fixed list of terms (tau, nu, phi, d) scaled by (2 gamma)^{-(l+s)/2}, s = tau+nu+phi.
#include <algorithm>
#include <cmath>
#include <vector>

#include "gto_tables.h"
#include "rijk_internal.h"

#define RIJK_API extern "C" __attribute__((visibility("default")))

namespace rijk {
namespace {

using gto_tab::LMAX;
constexpr int LTOT = 3 * LMAX;
constexpr int TET_MAX = (LTOT + 1) * (LTOT + 2) * (LTOT + 3) / 6;  // 455 entries with t+u+v <= 12
constexpr int NSPH = 245;            // sum over l <= 4 of (2l+1) ncart(l)
constexpr int TERM_KEYS = 2 * (LMAX + 1);
constexpr int TERM_STRIDE = 16;      // per key: offsets of m = 0 .. 15 (ncart(4) = 15) and the end
constexpr int GROUP_F = 24;          // per group: F_0 .. F_15 and the aux power table pw[0..7]
constexpr int ERI_THREADS = 128;

struct EriShell {
  double x, y, z;
  int l, nprim, prim0, off;
  int nfunc, pure, pad0, pad1;
};

struct EriTerm {
  short t, u, v, j;  // Hermite index of the term and the power j of (2 gamma)^-1
  int pad;
  double d;
};

struct EriLaunch {
  const EriShell* bra;
  const double* bexp;
  const double* bcoef;
  const int2* pairs;
  long npair;
  const EriShell* ket;
  const double* kexp;
  const double* kcoef;
  const int* kets;
  long nket;
  int la, lb, lc, G;
  int gsize;        // doubles of shared memory per group
  int mode;         // 0 packed rows (hi(hi+1)/2 + lo), 1 full rows (mu n + nu), 2 square (P, Q)
  long mu0, mu1;    // rows written (modes 0, 1)
  long rowbase;     // row index subtracted before storing
  long n;           // orbital functions (mode 1 row pitch in pairs)
  long ld;          // element pitch between stored rows
  double* out;
  const double* boys;
  const double* sph;
  const EriTerm* terms;
  const int* term_off;
  const int* tuv;
  const int* cart;
};

__host__ __device__ inline int tet(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
__host__ __device__ inline int ncart_d(int l) { return (l + 1) * (l + 2) / 2; }
__device__ __forceinline__ int tet_index(int t, int u, int v) {
  const int s = t + u + v, w = u + v;
  return s * (s + 1) * (s + 2) / 6 + w * (w + 1) / 2 + v;
}
__host__ __device__ inline int sph_off(int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += (2 * k + 1) * ncart_d(k);
  return o;
}

// F_m(T), m = 0 .. L, exactly as the host engine evaluates it (Taylor about the nearest grid
// point, downward recursion; F_0 and upward recursion past the grid).
__device__ void boys_eval(int L, double T, const double* __restrict__ tab, double* F) {
  constexpr double TMAX = gto_tab::BOYS_TMAX;
  constexpr int NPER = gto_tab::BOYS_NPER, MTAB = gto_tab::BOYS_MTAB;
  if (T < TMAX - 0.5 / NPER) {
    const int i = static_cast<int>(T * NPER + 0.5);
    const double dt = static_cast<double>(i) / NPER - T;
    const double* row = tab + static_cast<long>(i) * MTAB;
    double f = __ldg(row + L + 6);
    f = __ldg(row + L + 5) + f * dt / 6.0;
    f = __ldg(row + L + 4) + f * dt / 5.0;
    f = __ldg(row + L + 3) + f * dt / 4.0;
    f = __ldg(row + L + 2) + f * dt / 3.0;
    f = __ldg(row + L + 1) + f * dt / 2.0;
    f = __ldg(row + L) + f * dt;
    F[L] = f;
    const double e = exp(-T);
    for (int m = L; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + e) / (2 * m - 1);
  } else {
    const double e = exp(-T);
    F[0] = 0.5 * sqrt(gto_tab::PI / T);
    for (int m = 0; m < L; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2.0 * T);
  }
}

// 1-D Hermite expansion E[i][j][t] of a primitive product, i <= la, j <= lb, t < ts (= la+lb+2).
__device__ void hermite_1d_dev(int la, int lb, double p, double xpa, double xpb, double k0, double* E, int ts) {
  const double o2p = 0.5 / p;
  auto at = [&](int i, int j, int t) -> double& { return E[(i * (lb + 1) + j) * ts + t]; };
  for (int k = 0; k < (la + 1) * (lb + 1) * ts; ++k) E[k] = 0.0;
  at(0, 0, 0) = k0;
  for (int i = 0; i < la; ++i)
    for (int t = 0; t <= i + 1; ++t) {
      double v = xpa * at(i, 0, t) + (t + 1) * at(i, 0, t + 1);
      if (t > 0) v += o2p * at(i, 0, t - 1);
      at(i + 1, 0, t) = v;
    }
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j < lb; ++j)
      for (int t = 0; t <= i + j + 1; ++t) {
        double v = xpb * at(i, j, t) + (t + 1) * at(i, j, t + 1);
        if (t > 0) v += o2p * at(i, j, t - 1);
        at(i, j + 1, t) = v;
      }
}

__global__ void __launch_bounds__(ERI_THREADS) k_eri(const EriLaunch P) {
  extern __shared__ __align__(16) double sm_eri[];
  const int G = P.G;
  const int lane = threadIdx.x & 31;
  const int gl = threadIdx.x % G;
  const int gpb = blockDim.x / G;
  const int gloc = threadIdx.x / G;
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((lane / G) * G));
  const int la = P.la, lb = P.lb, lc = P.lc, Lab = la + lb, L = Lab + lc;
  const int nca = ncart_d(la), ncb = ncart_d(lb);
  const int ts = Lab + 2, nE1 = (la + 1) * (lb + 1) * ts;
  const int tL = tet(L), tLab = tet(Lab);
  double* g = sm_eri + static_cast<long>(gloc) * P.gsize;
  double* F = g;                         // F[0..15], pw at F + 16
  double* pw = g + 16;
  double* E = g + GROUP_F;               // 3 x nE1
  double* R0 = E + 3 * nE1;              // two R layers
  double* R1 = R0 + tL;
  double* W = R1 + tL;                   // nfc x tLab
  double* acc = W + ncart_d(lc) * tLab;  // nca x ncb x nfc
  const double sgn = (lc & 1) ? -1.0 : 1.0;
  const double two_pi_25 = 2.0 * 17.493418327624862;  // 2 pi^(5/2)

  const long ntask = P.npair * P.nket;
  const long stride = static_cast<long>(gridDim.x) * gpb;
  for (long task = static_cast<long>(blockIdx.x) * gpb + gloc; task < ntask; task += stride) {
    const long ip = task / P.nket;
    const long jc = task - ip * P.nket;
    const int2 pr = P.pairs[ip];
    const EriShell A = P.bra[pr.x];
    const EriShell B = P.bra[pr.y];
    const EriShell C = P.ket[P.kets[jc]];
    const int nfc = C.nfunc;
    const int nout = nca * ncb * nfc;
    const int nW = nfc * tLab;
    const int key = (C.pure ? LMAX + 1 : 0) + lc;
    const int* toff = P.term_off + key * (TERM_STRIDE + 1);
    for (int o = gl; o < nout; o += G) acc[o] = 0.0;
    const double ABx = A.x - B.x, ABy = A.y - B.y, ABz = A.z - B.z;
    const double r2 = ABx * ABx + ABy * ABy + ABz * ABz;
    for (int i = 0; i < A.nprim; ++i) {
      const double a = P.bexp[A.prim0 + i], ca = P.bcoef[A.prim0 + i];
      for (int j = 0; j < B.nprim; ++j) {
        const double b = P.bexp[B.prim0 + j], cb = P.bcoef[B.prim0 + j];
        const double p = a + b, mu = a * b / p;
        const double K = exp(-mu * r2);
        const double cc = ca * cb;
        if (fabs(cc * K) < 1e-22) continue;  // contributes below double precision (host rule)
        const double Px = (a * A.x + b * B.x) / p, Py = (a * A.y + b * B.y) / p, Pz = (a * A.z + b * B.z) / p;
        __syncwarp(gmask);  // the previous pair's readers of E and W are done
        for (int d = gl; d < 3; d += G) {
          const double pd = d == 0 ? Px : (d == 1 ? Py : Pz);
          const double ad = d == 0 ? A.x : (d == 1 ? A.y : A.z);
          const double bd = d == 0 ? B.x : (d == 1 ? B.y : B.z);
          hermite_1d_dev(la, lb, p, pd - ad, pd - bd, d == 0 ? K : 1.0, E + d * nE1, ts);
        }
        for (int o = gl; o < nW; o += G) W[o] = 0.0;
        for (int k = 0; k < C.nprim; ++k) {
          const double gam = P.kexp[C.prim0 + k], ck = P.kcoef[C.prim0 + k];
          const double al = p * gam / (p + gam);
          const double X = Px - C.x, Y = Py - C.y, Z = Pz - C.z;
          const double T = al * (X * X + Y * Y + Z * Z);
          if (gl == 0) {
            boys_eval(L, T, P.boys, F);
            const double pref = two_pi_25 / (p * gam * sqrt(p + gam)) * cc * ck * sgn;
            const double i2g = 1.0 / (2.0 * gam);
            double v = pref;
            for (int q = 0; q <= lc; ++q) { pw[q] = v; v *= i2g; }
          }
          __syncwarp(gmask);
          // R^n_tuv for n = L .. 0; layer n holds t+u+v <= L-n and reads layer n+1
          const double m2a = -2.0 * al;
          double* cur = R0;
          double* nxt = R1;
          for (int nn = L; nn >= 0; --nn) {
            const int cnt = tet(L - nn);
            for (int e = gl; e < cnt; e += G) {
              double r;
              if (e == 0) {
                double pwn = 1.0;
                for (int q = 0; q < nn; ++q) pwn *= m2a;
                r = pwn * F[nn];
              } else {
                const int c = __ldg(P.tuv + e);
                const int t = c & 0xff, u = (c >> 8) & 0xff, v = c >> 16;
                if (t > 0) {
                  r = X * nxt[tet_index(t - 1, u, v)];
                  if (t > 1) r += (t - 1) * nxt[tet_index(t - 2, u, v)];
                } else if (u > 0) {
                  r = Y * nxt[tet_index(t, u - 1, v)];
                  if (u > 1) r += (u - 1) * nxt[tet_index(t, u - 2, v)];
                } else {
                  r = Z * nxt[tet_index(t, u, v - 1)];
                  if (v > 1) r += (v - 1) * nxt[tet_index(t, u, v - 2)];
                }
              }
              cur[e] = r;
            }
            __syncwarp(gmask);
            double* tmp = cur;
            cur = nxt;
            nxt = tmp;
          }
          const double* R = nxt;  // layer 0
          for (int o = gl; o < nW; o += G) {
            const int m = o / tLab, e = o - m * tLab;
            const int c = __ldg(P.tuv + e);
            const int t = c & 0xff, u = (c >> 8) & 0xff, v = c >> 16;
            const int q1 = __ldg(toff + m + 1);
            double s = 0.0;
            for (int q = __ldg(toff + m); q < q1; ++q) {
              const EriTerm h = P.terms[q];
              s += h.d * pw[h.j] * R[tet_index(t + h.t, u + h.u, v + h.v)];
            }
            W[o] += s;
          }
          __syncwarp(gmask);  // W complete; F and R free for the next aux primitive
        }
        // acc[a][b][m] += sum_tuv Ex Ey Ez W[m][tuv]
        const double* Ex = E;
        const double* Ey = E + nE1;
        const double* Ez = E + 2 * nE1;
        for (int o = gl; o < nout; o += G) {
          const int m = o % nfc, ab = o / nfc;
          const int ib = ab % ncb, ia = ab / ncb;
          const int ka = __ldg(P.cart + la * 16 + ia), kb = __ldg(P.cart + lb * 16 + ib);
          const int ax = ka & 15, ay = (ka >> 4) & 15, az = ka >> 8;
          const int bx = kb & 15, by = (kb >> 4) & 15, bz = kb >> 8;
          const double* wm = W + m * tLab;
          double v = 0.0;
          for (int t = 0; t <= ax + bx; ++t) {
            const double et = Ex[(ax * (lb + 1) + bx) * ts + t];
            if (et == 0.0) continue;
            for (int u = 0; u <= ay + by; ++u) {
              const double eu = et * Ey[(ay * (lb + 1) + by) * ts + u];
              if (eu == 0.0) continue;
              for (int w = 0; w <= az + bz; ++w) v += eu * Ez[(az * (lb + 1) + bz) * ts + w] * wm[tet_index(t, u, w)];
            }
          }
          acc[o] += v;
        }
      }
    }
    __syncwarp(gmask);  // acc complete
    // bra Cartesian -> spherical, then store
    const int nfa = A.nfunc, nfb = B.nfunc;
    const double* ta = P.sph + sph_off(la);
    const double* tb = P.sph + sph_off(lb);
    for (int o = gl; o < nfa * nfb * nfc; o += G) {
      const int m = o % nfc, ab = o / nfc;
      const int fb = ab % nfb, fa = ab / nfb;
      double v = 0.0;
      const int ia0 = A.pure ? 0 : fa, ia1 = A.pure ? nca : fa + 1;
      const int ib0 = B.pure ? 0 : fb, ib1 = B.pure ? ncb : fb + 1;
      for (int ia = ia0; ia < ia1; ++ia) {
        const double wa = A.pure ? __ldg(ta + fa * nca + ia) : 1.0;
        if (wa == 0.0) continue;
        double sb = 0.0;
        for (int ib = ib0; ib < ib1; ++ib) {
          const double wb = B.pure ? __ldg(tb + fb * ncb + ib) : 1.0;
          sb += wb * acc[(ia * ncb + ib) * nfc + m];
        }
        v += wa * sb;
      }
      const long col = C.off + m;
      if (P.mode == 2) {
        P.out[(static_cast<long>(A.off + fa) - P.rowbase) * P.ld + col] = v;
      } else {
        const long mu = A.off + fa, nu = B.off + fb;
        if (P.mode == 0) {
          if (pr.x == pr.y && nu > mu) continue;
          const long hi = mu > nu ? mu : nu, lo = mu > nu ? nu : mu;
          if (hi < P.mu0 || hi >= P.mu1) continue;
          P.out[(hi * (hi + 1) / 2 + lo - P.rowbase) * P.ld + col] = v;
        } else {
          if (mu >= P.mu0 && mu < P.mu1) P.out[((mu - P.rowbase) * P.n + nu) * P.ld + col] = v;
          if (pr.x != pr.y && nu >= P.mu0 && nu < P.mu1) P.out[((nu - P.rowbase) * P.n + mu) * P.ld + col] = v;
        }
      }
    }
    __syncwarp(gmask);  // acc is reused by the group's next task
  }
}

// ------------------------------------------------------------------------ host side ----

struct HostBasis {
  std::vector<EriShell> sh;
  std::vector<double> exps, coefs;
  int nbf = 0, lmax = 0;
};

int load_basis(rijk_ctx* ctx, const rijk_basis_t* b, const char* what, HostBasis& out) {
  if (!b || b->nshell <= 0 || !b->l || !b->pure || !b->nprim || !b->xyz || !b->exps || !b->coefs)
    return set_err(ctx, RIJK_ERR_ARG, "%s basis: null arrays or no shells", what);
  out = HostBasis();
  int po = 0;
  for (int s = 0; s < b->nshell; ++s) {
    const int l = b->l[s], np = b->nprim[s];
    if (l < 0 || l > LMAX) return set_err(ctx, RIJK_ERR_ARG, "%s basis: shell %d has l = %d (0..4 supported)", what, s, l);
    if (np < 1) return set_err(ctx, RIJK_ERR_ARG, "%s basis: shell %d has no primitives", what, s);
    EriShell e{};
    e.x = b->xyz[3 * s];
    e.y = b->xyz[3 * s + 1];
    e.z = b->xyz[3 * s + 2];
    e.l = l;
    e.nprim = np;
    e.prim0 = static_cast<int>(out.exps.size());
    e.off = out.nbf;
    e.pure = b->pure[s] ? 1 : 0;
    e.nfunc = e.pure ? 2 * l + 1 : ncart_d(l);
    std::vector<double> nc(np);
    if (!gto_tab::normalise_shell(l, np, b->exps + po, b->coefs + po, nc.data()))
      return set_err(ctx, RIJK_ERR_ARG, "%s basis: shell %d has a non-positive exponent", what, s);
    out.exps.insert(out.exps.end(), b->exps + po, b->exps + po + np);
    out.coefs.insert(out.coefs.end(), nc.begin(), nc.end());
    out.nbf += e.nfunc;
    out.lmax = std::max(out.lmax, l);
    out.sh.push_back(e);
    po += np;
  }
  return RIJK_OK;
}

// Device copy of one basis: shells, exponents, coefficients (one allocation).
struct DevBasis {
  DeviceBuf buf;
  const EriShell* sh = nullptr;
  const double* exps = nullptr;
  const double* coefs = nullptr;
};

// Every upload goes through the context's stream (cudaMemcpyAsync; pageable sources are staged
// before the call returns).  That stream is non-blocking: a plain cudaMemcpy, on the legacy
// stream, would not order against the kernels that read the data and may still be in flight
// when they start.
int upload_basis(rijk_ctx* ctx, const HostBasis& h, DevBasis& d) {
  const size_t b0 = h.sh.size() * sizeof(EriShell), b1 = h.exps.size() * sizeof(double);
  std::vector<char> blob(b0 + 2 * b1);
  std::copy(reinterpret_cast<const char*>(h.sh.data()), reinterpret_cast<const char*>(h.sh.data()) + b0, blob.data());
  std::copy(reinterpret_cast<const char*>(h.exps.data()), reinterpret_cast<const char*>(h.exps.data()) + b1,
            blob.data() + b0);
  std::copy(reinterpret_cast<const char*>(h.coefs.data()), reinterpret_cast<const char*>(h.coefs.data()) + b1,
            blob.data() + b0 + b1);
  int rc = ensure(ctx, d.buf, blob.size(), "basis");
  if (rc) return rc;
  rc = cuda_check(ctx, cudaMemcpyAsync(d.buf.p, blob.data(), blob.size(), cudaMemcpyHostToDevice, ctx->stream),
                  "H2D basis");
  if (rc) return rc;
  char* p = static_cast<char*>(d.buf.p);
  d.sh = reinterpret_cast<const EriShell*>(p);
  d.exps = reinterpret_cast<const double*>(p + b0);
  d.coefs = reinterpret_cast<const double*>(p + b0 + b1);
  return RIJK_OK;
}

// Device tables shared by all launches: Boys grid, spherical transforms, aux term lists,
// Hermite index decode and Cartesian exponents.  Built once per context.
struct TabLayout {
  size_t boys, sph, terms, term_off, tuv, cart, total;
};

TabLayout tab_layout(size_t nterms) {
  TabLayout t{};
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t r = o;
    o = (o + bytes + 255) / 256 * 256;
    return r;
  };
  t.boys = take(sizeof(double) * gto_tab::BOYS_NT * gto_tab::BOYS_MTAB);
  t.sph = take(sizeof(double) * NSPH);
  t.terms = take(sizeof(EriTerm) * nterms);
  t.term_off = take(sizeof(int) * TERM_KEYS * (TERM_STRIDE + 1));
  t.tuv = take(sizeof(int) * TET_MAX);
  t.cart = take(sizeof(int) * (LMAX + 1) * 16);
  t.total = o;
  return t;
}

struct DevTables {
  const double* boys;
  const double* sph;
  const EriTerm* terms;
  const int* term_off;
  const int* tuv;
  const int* cart;
};

int ensure_tables(rijk_ctx* ctx, DevTables& dt) {
  // aux term lists: for (pure, l, m) the Hermite terms of the one-centre expansion at 2 gamma = 1
  std::vector<EriTerm> terms;
  std::vector<int> toff(TERM_KEYS * (TERM_STRIDE + 1), 0);
  const gto_tab::SphTables& S = gto_tab::sph();
  double a[LMAX + 1][LMAX + 2] = {};  // a[i][t]: E^{i0}_t at 2 gamma = 1
  a[0][0] = 1.0;
  for (int i = 0; i < LMAX; ++i)
    for (int t = 0; t <= i + 1; ++t) a[i + 1][t] = (t > 0 ? a[i][t - 1] : 0.0) + (t + 1) * a[i][t + 1];
  for (int pure = 0; pure < 2; ++pure)
    for (int l = 0; l <= LMAX; ++l) {
      const int key = pure * (LMAX + 1) + l, nc = ncart_d(l), nf = pure ? 2 * l + 1 : nc;
      for (int m = 0; m < nf; ++m) {
        toff[key * (TERM_STRIDE + 1) + m] = static_cast<int>(terms.size());
        double cube[LMAX + 1][LMAX + 1][LMAX + 1] = {};
        for (int lx = l; lx >= 0; --lx)
          for (int ly = l - lx; ly >= 0; --ly) {
            const int lz = l - lx - ly, c = gto_tab::cart_index(l, lx, ly);
            const double w = pure ? S.c[l][static_cast<size_t>(m) * nc + c] : (c == m ? 1.0 : 0.0);
            if (w == 0.0) continue;
            for (int t = 0; t <= lx; ++t)
              for (int u = 0; u <= ly; ++u)
                for (int v = 0; v <= lz; ++v) cube[t][u][v] += w * a[lx][t] * a[ly][u] * a[lz][v];
          }
        for (int t = 0; t <= l; ++t)
          for (int u = 0; u <= l - t; ++u)
            for (int v = 0; v <= l - t - u; ++v)
              if (cube[t][u][v] != 0.0) {
                EriTerm e{};
                e.t = static_cast<short>(t);
                e.u = static_cast<short>(u);
                e.v = static_cast<short>(v);
                e.j = static_cast<short>((l + t + u + v) / 2);
                e.d = cube[t][u][v];
                terms.push_back(e);
              }
      }
      for (int m = nf; m <= TERM_STRIDE; ++m) toff[key * (TERM_STRIDE + 1) + m] = static_cast<int>(terms.size());
    }
  const TabLayout lay = tab_layout(terms.size());
  if (!ctx->eri_tab.p) {
    std::vector<char> blob(lay.total, 0);
    std::vector<double> boys;
    gto_tab::boys_table_fill(boys);
    std::copy(boys.begin(), boys.end(), reinterpret_cast<double*>(blob.data() + lay.boys));
    double* sph = reinterpret_cast<double*>(blob.data() + lay.sph);
    for (int l = 0, o = 0; l <= LMAX; ++l)
      for (double v : S.c[l]) sph[o++] = v;
    std::copy(terms.begin(), terms.end(), reinterpret_cast<EriTerm*>(blob.data() + lay.terms));
    std::copy(toff.begin(), toff.end(), reinterpret_cast<int*>(blob.data() + lay.term_off));
    int* tuv = reinterpret_cast<int*>(blob.data() + lay.tuv);
    for (int s = 0, e = 0; s <= LTOT; ++s)
      for (int w = 0; w <= s; ++w)
        for (int v = 0; v <= w; ++v) tuv[e++] = (s - w) | ((w - v) << 8) | (v << 16);
    int* cart = reinterpret_cast<int*>(blob.data() + lay.cart);
    for (int l = 0; l <= LMAX; ++l)
      for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly)
          cart[l * 16 + gto_tab::cart_index(l, lx, ly)] = lx | (ly << 4) | ((l - lx - ly) << 8);
    int rc = ensure(ctx, ctx->eri_tab, lay.total, "integral tables");
    if (rc) return rc;
    rc = cuda_check(ctx, cudaMemcpyAsync(ctx->eri_tab.p, blob.data(), lay.total, cudaMemcpyHostToDevice, ctx->stream),
                    "H2D tables");
    if (rc) return rc;
  }
  const char* p = static_cast<const char*>(ctx->eri_tab.p);
  dt.boys = reinterpret_cast<const double*>(p + lay.boys);
  dt.sph = reinterpret_cast<const double*>(p + lay.sph);
  dt.terms = reinterpret_cast<const EriTerm*>(p + lay.terms);
  dt.term_off = reinterpret_cast<const int*>(p + lay.term_off);
  dt.tuv = reinterpret_cast<const int*>(p + lay.tuv);
  dt.cart = reinterpret_cast<const int*>(p + lay.cart);
  return RIJK_OK;
}

// Lanes per task for a class: enough to cover the widest stage without idling most of them.
int group_lanes(int la, int lb, int lc) {
  const int L = la + lb + lc;
  const int work = std::max({ncart_d(la) * ncart_d(lb) * ncart_d(lc), tet(L), ncart_d(lc) * tet(la + lb)});
  int G = 1;
  while (G < 32 && G * 3 < work) G *= 2;
  return G;
}

int group_doubles(int la, int lb, int lc) {
  const int Lab = la + lb, L = Lab + lc;
  int d = GROUP_F + 3 * (la + 1) * (lb + 1) * (Lab + 2) + 2 * tet(L) + ncart_d(lc) * tet(Lab) +
          ncart_d(la) * ncart_d(lb) * ncart_d(lc);
  return (d + 1) & ~1;
}

// Ket shells grouped by angular momentum, each group sorted by primitive count (tasks next to
// each other in a warp then share their loop trip counts).
struct KetLists {
  std::vector<int> idx;
  long start[LMAX + 2] = {};
};

KetLists ket_lists(const HostBasis& k) {
  KetLists out;
  for (int l = 0; l <= LMAX; ++l) {
    out.start[l] = static_cast<long>(out.idx.size());
    std::vector<int> v;
    for (int s = 0; s < static_cast<int>(k.sh.size()); ++s)
      if (k.sh[s].l == l) v.push_back(s);
    std::stable_sort(v.begin(), v.end(), [&](int x, int y) { return k.sh[x].nprim < k.sh[y].nprim; });
    out.idx.insert(out.idx.end(), v.begin(), v.end());
  }
  out.start[LMAX + 1] = static_cast<long>(out.idx.size());
  return out;
}

// Bra pair lists by class (l_A, l_B), concatenated, with class offsets.
struct PairLists {
  std::vector<int2> pairs;
  long start[(LMAX + 1) * (LMAX + 1) + 1] = {};
};

template <typename Keep>
void pair_lists(const std::vector<EriShell>& bra, const std::vector<int2>& cand, Keep keep, PairLists& out) {
  std::vector<int2> by[(LMAX + 1) * (LMAX + 1)];
  for (const int2& pr : cand)
    if (keep(pr)) by[bra[pr.x].l * (LMAX + 1) + bra[pr.y].l].push_back(pr);
  out.pairs.clear();
  for (int c = 0; c < (LMAX + 1) * (LMAX + 1); ++c) {
    out.start[c] = static_cast<long>(out.pairs.size());
    out.pairs.insert(out.pairs.end(), by[c].begin(), by[c].end());
  }
  out.start[(LMAX + 1) * (LMAX + 1)] = static_cast<long>(out.pairs.size());
}

// Launches every class of one output block.  pairs_dev holds PairLists::pairs on the device.
int launch_classes(rijk_ctx* ctx, const EriLaunch& base, const PairLists& pl, const int2* pairs_dev,
                   const KetLists& kl, const int* kets_dev, int* launches) {
  cudaStream_t s = ctx->stream;
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  for (int la = 0; la <= LMAX; ++la)
    for (int lb = 0; lb <= LMAX; ++lb) {
      const int c = la * (LMAX + 1) + lb;
      const long np = pl.start[c + 1] - pl.start[c];
      if (np == 0) continue;
      for (int lc = 0; lc <= LMAX; ++lc) {
        const long nk = kl.start[lc + 1] - kl.start[lc];
        if (nk == 0) continue;
        EriLaunch P = base;
        P.la = la;
        P.lb = lb;
        P.lc = lc;
        P.G = group_lanes(la, lb, lc);
        P.gsize = group_doubles(la, lb, lc);
        P.pairs = pairs_dev + pl.start[c];
        P.npair = np;
        P.kets = kets_dev + kl.start[lc];
        P.nket = nk;
        const size_t per_warp = static_cast<size_t>(32 / P.G) * P.gsize * sizeof(double);
        int warps = static_cast<int>(std::min<size_t>(ERI_THREADS / 32, static_cast<size_t>(maxsm) / per_warp));
        if (warps < 1) return set_err(ctx, RIJK_ERR_ARG, "integral class (%d %d|%d) needs too much shared memory", la, lb, lc);
        const size_t smem = per_warp * warps;
        if (smem > 48 * 1024) {
          cudaError_t e = cudaFuncSetAttribute(k_eri, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
          if (e != cudaSuccess) return cuda_check(ctx, e, "integral kernel shared memory");
        }
        const long gpb = static_cast<long>(warps) * 32 / P.G;
        const long ntask = np * nk;
        long blocks = (ntask + gpb - 1) / gpb;
        blocks = std::min<long>(blocks, 148L * 32);
        k_eri<<<static_cast<unsigned>(blocks), warps * 32, smem, s>>>(P);
        ++*launches;
      }
    }
  return cuda_check(ctx, cudaGetLastError(), "integral kernel launch");
}

EriLaunch base_launch(const DevTables& t) {
  EriLaunch P{};
  P.boys = t.boys;
  P.sph = t.sph;
  P.terms = t.terms;
  P.term_off = t.term_off;
  P.tuv = t.tuv;
  P.cart = t.cart;
  return P;
}

// Everything an integral call needs on the device.
struct EriPlan {
  HostBasis orb, aux;
  DevBasis dorb, daux, dauxu;  // dauxu: aux shells plus a unit s function (bra of (P|Q))
  DevTables tab{};
  KetLists kets;
  DeviceBuf kets_dev, pairs_dev;
  std::vector<int2> orb_pairs;  // all (A, B <= A)
};

void release_plan(EriPlan& p) {
  release(p.dorb.buf);
  release(p.daux.buf);
  release(p.dauxu.buf);
  release(p.kets_dev);
  release(p.pairs_dev);
}

int make_plan(rijk_ctx* ctx, const rijk_basis_t* orb, const rijk_basis_t* aux, EriPlan& p) {
  int rc;
  if ((rc = load_basis(ctx, aux, "aux", p.aux))) return rc;
  if (orb && (rc = load_basis(ctx, orb, "orbital", p.orb))) return rc;
  if ((rc = ensure_tables(ctx, p.tab))) return rc;
  if ((rc = upload_basis(ctx, p.aux, p.daux))) return rc;
  HostBasis au = p.aux;
  EriShell u{};
  u.l = 0;
  u.nprim = 1;
  u.prim0 = static_cast<int>(au.exps.size());
  u.off = 0;
  u.nfunc = 1;
  u.pure = 1;
  au.exps.push_back(0.0);  // exponent 0, coefficient 1: the constant function
  au.coefs.push_back(1.0);
  au.sh.push_back(u);
  if ((rc = upload_basis(ctx, au, p.dauxu))) return rc;
  if (orb && (rc = upload_basis(ctx, p.orb, p.dorb))) return rc;
  p.kets = ket_lists(p.aux);
  if ((rc = ensure(ctx, p.kets_dev, p.kets.idx.size() * sizeof(int), "ket list"))) return rc;
  if ((rc = cuda_check(ctx, cudaMemcpyAsync(p.kets_dev.p, p.kets.idx.data(), p.kets.idx.size() * sizeof(int),
                                            cudaMemcpyHostToDevice, ctx->stream), "H2D ket list")))
    return rc;
  if (orb) {
    const int ns = static_cast<int>(p.orb.sh.size());
    p.orb_pairs.reserve(static_cast<size_t>(ns) * (ns + 1) / 2);
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b <= a; ++b) p.orb_pairs.push_back(make_int2(a, b));
    if ((rc = ensure(ctx, p.pairs_dev, p.orb_pairs.size() * sizeof(int2), "pair list"))) return rc;
  }
  return RIJK_OK;
}

// (P|Q) into dV (naux x naux, pitch ld), asynchronous.
int eri2c_device(rijk_ctx* ctx, EriPlan& p, double* dV, long ld, int* launches) {
  const int na = static_cast<int>(p.aux.sh.size());
  std::vector<int2> cand(na);
  for (int a = 0; a < na; ++a) cand[a] = make_int2(a, na);  // (P, unit)
  PairLists pl;
  std::vector<EriShell> bra = p.aux.sh;
  EriShell u{};
  bra.push_back(u);
  pair_lists(bra, cand, [](const int2&) { return true; }, pl);
  DeviceBuf dp;
  int rc = ensure(ctx, dp, pl.pairs.size() * sizeof(int2), "2c pair list");
  if (rc) return rc;
  rc = cuda_check(ctx, cudaMemcpyAsync(dp.p, pl.pairs.data(), pl.pairs.size() * sizeof(int2), cudaMemcpyHostToDevice,
                                       ctx->stream), "H2D 2c pairs");
  if (!rc) {
    EriLaunch P = base_launch(p.tab);
    P.bra = p.dauxu.sh;
    P.bexp = p.dauxu.exps;
    P.bcoef = p.dauxu.coefs;
    P.ket = p.daux.sh;
    P.kexp = p.daux.exps;
    P.kcoef = p.daux.coefs;
    P.mode = 2;
    P.ld = ld;
    P.out = dV;
    rc = launch_classes(ctx, P, pl, static_cast<const int2*>(dp.p), p.kets, static_cast<const int*>(p.kets_dev.p),
                        launches);
    if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "two-centre integrals");
  }
  cudaStreamSynchronize(ctx->stream);  // no launch may still read the pair list
  release(dp);
  return rc;
}

// (mu nu|P) for the rows [mu0, mu1) into dout, asynchronous.  layout RIJK_LAYOUT_PACKED writes
// pair rows hi(hi+1)/2 + lo - rowbase (hi in [mu0, mu1)); RIJK_LAYOUT_NOPT_FULL writes rows
// (mu - mu0) n + nu for mu in [mu0, mu1).  Entries not written are left as they are.
int eri3c_rows(rijk_ctx* ctx, EriPlan& p, int layout, long mu0, long mu1, long rowbase, double* dout, long ld,
               int* launches) {
  const std::vector<EriShell>& sh = p.orb.sh;
  auto hits = [&](int s) { return sh[s].off < mu1 && sh[s].off + sh[s].nfunc > mu0; };
  PairLists pl;
  if (layout == RIJK_LAYOUT_PACKED)
    pair_lists(sh, p.orb_pairs, [&](const int2& pr) { return hits(pr.x); }, pl);
  else
    pair_lists(sh, p.orb_pairs, [&](const int2& pr) { return hits(pr.x) || hits(pr.y); }, pl);
  if (pl.pairs.empty()) return RIJK_OK;
  int rc = cuda_check(ctx, cudaMemcpyAsync(p.pairs_dev.p, pl.pairs.data(), pl.pairs.size() * sizeof(int2),
                                           cudaMemcpyHostToDevice, ctx->stream), "H2D 3c pairs");
  if (rc) return rc;
  EriLaunch P = base_launch(p.tab);
  P.bra = p.dorb.sh;
  P.bexp = p.dorb.exps;
  P.bcoef = p.dorb.coefs;
  P.ket = p.daux.sh;
  P.kexp = p.daux.exps;
  P.kcoef = p.daux.coefs;
  P.mode = layout == RIJK_LAYOUT_PACKED ? 0 : 1;
  P.mu0 = mu0;
  P.mu1 = mu1;
  P.rowbase = layout == RIJK_LAYOUT_PACKED ? rowbase : mu0;
  P.n = p.orb.nbf;
  P.ld = ld;
  P.out = dout;
  return launch_classes(ctx, P, pl, static_cast<const int2*>(p.pairs_dev.p), p.kets,
                        static_cast<const int*>(p.kets_dev.p), launches);
}

}  // namespace
}  // namespace rijk

using namespace rijk;

RIJK_API int rijk_eri2c(rijk_ctx* ctx, const rijk_basis_t* aux, double* PQ) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!PQ) return set_err(ctx, RIJK_ERR_ARG, "rijk_eri2c: null output");
  cudaSetDevice(ctx->device);
  EriPlan p;
  int rc = make_plan(ctx, nullptr, aux, p);
  const long na = p.aux.nbf;
  DeviceBuf V;
  int launches = 0;
  if (!rc) rc = ensure(ctx, V, static_cast<size_t>(na) * na * sizeof(double), "(P|Q)");
  if (!rc) rc = eri2c_device(ctx, p, static_cast<double*>(V.p), na, &launches);
  if (!rc)
    rc = cuda_check(ctx, cudaMemcpy(PQ, V.p, static_cast<size_t>(na) * na * sizeof(double), cudaMemcpyDeviceToHost),
                    "D2H (P|Q)");
  release(V);
  release_plan(p);
  return rc;
}

RIJK_API int rijk_eri3c(rijk_ctx* ctx, const rijk_basis_t* orb, const rijk_basis_t* aux, int layout, double* I3) {
  if (!ctx) return RIJK_ERR_ARG;
  if (!I3 || !orb) return set_err(ctx, RIJK_ERR_ARG, "rijk_eri3c: null argument");
  if (layout != RIJK_LAYOUT_NOPT_FULL && layout != RIJK_LAYOUT_PACKED)
    return set_err(ctx, RIJK_ERR_ARG, "rijk_eri3c: unknown layout %d", layout);
  cudaSetDevice(ctx->device);
  EriPlan p;
  int rc = make_plan(ctx, orb, aux, p);
  if (rc) { release_plan(p); return rc; }
  const long n = p.orb.nbf, naux = p.aux.nbf;
  // rows per block: at most ~1 GiB of device output
  const double row_bytes = static_cast<double>(layout == RIJK_LAYOUT_PACKED ? n : n) * naux * 8.0;
  long rows = std::max<long>(1, std::min<long>(n, static_cast<long>(1073741824.0 / row_bytes)));
  auto first_row = [&](long mu) { return layout == RIJK_LAYOUT_PACKED ? mu * (mu + 1) / 2 : mu * n; };
  DeviceBuf out;
  int launches = 0;
  for (long mu0 = 0; mu0 < n && !rc; mu0 += rows) {
    const long mu1 = std::min(n, mu0 + rows);
    const long r0 = first_row(mu0), cnt = first_row(mu1) - r0;
    const size_t bytes = static_cast<size_t>(cnt) * naux * sizeof(double);
    if ((rc = ensure(ctx, out, bytes, "3c block"))) break;
    cudaMemsetAsync(out.p, 0, bytes, ctx->stream);
    rc = eri3c_rows(ctx, p, layout, mu0, mu1, r0, static_cast<double*>(out.p), naux, &launches);
    if (!rc) rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "three-centre integrals");
    if (!rc) rc = cuda_check(ctx, cudaMemcpy(I3 + r0 * naux, out.p, bytes, cudaMemcpyDeviceToHost), "D2H 3c block");
  }
  release(out);
  release_plan(p);
  return rc;
}

RIJK_API int rijk_set_basis(rijk_ctx* ctx, const rijk_basis_t* orb, const rijk_basis_t* aux, int metric_form, long q0,
                            long q1) {
  rijk::NvtxRange range("rijk_set_basis");
  if (!ctx) return RIJK_ERR_ARG;
  if (!orb) return set_err(ctx, RIJK_ERR_ARG, "rijk_set_basis: null orbital basis");
  cudaSetDevice(ctx->device);
  EriPlan p;
  int rc = make_plan(ctx, orb, aux, p);
  if (rc) { release_plan(p); return rc; }
  const long naux = p.aux.nbf, n = p.orb.nbf;
  int launches = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  DeviceBuf V;
  float ms_ints = 0.f;
  rc = ensure(ctx, V, static_cast<size_t>(naux) * naux * sizeof(double), "(P|Q)");
  if (!rc) {
    cudaEventRecord(e0, ctx->stream);
    rc = eri2c_device(ctx, p, static_cast<double*>(V.p), naux, &launches);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    ms_ints += elapsed(e0, e1);
  }
  if (!rc) rc = set_metric_impl(ctx, static_cast<const double*>(V.p), cudaMemcpyDeviceToDevice, naux, metric_form);
  release(V);
  if (!rc && q1 > 0) rc = rijk_set_aux_range(ctx, q0, q1);
  if (!rc) {
    rc = set_3c_impl(ctx, n, naux, RIJK_LAYOUT_PACKED,
                     [&](long mu0, long mu1, long first, long, double* raw, long ldr) {
                       cudaEventRecord(e0, ctx->stream);
                       int r = eri3c_rows(ctx, p, RIJK_LAYOUT_PACKED, mu0, mu1, first, raw, ldr, &launches);
                       cudaEventRecord(e1, ctx->stream);
                       if (!r) r = cuda_check(ctx, cudaEventSynchronize(e1), "three-centre integrals");
                       ms_ints += elapsed(e0, e1);
                       return r;
                     });
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  release_plan(p);
  if (!rc) {
    ctx->stats.ms_setup_ints = ms_ints;
    ctx->stats.kernels_setup_ints = launches;
  }
  return rc;
}
