/*
 * gto_ints.h — host-side Gaussian integral engine (C ABI).
 *
 * Produces the inputs of the RI-JK Fock build: the orbital one-electron matrices, the
 * two-centre metric (P|Q) and the three-centre integrals (mu nu|P).  In the reference
 * these come from libint2 on the host:
 *   - (P|Q):      RI_V_calc            (src/libint_link.cpp:2049-2107), Engine(coulomb, xs_xs)
 *   - (mu nu|P):  calc_2el_AO_INTS_RI  (src/libint_link.cpp:2261-2350), Engine(coulomb, xs_xx)
 *   - S, T, V:    gen_1el_data         (src/molecule.cpp:3757-3800)
 * This engine is our own McMurchie-Davidson implementation (Hermite expansion, Boys
 * function from its series definition).  Functions are normalised like libint's
 * (primitive x^l normalisation, then contraction renormalised to unit norm); spherical
 * shells are real solid harmonics ordered m = -l..l.
 *
 * Every function returns 0 on success and a negative GTO_ERR_* code on failure.
 */
#ifndef GTO_INTS_H
#define GTO_INTS_H

#ifdef __cplusplus
extern "C" {
#endif

#define GTO_OK 0
#define GTO_ERR_ARG -1
#define GTO_ERR_LMAX -2
#define GTO_ERR_ALLOC -3

/* Layouts of the three-centre output. */
#define GTO_3C_NOPT_FULL 0   /* out[(mu*n + nu)*naux + P], full square: RI_AA of src/RI.cpp:69-71 */
#define GTO_3C_PACKED 1      /* out[(mu*(mu+1)/2 + nu)*naux + P], mu >= nu */

typedef struct gto_basis gto_basis;

/* Build a basis from flat shell arrays.  Shell s has angular momentum l[s], pure[s]
 * (1 = spherical), nprim[s] primitives whose exponents/library coefficients are the next
 * nprim[s] entries of exps/coefs, and centre xyz[3*s..3*s+2] in bohr. */
int gto_basis_create(gto_basis** out, int nshell, const int* l, const int* pure, const int* nprim,
                     const double* xyz, const double* exps, const double* coefs);
void gto_basis_destroy(gto_basis* b);
int gto_basis_nbf(const gto_basis* b);
int gto_basis_max_l(const gto_basis* b);
/* Normalised contraction coefficients as used in the integrals (same order as coefs). */
int gto_basis_norm_coefs(const gto_basis* b, double* out);
/* First basis-function index of every shell. */
int gto_basis_shell_offsets(const gto_basis* b, int* out);

/* n x n row-major one-electron matrices. */
int gto_overlap(const gto_basis* b, double* S);
int gto_kinetic(const gto_basis* b, double* T);
int gto_nuclear(const gto_basis* b, int natom, const double* Z, const double* xyz, double* V);

/* naux x naux two-centre Coulomb metric (P|Q). */
int gto_coulomb_2c(const gto_basis* aux, double* V);

/* Three-centre Coulomb integrals (mu nu|P) in one of the GTO_3C_* layouts. */
int gto_coulomb_3c(const gto_basis* orb, const gto_basis* aux, int layout, double* out);

/* Density of one atom (nuclear charge Z at xyz) for a superposition-of-atomic-densities start:
 * spherically averaged RHF with fractional occupations in the atom's orbital basis `orb`,
 * RI-JK in its fitting basis `aux`.  D (n x n) uses the reference's normalisation (trace of
 * D S = Z / 2); rows (at most n x n) receive nrows factor rows sqrt(f_k) v_k with
 * D = sum_k rows_k^T rows_k, usable as MO rows of a Fock build (the reference's SAD start,
 * src/sad_guess.cpp:165-215). */
int gto_atomic_density(const gto_basis* orb, const gto_basis* aux, double Z, const double* xyz, double* D,
                       double* rows, int* nrows);

/* The (2l+1) x ncart(l) row-major matrix C of the spherical functions of angular momentum l (0 .. 4)
 * in terms of the Cartesian ones of the same shell, Y_m = sum_c C[m][c] phi_c, with both normalised
 * as in the integrals (the map a Cartesian orbital basis is projected with, as the reference's
 * T_D5, src/molecule.cpp:4551-4680). */
int gto_cart_to_sph(int l, double* out);

/* Boys function F_m(T), m = 0..mmax (test hook). */
int gto_boys(int mmax, double T, double* F);

/* Threads used by the integral loops (0 = OpenMP default). */
void gto_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif
