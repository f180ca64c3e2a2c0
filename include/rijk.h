/*
 * rijk.h — C ABI of the B200 RI-JK Fock build (librijk.so).
 *
 * Drop-in for the reference's RI Fock-build routine and its set-up:
 *   rijk_set_metric   replaces RI_V_calc + S05_calc        src/libint_link.cpp:2049-2107, src/matr.cpp:372-401
 *   rijk_set_3c       replaces the RI_AA set-up of gen_RI_AA / regen_RI_AA
 *                                                          src/RI.cpp:34-101 (consumer of calc_2el_AO_INTS_RI,
 *                                                          src/libint_link.cpp:2261-2350)
 *   rijk_begin_3c, rijk_add_3c_block  the same, fed block by block from that shell loop
 *   rijk_set_basis    replaces gen_RI_AA whole, integrals included  src/RI.cpp:34-79
 *   rijk_eri2c        replaces RI_V_calc                            src/libint_link.cpp:2049-2107
 *   rijk_eri3c        replaces calc_2el_AO_INTS_RI                  src/libint_link.cpp:2261-2350
 *   rijk_mo_calc      replaces RI_data::MO_calc                     src/RI.cpp:469-587
 *   rijk_mo_ints_aaag replaces calc_2el_MO_INTS_AAAG_RI             src/RI.cpp:294-346
 *   rijk_soscf_hess_ints replaces calc_SOSCF_hess_INTS_RI           src/RI.cpp:348-450
 *   rijk_fock         replaces DM_to_F_transform_RI        src/RI.cpp:115-176 (declared include/RI.h)
 *                     and the J/K tail of calc_2el_MO_INTS_RI  src/RI.cpp:235-287
 *   rijk_fock_energy  F = H + (2J - K) c and the RHF energy   src/molecule.cpp:4407-4438, src/SCF.cpp:134
 *   rijk_scf          the RHF loop around it (DIIS variant)   src/SCF.cpp:78-223
 *   rijk_grad         adjoint of the Fock build (no reference counterpart: the reference
 *                     differentiates by finite differences, src/QM_calc.cpp:142)
 *
 * Conventions are the reference's: all matrices are host (or, for *_device calls, device)
 * double arrays in row-major order; D is normalised to 1 (D = sum_i C_i C_i^T over occupied
 * rows of MO, src/SCF.cpp:63-73) and is used as given (not symmetrised); MO holds one
 * orbital per row (n_c rows of n_ao); K is unscaled; J and K are full n x n.
 *
 * One context drives one GPU.  A context is not thread-safe.  Every function returns
 * RIJK_OK (0) or a negative RIJK_ERR_* code; rijk_last_error() gives the message.  Nothing
 * in the library calls exit() or aborts.
 *
 * With the environment variable RIJK_LOG set to a file name, every Fock build (rijk_fock; a
 * rijk_fock_device build at its rijk_sync) and every rijk_scf appends one JSON line to that file:
 * sizes, precision, device times, algorithmic FLOPs and bytes and their rates.  The main calls
 * are NVTX ranges of their own names for timeline tools.
 */
#ifndef RIJK_H
#define RIJK_H

#ifdef __cplusplus
extern "C" {
#endif

#define RIJK_OK 0
#define RIJK_ERR_ARG -1      /* null pointer, bad size or bad enum value                      */
#define RIJK_ERR_STATE -2    /* call order (e.g. rijk_fock before rijk_set_3c)                */
#define RIJK_ERR_CUDA -3     /* CUDA runtime error                                             */
#define RIJK_ERR_ALLOC -4    /* device memory exhausted                                        */
#define RIJK_ERR_SOLVER -5   /* metric factorisation failed (e.g. not positive definite)       */
#define RIJK_ERR_TIMEOUT -6  /* a bounded device-side wait ran out                             */
#define RIJK_ERR_NUMERIC -7  /* NaN or Inf met in an input or a result                        */
#define RIJK_ERR_CONVERGE -8 /* SCF did not converge within the iteration limit                */
#define RIJK_ERR_REDUCE -9   /* the caller's J/K reduction (rijk_scf_opts_t.reduce_jk) failed    */

/* Metric forms.  J and K agree in exact arithmetic (L^-T L^-1 = V^-1 = V^-1/2 V^-1/2). */
#define RIJK_METRIC_INVSQRT 0  /* V^-1/2 by eigendecomposition, eigenvalues <= 0 dropped (S05_calc) */
#define RIJK_METRIC_CHOLESKY 1 /* L^-1 with V = L L^T                                               */

/* Layouts of the three-centre integrals handed to rijk_set_3c. */
#define RIJK_LAYOUT_NOPT_FULL 0 /* I3[(mu*n + nu)*naux + P], full square: the reference's RI_AA */
#define RIJK_LAYOUT_PACKED 1    /* I3[(mu*(mu+1)/2 + nu)*naux + P], mu >= nu                    */

/* Arithmetic of one Fock build. */
#define RIJK_PREC_FP64 0  /* FP64 throughout: the drop-in form                                   */
#define RIJK_PREC_MIXED 1 /* exchange half-transform and K on tcgen05 tensor cores with split-BF16
                             (3-term) operands and FP32 accumulation; Coulomb in FP64          */
#define RIJK_PREC_FP64_TC 2 /* FP64 results, with K = X^T X on tcgen05 tensor cores: X^T split
                             into 8 int8 digit planes per row and split-K part (a power-of-two
                             exponent each), 36 exact s32 digit products, FP64 scaling and sums
                             (the Ozaki splitting scheme); J and the half-transform as FP64   */

typedef struct rijk_ctx rijk_ctx;

typedef struct {
  double ms_setup_metric; /* last rijk_set_metric, device time                             */
  double ms_setup_3c;     /* last rijk_set_3c, device time (metric contraction included)   */
  double ms_last_fock;    /* last Fock build, device time                                   */
  double ms_coulomb;      /* from its start until J is complete (the w and J passes)        */
  double ms_exchange;     /* from then until its end.  FP64 and FP64_TC builds run the
                             Coulomb pair beside the half-transform, so there the exchange
                             starts before J is complete; mixed builds run them in turn    */
  double flops_last_fock; /* algorithmic FLOPs of the last build                            */
  double bytes_last_fock; /* algorithmic HBM bytes of the last build                        */
  long n, naux, npad, ntile;
  long bytes_b;           /* device bytes of the fitted tensor B                            */
  long bytes_b_mixed;     /* device bytes of its split-BF16 copy (0 until first mixed build) */
  int kernels_last_fock;  /* kernels launched by the last build                             */
  int profiled_stages;    /* number of valid entries of ms_stage (0 unless profiling is on)  */
  double ms_stage[12];    /* device time of each kernel of the last build, in launch order   */
  char stage_names[12][24];
  double ms_setup_ints;   /* last rijk_set_basis: device time of the integral kernels          */
  int kernels_setup_ints; /* integral kernels it launched                                    */
  long q0, nq;            /* aux functions [q0, q0 + nq) held (all of them unless sliced)      */
  long grad_qchunk;       /* aux functions per chunk of the last rijk_grad (naux: one chunk)    */
  /* Device time of the stages of the last rijk_grad, summed over its aux chunks (with profiling
   * on): [0] the FP64 Fock build, energy and dE/dC, [1] X^Q recomputed in tiles (0 unless chunked),
   * [2] Y^Q and T^Q, [3] Gamma, [4] dE/d(P|mu nu) = M^T Gamma, [5] G = Gamma B, [6] -M^T G M.      */
  double ms_grad_stage[7];
  double ms_grad_total;   /* device time of rijk_grad before its host copies (profiling on)     */
} rijk_stats_t;

int rijk_create(rijk_ctx** ctx, int device);
int rijk_destroy(rijk_ctx* ctx);
/* Run on the caller's CUDA stream (a cudaStream_t) instead of the context's own.  An FP64 or FP64_TC
 * build also runs its Coulomb passes on a second stream the context owns: that stream waits on the
 * caller's stream at the start of the build, and the caller's stream waits on it before the build's
 * end, so work queued after the build on the caller's stream sees J and K. */
int rijk_set_stream(rijk_ctx* ctx, void* stream);
int rijk_last_error(const rijk_ctx* ctx, char* buf, int len);
/* Record a CUDA event around every kernel of a Fock build (for per-kernel timing); the kernels then
 * run one after another on one stream. */
int rijk_set_profiling(rijk_ctx* ctx, int on);
int rijk_get_stats(const rijk_ctx* ctx, rijk_stats_t* out);

/* (P|Q), naux x naux host array.  Factorises the metric on the GPU in FP64. */
int rijk_set_metric(rijk_ctx* ctx, const double* PQ, long naux, int metric_form);

/* Hold only the aux functions [q0, q1) of the fitted tensor (call after rijk_set_metric,
 * before rijk_set_3c).  J, K and rijk_mo_ints are sums over the aux index, so a Fock build of
 * such a context returns the slice's partial J and K; contexts on several GPUs that cover
 * [0, naux) give the full J and K after one all-reduce (sum).  rijk_scf runs on a slice with a
 * reduce_jk callback in its options (the sum over the ranks after every build); rijk_grad needs
 * the whole range. */
int rijk_set_aux_range(rijk_ctx* ctx, long q0, long q1);

/* Three-centre integrals (host array, layout RIJK_LAYOUT_*).  Forms the fitted tensor
 * B^Q_{mu nu} = sum_P M_QP (P|mu nu) on the GPU, stored packed (mu >= nu) in HBM. */
int rijk_set_3c(rijk_ctx* ctx, const double* I3, long n_ao, long naux, int layout);

/* The same fitted tensor from three-centre integrals handed over in blocks of orbital rows, for
 * callers whose (mu nu|P) does not fit in host memory at once (the reference's RI_AA is n^2 naux
 * doubles, 123 GB at (H2O)32 cc-pVTZ; it is filled by calc_2el_AO_INTS_RI's shell loop,
 * src/libint_link.cpp:2261-2350).  rijk_begin_3c starts one (after rijk_set_metric and any
 * rijk_set_aux_range); rijk_add_3c_block then takes the rows mu in [mu0, mu1) of the layout, the
 * ranges consecutive from mu0 = 0 and each block usable again by the caller when the call returns:
 *   RIJK_LAYOUT_NOPT_FULL  block[((mu - mu0) n_ao + nu) naux + P]
 *   RIJK_LAYOUT_PACKED     block[(mu (mu + 1) / 2 + nu - mu0 (mu0 + 1) / 2) naux + P], nu <= mu
 * Whole 64-row tile rows are contracted with the metric factor as they complete; the block that ends
 * at n_ao completes the fitted tensor, bit-identical to rijk_set_3c's.  An error, rijk_set_metric,
 * rijk_set_aux_range or rijk_set_3c abandons the stream (the context then has no fitted tensor). */
int rijk_begin_3c(rijk_ctx* ctx, long n_ao, long naux, int layout);
int rijk_add_3c_block(rijk_ctx* ctx, long mu0, long mu1, const double* block);

/* A contracted Gaussian basis as shell arrays, in the order of a basis-set file.  Coefficients
 * are as printed there; the library normalises them as libint does (x^l primitive
 * normalisation, unit-norm contraction).  Spherical shells are real solid harmonics in the
 * order m = -l .. l; Cartesian shells list x^a y^b z^c with a, then b, descending. */
typedef struct {
  int nshell;
  const int* l;         /* angular momentum per shell, 0 .. 4                        */
  const int* pure;      /* 1: spherical (2l+1 functions), 0: Cartesian               */
  const int* nprim;     /* primitives per shell                                      */
  const double* xyz;    /* shell centres in bohr, 3 per shell                        */
  const double* exps;   /* primitive exponents, all shells concatenated              */
  const double* coefs;  /* contraction coefficients, same order                      */
} rijk_basis_t;

/* (P|Q) of the aux basis computed on the GPU into a host naux x naux array. */
int rijk_eri2c(rijk_ctx* ctx, const rijk_basis_t* aux, double* PQ);

/* (mu nu|P) computed on the GPU into a host array in layout RIJK_LAYOUT_NOPT_FULL
 * (n^2 naux doubles) or RIJK_LAYOUT_PACKED (n(n+1)/2 naux doubles). */
int rijk_eri3c(rijk_ctx* ctx, const rijk_basis_t* orb, const rijk_basis_t* aux, int layout, double* I3);

/* gen_RI_AA on the GPU: (P|Q), the metric factor (RIJK_METRIC_*), (mu nu|P) and the fitted
 * tensor, with no integrals on the host and no host-to-device copy of them.  q1 > 0 keeps
 * only the aux functions [q0, q1) (as rijk_set_aux_range); q1 = 0 keeps all of them.
 * Equivalent to rijk_set_metric + rijk_set_aux_range + rijk_set_3c on the same integrals. */
int rijk_set_basis(rijk_ctx* ctx, const rijk_basis_t* orb, const rijk_basis_t* aux, int metric_form, long q0,
                   long q1);

/* The fitted tensor on disk (no reference counterpart: NOPT rebuilds RI_AA in every run).
 * rijk_save writes the metric factor and B (or the aux slice held) of a set-up context to a file;
 * rijk_load reads one into any context, which can then run Fock builds, rijk_grad and the MO
 * tensor calls without integrals.  The file carries a checksum: a damaged or truncated file gives
 * RIJK_ERR_ARG and leaves the context unchanged. */
int rijk_save(rijk_ctx* ctx, const char* path);
int rijk_load(rijk_ctx* ctx, const char* path);

/* Drop-in for DM_to_F_transform_RI(J, K, DM, MO, n_c, n_ao): host pointers, synchronous. */
int rijk_fock(rijk_ctx* ctx, const double* DM, const double* MO, long n_c, double* J, double* K, int precision);

/* Same on device pointers, asynchronous on the context's stream. */
int rijk_fock_device(rijk_ctx* ctx, const double* dDM, const double* dMO, long n_c, double* dJ, double* dK,
                     int precision);

/* Wait for the context's stream and report any error a kernel raised (RIJK_ERR_TIMEOUT when
 * a bounded device-side wait ran out); also refreshes the timing statistics. */
int rijk_sync(rijk_ctx* ctx);

/* Self-test of the bounded-wait error path (no reference counterpart).  Launches one warp on the
 * context's stream that allocates TMEM as the tcgen05 kernels do, waits on an mbarrier nothing ever
 * arrives on until `cycles` SM clock cycles (1000 .. 2e9) have passed, then raises the timeout bit,
 * frees the TMEM and returns.  Asynchronous; the next rijk_sync returns RIJK_ERR_TIMEOUT, and the
 * context stays usable. */
int rijk_selftest_wait_timeout(rijk_ctx* ctx, long long cycles);

/* Self-test of the allocation failure paths (no reference counterpart): after `after` more device
 * allocations of this context succeed, the next one fails with RIJK_ERR_ALLOC, as an exhausted
 * cudaMalloc would, and every later one too, until the hook is turned off with after < 0.  Only
 * allocations the library would really make count (a buffer already large enough is reused).  A
 * failed call leaves the context usable once allocations succeed again. */
int rijk_selftest_alloc_failure(rijk_ctx* ctx, long after);

/* Size of the fixed device scratch used by rijk_coulomb_noalloc (per GPU, held until exit). */
#define RIJK_NOALLOC_SCRATCH_BYTES (32L * 1024 * 1024)

/* No counterpart in the reference.  The Coulomb matrix J of rijk_fock_device, computed
 * without any device allocation.  It is for callers that cannot let the library call
 * cudaMalloc while their iterations run, for example a program that hands all of its GPU
 * memory to its own pool at start-up, or one that must not add an allocation (and the
 * device synchronisation it may bring) inside its loop.  The fitted tensor set up by
 * rijk_set_3c is the input; dDM (n x n) and dJ (n x n) are device pointers of the caller;
 * the call is asynchronous on the context's stream.  Working space comes from a fixed
 * RIJK_NOALLOC_SCRATCH_BYTES device array inside the library:
 *  - sizes that need more return RIJK_ERR_ARG (about n_ao <= 1980 fits);
 *  - all calls on one GPU share it, so calls that overlap on the GPU race;
 *  - rijk_create looks up the array's address on its device, which is when the array is
 *    allocated there (so create the context before handing the GPU's memory to a pool).
 * After rijk_set_aux_range the result is that slice's partial J, as with rijk_fock_device.
 * The call makes no cudaMalloc, cudaFree or allocating library call. */
int rijk_coulomb_noalloc(rijk_ctx* ctx, const double* dDM, double* dJ);

/* Options of rijk_scf (zero-initialised fields take the defaults given). */
typedef struct {
  int max_iter;           /* default 100                                                        */
  double conv_dm_rms;     /* converged when RMS(D_new - D) falls below this; default 1e-10     */
  int precision;          /* RIJK_PREC_FP64 or RIJK_PREC_FP64_TC (FP64 results throughout), or
                             RIJK_PREC_MIXED: mixed builds until the DIIS error falls below
                             switch_diis_err, RIJK_PREC_FP64 builds after that                */
  double switch_diis_err; /* default 1e-5; the switch also happens when the mixed-phase error has
                             not improved for 5 iterations or after max_iter / 2 mixed iterations */
  int diis_size;          /* default 8                                                          */
  int diis_keep_on_switch; /* 0 (default): restart DIIS at the switch to FP64 (measured faster);
                             1: keep the mixed-phase vectors until the history rolls over       */
  double lindep;          /* overlap eigenvalues below this are dropped; default 1e-10           */
  /* Optional start (host arrays): a density D0 (n x n) with factor rows R (guess_nrows x n),
   * D0 = R^T R, e.g. a superposition of atomic densities; its FP64 Fock build replaces the
   * core-Hamiltonian start (the reference's SAD start, src/sad_guess.cpp:199-201). */
  const double* guess_dm;
  const double* guess_rows;
  long guess_nrows;
  /* The converger (appended fields; zero = defaults). */
  int converger;          /* RIJK_CONV_DIIS (default) or RIJK_CONV_SOSCF, the reference's RHF step:
                             L-BFGS on the occupied-virtual rotations with the diagonal Hessian
                             4 (e_a - e_i), rotation I + X - X^T orthonormalised by Gram-Schmidt
                             (src/SCF.cpp:125-174, src/converger_2_1.cpp:55-125, src/l-bfgs_2_1.cpp);
                             or RIJK_CONV_DIIS_SOSCF: DIIS while the builds are mixed, the SOSCF
                             step (and its convergence test) from the switch to FP64 on, entered
                             as the reference enters it: one plain diagonalisation first         */
  double conv_grad;       /* SOSCF: converged when max |4 F_ai| < conv_grad; default 1e-7          */
  double conv_energy;     /* SOSCF: or when |E - E_previous| < conv_energy; default 1e-10          */
  int lbfgs_vectors;      /* SOSCF: curvature pairs kept, 1 .. 32; default min(n_mo, 20, max_iter)  */
  int density_by_eigenvectors; /* DIIS: 0 (default) takes each new density's occupied space from
                             trace-correcting purification of X^T F X (products only) and one
                             subspace step from the previous orbitals, falling back to the
                             eigensolver when either does not converge; 1 diagonalises every
                             step, as the reference (src/SCF.cpp:160-166).  Same densities to
                             rounding                                                        */
  int fp64_phase_precision; /* 0 (default): RIJK_PREC_FP64 builds after a mixed phase (and for a
                             closing build); RIJK_PREC_FP64_TC: the same FP64-accurate results
                             with K on the int8 tensor cores                                    */
  /* Optional orbital-space projector (appended fields; NULL = the whole AO space): an n_ao x
   * n_proj row-major host array T whose columns span the space the orbitals are confined to, as
   * the reference's Cartesian->spherical T_D5 (n_ao x n_ao_d5, make_D5_matr, src/molecule.cpp:4551-
   * 4680).  The orthogonaliser then comes from T^T S T (eigenvalues below lindep dropped), so every
   * diagonalisation runs in the projected space as diag_X_AO_in_MO does with D5 = 1
   * (src/molecule.cpp:4004-4050), while the Fock builds stay in the n_ao Cartesian AO basis.  MO
   * receives n_proj (less dropped) orbitals as rows of n_ao coefficients, the rest zero.        */
  const double* ao_projector;
  long n_proj;            /* 1 .. n_ao                                                          */
  /* Aux-sharded SCF (appended fields; NULL = one context holds every aux function).  Each rank's
   * context holds one slice of the aux functions (rijk_set_aux_range), so its Fock builds give
   * partial J and K.  rijk_scf calls reduce_jk(jk, count, stream, reduce_user) after every build,
   * with jk the device array [J | K] (count = 2 n_ao^2 doubles) written by work on `stream` (the
   * context's cudaStream_t).  The callback replaces jk in place by its sum over the ranks, either
   * enqueued on `stream` (an NCCL all-reduce) or complete when it returns (a host reduction after
   * synchronising the stream), and returns 0; any other value ends rijk_scf with RIJK_ERR_REDUCE.
   * Every rank calls rijk_scf with the same arguments.  The steps after the reduction use no
   * floating-point atomics, so equal J and K give equal decisions (DIIS, switch, convergence) on
   * every rank and the ranks reach the reduction the same number of times.  A context holding an
   * aux range needs reduce_jk; one holding every aux function calls it too when it is given (a
   * one-rank group).                                                                               */
  int (*reduce_jk)(double* jk, long count, void* stream, void* user);
  void* reduce_user;
} rijk_scf_opts_t;

#define RIJK_CONV_DIIS 0
#define RIJK_CONV_SOSCF 1
#define RIJK_CONV_DIIS_SOSCF 2

typedef struct {
  double energy;          /* E = tr(F D) + tr(H D) + e_nuc of the last FP64 Fock build, as the
                             reference reports it (src/SCF.cpp:134-156); a run that ends in the
                             mixed phase gets one more FP64 build for it                        */
  double dm_rms;          /* last RMS density change                                          */
  double diis_err;        /* last max |X^T (F D S - S D F) X|; in SOSCF steps, max |4 F_ai|     */
  int iterations;         /* Fock builds                                                       */
  int iterations_mixed;   /* of which in the mixed form                                        */
  int converged;
  int nmo;                /* orbitals kept after removing linear dependence                    */
  double ms_fock;         /* device time in Fock builds                                        */
  double ms_total;        /* wall time of rijk_scf                                             */
  double ms_build_phase;  /* wall time of the Fock-build + DIIS-error phase of the iterations    */
  double ms_diis_phase;   /* wall time of the Pulay extrapolation phase                         */
  double ms_diag_phase;   /* wall time of diagonalisation + new density                        */
  int history_len;        /* entries of the per-iteration trace below (first 128 iterations)   */
  double history_energy[128];
  double history_diis_err[128];  /* per build: the DIIS error, or max |4 F_ai| in SOSCF steps      */
  int history_mixed[128]; /* 1 where the iteration used the mixed form                          */
  double ms_setup_phase;  /* wall time before the first iteration: uploads, overlap
                             eigendecomposition, the guess's Fock build and diagonalisation     */
  double ms_final_phase;  /* wall time after the last iteration: the closing FP64 build (if any)
                             and the orbitals' diagonalisation and download                     */
  int purified;           /* DIIS steps whose occupied orbitals came from purification          */
} rijk_scf_result_t;

/* Restricted Hartree-Fock on the GPU around the Fock build: the reference's RHF loop
 * (src/SCF.cpp:78-223).  The converger is Pulay DIIS on F D S - S D F (default) or, with
 * opts->converger = RIJK_CONV_SOSCF, the reference's own SOSCF/L-BFGS orbital-rotation step and
 * convergence test (max |4 F_ai| or |dE|), or DIIS then SOSCF (RIJK_CONV_DIIS_SOSCF); all reach
 * the same energy.  MO holds the eigenvectors of the last FP64 Fock matrix (the reference's
 * closing diagonalisation, src/SCF.cpp:178).  H and S are n x n host
 * arrays; n_c occupied orbitals; the core-Hamiltonian guess (or opts' guess) starts it.
 * Diagonalisation, the converger's algebra and the energy are FP64 on the device.  MO (optional, n x n host) receives the orbitals, one per row, as the
 * reference's MO_VEC; E as in src/SCF.cpp:134.  The call's device work buffers, about
 * (16 + 2 diis_size) n^2 doubles, stay with the context for the next call until rijk_destroy. */
int rijk_scf(rijk_ctx* ctx, const double* H, const double* S, long n_c, double e_nuc, const rijk_scf_opts_t* opts,
             double* MO, rijk_scf_result_t* result);

/* Drop-in for calc_2el_MO_INTS_RI(n_ao, DM_D, J, K, MO_INTS, MO_VEC, MO_VEC1, MO_VEC2, n_c, n_a, t)
 * (src/RI.cpp:178-292; the CASSCF call at src/CAS.cpp:461): the active-space integrals
 *   MO_INTS[(b n_a + a) n_a^2 + d n_a + c] = sum_Q (C1 B^Q C2^T)_ab (C1 B^Q C2^T)_cd
 * with C1 = MO_VEC1, C2 = MO_VEC2 (n_a orbitals as rows, or as columns of an n_ao x n_a array
 * when t != 0), then, unless J or K is NULL, the core J and K of DM_D and the first n_c rows
 * of MO_VEC (as rijk_fock).  Host pointers; synchronous; FP64. */
int rijk_mo_ints(rijk_ctx* ctx, const double* DM_D, double* J, double* K, double* MO_INTS, const double* MO_VEC,
                 const double* MO_VEC1, const double* MO_VEC2, long n_c, long n_a, long t);

/* ---- MO-basis fitted tensors (post-SCF: CASSCF, perturbation theory) ----
 * (p a|Q) below is sum_{mu nu} C1[p][mu] C2[a][nu] B^Q_{mu nu}.  With RIJK_METRIC_INVSQRT it is the
 * reference's tensor; with the Cholesky form it differs by an orthogonal rotation of Q, and
 * every contraction over Q is the same.  Orbitals are rows of n_ao coefficients. */

/* out[(p*n2 + a)*naux + Q] for the rows of C1 (n1 x n_ao) and C2 (n2 x n_ao). */
int rijk_mo_tensor(rijk_ctx* ctx, const double* C1, long n1, const double* C2, long n2, double* out);

/* RI_data::MO_calc (src/RI.cpp:469-587): VEC holds n_cor core, n_act active and n_vac virtual
 * rows.  CC[(i n_cor + j)], VC[(v n_cor + j)], AA[(t n_act + u)], CA[(i n_act + u)] and
 * VA[(v n_act + u)], each times naux; any output may be NULL. */
int rijk_mo_calc(rijk_ctx* ctx, const double* VEC, long n_cor, long n_act, long n_vac, double* CC, double* VC,
                 double* AA, double* CA, double* VA);

/* calc_2el_MO_INTS_AAAG_RI (src/RI.cpp:294-346): MO_INTS[((t n_a + u) n_a + v) n_mo + x] = (tu|vx)
 * for active t, u, v (rows n_c .. n_c+n_a-1 of MO_VEC) and all n_mo rows x (the reference uses
 * n_mo = n_ao). */
int rijk_mo_ints_aaag(rijk_ctx* ctx, double* MO_INTS, const double* MO_VEC, long n_c, long n_a, long n_mo);

/* calc_SOSCF_hess_INTS_RI (src/RI.cpp:348-450): aa_J[(p n_a + t) n_a + u] = (pp|tu) and
 * aa_K[(p n_a + t) n_a + u] = (pt|pu) for all n_mo orbital rows p.  (The reference's cv_J / cv_K
 * arguments are never written by it and have no counterpart here.) */
int rijk_soscf_hess_ints(rijk_ctx* ctx, double* aa_J, double* aa_K, const double* MO_VEC, long n_c, long n_a,
                         long n_mo);

/* Aux functions per chunk of rijk_grad's Gamma stage (0, the default: all of them when HBM holds
 * Gamma for every aux function, else as many as it holds).  Below naux, each chunk's
 * half-transformed tensor is recomputed in tiles instead of read from the stored one. */
int rijk_set_grad_chunk(rijk_ctx* ctx, long q_per_chunk);

/* Adjoint of the Fock build (no reference counterpart; the reference differentiates by finite
 * differences, src/QM_calc.cpp:142).  For the orbitals MO (n_c rows of n, host) and D = C^T C:
 *   *E    = tr(F D) + tr(H D) + e_nuc with F = H + 2J - K (FP64 build; src/SCF.cpp:134)
 *   dEdC  = dE/dMO, n_c x n, = 4 C F (the orbital gradient)
 *   dEdI3 (optional) = dE/d(P|mu nu) for the packed pairs mu >= nu, laid out as
 *           RIJK_LAYOUT_PACKED ([pair][P]); a pair mu != nu stands for both (mu nu) and (nu mu)
 *   dEdPQ (optional) = dE/d(P|Q), naux x naux, entries V_PQ and V_QP taken as independent
 * Host pointers; synchronous. */
int rijk_grad(rijk_ctx* ctx, const double* MO, long n_c, const double* H, double e_nuc, double* E, double* dEdC,
              double* dEdI3, double* dEdPQ);

/* F = H + (2J - K) c (mc = 0/2) or H + (J - K) 2c (mc = 1), src/molecule.cpp:4418-4430, and
 * E = tr(F D) + tr(H D) + e_nuc (src/SCF.cpp:134); host pointers; F or E may be NULL. */
int rijk_fock_energy(rijk_ctx* ctx, const double* H, const double* DM, const double* J, const double* K, double c,
                     int mc, double e_nuc, double* F, double* E);

#ifdef __cplusplus
}
#endif
#endif
