"""Python binding of librijk.so (include/rijk.h), the B200 RI-JK Fock build.

The methods mirror the reference's RI interface (include/RI.h of the reference):

  FockBuilder.set_metric          RI_V_calc + S05_calc        src/libint_link.cpp:2049, src/matr.cpp:372
  FockBuilder.set_3c              RI_AA set-up of gen_RI_AA   src/RI.cpp:34-79
  FockBuilder.set_basis           gen_RI_AA with the integrals computed on the GPU
  FockBuilder.eri2c / eri3c       RI_V_calc / calc_2el_AO_INTS_RI   src/libint_link.cpp:2049-2107, :2261-2350
  FockBuilder.dm_to_f_transform_ri  DM_to_F_transform_RI      src/RI.cpp:115-176
  FockBuilder.calc_f_ao           F and E of calc_F_AO / RHF  src/molecule.cpp:4407-4438, src/SCF.cpp:134

Errors raise RijkError carrying the library's status code and message; there is no
fallback path: if librijk.so is missing the import of this module's functions fails.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OK = 0
ERR_ARG, ERR_STATE, ERR_CUDA, ERR_ALLOC, ERR_SOLVER, ERR_TIMEOUT, ERR_NUMERIC, ERR_CONVERGE = -1, -2, -3, -4, -5, -6, -7, -8
ERR_REDUCE = -9
METRIC_INVSQRT, METRIC_CHOLESKY = 0, 1
LAYOUT_NOPT_FULL, LAYOUT_PACKED = 0, 1
PREC_FP64, PREC_MIXED, PREC_FP64_TC = 0, 1, 2
CONV_DIIS, CONV_SOSCF, CONV_DIIS_SOSCF = 0, 1, 2

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


GRAD_STAGES = ("fock_energy_dEdC", "x_recompute", "y_t", "gamma", "d3c_M_gamma", "g_gamma_B", "dV_MtGM")


class Stats(ctypes.Structure):
    _fields_ = [("ms_setup_metric", ctypes.c_double), ("ms_setup_3c", ctypes.c_double),
                ("ms_last_fock", ctypes.c_double), ("ms_coulomb", ctypes.c_double),
                ("ms_exchange", ctypes.c_double), ("flops_last_fock", ctypes.c_double),
                ("bytes_last_fock", ctypes.c_double), ("n", ctypes.c_long), ("naux", ctypes.c_long),
                ("npad", ctypes.c_long), ("ntile", ctypes.c_long), ("bytes_b", ctypes.c_long),
                ("bytes_b_mixed", ctypes.c_long), ("kernels_last_fock", ctypes.c_int),
                ("profiled_stages", ctypes.c_int), ("ms_stage", ctypes.c_double * 12),
                ("stage_names", (ctypes.c_char * 24) * 12), ("ms_setup_ints", ctypes.c_double),
                ("kernels_setup_ints", ctypes.c_int), ("q0", ctypes.c_long), ("nq", ctypes.c_long),
                ("grad_qchunk", ctypes.c_long), ("ms_grad_stage", ctypes.c_double * 7),
                ("ms_grad_total", ctypes.c_double)]


class BasisT(ctypes.Structure):
    """rijk_basis_t: a contracted basis as shell arrays."""
    _fields_ = [("nshell", ctypes.c_int), ("l", ctypes.POINTER(ctypes.c_int)), ("pure", ctypes.POINTER(ctypes.c_int)),
                ("nprim", ctypes.POINTER(ctypes.c_int)), ("xyz", _dp), ("exps", _dp), ("coefs", _dp)]


def basis_t(basis):
    """rijk_basis_t over the shell arrays of an nopt_b200.ints.Basis (kept alive by the Basis)."""
    l, pu, npr, xyz, ex, co = basis.arrays
    ip = ctypes.POINTER(ctypes.c_int)
    return BasisT(len(l), l.ctypes.data_as(ip), pu.ctypes.data_as(ip), npr.ctypes.data_as(ip),
                  xyz.ctypes.data_as(_dp), ex.ctypes.data_as(_dp), co.ctypes.data_as(_dp))


# int reduce_jk(double* jk, long count, void* stream, void* user): the ranks' sum of [J | K] in place
REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, _dp, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p)


class ScfOpts(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("conv_dm_rms", ctypes.c_double), ("precision", ctypes.c_int),
                ("switch_diis_err", ctypes.c_double), ("diis_size", ctypes.c_int),
                ("diis_keep_on_switch", ctypes.c_int), ("lindep", ctypes.c_double),
                ("guess_dm", _dp), ("guess_rows", _dp), ("guess_nrows", ctypes.c_long),
                ("converger", ctypes.c_int), ("conv_grad", ctypes.c_double), ("conv_energy", ctypes.c_double),
                ("lbfgs_vectors", ctypes.c_int), ("density_by_eigenvectors", ctypes.c_int),
                ("fp64_phase_precision", ctypes.c_int), ("ao_projector", _dp), ("n_proj", ctypes.c_long),
                ("reduce_jk", REDUCE_FN), ("reduce_user", ctypes.c_void_p)]


class ScfResult(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("dm_rms", ctypes.c_double), ("diis_err", ctypes.c_double),
                ("iterations", ctypes.c_int), ("iterations_mixed", ctypes.c_int), ("converged", ctypes.c_int),
                ("nmo", ctypes.c_int), ("ms_fock", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("ms_build_phase", ctypes.c_double), ("ms_diis_phase", ctypes.c_double),
                ("ms_diag_phase", ctypes.c_double), ("history_len", ctypes.c_int),
                ("history_energy", ctypes.c_double * 128), ("history_diis_err", ctypes.c_double * 128),
                ("history_mixed", ctypes.c_int * 128), ("ms_setup_phase", ctypes.c_double),
                ("ms_final_phase", ctypes.c_double), ("purified", ctypes.c_int)]


class RijkError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("rijk error %d: %s" % (code, msg))
        self.code = code


def lib_path():
    return os.path.join(_HERE, "librijk.so")


def lib():
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise RuntimeError("librijk.so is not built (run python nopt_b200/build.py); there is no CPU fallback")
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        L.rijk_create.argtypes = [P(_vp), ctypes.c_int]
        L.rijk_destroy.argtypes = [_vp]
        L.rijk_set_stream.argtypes = [_vp, _vp]
        L.rijk_last_error.argtypes = [_vp, ctypes.c_char_p, ctypes.c_int]
        L.rijk_get_stats.argtypes = [_vp, P(Stats)]
        L.rijk_set_profiling.argtypes = [_vp, ctypes.c_int]
        L.rijk_set_metric.argtypes = [_vp, _dp, ctypes.c_long, ctypes.c_int]
        L.rijk_set_aux_range.argtypes = [_vp, ctypes.c_long, ctypes.c_long]
        L.rijk_set_3c.argtypes = [_vp, _dp, ctypes.c_long, ctypes.c_long, ctypes.c_int]
        L.rijk_begin_3c.argtypes = [_vp, ctypes.c_long, ctypes.c_long, ctypes.c_int]
        L.rijk_add_3c_block.argtypes = [_vp, ctypes.c_long, ctypes.c_long, _dp]
        L.rijk_eri2c.argtypes = [_vp, P(BasisT), _dp]
        L.rijk_eri3c.argtypes = [_vp, P(BasisT), P(BasisT), ctypes.c_int, _dp]
        L.rijk_set_basis.argtypes = [_vp, P(BasisT), P(BasisT), ctypes.c_int, ctypes.c_long, ctypes.c_long]
        L.rijk_mo_tensor.argtypes = [_vp, _dp, ctypes.c_long, _dp, ctypes.c_long, _dp]
        L.rijk_mo_calc.argtypes = [_vp, _dp, ctypes.c_long, ctypes.c_long, ctypes.c_long, _dp, _dp, _dp, _dp, _dp]
        L.rijk_mo_ints_aaag.argtypes = [_vp, _dp, _dp, ctypes.c_long, ctypes.c_long, ctypes.c_long]
        L.rijk_soscf_hess_ints.argtypes = [_vp, _dp, _dp, _dp, ctypes.c_long, ctypes.c_long, ctypes.c_long]
        L.rijk_set_grad_chunk.argtypes = [_vp, ctypes.c_long]
        L.rijk_save.argtypes = [_vp, ctypes.c_char_p]
        L.rijk_load.argtypes = [_vp, ctypes.c_char_p]
        L.rijk_fock.argtypes = [_vp, _dp, _dp, ctypes.c_long, _dp, _dp, ctypes.c_int]
        L.rijk_fock_device.argtypes = [_vp, _vp, _vp, ctypes.c_long, _vp, _vp, ctypes.c_int]
        L.rijk_sync.argtypes = [_vp]
        L.rijk_selftest_wait_timeout.argtypes = [_vp, ctypes.c_longlong]
        L.rijk_selftest_alloc_failure.argtypes = [_vp, ctypes.c_long]
        L.rijk_coulomb_noalloc.argtypes = [_vp, _vp, _vp]
        L.rijk_grad.argtypes = [_vp, _dp, ctypes.c_long, _dp, ctypes.c_double, _dp, _dp, _dp, _dp]
        L.rijk_mo_ints.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_long, ctypes.c_long, ctypes.c_long]
        L.rijk_scf.argtypes = [_vp, _dp, _dp, ctypes.c_long, ctypes.c_double, P(ScfOpts), _dp, P(ScfResult)]
        L.rijk_fock_energy.argtypes = [_vp, _dp, _dp, _dp, _dp, ctypes.c_double, ctypes.c_int, ctypes.c_double, _dp, _dp]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class FockBuilder:
    """One GPU context holding the fitted tensor B in HBM."""

    def __init__(self, device=0):
        h = _vp()
        rc = lib().rijk_create(ctypes.byref(h), int(device))
        if rc != OK:
            raise RijkError(rc, "rijk_create(device=%d) failed" % device)
        self._h = h
        self.n = self.naux = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().rijk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != OK:
            buf = ctypes.create_string_buffer(512)
            lib().rijk_last_error(self._h, buf, 512)
            raise RijkError(rc, buf.value.decode())

    def last_error(self):
        buf = ctypes.create_string_buffer(512)
        lib().rijk_last_error(self._h, buf, 512)
        return buf.value.decode()

    def set_stream(self, stream_ptr):
        self._check(lib().rijk_set_stream(self._h, _vp(int(stream_ptr))))

    def set_metric(self, V, form=METRIC_INVSQRT):
        V = _c(V)
        self._check(lib().rijk_set_metric(self._h, _p(V), V.shape[0], form))
        self.naux = V.shape[0]

    def set_aux_range(self, q0, q1):
        """Hold only aux functions [q0, q1): Fock builds then return that slice's partial J, K."""
        self._check(lib().rijk_set_aux_range(self._h, int(q0), int(q1)))

    def set_3c(self, I3, n, layout=LAYOUT_PACKED):
        I3 = _c(I3)
        self._check(lib().rijk_set_3c(self._h, _p(I3), int(n), I3.shape[-1], layout))
        self.n = n

    def begin_3c(self, n, naux, layout=LAYOUT_PACKED):
        """Start a streaming three-centre input (rijk_begin_3c)."""
        self._check(lib().rijk_begin_3c(self._h, int(n), int(naux), layout))
        self.n, self._s3 = n, (n, naux, layout)

    def add_3c_block(self, mu0, mu1, block):
        """Rows mu in [mu0, mu1) of the three-centre integrals in the layout given to begin_3c."""
        self._check(lib().rijk_add_3c_block(self._h, int(mu0), int(mu1), _p(_c(block))))

    def set_3c_streamed(self, I3, n, bounds, layout=LAYOUT_PACKED):
        """The fitted tensor from I3 handed over in the orbital-row ranges `bounds` ([(mu0, mu1), ...])."""
        naux = I3.shape[1]
        self.begin_3c(n, naux, layout)
        for mu0, mu1 in bounds:
            if layout == LAYOUT_NOPT_FULL:
                r0, r1 = mu0 * n, mu1 * n
            else:
                r0, r1 = mu0 * (mu0 + 1) // 2, mu1 * (mu1 + 1) // 2
            self.add_3c_block(mu0, mu1, I3[r0:r1])

    def set_basis(self, orb, aux, metric_form=METRIC_INVSQRT, q0=0, q1=0):
        """gen_RI_AA on the GPU: integrals, metric factor and fitted tensor from two Basis objects."""
        bo, ba = basis_t(orb), basis_t(aux)
        self._check(lib().rijk_set_basis(self._h, ctypes.byref(bo), ctypes.byref(ba), metric_form, int(q0), int(q1)))
        self.n, self.naux = orb.nbf, aux.nbf

    def eri2c(self, aux):
        """(P|Q) computed on the GPU (naux x naux)."""
        ba = basis_t(aux)
        V = np.empty((aux.nbf, aux.nbf))
        self._check(lib().rijk_eri2c(self._h, ctypes.byref(ba), _p(V)))
        return V

    def eri3c(self, orb, aux, layout=LAYOUT_PACKED):
        """(mu nu|P) computed on the GPU, in LAYOUT_PACKED ([pair][P]) or LAYOUT_NOPT_FULL ([mu][nu][P])."""
        bo, ba = basis_t(orb), basis_t(aux)
        n, naux = orb.nbf, aux.nbf
        shape = (n * (n + 1) // 2, naux) if layout == LAYOUT_PACKED else (n, n, naux)
        out = np.empty(shape)
        self._check(lib().rijk_eri3c(self._h, ctypes.byref(bo), ctypes.byref(ba), layout, _p(out)))
        return out

    def save(self, path):
        """Write the metric factor and fitted tensor to a file (rijk_save)."""
        self._check(lib().rijk_save(self._h, os.fsencode(path)))

    def load(self, path):
        """Read a file written by save into this context (rijk_load)."""
        self._check(lib().rijk_load(self._h, os.fsencode(path)))
        s = Stats()
        self._check(lib().rijk_get_stats(self._h, ctypes.byref(s)))
        self.n, self.naux = s.n, s.naux

    def mo_tensor(self, C1, C2):
        """(p a|Q) for the orbital rows of C1 and C2, shape (n1 * n2, naux)."""
        C1, C2 = _c(C1), _c(C2)
        out = np.empty((C1.shape[0] * C2.shape[0], self._naux()))
        self._check(lib().rijk_mo_tensor(self._h, _p(C1), C1.shape[0], _p(C2), C2.shape[0], _p(out)))
        return out

    def mo_calc(self, VEC, n_cor, n_act, n_vac):
        """RI_data::MO_calc: dict of the CC, VC, AA, CA, VA tensors ((p n2 + a), Q)."""
        VEC = _c(VEC)
        na = self._naux()
        shapes = {"CC": n_cor * n_cor, "VC": n_vac * n_cor, "AA": n_act * n_act, "CA": n_cor * n_act,
                  "VA": n_vac * n_act}
        out = {k: np.empty((v, na)) for k, v in shapes.items()}
        self._check(lib().rijk_mo_calc(self._h, _p(VEC), n_cor, n_act, n_vac, *[_p(out[k]) for k in
                                                                                    ("CC", "VC", "AA", "CA", "VA")]))
        return out

    def mo_ints_aaag(self, MO_VEC, n_c, n_a, n_mo=None):
        """calc_2el_MO_INTS_AAAG_RI: (tu|vx) as an (n_a^3, n_mo) array."""
        MO_VEC = _c(MO_VEC)
        n_mo = MO_VEC.shape[0] if n_mo is None else n_mo
        out = np.empty((n_a ** 3, n_mo))
        self._check(lib().rijk_mo_ints_aaag(self._h, _p(out), _p(MO_VEC), n_c, n_a, n_mo))
        return out

    def soscf_hess_ints(self, MO_VEC, n_c, n_a, n_mo=None):
        """calc_SOSCF_hess_INTS_RI: (aa_J, aa_K), each (n_mo, n_a^2)."""
        MO_VEC = _c(MO_VEC)
        n_mo = MO_VEC.shape[0] if n_mo is None else n_mo
        aJ, aK = np.empty((n_mo, n_a * n_a)), np.empty((n_mo, n_a * n_a))
        self._check(lib().rijk_soscf_hess_ints(self._h, _p(aJ), _p(aK), _p(MO_VEC), n_c, n_a, n_mo))
        return aJ, aK

    def _naux(self):
        s = Stats()
        self._check(lib().rijk_get_stats(self._h, ctypes.byref(s)))
        return s.nq

    def dm_to_f_transform_ri(self, DM, MO, n_c, precision=PREC_FP64, J=None, K=None):
        """(J, K) exactly as the reference's DM_to_F_transform_RI(J, K, DM, MO, n_c, n_ao)."""
        n = self.n
        DM = _c(DM)
        MO = _c(MO) if n_c > 0 else np.zeros((1, n))
        J = np.empty((n, n)) if J is None else J
        K = np.empty((n, n)) if K is None else K
        self._check(lib().rijk_fock(self._h, _p(DM), _p(MO), int(n_c), _p(J), _p(K), precision))
        return J, K

    def fock_device(self, dD, dMO, n_c, dJ, dK, precision=PREC_FP64):
        """Device-pointer form (ints from tensor.data_ptr()), asynchronous on the context stream."""
        self._check(lib().rijk_fock_device(self._h, _vp(dD), _vp(dMO), int(n_c), _vp(dJ), _vp(dK), precision))

    def scf(self, H, S, n_c, e_nuc, precision=PREC_FP64, conv_dm_rms=1e-10, switch_diis_err=1e-5, max_iter=100,
            diis_size=8, guess=None, diis_keep_on_switch=False, converger=CONV_DIIS, conv_grad=1e-7,
            conv_energy=1e-10, lbfgs_vectors=0, purify=True, fp64_phase=PREC_FP64, projector=None, reduce_jk=None):
        """RHF on the GPU (rijk_scf); guess = (D0, R) with D0 = R^T R (e.g. SystemIntegrals.sad()),
        None for the core-Hamiltonian start; converger CONV_DIIS, CONV_SOSCF (the reference's
        L-BFGS orbital rotations, converged on max|4 F_ai| < conv_grad or |dE| < conv_energy), or
        CONV_DIIS_SOSCF (DIIS while the builds are mixed, SOSCF from the switch to FP64 on).
        purify=False diagonalises X^T F X at every DIIS step (the reference's step); the default
        takes the occupied space from purification, with the eigensolver as its fallback.
        fp64_phase=PREC_FP64_TC makes the builds after a mixed phase FP64_TC ones.  projector (n x n_proj)
        confines the orbitals to the span of its columns, e.g. the Cartesian->spherical map of a
        Cartesian orbital basis (ints.d5_projector), as the reference's D5 treatment.
        reduce_jk(ptr, count, stream) sums the device array [J | K] (count doubles at ptr, written on
        the CUDA stream `stream`) over the ranks of an aux-sharded SCF, in place; an exception in it
        ends the SCF and is raised here (nopt_b200.parallel.ShardedFockBuilder.scf gives the NCCL one).
        Returns (E, MO rows, result dict)."""
        n = self.n
        o = ScfOpts(max_iter, conv_dm_rms, precision, switch_diis_err, diis_size, 1 if diis_keep_on_switch else 0,
                    1e-10)
        o.converger, o.conv_grad, o.conv_energy, o.lbfgs_vectors = converger, conv_grad, conv_energy, lbfgs_vectors
        o.density_by_eigenvectors = 0 if purify else 1
        o.fp64_phase_precision = 0 if fp64_phase == PREC_FP64 else fp64_phase
        if guess is not None:
            gD, gR = _c(guess[0]), _c(guess[1])
            o.guess_dm, o.guess_rows, o.guess_nrows = _p(gD), _p(gR), gR.shape[0]
        if projector is not None:
            T = _c(projector)
            o.ao_projector, o.n_proj = _p(T), T.shape[1]
        failure = []
        if reduce_jk is not None:
            def _cb(ptr, count, stream, user):
                try:
                    reduce_jk(ctypes.cast(ptr, ctypes.c_void_p).value, int(count), stream or 0)
                    return 0
                except BaseException as e:  # reported through RIJK_ERR_REDUCE, raised below
                    failure.append(e)
                    return 1
            o.reduce_jk = REDUCE_FN(_cb)  # kept alive by `o` for the call
        r = ScfResult()
        MO = np.zeros((n, n))
        rc = lib().rijk_scf(self._h, _p(_c(H)), _p(_c(S)), int(n_c), float(e_nuc), ctypes.byref(o), _p(MO),
                            ctypes.byref(r))
        if failure:
            raise failure[0]
        if rc != ERR_CONVERGE:  # not converged: the result (converged = 0) and its trace are returned
            self._check(rc)
        out = {k: getattr(r, k) for k, _ in ScfResult._fields_ if not k.startswith("history")}
        k = r.history_len
        out["history"] = [(r.history_energy[i], r.history_diis_err[i], r.history_mixed[i]) for i in range(k)]
        return r.energy, MO, out

    def calc_2el_mo_ints_ri(self, DM_D, MO_VEC, MO_VEC1, MO_VEC2, n_c, n_a, t=0, want_jk=True):
        """(MO_INTS (n_a^2 x n_a^2), J, K) as the reference's calc_2el_MO_INTS_RI (src/RI.cpp:178)."""
        n = self.n
        out = np.empty((n_a * n_a, n_a * n_a))
        J = np.empty((n, n)) if want_jk else None
        K = np.empty((n, n)) if want_jk else None
        D = _c(DM_D) if want_jk else None
        M0 = _c(MO_VEC) if (want_jk and n_c > 0) else None
        self._check(lib().rijk_mo_ints(self._h, _p(D), _p(J), _p(K), _p(out), _p(M0), _p(_c(MO_VEC1)),
                                       _p(_c(MO_VEC2)), int(n_c), int(n_a), int(t)))
        return out, J, K

    def set_grad_chunk(self, q_per_chunk):
        """Aux functions per chunk of grad's Gamma stage (0: automatic, from free HBM)."""
        self._check(lib().rijk_set_grad_chunk(self._h, int(q_per_chunk)))

    def grad(self, MO, n_c, H, e_nuc, want_3c=False, want_metric=False, out3=None, outV=None):
        """(E, dE/dMO (n_c x n), dE/d(P|mu nu) packed [pair][P] or None, dE/d(P|Q) or None).  out3 / outV
        (C-contiguous float64 arrays of those shapes) receive the last two instead of new arrays."""
        n = self.n
        MO = _c(MO[:n_c])
        E = ctypes.c_double(0.0)
        dC = np.empty((n_c, n))
        shape3, shapeV = (n * (n + 1) // 2, self.naux), (self.naux, self.naux)
        for o, sh in ((out3, shape3), (outV, shapeV)):
            if o is not None and (o.shape != sh or o.dtype != np.float64 or not o.flags.c_contiguous):
                raise ValueError("grad output array must be C-contiguous float64 of shape %s" % (sh,))
        d3 = (out3 if out3 is not None else np.empty(shape3)) if want_3c else None
        dV = (outV if outV is not None else np.empty(shapeV)) if want_metric else None
        self._check(lib().rijk_grad(self._h, _p(MO), int(n_c), _p(_c(H)), float(e_nuc), ctypes.byref(E), _p(dC),
                                    _p(d3), _p(dV)))
        return E.value, dC, d3, dV

    def sync(self):
        self._check(lib().rijk_sync(self._h))

    def selftest_alloc_failure(self, after):
        """After `after` more device allocations of this context, refuse the next ones with ERR_ALLOC
        (after < 0: off)."""
        self._check(lib().rijk_selftest_alloc_failure(self._h, int(after)))

    def selftest_wait_timeout(self, cycles):
        """Launch the bounded-wait self-test (a wait that runs out after `cycles` SM clocks); the
        next sync raises RijkError with ERR_TIMEOUT."""
        self._check(lib().rijk_selftest_wait_timeout(self._h, int(cycles)))

    def calc_f_ao(self, H, DM, J, K, c=1.0, mc=0, e_nuc=0.0):
        n = self.n
        F = np.empty((n, n))
        E = ctypes.c_double(0.0)
        self._check(lib().rijk_fock_energy(self._h, _p(_c(H)), _p(_c(DM)), _p(_c(J)), _p(_c(K)), c, mc, e_nuc,
                                           _p(F), ctypes.byref(E)))
        return F, E.value

    def set_profiling(self, on):
        self._check(lib().rijk_set_profiling(self._h, 1 if on else 0))

    def stats(self):
        s = Stats()
        self._check(lib().rijk_get_stats(self._h, ctypes.byref(s)))
        out = {k: getattr(s, k) for k, _ in Stats._fields_ if k not in ("ms_stage", "stage_names", "ms_grad_stage")}
        out["grad_stages"] = dict(zip(GRAD_STAGES, list(s.ms_grad_stage)))
        k = s.profiled_stages
        out["stages"] = {s.stage_names[i].value.decode(): s.ms_stage[i] for i in range(k)}
        return out
