"""Benchmark of the RI-JK Fock build on B200: Fock builds per second and SCF time.

Workload (default): water 32-mer (H2O)32, cc-pVTZ / cc-pVTZ-JKFIT (n = 1856, naux = 4448,
nocc = 160), seeded jittered 4x4x2 lattice.  A step is one Fock build (J and K) over the
resident fitted tensor B (63 GB, far larger than the 126 MB L2, so no flush is needed between
steps).  `value` is device-timed FP64 builds/s with the inputs in HBM; `e2e` is the same
metric through the drop-in C ABI call (pinned host D and C in, host J and K out; `e2e_pageable`
with plain pageable arrays, as the reference passes them); the mixed-precision form
(`mixed.value`, `mixed.speedup_vs_fp64`) and the SCF time to convergence are reported beside it.
The (H2O)16 cc-pVDZ workload and a CPU SCF time at (H2O)6 come as extra keys.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload NAME]

With N > 1 (torchrun) every rank runs an independent replica of the workload (the Fock
build of one molecule is a one-GPU problem): weak scaling, value = total builds/s.
`--impl reference` times the reference's CPU algorithm on all host threads: the oracle's
restatement of DM_to_F_transform_RI in the reference's dgemm order (the reference itself does not
build here), as whole builds where its full-square RI_AA fits in host memory, else one aux slice
of the build per step (every stage's share of that slice; see oracle sliced_step).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the dominant kernels at
# (H2O)16 cc-pVDZ, from one ncu capture of each (summaries under profiles/)
NCU_TRAFFIC = {("h2o16_dz", "xform_f64"): 1.290096e9 + 0.447404e9,
               ("h2o16_dz", "syrk_f64"): 0.457111e9 + 0.092111e9,
               ("h2o16_dz", "xform_tc"): 0.639337e9 + 0.202236e9,
               ("h2o16_dz", "syrk_tc"): 0.229277e9 + 0.004902e9,
               ("h2o16_dz", "syrk_i8"): 0.970246e9 + 0.088795e9,
               ("h2o16_dz", "coulomb_w_mixed"): 0.639341e9 + 0.004234e9,
               ("h2o16_dz", "coulomb_j_mixed"): 0.638610e9 + 0.010762e9,
               # (H2O)32 cc-pVTZ: the half-transform captured on a synthetic case with its orbital shape and
               # 256 aux functions (one launch, both 80-orbital batches: 4.469e9 read + 0.653e9 written),
               # scaled by aux functions (4448)
               ("h2o32_tz", "xform_f64"): (4.469058e9 + 0.652858e9) / 256 * 4448}
WORKLOAD_NAMES = {"h2o6_dz": "(H2O)6 cc-pVDZ/cc-pVDZ-JKFIT", "h2o16_dz": "(H2O)16 cc-pVDZ/cc-pVDZ-JKFIT",
                  "c40h82_dz": "C40H82 cc-pVDZ/cc-pVDZ-JKFIT", "h2o32_tz": "(H2O)32 cc-pVTZ/cc-pVTZ-JKFIT"}
METRIC = "RI-JK Fock builds/s (FP64 drop-in; mixed and SCF time beside it)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="h2o32_tz")
    ap.add_argument("--extra", default="h2o16_dz", help="second workload reported under its own key ('none': skip)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-scf", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--cpu-slices", type=int, default=12,
                    help="aux slices of the CPU arm when the full-square RI_AA does not fit host memory")
    ap.add_argument("--metric", default="invsqrt", choices=["invsqrt", "cholesky"],
                    help="metric factor of the fitted tensor: V^-1/2 (the reference's S05_calc) or L^-1")
    ap.add_argument("--setup", default="gpu", choices=["gpu", "host"],
                    help="gpu: integrals on the device (rijk_set_basis); host: host integrals + rijk_set_3c")
    ap.add_argument("--shard", default="replicas", choices=["replicas", "q"],
                    help="N > 1: independent replicas (weak scaling), or one molecule with the aux index "
                         "split over the ranks and J, K all-reduced (strong scaling)")
    return ap.parse_args()


class SyntheticSystem:
    """Seeded random inputs of a chosen size (workload "rand:n=..,naux=..,nocc=.."): packed
    three-centre entries ~ N(0,1) e^{-|mu-nu|/n}, a well-conditioned metric, a random symmetric H and
    S = 1.  For kernel timing and profiling at sizes the molecules do not give; no SCF."""

    def __init__(self, spec, seed):
        kv = dict(x.split("=") for x in spec.split(","))
        self.n, self.naux, self.nocc = int(kv["n"]), int(kv["naux"]), int(kv["nocc"])
        rng = np.random.default_rng(seed)
        n, na = self.n, self.naux
        A = rng.normal(size=(na, na))
        self.V = A @ A.T / na + np.eye(na)
        mu, nu = np.tril_indices(n)
        self.I3 = rng.normal(size=(mu.size, na)) * np.exp(-np.abs(mu - nu) / n)[:, None]
        Hm = rng.normal(size=(n, n))
        self.H = (Hm + Hm.T) / np.sqrt(n)
        self.S = np.eye(n)
        self.Enuc = 0.0
        self.orb = self.aux = None
        self.synthetic = True


def build_system(workload, seed, ri_integrals=True):
    from nopt_b200 import ints
    from nopt_b200.molecules import WORKLOADS
    if workload.startswith("rand:"):
        t = time.time()
        si = SyntheticSystem(workload[5:], seed)
        return si, time.time() - t, (None, None)
    fac, ob, ab = WORKLOADS[workload]
    mol = fac(seed)
    t = time.time()
    si = ints.SystemIntegrals(mol, ob, ab, layout=ints.LAYOUT_PACKED, ri_integrals=ri_integrals)
    return si, time.time() - t, (ob, ab)


def core_guess(si):
    """Orbitals of the core Hamiltonian (rows = orbitals), orthonormal in S."""
    s, U = np.linalg.eigh(si.S)
    X = U / np.sqrt(s)
    e, Cp = np.linalg.eigh(X.T @ si.H @ X)
    MO = (X @ Cp).T.copy()
    DM = MO[:si.nocc].T @ MO[:si.nocc]
    return DM, MO


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.lines, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU arm ------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import rijk_oracle as O
    return O


def _blas_threads():
    from threadpoolctl import threadpool_info
    return max([p.get("num_threads", 1) for p in threadpool_info()] or [1])


def workload_shape(workload, seed):
    """(n, naux, nocc) of a workload without computing any integral."""
    if workload.startswith("rand:"):
        kv = dict(x.split("=") for x in workload[5:].split(","))
        return int(kv["n"]), int(kv["naux"]), int(kv["nocc"])
    from nopt_b200 import ints
    from nopt_b200.molecules import WORKLOADS
    fac, ob, ab = WORKLOADS[workload]
    mol = fac(seed)
    return ints.Basis.for_molecule(ob, mol).nbf, ints.Basis.for_molecule(ab, mol).nbf, mol.nelec // 2


def host_available():
    with open("/proc/meminfo") as f:
        for line in f:
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    return 0


def cpu_arm_plan(workload, seed, nslices):
    """("full", bytes) when the reference's full-square RI_AA and its half-transformed copies fit in
    70% of the host's available memory; ("sliced", bytes) when one aux slice and RI_CA do;
    ("unavailable", reason) otherwise."""
    n, naux, nocc = workload_shape(workload, seed)
    full = n * (n + 1) // 2 * naux * 8 + n * n * naux * 8 + 2 * nocc * n * naux * 8
    avail = host_available()
    if full <= 0.7 * avail:
        return "full", full
    sliced = nocc * n * naux * 8 + 2.2 * n * n * (naux / max(nslices, 1)) * 8 + n * n * 8 * 4
    if sliced <= 0.7 * avail:
        return "sliced", sliced
    return "unavailable", ("the CPU arm needs %.0f GB of host memory even with %d aux slices; %.0f GB are available"
                           % (sliced / 1e9, nslices, avail / 1e9))


def cpu_full(si, DM, MO, steps=None, warmup=1, budget_s=None):
    """Whole builds of the oracle's DM_to_F_transform_RI (NOPT layout) on all host threads: either
    `steps` builds after `warmup`, or as many as fit in budget_s.  Returns (builds/s, builds, seconds, note)."""
    O = _oracle()
    RI = O.unpack_3c(si.I3, si.n)
    Vm05, _ = O.s05_calc(si.V)
    for _ in range(max(warmup, 1)):
        O.dm_to_f_transform_ri(RI, Vm05, DM, MO, si.nocc, si.n)
    t0 = time.perf_counter()
    k = 0
    while True:
        O.dm_to_f_transform_ri(RI, Vm05, DM, MO, si.nocc, si.n)
        k += 1
        el = time.perf_counter() - t0
        if (steps is not None and k >= steps) or (steps is None and (el > budget_s or k >= 50)):
            break
    return k / el, k, el, "%d whole builds in NOPT layout (RI_AA %.2f GB) after %d untimed" % (
        k, RI.nbytes / 1e9, max(warmup, 1))


def cpu_sliced(si, DM, MO, nslices, steps, warmup):
    """The oracle's aux-sliced restatement of DM_to_F_transform_RI: untimed set-up (V^-1/2, and
    RI_CA and the Coulomb coefficients from every raw slice of (mu nu|P) computed by the host
    integral engine), then `steps` timed repetitions of one slice's share of the build.  A slice
    of s of the naux aux functions carries s / naux of every stage's products, so builds/s =
    (s / naux) / (seconds per slice step).  Returns (builds/s, steps, seconds, note, set-up s)."""
    from nopt_b200 import ints
    O = _oracle()
    n, naux, nocc = si.n, si.naux, si.nocc
    t0 = time.perf_counter()
    V = si.V if si.V is not None else ints.coulomb_2c(si.aux)
    Vm05, _ = O.s05_calc(V)
    bounds = ints.aux_slice_bounds(si.aux, nslices)
    mid = len(bounds) // 2
    keep = {}

    def raw(p0, p1):
        A = ints.coulomb_3c_aux_range(si.orb, si.aux, p0, p1)
        if (p0, p1) == bounds[mid]:
            keep["A"] = A
        return A

    RI_CA, RI_Jv = O.sliced_setup(raw, bounds, Vm05, DM, MO, nocc, n)
    p0, p1 = bounds[mid]
    A = keep.pop("A")
    t_setup = time.perf_counter() - t0
    for _ in range(max(warmup, 1)):
        O.sliced_step(A, p0, p1, RI_CA, RI_Jv, Vm05, DM, MO, nocc, n)
    t0 = time.perf_counter()
    for _ in range(steps):
        O.sliced_step(A, p0, p1, RI_CA, RI_Jv, Vm05, DM, MO, nocc, n)
    el = time.perf_counter() - t0
    frac = (p1 - p0) / naux
    note = ("%d steps, each the share of aux slice [%d, %d) (%d of %d aux functions, %.4f of a build) of every stage "
            "of the reference's build, in its dgemm order; the full-square RI_AA (%.0f GB) does not fit in host "
            "memory, so it is held one slice (%.1f GB) at a time and RI_CA (%.1f GB) whole" %
            (steps, p0, p1, p1 - p0, naux, frac, n * n * naux * 8 / 1e9, A.nbytes / 1e9, RI_CA.nbytes / 1e9))
    return frac * steps / el, steps, el, note, t_setup


def config_of(workload, n, naux, nocc, world, sharded, seed):
    """The `config` object of both arms' JSON lines."""
    nt = (n + 63) // 64
    bytes_b = naux * (nt * (nt + 1) // 2) * 4096 * 8
    name = WORKLOAD_NAMES.get(workload)
    if name is None:
        name = ("synthetic " + workload[5:].replace(",", " ") + " (random packed B ~ N(0,1) e^-|mu-nu|/n)"
                if workload.startswith("rand:") else workload)
    return {"workload": name, "n": n, "naux": naux, "nocc": nocc,
            "parallelism": ("aux-sharded x%d" % world) if sharded else ("replicas x%d" % world if world > 1 else "single"),
            "l2": "inputs larger than L2 (B = %.2f GB)" % (bytes_b / 1e9), "seed": seed}


def run_reference(args, rank, world):
    if rank != 0:
        return
    n, naux, nocc = workload_shape(args.workload, args.seed)
    cfg = config_of(args.workload, n, naux, nocc, world, args.shard == "q" and world > 1, args.seed)
    mode, need = cpu_arm_plan(args.workload, args.seed, args.cpu_slices)
    if mode == "unavailable":
        print(json.dumps({"impl": "reference", "unavailable": need}), flush=True)
        return
    si, tint, (ob, ab) = build_system(args.workload, args.seed, ri_integrals=(mode == "full"))
    DM, MO = core_guess(si)
    setup = None
    if mode == "full":
        v, k, el, note = cpu_full(si, DM, MO, steps=args.steps, warmup=args.warmup)
    else:
        v, k, el, note, setup = cpu_sliced(si, DM, MO, args.cpu_slices, args.steps, args.warmup)
    threads = _blas_threads()
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "builds/s", "n_gpus": 0, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
           "cpu_baseline": {"value": v, "unit": "builds/s", "cores": threads, "kind": "port",
                            "sample": note + " (oracle restatement; the reference needs libint2/Eigen/Boost/LAPACKE, "
                                             "absent here)"},
           "e2e": {"value": v, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "setup_s": {"host_integrals": tint, "sliced_setup": setup}}
    print(json.dumps(out), flush=True)


def cpu_baseline_for(si, DM, MO, workload, seed, nslices, budget_s):
    """cpu_baseline object of our arm: whole builds within budget_s where they fit, else two slice steps."""
    mode, need = cpu_arm_plan(workload, seed, nslices)
    if mode == "unavailable":
        return {"skipped": need}
    if mode == "full":
        v, k, el, note = cpu_full(si, DM, MO, budget_s=budget_s)
    else:
        v, k, el, note, _ = cpu_sliced(si, DM, MO, nslices, 2, 1)
    return {"value": v, "unit": "builds/s", "cores": _blas_threads(), "kind": "port", "sample": note}


# ------------------------------------------------------------------ GPU arm ------
def grad_report(fb, si, MOc, nocc, fp64_peak, reps=3):
    """rijk_grad (E, dE/dC, dE/d(P|mu nu) packed, dE/d(P|Q); host outputs): wall time per call, and
    the device time, FLOPs and FP64 roofline fraction of each stage (profiling events)."""
    # outputs allocated once and reused, as a caller keeps its gradient arrays between calls (new
    # arrays would put the first-touch page faults of GBs of host memory into every call)
    out3 = np.empty((si.n * (si.n + 1) // 2, si.naux))
    outV = np.empty((si.naux, si.naux))
    kw = dict(want_3c=True, want_metric=True, out3=out3, outV=outV)
    fb.grad(MOc, nocc, si.H, si.Enuc, **kw)  # first call: module loads, first touch of the outputs
    t0 = time.perf_counter()
    for _ in range(reps):
        fb.grad(MOc, nocc, si.H, si.Enuc, **kw)
    wall = (time.perf_counter() - t0) / reps
    fb.set_profiling(True)
    fb.grad(MOc, nocc, si.H, si.Enuc, **kw)
    fb.set_profiling(False)
    st = fb.stats()
    n, naux = si.n, si.naux
    npad = st["npad"]
    noccp = (nocc + 15) // 16 * 16
    te = st["ntile"] * 4096
    chunked = st["grad_qchunk"] < naux
    flops = {"x_recompute": 2.0 * noccp * npad * npad * naux if chunked else 0.0,
             "y_t": 4.0 * noccp * noccp * npad * naux, "gamma": 2.0 * te * noccp * naux,
             "d3c_M_gamma": 2.0 * te * naux * naux, "g_gamma_B": 2.0 * te * naux * naux, "dV_MtGM": 4.0 * naux ** 3}
    stages = {}
    for k, ms in st["grad_stages"].items():
        e = {"ms": ms}
        if k in flops and ms > 0 and flops[k] > 0:
            e["tflops"] = flops[k] / (ms * 1e-3) / 1e12
            e["frac_of_fp64_peak"] = e["tflops"] / fp64_peak
        stages[k] = e
    top = max((k for k in stages if k in flops), key=lambda k: stages[k]["ms"])
    return {"wall_ms": 1e3 * wall, "device_ms": st["ms_grad_total"], "aux_chunk": st["grad_qchunk"],
            "recompute_path": bool(chunked), "stages": stages, "top_stage": top,
            "flops": sum(flops.values()), "fp64_peak_tflops": fp64_peak,
            "what": "rijk_grad through the C ABI: E, dE/dC, dE/d(P|mu nu) (packed) and dE/d(P|Q) to host memory; "
                    "device_ms = its kernels before the host copies (stage events), wall_ms includes the copies "
                    "(%.2f GB, into pageable arrays reused between calls) and the call's device buffer allocation"
                    % ((n * (n + 1) // 2 * naux + naux * naux) * 8 / 1e9)}


def c40h82_grad(seed, dev, fp64_peak, chunk=1200):
    """The C40H82 cc-pVDZ adjoint case: mixed -> FP64 SCF, then rijk_grad with Gamma in aux chunks and
    X^Q recomputed in tiles (the path taken when HBM cannot hold Gamma for every aux function)."""
    from nopt_b200 import rijk
    si, _, _ = build_system("c40h82_dz", seed, ri_integrals=False)
    with rijk.FockBuilder(dev.index) as fb:
        fb.set_basis(si.orb, si.aux, rijk.METRIC_INVSQRT)
        t0 = time.perf_counter()
        E, MOc, r = fb.scf(si.H, si.S, si.nocc, si.Enuc, precision=rijk.PREC_MIXED, guess=si.sad(),
                           converger=rijk.CONV_DIIS_SOSCF)
        t_scf = time.perf_counter() - t0
        fb.set_grad_chunk(chunk)
        g = grad_report(fb, si, MOc, si.nocc, fp64_peak, reps=1)
    g.update({"workload": WORKLOAD_NAMES["c40h82_dz"], "scf_seconds_first_call": t_scf, "energy": E,
              "scf_builds": r["iterations"], "scf_builds_mixed": r["iterations_mixed"]})
    return g


def extra_workload(name, seed, dev, steps, want_cpu, budget_s, fp64_peak):
    """A second workload on a fresh context: FP64 and mixed builds/s (device-timed), e2e through
    rijk_fock, SCF times, the adjoint's time, and the CPU arm's builds/s."""
    import ctypes
    import torch
    from nopt_b200 import rijk
    si, _, _ = build_system(name, seed, ri_integrals=True)
    DM, MO = core_guess(si)
    n, nocc = si.n, si.nocc
    stream = torch.cuda.current_stream(dev)
    out = {"workload": WORKLOAD_NAMES.get(name, name), "n": n, "naux": si.naux, "nocc": nocc}
    with rijk.FockBuilder(dev.index) as fb:
        fb.set_stream(stream.cuda_stream)
        fb.set_basis(si.orb, si.aux, rijk.METRIC_INVSQRT)
        dD = torch.from_numpy(DM).to(dev)
        dMO = torch.from_numpy(MO[:nocc].copy()).to(dev)
        dJ = torch.empty((n, n), dtype=torch.float64, device=dev)
        dK = torch.empty((n, n), dtype=torch.float64, device=dev)

        def timed(prec):
            for _ in range(3):
                fb.fock_device(dD.data_ptr(), dMO.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), prec)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fb.fock_device(dD.data_ptr(), dMO.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), prec)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            return e0.elapsed_time(e1) / steps

        ms64 = timed(rijk.PREC_FP64)
        msmx = timed(rijk.PREC_MIXED)
        out["fp64"] = {"value": 1e3 / ms64, "unit": "builds/s", "ms_per_step": ms64}
        out["mixed"] = {"value": 1e3 / msmx, "unit": "builds/s", "ms_per_step": msmx, "speedup_vs_fp64": ms64 / msmx}
        hD = torch.from_numpy(DM).pin_memory()
        hMO = torch.from_numpy(MO[:nocc].copy()).pin_memory()
        hJ = torch.empty((n, n), dtype=torch.float64).pin_memory()
        hK = torch.empty((n, n), dtype=torch.float64).pin_memory()
        P = ctypes.POINTER(ctypes.c_double)
        pD, pMO, pJ, pK = [ctypes.cast(t.data_ptr(), P) for t in (hD, hMO, hJ, hK)]
        L = rijk.lib()
        fb._check(L.rijk_fock(fb._h, pD, pMO, nocc, pJ, pK, rijk.PREC_FP64))
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(steps):
            fb._check(L.rijk_fock(fb._h, pD, pMO, nocc, pJ, pK, rijk.PREC_FP64))
        out["e2e"] = {"value": steps / (time.perf_counter() - t0), "unit": "builds/s",
                      "h2d_bytes_per_step": int((n * n + nocc * n) * 8), "d2h_bytes_per_step": int(2 * n * n * 8)}
        # the same with plain pageable numpy arrays, as the reference passes them
        pgD, pgMO = np.ascontiguousarray(DM), np.ascontiguousarray(MO[:nocc])
        pgJ, pgK = np.empty((n, n)), np.empty((n, n))
        args_pg = [ctypes.cast(a.ctypes.data, P) for a in (pgD, pgMO, pgJ, pgK)]
        fb._check(L.rijk_fock(fb._h, args_pg[0], args_pg[1], nocc, args_pg[2], args_pg[3], rijk.PREC_FP64))
        t0 = time.perf_counter()
        for _ in range(steps):
            fb._check(L.rijk_fock(fb._h, args_pg[0], args_pg[1], nocc, args_pg[2], args_pg[3], rijk.PREC_FP64))
        out["e2e_pageable"] = {"value": steps / (time.perf_counter() - t0), "unit": "builds/s"}
        guess = si.sad()
        scf = {}
        fb.scf(si.H, si.S, nocc, si.Enuc, guess=guess)  # untimed first call
        for key, prec, conv in (("fp64", rijk.PREC_FP64, rijk.CONV_DIIS),
                                ("diis_mixed_then_soscf_fp64", rijk.PREC_MIXED, rijk.CONV_DIIS_SOSCF)):
            best = None
            for _ in range(3):
                t0 = time.perf_counter()
                E, _, r = fb.scf(si.H, si.S, nocc, si.Enuc, precision=prec, guess=guess, converger=conv)
                t = time.perf_counter() - t0
                if best is None or t < best[0]:
                    best = (t, E, r)
            r = best[2]
            # where the time goes at this size: the library's own clocks of the fastest run
            scf[key] = {"seconds": best[0], "energy": best[1], "iterations": r["iterations"],
                        "iterations_mixed": r["iterations_mixed"], "ms_fock": r["ms_fock"],
                        "ms_setup": r["ms_setup_phase"], "ms_build_and_error": r["ms_build_phase"],
                        "ms_diis": r["ms_diis_phase"], "ms_density": r["ms_diag_phase"],
                        "ms_final": r["ms_final_phase"], "purified_steps": r["purified"]}
        scf["diis_mixed_then_soscf_fp64"]["abs_dE_vs_fp64"] = abs(scf["diis_mixed_then_soscf_fp64"]["energy"] -
                                                                  scf["fp64"]["energy"])
        out["scf"] = scf
        # the adjoint (rijk_grad) at the converged FP64 orbitals: E, dE/dC, dE/d(P|mu nu), dE/d(P|Q)
        E, MOc, _ = fb.scf(si.H, si.S, nocc, si.Enuc, guess=guess)
        out["grad"] = grad_report(fb, si, MOc, nocc, fp64_peak)

    if want_cpu:
        out["cpu_baseline"] = cpu_baseline_for(si, DM, MO, name, seed, 12, budget_s)
        if "value" in out["cpu_baseline"]:
            out["ratio_e2e_vs_cpu"] = out["e2e"]["value"] / out["cpu_baseline"]["value"]
    return out


def scf_cpu_small(seed, dev):
    """SCF time to convergence of the reference's algorithm on the host (the oracle's RHF with its
    restated Fock build, whole builds in NOPT layout, all threads) beside rijk_scf on the GPU, for the
    (H2O)6 cc-pVDZ/cc-pVDZ-JKFIT workload the reference runs as-is; the same SAD start and the same
    criterion (density RMS change < 1e-10)."""
    from nopt_b200 import ints, rijk
    O = _oracle()
    si, _, _ = build_system("h2o6_dz", seed, ri_integrals=True)
    RI = O.unpack_3c(si.I3, si.n)
    guess = si.sad()
    t0 = time.perf_counter()
    Vm05, _ = O.s05_calc(si.V)
    Ec, _, _, _, itc = O.scf_rhf(si.S, si.H, RI, Vm05, si.nocc, si.Enuc, conv_dm=1e-10, guess=guess)
    tc = time.perf_counter() - t0
    with rijk.FockBuilder(dev.index) as fb:
        fb.set_basis(si.orb, si.aux, rijk.METRIC_INVSQRT)
        fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess)
        best = None
        for _ in range(3):
            t0 = time.perf_counter()
            Eg, _, r = fb.scf(si.H, si.S, si.nocc, si.Enuc, guess=guess)
            t = time.perf_counter() - t0
            best = (t, Eg, r["iterations"]) if best is None or t < best[0] else best
    return {"workload": WORKLOAD_NAMES["h2o6_dz"], "cpu_seconds": tc, "cpu_builds": itc + 2, "cpu_energy": Ec,
            "cpu_cores": _blas_threads(), "gpu_seconds": best[0], "gpu_builds": best[2], "gpu_energy": best[1],
            "abs_dE": abs(Ec - best[1]), "speedup": tc / best[0],
            "note": "CPU: oracle RHF/DIIS with the restated DM_to_F_transform_RI (V^-1/2 set-up included, integrals "
                    "not); GPU: rijk_scf FP64 DIIS after rijk_set_basis, fastest of three"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1 or "RANK" in os.environ:  # launched by torchrun (a one-rank group included)
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist is not None:
            dist.destroy_process_group()
        return

    from nopt_b200 import rijk
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    synthetic = args.workload.startswith("rand:")
    if synthetic:  # no basis: integrals come from the seeded generator, set up through rijk_set_3c
        args.setup, args.no_scf = "host", True
    want_cpu = not args.no_cpu and rank == 0 and world == 1
    mode, _ = cpu_arm_plan(args.workload, args.seed, args.cpu_slices) if want_cpu else ("none", None)
    if args.setup == "host":
        n_, naux_, _ = workload_shape(args.workload, args.seed)
        packed = n_ * (n_ + 1) // 2 * naux_ * 8
        if packed > 0.7 * host_available():
            raise SystemExit("--setup host needs %.0f GB of host memory for (mu nu|P); use --setup gpu" % (packed / 1e9))
    # host RI integrals only where something needs them: the host set-up path or a whole-build CPU arm
    need_host_ri = args.setup == "host" or mode == "full"
    si, tint, (ob, ab) = build_system(args.workload, args.seed, ri_integrals=need_host_ri)
    DM, MO = core_guess(si)
    n, naux, nocc = si.n, si.naux, si.nocc
    stream = torch.cuda.current_stream(dev)
    fb = rijk.FockBuilder(local)
    fb.set_stream(stream.cuda_stream)
    sharded = args.shard == "q" and dist is not None
    q = (0, 0)
    if sharded:
        from nopt_b200.parallel import aux_slices
        q = aux_slices(naux, world)[rank]
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    form = rijk.METRIC_CHOLESKY if args.metric == "cholesky" else rijk.METRIC_INVSQRT
    if args.setup == "gpu":  # integrals, metric factor and B all on the device (rijk_set_basis)
        fb.set_basis(si.orb, si.aux, form, *q)
    else:  # host integrals up, metric factor and B on the device
        fb.set_metric(si.V, form)
        if sharded:
            fb.set_aux_range(*q)
        fb.set_3c(si.I3, n)
    t_setup = time.perf_counter() - t0
    st0 = fb.stats()

    dD = torch.from_numpy(DM).to(dev)
    dMO = torch.from_numpy(MO[:nocc].copy()).to(dev)
    dJK = torch.empty((2, n, n), dtype=torch.float64, device=dev)  # J and K in one buffer: one collective
    dJ, dK = dJK[0], dJK[1]

    def build(prec):
        fb.fock_device(dD.data_ptr(), dMO.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), prec)
        if sharded:  # partial J, K of this rank's aux slice -> full J, K (NCCL on the same stream)
            dist.all_reduce(dJK)

    def timed(prec, steps, warm):
        for _ in range(warm):
            build(prec)
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            build(prec)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        ms = e0.elapsed_time(e1) / steps
        if dist is not None:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    with ClockSampler(local) as clk:
        ms = timed(rijk.PREC_FP64, args.steps, max(args.warmup, 3))
    st = fb.stats()
    launches = st["kernels_last_fock"] * args.steps
    value = (1 if sharded else world) * 1e3 / ms

    # end to end through the drop-in call: host D, C in; host J, K out.  Pinned buffers, and
    # plain pageable arrays as the reference passes them (J and K are new[]'d per call there,
    # src/molecule.cpp:4409-4415).
    import ctypes
    P = ctypes.POINTER(ctypes.c_double)
    L = rijk.lib()

    def e2e(hD, hMO, hJ, hK, steps):
        pD, pMO, pJ, pK = [ctypes.cast(p, P) for p in (hD, hMO, hJ, hK)]
        for _ in range(2):
            fb._check(L.rijk_fock(fb._h, pD, pMO, nocc, pJ, pK, rijk.PREC_FP64))
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fb._check(L.rijk_fock(fb._h, pD, pMO, nocc, pJ, pK, rijk.PREC_FP64))
            if sharded:  # the host matrices of all ranks summed through the GPU
                Jt = torch.from_numpy(np.ctypeslib.as_array(ctypes.cast(hJ, P), (n, n)))
                Kt = torch.from_numpy(np.ctypeslib.as_array(ctypes.cast(hK, P), (n, n)))
                tj, tk = Jt.to(dev), Kt.to(dev)
                dist.all_reduce(tj)
                dist.all_reduce(tk)
                Jt.copy_(tj.cpu())
                Kt.copy_(tk.cpu())
        e1.record(stream)
        torch.cuda.synchronize(dev)
        t = e0.elapsed_time(e1) / steps
        if dist is not None:
            tt = torch.tensor([t], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt.item())
        return t

    hD = torch.from_numpy(DM).pin_memory()
    hMO = torch.from_numpy(MO[:nocc].copy()).pin_memory()
    hJ = torch.empty((n, n), dtype=torch.float64).pin_memory()
    hK = torch.empty((n, n), dtype=torch.float64).pin_memory()
    ms_e2e = e2e(hD.data_ptr(), hMO.data_ptr(), hJ.data_ptr(), hK.data_ptr(), args.steps)
    pgD, pgMO = np.ascontiguousarray(DM), np.ascontiguousarray(MO[:nocc])
    pgJ, pgK = np.empty((n, n)), np.empty((n, n))
    psteps = max(3, args.steps // 4)
    ms_e2e_pg = e2e(pgD.ctypes.data, pgMO.ctypes.data, pgJ.ctypes.data, pgK.ctypes.data, psteps)

    # per-kernel device times (events around each launch on the launching stream)
    def stage_times(prec, reps=5):
        fb.set_profiling(True)
        acc = {}
        for _ in range(reps):
            fb.fock_device(dD.data_ptr(), dMO.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), prec)
            fb.sync()
            for k, v in fb.stats()["stages"].items():
                acc.setdefault(k, []).append(v)
        fb.set_profiling(False)
        return {k: float(np.median(v)) for k, v in acc.items()}

    stage_ms = stage_times(rijk.PREC_FP64)
    top = max(stage_ms, key=stage_ms.get)

    peaks = json.load(open(PEAKS)) if os.path.exists(PEAKS) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    # FP64 peak: cuBLAS DGEMM measured on this GPU (the measured-peaks file has no FP64 figure)
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e9
    for _ in range(3):
        e0.record(stream)
        torch.matmul(a, b)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    fp64_peak = 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    del a, b
    ntile, npad = st0["ntile"], st0["npad"]
    noccp = (nocc + 15) // 16 * 16
    tile_elems = ntile * 4096
    algo = {
        "coulomb_w": ("hbm", tile_elems * naux * 8.0),
        "coulomb_j": ("hbm", tile_elems * naux * 8.0),
        "xform_f64": ("tensor", 2.0 * noccp * npad * npad * naux),
        "syrk_f64": ("tensor", float(npad) * (npad + 64) * noccp * naux),
    }
    kind, amount = algo.get(top, ("hbm", 0.0))
    if kind == "hbm":
        achieved = amount / (stage_ms[top] * 1e-3) / 1e9
        roof = {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": None, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
    else:
        achieved = amount / (stage_ms[top] * 1e-3) / 1e12
        roof = {"kernel": top, "bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "traffic": NCU_TRAFFIC.get((args.workload, top)),
                "traffic_note": "DRAM bytes of the stage (all its launches) from ncu captures (profiles/); "
                                "algorithmic: read B once, write XT once = %.3e" % (
                                    tile_elems * naux * 8.0 + npad * naux * noccp * 8.0),
                "peak_source": "FP64 DMMA: cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in MEASURED_PEAKS.json)"}
    cw = stage_ms.get("coulomb_w", 0.0) + stage_ms.get("coulomb_j", 0.0)
    coul = {"achieved_gbs": 2 * tile_elems * naux * 8.0 / (cw * 1e-3) / 1e9 if cw else None, "peak_gbs": hbm}
    if coul["achieved_gbs"]:
        coul["frac"] = coul["achieved_gbs"] / hbm

    # mixed precision form (tcgen05 split-BF16 exchange, FP64 Coulomb)
    mixed = None
    try:
        with ClockSampler(local) as mclk:
            msm = timed(rijk.PREC_MIXED, args.steps, 3)
        fb.sync()
        Km = dK.cpu().numpy().copy()
        fb.fock_device(dD.data_ptr(), dMO.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), rijk.PREC_FP64)
        fb.sync()
        K64 = dK.cpu().numpy()
        mstages = stage_times(rijk.PREC_MIXED)
        mtop = max(mstages, key=mstages.get)
        mixed = {"value": (1 if sharded else world) * 1e3 / msm, "unit": "builds/s", "ms_per_step": msm,
                 "speedup_vs_fp64": ms / msm,
                 "max_abs_dK_vs_fp64": float(np.max(np.abs(Km - K64))),
                 "exchange_energy_err": float(abs(np.sum(DM * (Km - K64)))),
                 "stage_ms": mstages, "top_kernel": mtop, "clocks": mclk.summary(),
                 "gpu_launches": fb.stats()["kernels_last_fock"] * args.steps}
        # every mixed kernel against its roofline; the tensor peak is the sustained (power-capped)
        # figure when the clocks sampled during the mixed timing show the power cap, else the burst one
        capped = "sw_power_cap" in (mclk.summary().get("reasons") or [])
        tpk = peaks.get("bf16_tflops_sustained" if capped else "bf16_tflops", 1590.0)
        tsrc = "MEASURED_PEAKS.json " + ("bf16_tflops_sustained (sw_power_cap seen)" if capped else "bf16_tflops")
        npad2 = ((npad + 127) // 128) * 128
        nb = npad2 // 128
        flops = {"xform_tc": 3 * 2.0 * noccp * npad2 * npad2 * naux,
                 "syrk_tc": 3 * 2.0 * naux * noccp * 128 * 128 * nb * (nb + 1) / 2,
                 "syrk_tc2": 3 * 2.0 * naux * noccp * 128 * 128 * nb * (nb + 1) / 2}
        mbytes = tile_elems * naux * 4.0  # hi + lo bf16 planes of the stored tiles
        xt_bytes = npad2 * naux * noccp * 4.0  # the split X^T, hi + lo
        ntile2 = nb * 2 * (nb * 2 + 1) // 2
        tbytes = {"xform_tc": mbytes + xt_bytes,  # read the split B once, write X^T once
                  "syrk_tc": xt_bytes + ntile2 * 4096 * 8.0,  # read X^T once, write K once
                  "syrk_tc2": xt_bytes + ntile2 * 4096 * 8.0}
        roofs = {}
        for k, v in mstages.items():
            if k in flops and v > 0:
                # the binding roofline of the two: tensor time or HBM time of the algorithmic bytes
                t_tc, t_mem = flops[k] / (tpk * 1e12), tbytes[k] / (hbm * 1e9)
                if t_tc >= t_mem:
                    ach = flops[k] / (v * 1e-3) / 1e12
                    roofs[k] = {"bound": "tensor", "achieved": ach, "peak": tpk, "unit": "TFLOP/s", "frac": ach / tpk,
                                "peak_source": tsrc, "bytes_frac": t_mem / (v * 1e-3)}
                else:
                    bw = tbytes[k] / (v * 1e-3) / 1e9
                    roofs[k] = {"bound": "hbm", "achieved": bw, "peak": hbm, "unit": "GB/s", "frac": bw / hbm,
                                "peak_source": "MEASURED_PEAKS.json hbm_gbs", "tensor_frac": t_tc / (v * 1e-3)}
            elif k in ("coulomb_w_mixed", "coulomb_j_mixed") and v > 0:
                bw = mbytes / (v * 1e-3) / 1e9
                roofs[k] = {"bound": "hbm", "achieved": bw, "peak": hbm, "unit": "GB/s", "frac": bw / hbm,
                            "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
        for k in roofs:
            roofs[k]["traffic"] = NCU_TRAFFIC.get((args.workload, k))
        mixed["rooflines"] = roofs
        if mtop in roofs:
            mixed["roofline"] = dict(roofs[mtop], kernel=mtop)
    except rijk.RijkError as e:
        mixed = {"unavailable": str(e)}

    # the FP64 form with K on tcgen05 tensor cores from int8 digit planes (RIJK_PREC_FP64_TC, opt-in)
    fp64tc = None
    if not sharded:
        try:
            mst = timed(rijk.PREC_FP64_TC, args.steps, 3)
            fb.sync()
            Kt = dK.cpu().numpy().copy()
            fb.fock_device(dD.data_ptr(), dMO.data_ptr(), nocc, dJ.data_ptr(), dK.data_ptr(), rijk.PREC_FP64)
            fb.sync()
            K64t = dK.cpu().numpy()
            fp64tc = {"value": 1e3 / mst, "unit": "builds/s", "ms_per_step": mst, "speedup_vs_fp64": ms / mst,
                      "max_abs_dK_vs_fp64": float(np.max(np.abs(Kt - K64t))),
                      "stage_ms": stage_times(rijk.PREC_FP64_TC),
                      "note": "slice_x = the int8 digits of X^T (8 per element); syrk_i8 = K from 36 exact s32 "
                              "digit products; J and the half-transform as the FP64 form"}
        except rijk.RijkError as e:
            fp64tc = {"unavailable": str(e)}

    # per-iteration errors of the mixed form along an FP64 SCF path: at each iteration's density both
    # forms are built; max |dJ|, max |dK| and the energy difference tr((2 dJ - dK) D) are recorded
    if isinstance(mixed, dict) and "unavailable" not in mixed and not sharded and not synthetic:
        s_, U_ = np.linalg.eigh(si.S)
        Xo = U_[:, s_ > 1e-10] / np.sqrt(s_[s_ > 1e-10])
        D0, R0 = si.sad()
        Jg, Kg = fb.dm_to_f_transform_ri(D0, R0, R0.shape[0])
        F = si.H + 2 * Jg - Kg
        rows = []
        nit = 12 if n <= 1024 else 6
        for it in range(nit):
            e_, Cp = np.linalg.eigh(Xo.T @ F @ Xo)
            Cm = (Xo @ Cp).T[:nocc].copy()
            Dm = Cm.T @ Cm
            J64, K64 = fb.dm_to_f_transform_ri(Dm, Cm, nocc, rijk.PREC_FP64)
            Jmx, Kmx = fb.dm_to_f_transform_ri(Dm, Cm, nocc, rijk.PREC_MIXED)
            dJm, dKm = Jmx - J64, Kmx - K64
            E64 = float(np.sum(Dm * (2 * si.H + 2 * J64 - K64))) + si.Enuc
            rows.append({"iteration": it, "energy_fp64": E64, "max_abs_dJ": float(np.max(np.abs(dJm))),
                         "max_abs_dK": float(np.max(np.abs(dKm))), "dE": float(np.sum(Dm * (2 * dJm - dKm)))})
            F = si.H + 2 * J64 - K64
        mixed["per_iteration"] = rows
        mixed["per_iteration_note"] = ("FP64 SCF path from the SAD start (plain diagonalisation); at each density the "
                                       "mixed build against the FP64 build, which matches the oracle to 1e-9")

    # SCF to convergence on the GPU (rijk_scf): FP64, and mixed builds switching to FP64
    scf = None
    if sharded:
        scf = {"skipped": "the SCF driver needs every aux function in one context"}
    elif not args.no_scf:
        out = {}
        E64 = None
        t0 = time.perf_counter()
        guess = si.sad()  # superposition of atomic densities (host, once per geometry)
        t_guess = time.perf_counter() - t0
        big = n > 1024
        fb.scf(si.H, si.S, nocc, si.Enuc, guess=guess)  # untimed first calls (work buffers, solver set-up)
        fb.scf(si.H, si.S, nocc, si.Enuc, guess=guess, converger=rijk.CONV_SOSCF)
        runs = [("fp64", rijk.PREC_FP64, rijk.CONV_DIIS), ("mixed_then_fp64", rijk.PREC_MIXED, rijk.CONV_DIIS),
                ("soscf_fp64", rijk.PREC_FP64, rijk.CONV_SOSCF),
                ("diis_mixed_then_soscf_fp64", rijk.PREC_MIXED, rijk.CONV_DIIS_SOSCF),
                ("diis_mixed_then_soscf_fp64tc", rijk.PREC_MIXED, rijk.CONV_DIIS_SOSCF)]
        if not big:
            runs.insert(3, ("soscf_mixed_then_fp64", rijk.PREC_MIXED, rijk.CONV_SOSCF))
        reps = 2 if big else 3
        for name, prec, conv in runs:
            # the last variant's FP64-accurate phase uses FP64_TC builds (K on the int8 tensor cores)
            fp64_phase = rijk.PREC_FP64_TC if name.endswith("fp64tc") else rijk.PREC_FP64
            el = None
            for _ in range(reps):  # the fastest of the runs: host-side latencies make single SCF timings noisy
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                E, _, r = fb.scf(si.H, si.S, nocc, si.Enuc, precision=prec, conv_dm_rms=1e-10, guess=guess,
                                 converger=conv, fp64_phase=fp64_phase)
                t = time.perf_counter() - t0
                if el is None or t < el:
                    el, r_best = t, r
            r = r_best
            out[name] = {"seconds": el, "iterations": r["iterations"], "iterations_mixed": r["iterations_mixed"],
                         "energy": E, "ms_fock": r["ms_fock"], "ms_diag": r["ms_diag_phase"],
                         "ms_inside": r["ms_total"], "ms_setup": r["ms_setup_phase"],
                         "ms_final": r["ms_final_phase"], "purified": r["purified"],
                         "converged": bool(r["converged"])}
            if name == "fp64":
                E64 = E
            else:
                out[name]["abs_dE_vs_fp64"] = abs(E - E64)
        out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds"] / min(
            out[k]["seconds"] for k in out if k.startswith(("mixed", "diis_mixed", "soscf_mixed")))
        out["criterion"] = ("DIIS: density RMS change < 1e-10; SOSCF (the reference's converger): max|4 F_ai| < 1e-7 "
                            "or |dE| < 1e-10; mixed runs switch to FP64 when the DIIS error / max|4 F_ai| < 1e-5; "
                            "diis_mixed_then_soscf_fp64: DIIS over the mixed builds, the SOSCF step and test after "
                            "the switch")
        out["start"] = "superposition of atomic densities (%.2f s on the host, not in the SCF time)" % t_guess
        out["timing"] = ("wall time of rijk_scf, the fastest of %d runs (ms_inside: the library's own clock of "
                         "that run, without argument checks and buffer release; ms_setup: before the first "
                         "iteration, uploads, overlap eigendecomposition and the guess's build and diagonalisation; "
                         "ms_final: after the last iteration, closing build and orbitals)" % reps)
        scf = out
    fb.close()
    del dD, dMO, dJ, dK, dJK
    torch.cuda.empty_cache()

    cpu = None
    if want_cpu:
        cpu = cpu_baseline_for(si, DM, MO, args.workload, args.seed, args.cpu_slices, args.cpu_seconds)

    extra = scf_small = grad_c40 = None
    if rank == 0 and world == 1 and not synthetic and args.extra not in ("none", "", args.workload):
        extra = extra_workload(args.extra, args.seed, dev, max(5, args.steps // 2), want_cpu, args.cpu_seconds / 2,
                               fp64_peak)
        if want_cpu and not args.no_scf:
            scf_small = scf_cpu_small(args.seed, dev)
        if not args.no_scf:
            grad_c40 = c40h82_grad(args.seed, dev, fp64_peak)

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
               "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
               "scaling": "strong" if sharded else "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": config_of(args.workload, n, naux, nocc, world, sharded, args.seed),
               "e2e": {"value": (1 if sharded else world) * 1e3 / ms_e2e, "unit": "builds/s",
                       "h2d_bytes_per_step": int((n * n + nocc * n) * 8), "d2h_bytes_per_step": int(2 * n * n * 8),
                       "host_buffers": "pinned"},
               "e2e_pageable": {"value": (1 if sharded else world) * 1e3 / ms_e2e_pg, "unit": "builds/s",
                                "steps": psteps, "host_buffers": "pageable numpy arrays"},
               "gpu_launches": launches,
               "roofline": roof, "coulomb_roofline": coul, "stage_ms": stage_ms,
               "mixed": mixed, "fp64_tc": fp64tc, "scf": scf, "cpu_baseline": cpu, "clocks": clk.summary(),
               "setup": {"path": "rijk_set_basis (GPU integrals)" if args.setup == "gpu" else "host integrals + rijk_set_3c",
                         "metric": "V^-1/2" if args.metric == "invsqrt" else "L^-1 (Cholesky)",
                         "wall_s": t_setup,
                         "gpu_integrals_ms": st0["ms_setup_ints"] if args.setup == "gpu" else None,
                         "metric_ms": st0["ms_setup_metric"], "b_ms": st0["ms_setup_3c"],
                         "host_integrals_s": tint, "host_ri_integrals": need_host_ri}}
        if cpu and "value" in cpu:
            out["ratio_vs_cpu"] = {"value": value / cpu["value"], "e2e": out["e2e"]["value"] / cpu["value"]}
        if extra is not None:
            out["extra_" + args.extra] = extra
        if scf_small is not None:
            out["scf_cpu_vs_gpu_h2o6"] = scf_small
        if grad_c40 is not None:
            out["grad_c40h82"] = grad_c40
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
