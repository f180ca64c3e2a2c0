"""Build recipe for the native libraries, in-tree.

  nopt_b200/libgto_ints.so   host integral engine (g++, OpenMP)
  nopt_b200/librijk.so       the RI-JK Fock build: sm_100a kernels + C ABI (nvcc)

Everything is compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INC = os.path.join(ROOT, "include")
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SOURCES = ["host/gto_ints.cpp", "host/gto_guess.cpp"]
CUDA_SOURCES = [
    "rijk/rijk_api.cu",
    "rijk/k_pack.cu",
    "rijk/k_metric.cu",
    "rijk/k_coulomb.cu",
    "rijk/k_exchange_f64.cu",
    "rijk/k_exchange_tc.cu",
    "rijk/k_exchange_i8.cu",
    "rijk/k_scf.cu",
    "rijk/k_adjoint.cu",
    "rijk/k_moints.cu",
    "rijk/rijk_noalloc.cu",
    "rijk/k_eri.cu",
    "rijk/k_mo_ri.cu",
    "rijk/rijk_cache.cu",
    "rijk/rijk_selftest.cu",
    "rijk/k_gemm.cu",
    "rijk/rijk_stream3c.cu",
]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = list(srcs)
    for d in (INC, os.path.join(CSRC, "rijk"), os.path.join(CSRC, "host")):
        if os.path.isdir(d):
            deps += [os.path.join(d, f) for f in os.listdir(d)]
    return any(os.path.getmtime(s) > t for s in deps if os.path.exists(s))


def build_host(force=False):
    out = os.path.join(HERE, "libgto_ints.so")
    srcs = [os.path.join(CSRC, s) for s in HOST_SOURCES]
    if force or _stale(out, srcs):
        _run(["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17", "-Wall",
              "-I" + INC] + srcs + ["-o", out])
    return out


def _headers():
    out = []
    for d in (INC, os.path.join(CSRC, "rijk"), os.path.join(CSRC, "host")):
        if os.path.isdir(d):
            out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return out


def build_cuda(force=False, extra=()):
    """Compiles each stale object (older than its source or any header) in parallel, then links."""
    from concurrent.futures import ThreadPoolExecutor
    out = os.path.join(HERE, "librijk.so")
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    hdr_t = max([os.path.getmtime(h) for h in _headers()] or [0.0])
    jobs, objs = [], []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t):
            jobs.append([NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                         "-Xcompiler", "-fvisibility=hidden", "-I" + INC,
                                         "-I" + os.path.join(CSRC, "rijk"), "-I" + os.path.join(CSRC, "host"),
                                         "--expt-relaxed-constexpr", "-c", s, "-o", o] + list(extra))
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(_run, jobs))
    if jobs or not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(o) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-lcusolver", "-lcublas", "-lcudart"])
    return out


def build(force=False):
    build_host(force)
    build_cuda(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
