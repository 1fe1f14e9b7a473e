"""Builds the engine's shared library scamper_b200/libgpumc.so with nvcc for
sm_100a (and the CPU oracle used by the tests, when asked).  The library is
built in-tree so that it travels with the repository snapshot."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["capi.cu", "sim.cu", "server.cu", "sweep_discrete.cu", "sweep_o3.cu",
           "sweep_msc.cu", "lattice_ops.cu", "noalloc.cu",
           "sweep_ising_bits.cu", "sweep_potts_bits.cu", "cluster.cu"]
LIB = os.path.join(HERE, "libgpumc.so")
LIB_BOUNDS = os.path.join(HERE, "libgpumc_bounds.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr", "-static-global-template-stub=false",
         "-I", os.path.join(ROOT, "include")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force=False, verbose=False, jobs=None, bounds=False):
    """Builds libgpumc.so, or with bounds=True the bounds-checked
    libgpumc_bounds.so (-DGPUMC_DEBUG_BOUNDS: out-of-range accesses of the
    kernels are skipped and counted, gpumc_debug_bounds reports them)."""
    lib = LIB_BOUNDS if bounds else LIB
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "gpumc.h")]
    if not force and not _stale(lib, deps):
        return lib
    objdir = os.path.join(HERE, "_build_bounds" if bounds else "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    extra = ["-DGPUMC_DEBUG_BOUNDS"] if bounds else []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [NVCC, *FLAGS, *extra, "-rdc=false", "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib, *objs,
           "-Xcompiler", "-fPIC", "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    subprocess.run(cmd, check=True)
    return lib


def build_oracle():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return os.path.join(ROOT, "oracle", "liboracle.so")


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True, bounds="--bounds" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle()
