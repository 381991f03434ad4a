"""Build libsoup_b200.so in-tree with nvcc for sm_100a.

    python build.py            # incremental: objects are rebuilt when a source or header changed

Objects go to csrc/_build/, the library to the package directory (beside _abi.py).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(PKG, "libsoup_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "--expt-relaxed-constexpr",
         "-ccbin", "/usr/bin/g++"]
SOURCES = ["soup_capi.cu", "kernels_grid.cu", "kernels_force.cu", "kernels_step.cu", "kernels_bonds.cu",
           "kernels_sweep.cu", "kernels_analysis.cu", "kernels_observables.cu", "kernels_adjoint.cu", "kernels_noalloc.cu", "host_init.cpp"]
HEADERS = ["soup_internal.h", "soup_common.cuh", os.path.join("..", "..", "include", "soup_b200.h")]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(HERE, h) for h in HEADERS]
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, extra=None):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    procs = []
    for s in SOURCES:
        src = os.path.join(HERE, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if _stale(obj, src):
            cmd = [NVCC] + ARCH + FLAGS + (extra or []) + ["-c", src, "-o", obj]
            if s.endswith(".cpp"):
                cmd = [NVCC] + FLAGS + ["-x", "c++", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(out.decode())
        elif verbose and out:
            sys.stdout.write(out.decode())
    if failed:
        raise RuntimeError("nvcc failed")
    if procs or not os.path.exists(OUT):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-cudart", "static", "-ccbin", "/usr/bin/g++"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
