"""Build libdrift_pt.so in-tree with nvcc for sm_100a.

    python -m drift_b200.build

The library is loaded by ``drift_b200._lib`` through ctypes. It is built in the package directory
(not pip-installed, not a JIT cache) so that the built file travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_PATH = os.path.join(HERE, "libdrift_pt.so")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = ["dpt_host.cpp", "dpt_kernels.cu", "dpt_capi.cu", "dpt_noalloc.cu", "dpt_batched.cu", "dpt_multispin.cu",
           "dpt_sk_host.cpp", "dpt_sk.cu", "dpt_gemm.cu", "dpt_made.cu", "dpt_gms_host.cpp", "dpt_gms.cu",
           "dpt_batch_mh.cu", "dpt_batch_host.cpp", "dpt_unit_host.cpp"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdrift_pt.so")
    return cand


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


CLI_PATH = os.path.join(HERE, "ising_pt")


def build_cli(force: bool = False, verbose: bool = False) -> str:
    """The `ising_pt` command-line twin of the reference executable, linked against libdrift_pt.so."""
    src = os.path.join(CSRC, "ising_pt_cli.cpp")
    deps = [src, LIB_PATH, os.path.join(os.path.dirname(HERE), "include", "drift_pt.h")]
    if not force and not _stale(CLI_PATH, deps):
        return CLI_PATH
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        raise RuntimeError("a C++ compiler is required to build the ising_pt command")
    cmd = [cxx, "-O2", "-std=c++17", "-o", CLI_PATH + ".tmp", src, "-L" + HERE, "-ldrift_pt",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building ising_pt failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    os.replace(CLI_PATH + ".tmp", CLI_PATH)
    return CLI_PATH


# A profiling build of the same sources with the dense kernel's hand-off stamps compiled in
# (drift_b200/sk_stamps.py reads them); the product library never has them.
SK_STAMP_LIB_PATH = os.path.join(HERE, "libdrift_pt_skstamp.so")


def build(force: bool = False, verbose: bool = False, sk_stamps: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "drift_pt.h"))
    out = SK_STAMP_LIB_PATH if sk_stamps else LIB_PATH
    if not force and not _stale(out, deps):
        return out
    tmp = out + ".tmp"
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH_FLAGS, "-lineinfo", "-shared", *(["-DDPT_SK_STAMPS"] if sk_stamps else []),
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fvisibility=hidden",
           "--expt-relaxed-constexpr", "-o", tmp, *srcs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    if "--sk-stamps" in sys.argv:
        print(build(force="--force" in sys.argv, verbose=True, sk_stamps=True))
    else:
        print(build(force="--force" in sys.argv, verbose=True))
        print(build_cli(force="--force" in sys.argv, verbose=True))
