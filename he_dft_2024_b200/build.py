"""Build libhedft.so (sm_100a) in-tree with nvcc.

The library is the product path: hand-written CUDA kernels behind the C-ABI of include/he_dft.h.
It is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).

The build runs in two parallel stages:

1. the host translation units (he_dft.cu, he_noalloc.cu): the C-ABI, the orchestration and the
   light kernels.  They see the heavy kernel templates of csrc/kernels.cuh (stencils, FFT passes)
   as declarations only, so every heavy kernel they launch is an undefined symbol of their
   objects;
2. kernel translation units written into _build/: each defines HE_KERNEL_TU, includes
   kernels.cuh and explicitly instantiates a share of those undefined kernels (read with nm,
   demangled with c++filt), so exactly the launched kernels are compiled, spread over the
   machine's cores.

The objects are then linked into one shared library.
"""
import os
import re
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhedft.so")
SOURCES = ["he_dft.cu", "he_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# kernel templates instantiated in the kernel translation units (declared only in the host ones)
HEAVY = re.compile(r"^void he::(k_stencil|k_xpass|k_xpass_c|k_ypass|k_ypass_reg|k_zconv|k_zconv_reg|"
                   r"k_zmix|k_yzconv|k_xy_r2c|k_xy_c2r_pot|k_xy_c2r2_corr)<")


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_source_mtime():
    newest = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                newest = max(newest, os.path.getmtime(os.path.join(d, f)))
    return max(newest, os.path.getmtime(os.path.abspath(__file__)))


def _flags(extra):
    return [nvcc_path(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
            "-static-global-template-stub=false", "-Xcompiler", "-fPIC",
            "-I", os.path.join(ROOT, "include"), "-I", CSRC, *extra]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed: " + " ".join(cmd[-3:]))
    return r.stdout + r.stderr


def _undefined_kernels(objs):
    """Demangled signatures of the heavy kernels the objects launch but do not define."""
    found = set()
    for o in objs:
        mangled = subprocess.run(["nm", "-u", o], capture_output=True, text=True, check=True).stdout
        names = [ln.split()[-1] for ln in mangled.splitlines() if ln.strip()]
        dem = subprocess.run(["c++filt"], input="\n".join(names), capture_output=True, text=True,
                             check=True).stdout.splitlines()
        found.update(d for d in dem if HEAVY.match(d))
    return sorted(found)


def _kernel_units(sigs, nunits):
    """Write the kernel translation units; signature k goes to unit k mod nunits (each family
    spreads over every unit)."""
    os.makedirs(BUILD, exist_ok=True)
    paths = []
    for u in range(nunits):
        body = [f"// Generated by build.py: explicit instantiations, unit {u + 1} of {nunits}.",
                "#define HE_KERNEL_TU", '#include "kernels.cuh"', ""]
        body += ["template __global__ " + s + ";" for s in sigs[u::nunits]]
        path = os.path.join(BUILD, f"kernels_{u}.cu")
        with open(path, "w") as f:
            f.write("\n".join(body) + "\n")
        paths.append(path)
    return paths


def build(force=False, verbose=False, extra=(), jobs=None):
    """Compile libhedft.so unless it is newer than every source."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_source_mtime():
        return LIB
    jobs = jobs or min(16, max(2, os.cpu_count() or 2))
    os.makedirs(BUILD, exist_ok=True)
    base = _flags(extra)
    host_objs = [os.path.join(BUILD, s.replace(".cu", ".o")) for s in SOURCES]
    log = []
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        log += ex.map(lambda so: _run(base + ["-c", "-o", so[1], os.path.join(CSRC, so[0])], verbose),
                      zip(SOURCES, host_objs))
        sigs = _undefined_kernels(host_objs)
        units = _kernel_units(sigs, max(1, min(jobs, len(sigs))))
        kern_objs = [u[:-3] + ".o" for u in units]
        log += ex.map(lambda uo: _run(base + ["-c", "-o", uo[1], uo[0]], verbose), zip(units, kern_objs))
    _run([nvcc_path(), *ARCH, "-shared", "-o", LIB + ".tmp", *host_objs, *kern_objs], verbose)
    if verbose:
        out = "".join(log).strip()
        if out:
            print(out)
        print(f"{len(sigs)} kernel instantiations in {len(units)} units")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=("-Xptxas", "-v") if "--ptxas" in sys.argv else ())
