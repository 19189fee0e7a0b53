"""Build the libraries for sm_100a: ``msmpb_b200/libmsmpb.so`` (MSM) and
``msmpb_b200/libpme.so`` (the smooth-PME comparator).

Every .cu/.cpp under msmpb_b200/csrc (and csrc/pme) is compiled with nvcc
(``-gencode arch=compute_100a,code=sm_100a -lineinfo``) into
msmpb_b200/_build/. libmsmpb.so links the engine and kernels with the MSM C
ABI (forcefield.h, msmpb_b200.h: ff_api.cpp, batch.cpp, noalloc.cu);
libpme.so links the same engine and kernels with the PME C ABI (pme.h,
pme_b200.h: csrc/pme/). The two export the same FF_* names for their own
methods, as the reference's two builds do. CUDA runtime is linked
statically so the libraries load on any box with the driver.

Usage: python -m msmpb_b200.build [--force] [-j N] [--verbose]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmsmpb.so")
PME_LIB = os.path.join(PKG, "libpme.so")
PME_SRC = os.path.join(CSRC, "pme")
# MSM C ABI, not linked into libpme.so
MSM_ONLY = ("ff_api.cpp", "batch.cpp", "noalloc.cu")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O3", "--expt-relaxed-constexpr",
         "-I", INCLUDE, "-I", CSRC]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def sources():
    out = []
    for d in (CSRC, PME_SRC):
        for f in sorted(os.listdir(d)):
            if f.endswith((".cu", ".cpp")):
                out.append(os.path.join(d, f))
    return out


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
          if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)
           if f.endswith(".h")]
    return hs


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0)


def _compile(src, obj, verbose, extra):
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return r.stderr


def build(force=False, jobs=None, verbose=False, extra=None):
    extra = list(extra or [])
    os.makedirs(BUILD, exist_ok=True)
    hdr_time = _newest(headers())
    srcs = sources()
    todo = []
    objs = []
    for s in srcs:
        obj = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(obj)
        if (force or not os.path.exists(obj) or
                os.path.getmtime(obj) < max(os.path.getmtime(s), hdr_time)):
            todo.append((s, obj))
    jobs = jobs or min(8, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, s, o, verbose, extra) for s, o in todo]
        for f in futs:
            msg = f.result()
            if verbose and msg:
                print(msg)
    msm_objs = [o for s, o in zip(srcs, objs) if os.path.dirname(s) == CSRC]
    pme_objs = [o for s, o in zip(srcs, objs)
                if os.path.basename(s) not in MSM_ONLY]
    for lib, lobjs in ((LIB, msm_objs), (PME_LIB, pme_objs)):
        if todo or not os.path.exists(lib) or os.path.getmtime(lib) < _newest(lobjs):
            cmd = [nvcc(), *ARCH, "-shared", "-o", lib, *lobjs, "-cudart", "static"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas else []
    try:
        print(build(a.force or a.ptxas, a.j, a.verbose or a.ptxas, extra))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
