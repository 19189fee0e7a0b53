"""Build the reference MSM library into oracle/_ref/ (test infrastructure only).

The reference (hkayabilisim/msmpb, MIT) is plain C99: code/forcefield0.c,
code/forcefield1.c, code/forcefield.h and the driver code/msmpb.c. Its only
external dependency, FFTW3 (environment/Dockerfile:10, unpinned Ubuntu 18.04
``libfftw3-dev``), is absent here, so the project-written FFT in
oracle/fftw_shim/ stands in for the five FFTW symbols it uses.

forcefield0.c and msmpb.c compile unmodified from where they lie. forcefield1.c
gets two minimal index patches, written to oracle/_ref/src/ (git-ignored, never
committed):

* P1 (code/forcefield1.c:195-204): at maxLevel == 1 the grid-energy loop must
  index q[1] with the (nu-1) padding / (nu/2-1) offset that anterpolate()
  allocated and filled (code/forcefield1.c:143, :339-345).
* P2 (code/forcefield1.c:504-514): at maxLevel > 1 restrict_() writes the top
  level unpadded (code/forcefield1.c:408-415 with sd = of = 0), so FFTg2g must
  read it unpadded.

With both patches the build reproduces the published Box44 energies of
results/TableII.json and results/Figure6.json. The unpatched library is also
built, to report the deviation.

Outputs (all under oracle/_ref/):
  libmsmpb_ref.so            patched library (+ ``struct O o`` definition)
  libmsmpb_ref_unpatched.so  unpatched library
  msmpb_ref                  the reference CLI driver over the patched sources
  msmpb_dropin               the same driver source, unmodified, compiled against
                             this project's include/forcefield.h and linked to
                             msmpb_b200/libmsmpb.so (the drop-in check of the CLI)
  libpme_ref.so              the reference smooth-PME comparator (code/pme0.c,
                             code/pme1.c, unmodified) with the FFT shim
  pme_ref                    its CLI driver (code/pme.c) over those sources
  pme_dropin                 code/pme.c, unmodified, compiled against this
                             project's include/pme.h and linked to
                             msmpb_b200/libpme.so
  src/lib/                   the sources of the patched library (forcefield0.c
                             and forcefield.h copied, forcefield1.c patched),
                             so that ``build_native()`` can rebuild it where
                             the reference tree is absent
  native/libmsmpb_ref_native.so  that rebuild with -march=native for the host
                             it runs on (made on demand by bench.py's CPU arms)

Usage: python oracle/build_ref.py [--reference DIR]   (default: $MSMPB_REFERENCE)
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "fftw_shim")

P1_ANCHOR = "  int ofz = padz / 2 ;\n"
P1_ADD = ("  if (ff->maxLevel == 1) { padx = pady = padz = nu - 1;"
          " ofx = ofy = ofz = nu/2 - 1; }\n")
P2_ANCHOR = "  int ofz = nu/2 - 1;\n"
P2_ADD = ("  int px = nu - 1, py = nu - 1, pz = nu - 1;\n"
          "  if (ff->maxLevel > 1) { ofx = ofy = ofz = 0; px = py = pz = 0; }\n")
P2_OLD = "ql[((i+ofx)*(gd.y + nu-1) + (j+ofy))*(gd.z + nu - 1) + k + ofz]"
P2_NEW = "ql[((i+ofx)*(gd.y + py) + (j+ofy))*(gd.z + pz) + k + ofz]"

CFLAGS = ["-O3", "-std=gnu11", "-fPIC", "-w"]

# where the reference project lies: the MSMPB_REFERENCE environment variable,
# else the read-only checkout of this build container
REFERENCE = os.environ.get("MSMPB_REFERENCE", "/root/reference")


def _replace_once(text, old, new):
    if text.count(old) != 1:
        raise RuntimeError("patch anchor not found exactly once: %r" % old)
    return text.replace(old, new)


def patch_forcefield1(src_text):
    text = src_text.replace("\r\n", "\n")
    text = _replace_once(text, P1_ANCHOR, P1_ANCHOR + P1_ADD)
    text = _replace_once(text, P2_ANCHOR, P2_ANCHOR + P2_ADD)
    text = _replace_once(text, P2_OLD, P2_NEW)
    return text


def run(cmd):
    subprocess.run(cmd, check=True)


def build(reference_root=REFERENCE, quiet=False):
    code = os.path.join(reference_root, "code")
    ff0 = os.path.join(code, "forcefield0.c")
    ff1 = os.path.join(code, "forcefield1.c")
    drv = os.path.join(code, "msmpb.c")
    if not all(os.path.exists(p) for p in (ff0, ff1, drv)):
        if not quiet:
            print("build_ref: reference sources not present; skipped")
        return False
    src_dir = os.path.join(OUT, "src")
    os.makedirs(src_dir, exist_ok=True)
    with open(ff1, "r", newline="") as f:
        patched = patch_forcefield1(f.read())
    ff1p = os.path.join(src_dir, "forcefield1_patched.c")
    with open(ff1p, "w") as f:
        f.write(patched)
    glue = os.path.join(src_dir, "ref_glue.c")
    with open(glue, "w") as f:
        f.write('#include "forcefield.h"\n'
                '/* the library reads o.test (code/forcefield0.c:469); the\n'
                '   drivers define o (code/msmpb.c:9), a bare library must */\n'
                'struct O o = {"none"};\n')
    # the library's sources in a directory of their own (the drop-in driver
    # copies below must not see the reference header beside them)
    lib_src = os.path.join(src_dir, "lib")
    os.makedirs(lib_src, exist_ok=True)
    for f in ("forcefield0.c", "forcefield.h"):
        shutil.copy(os.path.join(code, f), os.path.join(lib_src, f))
    for f in ("forcefield1_patched.c", "ref_glue.c"):
        shutil.copy(os.path.join(src_dir, f), os.path.join(lib_src, f))
    inc = ["-I", SHIM, "-I", code]
    fft = os.path.join(SHIM, "fft_shim.c")
    cc = os.environ.get("CC", "gcc")
    run([cc, *CFLAGS, "-shared", *inc, ff0, ff1p, fft, glue, "-lm",
         "-o", os.path.join(OUT, "libmsmpb_ref.so")])
    run([cc, *CFLAGS, "-shared", *inc, ff0, ff1, fft, glue, "-lm",
         "-o", os.path.join(OUT, "libmsmpb_ref_unpatched.so")])
    run([cc, *CFLAGS, *inc, drv, ff0, ff1p, fft, "-lm",
         "-o", os.path.join(OUT, "msmpb_ref")])
    # the unmodified driver against this project's header and library; a
    # scratch copy, so that its quoted include finds include/forcefield.h
    root = os.path.dirname(HERE)
    our_lib_dir = os.path.join(root, "msmpb_b200")
    if os.path.exists(os.path.join(our_lib_dir, "libmsmpb.so")):
        drv_copy = os.path.join(src_dir, "msmpb_dropin.c")
        shutil.copy(drv, drv_copy)
        run([cc, "-O2", "-std=gnu11", "-w", "-I", os.path.join(root, "include"), drv_copy,
             "-L", our_lib_dir, "-lmsmpb", "-lm", "-Wl,-rpath,$ORIGIN/../../msmpb_b200",
             "-o", os.path.join(OUT, "msmpb_dropin")])
    build_pme(code, src_dir, inc, fft, cc, root)
    if not quiet:
        print("build_ref: built", OUT)
    return True


def build_native(quiet=True):
    """Rebuild the patched reference library from oracle/_ref/src/ with
    ``-O3 -march=native`` for the host this runs on (the portable build above
    uses -O3 only, since it may run on another machine). Returns the library
    path, or None when the sources or the compiler are missing."""
    src_dir = os.path.join(OUT, "src", "lib")
    srcs = [os.path.join(src_dir, f) for f in
            ("forcefield0.c", "forcefield1_patched.c", "ref_glue.c")]
    if not all(os.path.exists(p) for p in srcs + [os.path.join(src_dir, "forcefield.h")]):
        return None
    out_dir = os.path.join(OUT, "native")
    os.makedirs(out_dir, exist_ok=True)
    lib = os.path.join(out_dir, "libmsmpb_ref_native.so")
    cc = os.environ.get("CC", "gcc")
    cmd = [cc, *CFLAGS, "-march=native", "-shared", "-I", SHIM, "-I", src_dir, *srcs,
           os.path.join(SHIM, "fft_shim.c"), "-lm", "-o", lib + ".tmp"]
    try:
        subprocess.run(cmd, check=True, capture_output=quiet)
        os.replace(lib + ".tmp", lib)
    except (OSError, subprocess.CalledProcessError):
        return None
    return lib


def build_pme(code, src_dir, inc, fft, cc, root):
    """The PME comparator: library, driver and drop-in driver."""
    p0, p1, drv = (os.path.join(code, f) for f in ("pme0.c", "pme1.c", "pme.c"))
    if not all(os.path.exists(p) for p in (p0, p1, drv)):
        return
    glue = os.path.join(src_dir, "pme_glue.c")
    with open(glue, "w") as f:
        f.write('#include "pme.h"\n'
                '/* the drivers define o (code/pme.c:9); a bare library must */\n'
                'struct O o = {"none"};\n')
    run([cc, *CFLAGS, "-shared", *inc, p0, p1, fft, glue, "-lm",
         "-o", os.path.join(OUT, "libpme_ref.so")])
    run([cc, *CFLAGS, *inc, drv, p0, p1, fft, "-lm", "-o", os.path.join(OUT, "pme_ref")])
    our_lib_dir = os.path.join(root, "msmpb_b200")
    if os.path.exists(os.path.join(our_lib_dir, "libpme.so")):
        drv_copy = os.path.join(src_dir, "pme_dropin.c")
        shutil.copy(drv, drv_copy)
        run([cc, "-O2", "-std=gnu11", "-w", "-I", os.path.join(root, "include"), drv_copy,
             "-L", our_lib_dir, "-l:libpme.so", "-lm", "-Wl,-rpath,$ORIGIN/../../msmpb_b200",
             "-o", os.path.join(OUT, "pme_dropin")])


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REFERENCE)
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args()
    if a.clean and os.path.isdir(OUT):
        shutil.rmtree(OUT)
    sys.exit(0 if build(a.reference) else 1)
