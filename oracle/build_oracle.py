"""Build recipe for the oracle (test infrastructure only).

* ``oracle/liblu2oracle.so``: the plain-C restatement ``lu2_oracle.c``.
* ``oracle/_ref/``: the UNMODIFIED reference sources (telmin/lu2), compiled
  where they lie under the reference checkout, together with
  ``ref_harness.c``, into two shared libraries:

  - ``libref_lu2_shipped.so``: the reference as shipped;
  - ``libref_lu2_fixed.so``: the same, except that ``lu2tlib.c`` is first
    copied into ``oracle/_ref/`` with the one-token fix
    ``findpivot(n,a,ii)`` -> ``findpivot(n,a+ip,ii)`` (the pivot of the
    second column of each 2-column leaf is then searched in that column).

  The reference's own build system is not run.  It needs only a CBLAS for
  ``cblas_dgemm``/``cblas_idamax``; ``oracle/refinc/cblas.h`` declares them and
  the OpenBLAS 0.3.15 shared library that ships inside the Python environment
  (opencv-python-headless wheel) defines them.  Compile flags follow the
  reference's Makefile.common:39-40,85-86 (-O2 -DTIMETEST -DREAL=double
  -fopenmp, -funroll-loops for lu2lib.c).

``oracle/_ref/`` is git-ignored; it travels to GPU machines with the working
tree, where the reference checkout does not exist.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the telmin/lu2 checkout: LU2_REFERENCE_DIR, else a directory "reference"
# beside this repository
REF_DIR = os.environ.get("LU2_REFERENCE_DIR",
                         os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
OUT_DIR = os.path.join(HERE, "_ref")

REF_SOURCES = ["lu2lib.c", "timerlib.c", "second.c", "lu2_mp_nompi.c"]


def find_openblas() -> str | None:
    """Locate an unprefixed-CBLAS OpenBLAS shared library in this environment."""
    roots = {sys.prefix, os.path.dirname(os.path.dirname(os.__file__))}
    pats = []
    for r in roots:
        pats += glob.glob(os.path.join(r, "lib", "python3*", "site-packages", "*.libs", "libopenblas*.so*"))
    for p in sorted(pats):
        try:
            out = subprocess.run(["nm", "-D", "--defined-only", p], capture_output=True, text=True).stdout
        except OSError:
            continue
        if " cblas_dgemm" in out and " cblas_idamax" in out and " openblas_set_num_threads" in out:
            return p
    return None


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def build_oracle(verbose: bool = False) -> str:
    out = os.path.join(HERE, "liblu2oracle.so")
    src = os.path.join(HERE, "lu2_oracle.c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-std=gnu11", "-o", out, src, "-lm"])
        if verbose:
            print("built", out)
    return out


def build_ref(verbose: bool = False) -> dict:
    """Compile the reference into oracle/_ref/.  Returns {'shipped': path, 'fixed': path}
    or raises RuntimeError when the reference or OpenBLAS is absent."""
    if not os.path.isdir(REF_DIR):
        raise RuntimeError("reference sources not present at %s" % REF_DIR)
    blas = find_openblas()
    if blas is None:
        raise RuntimeError("no OpenBLAS with an unprefixed CBLAS found")
    os.makedirs(OUT_DIR, exist_ok=True)
    cflags = ["-O2", "-fPIC", "-w", "-std=gnu89", "-fopenmp", "-DTIMETEST", "-DUNIX", "-DREAL=double",
              "-I" + os.path.join(HERE, "refinc"), "-I" + REF_DIR]
    objs = []
    for s in REF_SOURCES:
        o = os.path.join(OUT_DIR, s.replace(".c", ".o"))
        extra = ["-funroll-loops"] if s == "lu2lib.c" else []
        _run(["gcc"] + extra + cflags + ["-c", os.path.join(REF_DIR, s), "-o", o])
        objs.append(o)
    lu2o = os.path.join(OUT_DIR, "lu2_nomain.o")
    _run(["gcc"] + cflags + ["-Dmain=lu2_reference_main", "-c", os.path.join(REF_DIR, "lu2.c"), "-o", lu2o])
    tlib = os.path.join(OUT_DIR, "lu2tlib.o")
    _run(["gcc"] + cflags + ["-c", os.path.join(REF_DIR, "lu2tlib.c"), "-o", tlib])
    # the fixed variant: a patched copy of lu2tlib.c in the build directory
    with open(os.path.join(REF_DIR, "lu2tlib.c")) as f:
        text = f.read()
    bug = "findpivot(n,a,ii)"
    if text.count(bug) != 1:
        raise RuntimeError("expected exactly one '%s' in lu2tlib.c" % bug)
    fixed_src = os.path.join(OUT_DIR, "lu2tlib_fixed.c")
    with open(fixed_src, "w") as f:
        f.write(text.replace(bug, "findpivot(n,a+ip,ii)"))
    tlibf = os.path.join(OUT_DIR, "lu2tlib_fixed.o")
    _run(["gcc"] + cflags + ["-c", fixed_src, "-o", tlibf])
    harn = os.path.join(OUT_DIR, "ref_harness.o")
    _run(["gcc", "-O2", "-fPIC", "-std=gnu11", "-c", os.path.join(HERE, "ref_harness.c"), "-o", harn])
    blas_dir = os.path.dirname(blas)
    res = {}
    for name, t in (("shipped", tlib), ("fixed", tlibf)):
        so = os.path.join(OUT_DIR, "libref_lu2_%s.so" % name)
        _run(["gcc", "-shared", "-fopenmp", "-o", so, harn, lu2o, t] + objs +
             [blas, "-Wl,--disable-new-dtags,-rpath," + blas_dir, "-lpthread", "-lm"])
        res[name] = so
    with open(os.path.join(OUT_DIR, "BUILD_INFO.txt"), "w") as f:
        f.write("reference: %s\nopenblas: %s\n" % (REF_DIR, blas))
    if os.path.exists(GPU_LIB):
        res.update(build_dropin(cflags, objs, lu2o, tlib, blas, verbose))
    if verbose:
        print("built", res)
    return res


GPU_LIB = os.path.join(os.path.dirname(HERE), "lu2_b200", "liblu2gpu.so")


def build_dropin(cflags: list[str], objs: list[str], lu2o: str, tlib: str, blas: str, verbose: bool) -> dict:
    """The reference's own programs linked against the GPU library, as a
    maintainer would link them (no reference source is edited):

    * ``lu2_gdr``: the reference's GDR build (Makefile.common:47-48, 69-70,
      87-88: lu2.o lu2tlib.o ... lu2lib_gdr.o gdrdgemm.o, lu2lib.c with
      -DUSEGDR) with liblu2gpu.so in place of the GRAPE-DR library
      ($(GDRLIBS)): mydgemm sends k > 512 products through mygdrdgemm to the
      GPU's gdr_dgemm_ (lu2lib.c:2097-2100).
    * ``libref_lu2_gdr.so``: the same objects with ref_harness.c instead of
      main, so tests can read its pivots and x.
    * ``lu2_gpu``: lu2.c's main with lumcolumn from liblu2gpu.so: lu2.c built
      with -Dlumcolumn=lumcolumn_cpu, that symbol weakened, and
      dropin_lumcolumn.c's strong lumcolumn_cpu forwarding to the library.
    """
    lib_dir = os.path.dirname(GPU_LIB)
    gdr_lib = os.path.join(OUT_DIR, "lu2lib_gdr.o")
    _run(["gcc", "-funroll-loops"] + cflags + ["-DUSEGDR", "-c", os.path.join(REF_DIR, "lu2lib.c"), "-o", gdr_lib])
    gdrdgemm = os.path.join(OUT_DIR, "gdrdgemm.o")
    _run(["gcc"] + cflags + ["-c", os.path.join(REF_DIR, "gdrdgemm.c"), "-o", gdrdgemm])
    lu2main = os.path.join(OUT_DIR, "lu2_main.o")
    _run(["gcc"] + cflags + ["-c", os.path.join(REF_DIR, "lu2.c"), "-o", lu2main])
    base = [o for o in objs if not o.endswith("lu2lib.o")]  # timerlib, second, lu2_mp_nompi
    gpu_link = ["-L" + lib_dir, "-llu2gpu", "-Wl,--disable-new-dtags,-rpath,$ORIGIN/../../lu2_b200"]
    blas_link = [blas, "-Wl,-rpath," + os.path.dirname(blas), "-lpthread", "-lm"]
    out = {}
    exe = os.path.join(OUT_DIR, "lu2_gdr")
    _run(["gcc", "-fopenmp", "-o", exe, lu2main, tlib, gdr_lib, gdrdgemm] + base + gpu_link + blas_link)
    out["lu2_gdr"] = exe
    so = os.path.join(OUT_DIR, "libref_lu2_gdr.so")
    harn = os.path.join(OUT_DIR, "ref_harness.o")
    _run(["gcc", "-shared", "-fopenmp", "-o", so, harn, lu2o, tlib, gdr_lib, gdrdgemm] + base + gpu_link + blas_link)
    out["gdr"] = so
    gpumain = os.path.join(OUT_DIR, "lu2_gpu_main.o")
    _run(["gcc"] + cflags + ["-Dlumcolumn=lumcolumn_cpu", "-c", os.path.join(REF_DIR, "lu2.c"), "-o", gpumain])
    _run(["objcopy", "--weaken-symbol=lumcolumn_cpu", gpumain])
    shim = os.path.join(OUT_DIR, "dropin_lumcolumn.o")
    _run(["gcc", "-O2", "-fPIC", "-c", os.path.join(HERE, "dropin_lumcolumn.c"), "-o", shim])
    exe2 = os.path.join(OUT_DIR, "lu2_gpu")
    lu2lib = [o for o in objs if o.endswith("lu2lib.o")]
    _run(["gcc", "-fopenmp", "-o", exe2, gpumain, shim, tlib] + lu2lib + base + gpu_link + blas_link)
    out["lu2_gpu"] = exe2
    if verbose:
        print("built", out)
    return out


def main() -> int:
    build_oracle(verbose=True)
    try:
        build_ref(verbose=True)
    except RuntimeError as e:
        print("oracle/_ref not built:", e)
    return 0


if __name__ == "__main__":
    sys.exit(main())
