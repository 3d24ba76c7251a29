"""Build recipe for the compiled SIFEL reference used as a checker.

Test infrastructure only: nothing in the product library imports, links or
runs what this script builds.  It compiles SIFEL's own GEFEL, MEFEL and TRFEL
sources *where they lie* in the read-only reference checkout with plain
``g++`` (the reference's Makefiles are read only to learn their ``SRCS``
lists; their build system is not run) and writes every output under
``oracle/_ref/``:

* ``obj/<module>/*.o``                 -- one object per reference source;
* ``libgef.a``, ``libmef.a``, ``libtrf.a`` -- static archives of the above;
* ``mefel_ref`` / ``trfel_ref``          -- the reference programs, unchanged
  ``main`` from ``MEFEL/SRC/mefel.cpp`` and ``TRFEL/SRC/trfel.cpp``;
* ``mefel_dump`` / ``trfel_dump``        -- in-process harnesses
  (``oracle/ref_harness_mefel.cpp``, ``oracle/ref_harness_trfel.cpp``) that
  run the reference pipeline on a deck and dump K, f, u and timings;
* ``libsifelref.so``                   -- GEFEL compiled position-independent
  plus ``oracle/ref_solver_capi.cpp``: a C entry point into the reference's
  own ``symcomprow::cg_prec`` / ``comprow::cg_prec`` for timing the CPU
  baseline on exactly the arrays the GPU path receives;
* ``mefel_dump_gpu`` / ``trfel_dump_gpu`` -- the MEFEL / TRFEL harness and
  SIFEL's objects linked with the drop-in binding
  ``ssf_b200/integration/sifel_gpu_shim.cpp`` (``-Wl,--wrap`` of
  ``symcomprow::cg_prec``) and, for MEFEL, the assembly binding
  ``ssf_b200/integration/sifel_gpu_assembly.cpp`` (``-Wl,--wrap`` of
  ``stiffness_matrix``): SIFEL's own front end on a deck, with the assembly
  and the solves on the GPU.  Run only by the drop-in tests.

Only one compile-environment shim is needed: ``GEFEL/cc.cpp`` includes
``umfpack.h`` unconditionally although every use sits under ``INC_CHMD``;
``oracle/ref_compat/umfpack.h`` is an empty stand-in placed on the include
path.  No reference file is copied or modified.

Usage:  python oracle/build_ref.py [--ref PATH] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# where the reference's sources lie; SIFEL_REFERENCE overrides it
DEFAULT_REF = os.environ.get("SIFEL_REFERENCE", "/root/reference/SIFEL")

CXX = os.environ.get("CXX", "g++")
# Flags follow the reference's optimized build (Makefile.in: OPTCFLAGS -O3 plus
# COMPATFLAGS -std=c++11); -fPIC so GEFEL can also go into libsifelref.so.
CXXFLAGS = ["-O3", "-std=c++11", "-w", "-fPIC", "-fno-omit-frame-pointer"]

# module -> (source dir relative to SIFEL root, include dirs, makefile)
MODULES = {
    "cmlfile": ("GEFEL/CMLFILE", []),
    "randy": ("GEFEL/RANDY", []),
    "parser": ("GEFEL/PARSER", []),
    "optim": ("GEFEL/OPTIM", ["GEFEL/CMLFILE", "GEFEL/RANDY", "GEFEL", "GEFEL/PARSER"]),
    "sparse": ("GEFEL/SPARSE", ["GEFEL", "GEFEL/PARSER", "GEFEL/SPARSE"]),
    "gefel": ("GEFEL", ["GEFEL/OPTIM", "GEFEL/RANDY", "GEFEL/CMLFILE", "GEFEL/PARSER", "GEFEL/SPARSE"]),
    "mefel": ("MEFEL/SRC", ["GEFEL", "GEFEL/PARSER", "GEFEL/OPTIM", "GEFEL/RANDY", "GEFEL/CMLFILE"]),
    "trfel": ("TRFEL/SRC", ["GEFEL", "GEFEL/PARSER", "GEFEL/OPTIM", "GEFEL/RANDY", "GEFEL/CMLFILE"]),
}
GEFEL_PARTS = ["cmlfile", "randy", "parser", "optim", "sparse", "gefel"]


def srcs_of(makefile: str) -> list[str]:
    """Return the de-duplicated ``SRCS`` list of one reference Makefile."""
    out: list[str] = []
    with open(makefile) as fh:
        for line in fh:
            s = line.split("#", 1)[0]
            m = re.match(r"\s*SRCS\s*\+?=\s*(.*)$", s)
            if not m:
                continue
            for tok in m.group(1).split():
                if tok.endswith(".cpp") and tok not in out:
                    out.append(tok)
    return out


def compile_one(args):
    src, obj, incs = args
    if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src):
        return obj, None
    cmd = [CXX, *CXXFLAGS, *[f"-I{i}" for i in incs], "-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, " ".join(cmd) + "\n" + p.stderr[-4000:]
    return obj, None


def run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise SystemExit(" ".join(cmd) + "\n" + p.stdout[-2000:] + p.stderr[-4000:])


def build(ref: str, jobs: int) -> None:
    ref = os.path.abspath(ref)
    if not os.path.isdir(os.path.join(ref, "GEFEL")):
        raise SystemExit(f"reference tree not found at {ref}")
    os.makedirs(OUT, exist_ok=True)
    compat = os.path.join(HERE, "ref_compat")
    tasks = []
    objs: dict[str, list[str]] = {}
    for mod, (sdir, incs) in MODULES.items():
        d = os.path.join(ref, sdir)
        odir = os.path.join(OUT, "obj", mod)
        os.makedirs(odir, exist_ok=True)
        inc_abs = [compat, d] + [os.path.join(ref, i) for i in incs]
        objs[mod] = []
        for s in srcs_of(os.path.join(d, "Makefile")):
            src = os.path.join(d, s)
            obj = os.path.join(odir, s[:-4] + ".o")
            objs[mod].append(obj)
            tasks.append((src, obj, inc_abs))
    # the two reference mains
    mains = {
        "mefel": os.path.join(ref, "MEFEL/SRC/mefel.cpp"),
        "trfel": os.path.join(ref, "TRFEL/SRC/trfel.cpp"),
    }
    main_objs = {}
    for mod, src in mains.items():
        obj = os.path.join(OUT, "obj", mod + "_main.o")
        inc_abs = [compat, os.path.dirname(src)] + [os.path.join(ref, i) for i in MODULES[mod][1]]
        tasks.append((src, obj, inc_abs))
        main_objs[mod] = obj
    # harnesses (our own sources, compiled against the reference headers)
    harness = {
        "mefel": os.path.join(HERE, "ref_harness_mefel.cpp"),
        "trfel": os.path.join(HERE, "ref_harness_trfel.cpp"),
        "capi": os.path.join(HERE, "ref_solver_capi.cpp"),
    }
    harness_objs = {}
    for key, src in harness.items():
        mod = "gefel" if key == "capi" else key
        sdir = MODULES[mod][0]
        obj = os.path.join(OUT, "obj", f"harness_{key}.o")
        inc_abs = [compat, os.path.join(ref, sdir)] + [os.path.join(ref, i) for i in MODULES[mod][1]]
        tasks.append((src, obj, inc_abs))
        harness_objs[key] = obj

    errs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, err in ex.map(compile_one, tasks):
            if err:
                errs.append(err)
    if errs:
        raise SystemExit("reference compile failed:\n" + "\n".join(errs[:3]))

    libgef = os.path.join(OUT, "libgef.a")
    libmef = os.path.join(OUT, "libmef.a")
    libtrf = os.path.join(OUT, "libtrf.a")
    for lib, mods in ((libgef, GEFEL_PARTS), (libmef, ["mefel"]), (libtrf, ["trfel"])):
        if os.path.exists(lib):
            os.remove(lib)
        run(["ar", "rcs", lib] + [o for m in mods for o in objs[m]])
    syslibs = ["-lm", "-rdynamic", "-ldl"]
    run([CXX, "-o", os.path.join(OUT, "mefel_ref"), main_objs["mefel"], libmef, libgef, *syslibs])
    run([CXX, "-o", os.path.join(OUT, "trfel_ref"), main_objs["trfel"], libtrf, libgef, *syslibs])
    run([CXX, "-o", os.path.join(OUT, "mefel_dump"), harness_objs["mefel"], libmef, libgef, *syslibs])
    run([CXX, "-o", os.path.join(OUT, "trfel_dump"), harness_objs["trfel"], libtrf, libgef, *syslibs])
    gef_objs = [o for m in GEFEL_PARTS for o in objs[m]]
    run([CXX, "-shared", "-o", os.path.join(OUT, "libsifelref.so"), harness_objs["capi"],
         *gef_objs, "-lm", "-ldl"])
    build_dropin(ref, harness_objs["mefel"], libmef, libgef, syslibs, harness_objs["trfel"], libtrf)


WRAP = "_ZN10symcomprow7cg_precEPdS0_ldRlRddlldP7ISolver"
WRAP_ASM = "_Z16stiffness_matrixl"  # stiffness_matrix(long), MEFEL/SRC/globmat.cpp:41


def build_dropin(ref, harness_obj, libmef, libgef, syslibs, trfel_obj=None, libtrf=None):
    """mefel_dump_gpu / trfel_dump_gpu: the same harnesses and SIFEL objects,
    linked with the drop-in binding (ssf_b200/integration/sifel_gpu_shim.cpp)
    so that symcomprow::cg_prec -- MEFEL's load-case solves and every TRFEL
    time step's solve -- runs on the GPU through libsifelgpu.so; the MEFEL
    program also takes the assembly binding
    (ssf_b200/integration/sifel_gpu_assembly.cpp: stiffness_matrix on the GPU)."""
    root = os.path.dirname(HERE)
    lib_dir = os.path.join(root, "ssf_b200")
    if not os.path.exists(os.path.join(lib_dir, "libsifelgpu.so")):
        return
    shim = os.path.join(root, "ssf_b200", "integration", "sifel_gpu_shim.cpp")
    shim_obj = os.path.join(OUT, "obj", "sifel_gpu_shim.o")
    run([CXX, *CXXFLAGS, f"-I{os.path.join(ref, 'GEFEL')}", f"-I{os.path.join(ref, 'GEFEL', 'SPARSE')}",
         f"-I{os.path.join(root, 'include')}", f"-I{os.path.join(HERE, 'ref_compat')}", "-c", shim, "-o", shim_obj])
    asm = os.path.join(root, "ssf_b200", "integration", "sifel_gpu_assembly.cpp")
    asm_obj = os.path.join(OUT, "obj", "sifel_gpu_assembly.o")
    inc = [os.path.join(ref, d) for d in MODULES["mefel"][1]] + [os.path.join(ref, MODULES["mefel"][0])]
    run([CXX, *CXXFLAGS, *[f"-I{d}" for d in inc], f"-I{os.path.join(ref, 'GEFEL', 'SPARSE')}",
         f"-I{os.path.join(root, 'include')}", f"-I{os.path.join(HERE, 'ref_compat')}", "-c", asm, "-o", asm_obj])
    run([CXX, "-o", os.path.join(OUT, "mefel_dump_gpu"), harness_obj, shim_obj, asm_obj, libmef, libgef,
         f"-Wl,--wrap={WRAP}", f"-Wl,--wrap={WRAP_ASM}", f"-L{lib_dir}", "-lsifelgpu",
         "-Wl,-rpath,$ORIGIN/../../ssf_b200", *syslibs])
    if trfel_obj is not None:
        run([CXX, "-o", os.path.join(OUT, "trfel_dump_gpu"), trfel_obj, shim_obj, libtrf, libgef,
             f"-Wl,--wrap={WRAP}", f"-L{lib_dir}", "-lsifelgpu", "-Wl,-rpath,$ORIGIN/../../ssf_b200", *syslibs])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args()
    build(a.ref, a.j)
    print("reference built into", OUT)


if __name__ == "__main__":
    main()
