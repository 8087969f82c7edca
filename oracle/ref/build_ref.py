"""Build the reference's own FAC solver into oracle/_ref/ (test
infrastructure only: it generates the golden fixtures that pin the oracle).

    python oracle/ref/build_ref.py [--ref /root/reference] [--jobs N]

The reference's CMake build cannot run here (its BLT submodule is empty and
there is no Fortran compiler, m4 or MPI), so this recipe does by hand what
the configure step and the compilers would:

1. SAMRAI_config.h from the reference's template for a serial build
   (mkconfig.py) and an include tree whose SAMRAI/<pkg> entries link to the
   reference's source directories;
2. every .C unit of tbox, hier, pdat, geom, xfer, math, solv, mesh and
   appu compiled with g++ (the four template-implementation units that
   headers include are skipped);
3. the Fortran kernels those packages call: the m4 templates expanded
   (m4lite.py, as cmake/SetupM4.cmake runs m4) and every routine of the
   kernel files translated to C (f77c.py), compiled with gcc;
4. abort() stubs for the Fortran symbols the compiled units reference but
   the FAC path never calls (complex data, other centerings);
5. fac_ref_driver.C linked with all of it: oracle/_ref/fac_ref_driver;
   and, when the CUDA library is built, the same driver on the drop-in
   operators (samrai_b200/dropin): oracle/_ref/fac_dropin_driver;
6. br_ref_driver.C (tagging and Berger-Rigoutsos clustering) linked with
   the same objects and the reference's FAC_adaptive test problem
   (source/test/FAC_adaptive, all but its main.C), whose adaption estimate
   it calls: oracle/_ref/br_ref_driver.

Nothing is copied from the reference into the repository: the generated
files and objects live under oracle/_ref/, which git ignores.  Everything is
compiled with -ffp-contract=off, so products and sums round separately as
in the Fortran.
"""
import argparse
import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(os.path.dirname(HERE), "_ref")
PKGS = ["tbox", "hier", "pdat", "geom", "xfer", "math", "solv", "mesh", "appu"]
SKIP = {"pdat/ArrayDataOperationUtilities.C", "pdat/CopyOperation.C", "pdat/SumOperation.C",
        "tbox/MathUtilities.C"}
CXXFLAGS = ["-std=c++11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-w"]
CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-w"]
# Fortran kernel sources: plain .f, and m4 templates with the directory
# their include()s name
FORTRAN = ["solv/fortran/solv_cellpoissonfacops2d.f", "solv/fortran/solv_cellpoissonfacops3d.f",
           "solv/fortran/solv_cartesianrobinbchelper2d.f",
           "solv/fortran/solv_cartesianrobinbchelper3d.f"]
M4 = ["geom/fortran/geom_cartrefine2d.m4", "geom/fortran/geom_cartrefine3d.m4",
      "geom/fortran/geom_cartcoarsen2d.m4", "geom/fortran/geom_cartcoarsen3d.m4",
      "pdat/fortran/pdat_conrefine2d.m4", "pdat/fortran/pdat_conrefine3d.m4",
      "pdat/fortran/pdat_concoarsen2d.m4", "pdat/fortran/pdat_concoarsen3d.m4",
      "pdat/fortran/pdat_lintimint2d.m4", "pdat/fortran/pdat_lintimint3d.m4"]


def newer(src, dst):
    return not os.path.exists(dst) or os.path.getmtime(src) > os.path.getmtime(dst)


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"failed: {' '.join(cmd)}\n{r.stderr[-4000:]}")
    return r.stdout


def include_tree(ref):
    inc = os.path.join(OUT, "include")
    sys.path.insert(0, HERE)
    import mkconfig
    mkconfig.main(ref, inc)
    for p in os.listdir(os.path.join(ref, "source", "SAMRAI")):
        src = os.path.join(ref, "source", "SAMRAI", p)
        if os.path.isdir(src):
            dst = os.path.join(inc, "SAMRAI", p)
            if os.path.islink(dst):
                os.unlink(dst)
            os.symlink(src, dst)
    return inc


def compile_cxx(ref, inc, jobs):
    objs, work = [], []
    for pkg in PKGS:
        d = os.path.join(ref, "source", "SAMRAI", pkg)
        for f in sorted(os.listdir(d)):
            if not f.endswith(".C") or f"{pkg}/{f}" in SKIP:
                continue
            src = os.path.join(d, f)
            obj = os.path.join(OUT, "obj", pkg, f[:-2] + ".o")
            objs.append(obj)
            if newer(src, obj):
                work.append((src, obj))
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    for pkg in PKGS:
        os.makedirs(os.path.join(OUT, "obj", pkg), exist_ok=True)

    def one(job):
        src, obj = job
        run(["g++", *CXXFLAGS, "-I" + inc, "-c", src, "-o", obj])
        return src

    print(f"build_ref: compiling {len(work)} of {len(objs)} reference units", flush=True)
    with cf.ThreadPoolExecutor(jobs) as ex:
        for i, _ in enumerate(ex.map(one, work)):
            if (i + 1) % 50 == 0:
                print(f"build_ref: {i + 1}/{len(work)}", flush=True)
    return objs


def compile_kernels(ref):
    sys.path.insert(0, HERE)
    import f77c
    import m4lite
    gen = os.path.join(OUT, "gen")
    os.makedirs(gen, exist_ok=True)
    root = os.path.join(ref, "source", "SAMRAI")
    texts = []
    for f in FORTRAN:
        with open(os.path.join(root, f)) as fh:
            texts.append(fh.read())
    for f in M4:
        defs = {"FORTDIR": os.path.join(root, os.path.dirname(f)),
                "PDAT_FORTDIR": os.path.join(root, "pdat", "fortran")}
        t = m4lite.expand_file(os.path.join(root, f), defs)
        with open(os.path.join(gen, os.path.basename(f)[:-3] + ".f"), "w") as fh:
            fh.write(t)
        texts.append(t)
    chunks, names = [f77c.PRELUDE], []
    with open(os.path.join(gen, "f77c.log"), "w") as log:
        for t in texts:
            c, n = f77c.translate(t, log=log)
            chunks += c
            names += n
    src = os.path.join(gen, "kernels.c")
    with open(src, "w") as fh:
        fh.write("\n\n".join(chunks) + "\n")
    obj = os.path.join(gen, "kernels.o")
    run(["gcc", *CFLAGS, "-c", src, "-o", obj])
    # the same kernels as a shared library, for tests that call the
    # reference's routines one by one
    run(["gcc", *CFLAGS, "-fPIC", "-shared", src, "-o", os.path.join(OUT, "libref_kernels.so"),
         "-lm"])
    print(f"build_ref: {len(names)} Fortran routines translated", flush=True)
    return obj


def symbols(objs, defined):
    flag = "--defined-only" if defined else "-u"
    out = set()
    for i in range(0, len(objs), 200):
        txt = run(["nm", flag, *objs[i:i + 200]])
        for line in txt.splitlines():
            parts = line.split()
            if parts and not line.endswith(":"):
                out.add(parts[-1])
    return out


def stubs(objs, name="stubs"):
    """abort() stubs for Fortran symbols (lower case, one trailing
    underscore) referenced but defined nowhere."""
    und = symbols(objs, False) - symbols(objs, True)
    f77 = sorted(s for s in und if re.fullmatch(r"[a-z][a-z0-9]*_", s))
    gen = os.path.join(OUT, "gen")
    src = os.path.join(gen, name + ".c")
    with open(src, "w") as fh:
        fh.write("/* Fortran routines the FAC path never calls. */\n#include <stdio.h>\n"
                 "#include <stdlib.h>\n")
        for s in f77:
            fh.write(f'void {s}(void) {{ fprintf(stderr, "{s} not built\\n"); abort(); }}\n')
    obj = os.path.join(gen, name + ".o")
    run(["gcc", *CFLAGS, "-c", src, "-o", obj])
    print(f"build_ref: {len(f77)} Fortran symbols stubbed", flush=True)
    return obj


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SAMRAI_REFERENCE", "/root/reference"))
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args()
    if not os.path.isdir(os.path.join(a.ref, "source", "SAMRAI")):
        print(f"build_ref: no reference tree at {a.ref}", file=sys.stderr)
        return 1
    inc = include_tree(a.ref)
    objs = compile_cxx(a.ref, inc, a.jobs)
    kobj = compile_kernels(a.ref)
    drv_src = os.path.join(HERE, "fac_ref_driver.C")
    drv_obj = os.path.join(OUT, "obj", "fac_ref_driver.o")
    run(["g++", *CXXFLAGS, "-I" + inc, "-c", drv_src, "-o", drv_obj])
    sobj = stubs(objs + [kobj, drv_obj])
    # every object linked (not an archive), so that the units that only
    # register start-up/shut-down handlers through static objects are kept
    exe = os.path.join(OUT, "fac_ref_driver")
    run(["g++", "-o", exe, drv_obj, *objs, kobj, sobj, "-lm"])
    print(f"build_ref: {exe}", flush=True)
    dropin(inc, objs + [kobj, sobj])
    br_driver(a.ref, inc, objs + [kobj], a.jobs)
    return 0


def br_driver(ref, inc, objs, jobs):
    """br_ref_driver: the reference's AdaptivePoisson tagging and its
    BergerRigoutsos box generator on one level."""
    tdir = os.path.join(ref, "source", "test", "FAC_adaptive")
    odir = os.path.join(OUT, "obj", "FAC_adaptive")
    os.makedirs(odir, exist_ok=True)
    flags = [*CXXFLAGS, "-I" + inc, "-I" + tdir]
    work, tobjs = [], []
    for f in sorted(os.listdir(tdir)):
        if not f.endswith(".C") or f == "main.C":
            continue
        src, obj = os.path.join(tdir, f), os.path.join(odir, f[:-2] + ".o")
        tobjs.append(obj)
        if newer(src, obj):
            work.append((src, obj))
    with cf.ThreadPoolExecutor(jobs) as ex:
        list(ex.map(lambda j: run(["g++", *flags, "-c", j[0], "-o", j[1]]), work))
    drv_obj = os.path.join(OUT, "obj", "br_ref_driver.o")
    run(["g++", *flags, "-c", os.path.join(HERE, "br_ref_driver.C"), "-o", drv_obj])
    sobj = stubs(objs + tobjs + [drv_obj], name="br_stubs")
    exe = os.path.join(OUT, "br_ref_driver")
    run(["g++", "-o", exe, drv_obj, *tobjs, *objs, sobj, "-lm"])
    print(f"build_ref: {exe}", flush=True)


def dropin(inc, objs):
    """fac_dropin_driver: the driver with the reference's CellPoissonFACOps
    replaced by samrai_b200's B200CellPoissonFACOps (compiled here against
    the reference's headers), linked with the CUDA library; skipped when
    that library is not built."""
    root = os.path.dirname(os.path.dirname(HERE))
    lib_dir = os.path.join(root, "samrai_b200", "_build")
    if not os.path.exists(os.path.join(lib_dir, "libsamrai_fac_b200.so")):
        print("build_ref: no CUDA library, fac_dropin_driver not built", flush=True)
        return
    src_dir = os.path.join(root, "samrai_b200", "dropin")
    flags = [*CXXFLAGS, "-I" + inc, "-I" + src_dir, "-I" + os.path.join(root, "include")]
    ops_obj = os.path.join(OUT, "obj", "B200CellPoissonFACOps.o")
    run(["g++", *flags, "-c", os.path.join(src_dir, "B200CellPoissonFACOps.C"), "-o", ops_obj])
    drv_obj = os.path.join(OUT, "obj", "fac_dropin_driver.o")
    run(["g++", *flags, "-DWITH_B200_OPS", "-c", os.path.join(HERE, "fac_ref_driver.C"), "-o",
         drv_obj])
    exe = os.path.join(OUT, "fac_dropin_driver")
    run(["g++", "-o", exe, drv_obj, ops_obj, *objs, "-L" + lib_dir, "-lsamrai_fac_b200",
         "-Wl,-rpath,$ORIGIN/../../samrai_b200/_build", "-lm"])
    print(f"build_ref: {exe}", flush=True)


if __name__ == "__main__":
    sys.exit(main())
