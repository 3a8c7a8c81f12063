"""Builds CHarm 0.4.9 itself (the reference CPU implementation) from its
sources into oracle/_ref/, for use as a checker and as the timed CPU
baseline.  Test infrastructure: nothing in the charm_b200 package loads what
this writes.

    python oracle/build_ref.py [--reference DIR] [-j N] [--variants ...]

CHarm's own build system (autotools) is not run.  This recipe does by hand
the three things its configure step does for this path:

  * instantiates the public headers from CHarm's templates
    (src/<module>/<module>.h.in -> charm/charm<P>_<module>.h and
    src/charm.h.in -> charm/charm<P>.h, configure.ac:730-745), replacing
    @P@ / @PC@ / @RDT@ (precision prefix, upper-case prefix, real type,
    configure.ac:197-199,219-221,256-258), @WITH_MPI@ = @WITH_MPFR@ = 0 and
    the version numbers;
  * writes config.h with the macros the sources test (precision, SIMD
    width, OpenMP, aligned allocation, isfinite; config.h.in);
  * compiles the unconditional source list of every module's Makefile.am
    (`libcharm@P@_<module>_la_SOURCES`; src/mpi and src/mpfr are left out,
    as configure does without --enable-mpi / --enable-mpfr) with the flags
    `--enable-openmp --enable-avx-512` / `--enable-avx2` and
    CFLAGS="-O3 -ffast-math" give (configure.ac:385-392, 503), and links
    them with oracle/fftw_shim (FFTW 3 is an external library that is not
    installed here) into one shared library per variant.

Variants (oracle/_ref/<file>):

  d_avx512  libcharm_d_avx512.so  double, AVX-512, OpenMP, -O3 -ffast-math
  d_avx2    libcharm_d_avx2.so    double, AVX2,    OpenMP, -O3 -ffast-math
  q         libcharmq.so          __float128 (quad), OpenMP, -O2 (CHarm
                                  allows no SIMD in quad precision)
  f         libcharmf.so          float, AVX2, OpenMP, -O3 -ffast-math

Sources are read where they lie under the reference tree; outputs go only
to oracle/_ref/.
"""
import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "fftw_shim")

MODULES = ["crd", "err", "glob", "integ", "leg", "misc", "sha", "shc", "shs",
           "simd", "xnum", "gfm"]
TEMPLATES = {"charm.h.in": ""}
for _m in ["crd", "err", "integ", "leg", "misc", "sha", "shc", "shs", "gfm",
           "mpi", "glob"]:
    TEMPLATES["%s/%s.h.in" % (_m, _m)] = "_" + _m

VARIANTS = {
    "d_avx512": dict(P="", PC="", RDT="double", prec=1, simd="HAVE_AVX512F",
                     cflags=["-O3", "-ffast-math", "-mavx512f", "-mavx512dq"],
                     lib="libcharm_d_avx512.so"),
    "d_avx2": dict(P="", PC="", RDT="double", prec=1, simd="HAVE_AVX2",
                   cflags=["-O3", "-ffast-math", "-mavx2", "-mfma"],
                   lib="libcharm_d_avx2.so"),
    "q": dict(P="q", PC="Q", RDT="__float128", prec=3, simd=None,
              cflags=["-O2"], lib="libcharmq.so"),
    "f": dict(P="f", PC="F", RDT="float", prec=2, simd="HAVE_AVX2",
              cflags=["-O3", "-ffast-math", "-mavx2", "-mfma"],
              lib="libcharmf.so"),
}


def version(ref):
    v = open(os.path.join(ref, "VERSION")).read().strip()
    parts = (v.split(".") + ["0", "0", "0"])[:3]
    return v, parts


def sources(ref, module):
    """The unconditional `libcharm@P@_<module>_la_SOURCES = a.c \\ b.c ...`
    list of src/<module>/Makefile.am."""
    text = open(os.path.join(ref, "src", module, "Makefile.am")).read()
    m = re.search(r"^libcharm@P@_%s_la_SOURCES\s*=\s*((?:.*\\\n)*.*)$" % module,
                  text, re.M)
    if not m:
        raise RuntimeError("no source list in src/%s/Makefile.am" % module)
    return [t for t in m.group(1).replace("\\\n", " ").split() if t.endswith(".c")]


def gen_headers(ref, v, gen):
    ver, (ma, mi, pa) = version(ref)
    subs = {"@P@": v["P"], "@PC@": v["PC"], "@RDT@": v["RDT"],
            "@WITH_MPI@": "0", "@WITH_MPFR@": "0", "@CHARM_MAJOR@": ma,
            "@CHARM_MINOR@": mi, "@CHARM_PATCH@": pa,
            "@CHARM_PATCH_NUMBER@": re.sub(r"\D", "", pa) or "0"}
    os.makedirs(os.path.join(gen, "charm"), exist_ok=True)
    os.makedirs(os.path.join(gen, "src"), exist_ok=True)
    for m in MODULES:
        os.makedirs(os.path.join(gen, "src", m), exist_ok=True)
    for tmpl, suffix in TEMPLATES.items():
        text = open(os.path.join(ref, "src", tmpl)).read()
        for k, val in subs.items():
            text = text.replace(k, val)
        left = re.findall(r"@[A-Z_]+@", text)
        if left:
            raise RuntimeError("unreplaced %s in %s" % (sorted(set(left)), tmpl))
        name = "charm%s%s.h" % (v["P"], suffix)
        open(os.path.join(gen, "charm", name), "w").write(text)
    # config.h: the macros of config.h.in that this path's sources test
    d = {"HAVE_OPENMP": 1, "HAVE_ISFINITE": 1, "HAVE_POSIX_MEMALIGN": 1,
         "HAVE_ALIGNED_ALLOC": 1, "HAVE_MM_MALLOC_H": 1, "HAVE_LIBM": 1,
         "HAVE_CLOCK_GETTIME": 1, "HAVE_STDINT_H": 1, "HAVE_STDLIB_H": 1,
         "HAVE_STRING_H": 1, "HAVE_INTTYPES_H": 1, "STDC_HEADERS": 1,
         "HAVE_FFTW_VERSION": 1}
    if v["prec"] == 1:
        d["HAVE_LIBFFTW3"] = 1
    elif v["prec"] == 2:
        d["HAVE_LIBFFTW3F"] = 1
        d["CHARM_FLOAT"] = 1
    else:
        d["HAVE_LIBFFTW3Q"] = 1
        d["HAVE_LIBQUADMATH"] = 1
        d["CHARM_QUAD"] = 1
    if v["simd"]:
        d[v["simd"]] = 1
    lines = ["#ifndef __CONFIG_H__", "#define __CONFIG_H__"]
    lines += ["#define %s %s" % kv for kv in sorted(d.items())]
    lines += ['#define PACKAGE "charm"', '#define VERSION "%s"' % ver,
              '#define PACKAGE_VERSION "%s"' % ver,
              '#define _CHARM_CC "gcc"',
              '#define _CHARM_CFLAGS "%s"' % " ".join(v["cflags"]),
              '#define _CHARM_CPPFLAGS ""', '#define _CHARM_LDFLAGS ""',
              '#define _CHARM_LIBS "-lfftw3 (oracle shim) -lm"',
              "#endif", ""]
    open(os.path.join(gen, "config.h"), "w").write("\n".join(lines))


def run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError("%s\n%s" % (" ".join(cmd), r.stdout[-4000:]))
    return r.stdout


def build_variant(ref, name, jobs):
    v = VARIANTS[name]
    root = os.path.join(OUT, "build", name)
    gen = os.path.join(root, "gen")
    obj = os.path.join(root, "obj")
    os.makedirs(obj, exist_ok=True)
    gen_headers(ref, v, gen)
    # -I<ref>/charm is CHarm's own AM_CPPFLAGS (src/*/Makefile.am); some
    # headers include "../src/<module>/..." relative to it
    inc = ["-I" + gen, "-I" + os.path.join(gen, "src"), "-I" + SHIM,
           "-I" + os.path.join(ref, "charm")]
    flags = ["-std=gnu11", "-fPIC", "-fopenmp", "-DHAVE_CONFIG_H", "-w"] + v["cflags"]
    jobs_list = []
    for m in MODULES:
        mod_inc = ["-I" + os.path.join(gen, "src", m),
                   "-I" + os.path.join(ref, "src", m)]
        for src in sources(ref, m):
            o = os.path.join(obj, "%s__%s.o" % (m, src[:-2]))
            jobs_list.append(["gcc", "-c"] + flags + inc + mod_inc +
                             [os.path.join(ref, "src", m, src), "-o", o])
    shim_o = os.path.join(obj, "fftw_shim.o")
    jobs_list.append(["gcc", "-c", "-std=gnu11", "-fPIC", "-fopenmp-simd",
                      "-DSHIM_PREC=%d" % v["prec"], "-I" + SHIM] +
                     [f for f in v["cflags"]] +
                     [os.path.join(SHIM, "fftw_shim.c"), "-o", shim_o])
    with cf.ThreadPoolExecutor(jobs) as ex:
        list(ex.map(run, jobs_list))
    objs = [j[j.index("-o") + 1] for j in jobs_list]
    lib = os.path.join(OUT, v["lib"])
    libs = ["-lm", "-lgomp"] + (["-lquadmath"] if v["prec"] == 3 else [])
    tmp = lib + ".tmp"
    run(["gcc", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-Wl,-z,defs",
         "-o", tmp] + objs + libs)
    os.replace(tmp, lib)
    # the objects and generated headers are not needed once linked
    shutil.rmtree(root, ignore_errors=True)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="root of the CHarm 0.4.9 source tree")
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--variants", nargs="*", default=list(VARIANTS))
    a = ap.parse_args(argv)
    ref = os.path.abspath(a.reference)
    if not os.path.isfile(os.path.join(ref, "src", "shs", "shs_point.c")):
        sys.exit("build_ref: %s does not look like the CHarm source tree" % ref)
    for name in a.variants:
        print(build_variant(ref, name, a.j), flush=True)


if __name__ == "__main__":
    main()
