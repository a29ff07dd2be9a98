#!/usr/bin/env python3
"""Build the reference libflame (CPU, f2c built-in BLAS) straight from its
sources with gcc, without running the reference's configure/make.

Test infrastructure only.  The product never links or loads what this
produces; the parity tests and the CPU-baseline leg of bench.py do.

Inputs : the reference source tree (default /root/reference, read-only) and
         the hand-written configuration header oracle/ref_config/FLA_config.h.
Outputs: oracle/_ref/libflame_ref.so        (flat FLA_* + lapack2flame, serial)
         oracle/_ref/libflame_ref_smp.so    (same + SuperMatrix/OpenMP, for the
                                             multi-threaded CPU baseline)
         oracle/_ref/libflame_ref_openblas.so (--openblas: the serial objects
                                             without the built-in f2c BLAS, their
                                             BLAS references renamed to SciPy's
                                             bundled LP64 OpenBLAS, whose
                                             exports carry a scipy_ prefix: the
                                             fast multi-threaded CPU baseline)
Objects go to oracle/_ref/obj*/.  Nothing is written into the reference tree.

Which reference sources are compiled: every .c under the directories listed
in CORE_DIRS (object runtime, control trees, BLIS-1 glue, built-in f2c BLAS,
the FLAME BLAS/LAPACK operation trees, lapack2flame and its argument checks)
plus the f2c LAPACK files named in oracle/ref_f2c_files.txt (the closure of
what dposv_/dgesv_/dsposv_/dsgesv_ and lapack2flame call), skipping the
GPU/HIP offload, Matlab and old/ subtrees.
"""
import os, sys, subprocess, argparse, concurrent.futures as cf

HERE = os.path.dirname(os.path.abspath(__file__))
# where this container mounts the reference sources (read-only)
DEFAULT_REF = "/root/reference"
CORE_DIRS = [
    "src/base/flamec/main", "src/base/flamec/control", "src/base/flamec/blis",
    "src/base/flamec/util", "src/base/flamec/check", "src/base/flamec/wrappers",
    "src/base/flamec/hierarchy", "src/base/flamec/supermatrix/main",
    "src/flablas", "src/blas", "src/lapack", "src/map/lapack2flamec",
    "src/map/common/lapackcheck",
]
SKIP_PARTS = {"gpu", "hip", "old", "matlab", "octave", "flatex", "test", "openflame"}


def header_dirs(ref):
    dirs = set()
    for root, dnames, fnames in os.walk(os.path.join(ref, "src")):
        parts = set(os.path.relpath(root, ref).split(os.sep))
        if parts & (SKIP_PARTS - {"gpu", "hip"}):
            continue
        if any(f.endswith(".h") for f in fnames):
            dirs.add(root)
    return sorted(dirs)


def sources(ref, f2c_list):
    srcs = []
    for d in CORE_DIRS:
        for root, dnames, fnames in os.walk(os.path.join(ref, d)):
            parts = set(os.path.relpath(root, ref).split(os.sep))
            if parts & SKIP_PARTS:
                continue
            srcs += [os.path.join(root, f) for f in sorted(fnames) if f.endswith(".c")]
    srcs.append(os.path.join(HERE, "ref_shim.c"))
    if f2c_list:
        f2c_dir = os.path.join(ref, "src/map/common/lapacksrc")
        for name in f2c_list:
            srcs.append(os.path.join(f2c_dir, name))
    return srcs


def compile_one(args):
    src, obj, flags = args
    if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src):
        return src, 0, ""
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    p = subprocess.run(["gcc", "-c", src, "-o", obj] + flags,
                       capture_output=True, text=True)
    return src, p.returncode, p.stderr[-2000:]


def build(ref, out, smp, f2c_list, jobs):
    tag = "smp" if smp else "serial"
    objdir = os.path.join(out, "obj_" + tag)
    inc = ["-I" + os.path.join(HERE, "ref_config")] + ["-I" + d for d in header_dirs(ref)]
    flags = ["-O2", "-fPIC", "-w", "-fno-strict-aliasing", "-std=gnu99", "-D_GNU_SOURCE"] + inc
    if smp:
        flags += ["-DFLA_REF_SUPERMATRIX", "-fopenmp"]
    srcs = sources(ref, f2c_list)
    jobs_list = []
    for s in srcs:
        rel = os.path.relpath(s, ref) if s.startswith(ref) else "shim/" + os.path.basename(s)
        jobs_list.append((s, os.path.join(objdir, rel[:-2] + ".o"), flags))
    failed = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for src, rc, err in ex.map(compile_one, jobs_list):
            if rc != 0:
                failed.append((src, err))
    if failed:
        for src, err in failed[:10]:
            print("FAILED", src, "\n", err, file=sys.stderr)
        print("\n".join(s for s, _ in failed), file=sys.stderr)
        raise SystemExit("%d reference files failed to compile" % len(failed))
    lib = os.path.join(out, "libflame_ref_smp.so" if smp else "libflame_ref.so")
    objs = [j[1] for j in jobs_list]
    rsp = os.path.join(out, "objs_%s.rsp" % tag)
    with open(rsp, "w") as f:
        f.write("\n".join(objs))
    cmd = ["gcc", "-shared", "-o", lib, "@" + rsp, "-lm"]
    if smp:
        cmd.append("-fopenmp")
    subprocess.run(cmd, check=True)
    return lib


def openblas_lib():
    """SciPy's bundled OpenBLAS (LP64, Fortran symbols prefixed scipy_)."""
    import glob
    import scipy
    d = os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs"))
    libs = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
    if not libs:
        raise SystemExit("SciPy's bundled OpenBLAS not found under " + d)
    return libs[0]


def build_openblas(ref, out):
    """Relink the serial objects, minus src/flablas (the built-in BLAS; only
    its lsame.c reads FLA_ENABLE_BUILTIN_BLAS; its f2c runtime helpers under
    f2c/other/util stay), against OpenBLAS: every
    symbol the objects reference but do not define and that OpenBLAS exports
    as scipy_<name> is renamed to it (objcopy --redefine-syms on one
    relocatable object)."""
    ob = openblas_lib()
    objdir = os.path.join(out, "obj_serial")
    objs = []
    for root, _, fnames in os.walk(objdir):
        rel = os.path.relpath(root, objdir)
        # keep the f2c runtime helpers (complex conjugate / imaginary part)
        if rel.startswith(os.path.join("src", "flablas")) and \
                not rel.startswith(os.path.join("src", "flablas", "f2c", "other", "util")):
            continue
        objs += [os.path.join(root, f) for f in fnames if f.endswith(".o")]
    rsp = os.path.join(out, "objs_openblas.rsp")
    with open(rsp, "w") as f:
        f.write("\n".join(sorted(objs)))
    combined = os.path.join(out, "libflame_ref_openblas.o")
    subprocess.run(["ld", "-r", "-o", combined, "@" + rsp], check=True)
    undef = subprocess.run(["nm", "-u", combined], capture_output=True, text=True, check=True).stdout.split()
    undef = {u for u in undef if u not in ("U", "w")}
    exported = subprocess.run(["nm", "-D", "--defined-only", ob], capture_output=True, text=True,
                              check=True).stdout.split()
    exported = {e for e in exported if e.startswith("scipy_")}
    pairs = sorted((u, "scipy_" + u) for u in undef if "scipy_" + u in exported)
    mp = os.path.join(out, "openblas_redefine.txt")
    with open(mp, "w") as f:
        f.write("".join("%s %s\n" % p for p in pairs))
    subprocess.run(["objcopy", "--redefine-syms=" + mp, combined], check=True)
    lib = os.path.join(out, "libflame_ref_openblas.so")
    subprocess.run(["gcc", "-shared", "-o", lib, combined, ob, "-Wl,-rpath," + os.path.dirname(ob), "-lm"],
                   check=True)
    print("renamed %d BLAS/LAPACK references to OpenBLAS" % len(pairs))
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("LIBFLAME_REF_DIR") or DEFAULT_REF,
                    help="reference source tree (default: $LIBFLAME_REF_DIR, else %s)" % DEFAULT_REF)
    ap.add_argument("--if-present", action="store_true",
                    help="exit quietly when the reference tree is absent")
    ap.add_argument("--out", default=os.path.join(HERE, "_ref"))
    ap.add_argument("--smp", action="store_true", help="also build the SuperMatrix/OpenMP library")
    ap.add_argument("--openblas", action="store_true",
                    help="also build libflame_ref_openblas.so (reference over SciPy's OpenBLAS)")
    ap.add_argument("-j", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args()
    if not os.path.isdir(os.path.join(a.ref, "src")):
        if a.if_present:
            print("reference tree not found at %s: checker library not built" % a.ref)
            return
        raise SystemExit("reference tree not found at " + a.ref)
    with open(os.path.join(HERE, "ref_f2c_files.txt")) as f:
        f2c_list = [l.strip() for l in f if l.strip() and not l.startswith("#")]
    os.makedirs(a.out, exist_ok=True)
    print(build(a.ref, a.out, False, f2c_list, a.j))
    if a.smp:
        print(build(a.ref, a.out, True, f2c_list, a.j))
    if a.openblas:
        print(build_openblas(a.ref, a.out))


if __name__ == "__main__":
    main()
