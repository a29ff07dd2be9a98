"""Build libflame_b200.so in-tree with nvcc for sm_100a.

    python -m libflame_b200.build        (or libflame_b200.build.build())

Every .cu file under libflame_b200/csrc is compiled (in parallel) and linked
into libflame_b200/libflame_b200.so with the CUDA runtime linked statically,
so the library only needs the NVIDIA driver at run time.  Objects go to
libflame_b200/_build/.  A file is recompiled when it or any header in csrc/
or include/ is newer than its object.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libflame_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC, "-diag-suppress", "177"]


def nvcc():
    for cand in [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]:
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(args):
    src, obj, force = args
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return src, 0, ""
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    return src, p.returncode, p.stdout + p.stderr


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = [(s, os.path.join(BUILD, os.path.basename(s)[:-3] + ".o"), force) for s in srcs]
    with cf.ThreadPoolExecutor(min(len(jobs), os.cpu_count() or 4)) as ex:
        res = list(ex.map(_compile, jobs))
    failed = [(s, out) for s, rc, out in res if rc != 0]
    for s, out in failed:
        sys.stderr.write("nvcc failed for %s\n%s\n" % (s, out))
    if failed:
        raise RuntimeError("libflame_b200 build failed")
    if verbose:
        for s, rc, out in res:
            if out.strip():
                sys.stderr.write(out)
    objs = [j[1] for j in jobs]
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
