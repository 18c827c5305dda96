"""Builds libmclics_b200.so in-tree with nvcc for sm_100a (B200).

    python -m mclics_b200.build [--force]

Objects go to mclics_b200/_build/, the library to mclics_b200/libmclics_b200.so, the command-line program to
mclics_b200/mclics_b200. kernels_ref8.cu (the reference-order replay kernel) is compiled with -fmad=false so that
its arithmetic rounds like the reference's x86-64 build.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmclics_b200.so")
EXE = os.path.join(HERE, "mclics_b200")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
          "-I" + os.path.join(HERE, "..", "include")] + ARCH
PER_FILE = {"kernels_ref8.cu": ["-fmad=false"]}
SOURCES = ["sweep_pass_ghrl.cu", "sweep_pass_ghrl_chiral.cu", "sweep_pass_pear.cu", "sweep_pass_ll.cu",
           "sweep_fused_ghrl.cu", "sweep_fused_pear.cu", "sweep_fused_ll.cu", "learned.cu", "kernels.cu",
           "kernels_ref8.cu", "sweep_fused.cu", "observe_static.cu", "extras.cu", "engine.cpp", "driver.cpp"]  # slowest first: they start compiling first


def nvcc():
    for p in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if p and os.path.exists(p):
            return p
    raise RuntimeError("nvcc not found")


def _deps_newer(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    heads = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    heads.append(os.path.join(HERE, "..", "include", "mclics_b200.h"))
    return any(os.path.getmtime(p) > t for p in [src] + heads)


def _compile(src, verbose):
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if not _deps_newer(obj, path):
        return obj
    cmd = [nvcc()] + COMMON + PER_FILE.get(src, []) + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd[1:1] = ["-x", "cu"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if force:
        for s in srcs:
            p = os.path.join(BUILD, s + ".o")
            if os.path.exists(p):
                os.remove(p)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    main_src = os.path.join(CSRC, "main.cpp")
    if os.path.exists(main_src) and (force or not os.path.exists(EXE) or os.path.getmtime(LIB) > os.path.getmtime(EXE)
                                     or os.path.getmtime(main_src) > os.path.getmtime(EXE)):
        cmd = [nvcc(), "-O2", "-std=c++17", "-I" + os.path.join(HERE, "..", "include"), main_src, "-o", EXE,
               "-L" + HERE, "-lmclics_b200", "-Xlinker", "-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("CLI link failed:\n%s%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.v))
    sys.exit(0)
