"""Build recipe of libpppm_b200.so (sm_100a) and the C++ scene host.

Compiles every csrc/*.cu for sm_100a with nvcc and links them into
pppm-tdbem_b200/lib/libpppm_b200.so; builds the scene host executable
pppm-tdbem_b200/bin/pppm_demo against it.  Objects are cached in lib/obj and rebuilt
when a source or header is newer.  Run as a script or through __graft_entry__.build().
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
INC = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --use_fast_math: the FP32 path reproduces the reference's arithmetic, which is built with
# it (approximate float division/sqrt, flush-to-zero, fast sin/cos/exp); double arithmetic
# is unaffected.
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--use_fast_math", "-Xcompiler", "-fPIC",
              "-Xptxas", "-O3", "-I" + INC, "-I" + CSRC]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def build_library(verbose=False):
    os.makedirs(os.path.join(LIB, "obj"), exist_ok=True)
    sources = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(INC, "pppm_b200.h"))
    objs, jobs = [], []
    for src in sources:
        s = os.path.join(CSRC, src)
        o = os.path.join(LIB, "obj", src[:-3] + ".o")
        objs.append(o)
        if _newer(o, [s] + headers):
            jobs.append(["nvcc"] + ARCH + NVCC_FLAGS + ["-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for r in ex.map(_run, jobs):
            if verbose and r.stderr:
                print(r.stderr)
    so = os.path.join(LIB, "libpppm_b200.so")
    if _newer(so, objs):
        _run(["nvcc"] + ARCH + ["-shared", "-o", so] + objs + ["-lcudart"])
    return so


def build_host(so):
    os.makedirs(BIN, exist_ok=True)
    srcs = sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp")) if os.path.isdir(HOST) else []
    if not srcs:
        return None
    exe = os.path.join(BIN, "pppm_demo")
    hdrs = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")]
    if _newer(exe, srcs + hdrs + [so]):
        _run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + INC, "-I" + HOST, "-o", exe] + srcs +
             ["-L" + LIB, "-lpppm_b200", "-Wl,-rpath,$ORIGIN/../lib"])
    return exe


def build(verbose=False):
    so = build_library(verbose)
    build_host(so)
    return so


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
