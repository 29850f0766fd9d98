"""Build libdisorder.so (sm_100a) in-tree with nvcc.

Usage: python -m disorder_b200.build [--debug]
Objects go to _build/ at the repository root; the shared library is written
next to this file as disorder_b200/libdisorder.so. --debug builds the
device index checks in (-DDISORDER_CHECKS: every checked index outside its
array is recorded and skipped, and disorder_synchronize reports it) into
disorder_b200/libdisorder_checks.so (objects in _build_checks/); the package
loads it instead when DISORDER_LIB=checks.
"""

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdisorder.so")
LIB_CHECKS = os.path.join(HERE, "libdisorder_checks.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build(debug=False, verbose=False, jobs=8):
    bdir = os.path.join(ROOT, "_build_checks" if debug else "_build")
    lib_out = LIB_CHECKS if debug else LIB
    os.makedirs(bdir, exist_ok=True)
    flags = ARCH + ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                    "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]
    if debug:
        flags += ["-DDISORDER_CHECKS=1"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    objs = []
    cmds = []
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "disorder.h"))
    newest_dep = max(os.path.getmtime(d) for d in deps)
    for s in sources():
        o = os.path.join(bdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if (not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), newest_dep)
                or verbose):
            cmds.append([nvcc()] + flags + ["-c", s, "-o", o])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for cmd, r in ex.map(run, cmds):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
    link = [nvcc()] + ARCH + ["-shared", "-o", lib_out] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return lib_out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.debug, a.verbose))
