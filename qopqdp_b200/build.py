"""Build libqop_b200.so (the C-ABI library) from csrc/*.cu for sm_100a.

Objects go to qopqdp_b200/_build/, the shared library to qopqdp_b200/lib/.
Rebuilds only the translation units whose source or shared headers changed.
Usage: python -m qopqdp_b200.build [-j N] [--force]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libqop_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "-I", INCLUDE, "-I", CSRC,
]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "qop.h"))
    hs.append(os.path.join(INCLUDE, "qop_b200.h"))
    return [h for h in hs if os.path.exists(h)]


def _compile(src, obj, extra):
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return r.stderr


def build(jobs=None, force=False, verbose=False, extra=None):
    """Compile every csrc/*.cu and link libqop_b200.so; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    extra = list(extra or [])
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [os.path.getmtime(__file__)])
    todo, objs = [], []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s[:-3] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_mtime):
            todo.append((src, obj))
    jobs = jobs or min(8, os.cpu_count() or 4)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = {ex.submit(_compile, s, o, extra): s for s, o in todo}
            for f in cf.as_completed(futs):
                msg = f.result()
                if verbose and msg.strip():
                    print(msg, file=sys.stderr)
    if todo or not os.path.exists(LIB) or force:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else []
    print(build(a.j, a.force or a.ptxas_v, a.v or a.ptxas_v, extra))


if __name__ == "__main__":
    main()
