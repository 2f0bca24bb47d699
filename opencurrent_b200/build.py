"""Build libocu_b200.so in-tree with nvcc for sm_100a.

    python -m opencurrent_b200.build          # incremental
    python -m opencurrent_b200.build --clean

Every translation unit is compiled with --fmad=false: products and sums are rounded exactly as
the reference expressions are written, which is what makes the kernels bit-compatible with the
CPU oracle.  Objects go to _build/ (git-ignored); the shared library lands next to this file.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build", "ocu_b200")
LIB = os.path.join(PKG, "libocu_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O2", "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]
    return max(os.path.getmtime(h) for h in hs)


def compile_one(src, force, verbose):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    path = os.path.join(CSRC, src)
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) > max(os.path.getmtime(path), headers_mtime())):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + ["-c", path, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stdout + r.stderr
    return obj, (r.stdout + r.stderr) if verbose else None


def build(force=False, verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: compile_one(s, force, verbose), srcs))
    errors = [msg for (obj, msg) in results if msg and "error" in msg.lower()]
    for (obj, msg) in results:
        if msg and verbose:
            sys.stderr.write(msg)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    objs = [o for (o, _) in results]
    if (force or not os.path.exists(LIB)
            or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register/spill info")
    a = ap.parse_args()
    if a.clean:
        shutil.rmtree(BUILD, ignore_errors=True)
        if os.path.exists(LIB):
            os.remove(LIB)
        return
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
