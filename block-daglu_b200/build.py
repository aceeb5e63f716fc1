"""Builds libbdlu.so in-tree: the C ABI, host analysis and the sm_100a kernels.

    python block-daglu_b200/build.py [--force]

Objects go to block-daglu_b200/_build/, the library to block-daglu_b200/lib/.
Device code is compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a);
host code with -ffp-contract=off so that the host-side factor assembly performs
the same unfused arithmetic as the reference's dense micro-kernel.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libbdlu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
CUDA_INC = "/usr/local/cuda/include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
          "-Xcompiler", "-fPIC,-ffp-contract=off,-Wall"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cpp", ".cu")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    for dp, _, fs in os.walk(inc):
        hs += [os.path.join(dp, f) for f in fs if f.endswith(".h")]
    return hs


def compile_one(src, force):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [NVCC] + COMMON + ARCH + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [CXX, "-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-Wall", "-I" + os.path.join(ROOT, "include"),
               "-I" + CSRC, "-I" + CUDA_INC, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr)
    return obj, None


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: compile_one(s, force), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("libbdlu build failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, "-shared"] + ARCH + ["-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("libbdlu link failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
