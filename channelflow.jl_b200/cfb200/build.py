"""Build libcfb200.so in-tree for sm_100a with nvcc (no JIT, no CPU fallback).

The kernels of each compile-time size are instantiated in their own object
(csrc/cf_inst_col.cu once per Chebyshev length, csrc/cf_inst_fft.cu once per
padded length); the objects compile in parallel into csrc/../_build and link
with the host code (csrc/cf_engine.cu) into cfb200/libcfb200.so.
"""
import os
import re
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
SRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
OUT = os.path.join(HERE, "libcfb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]


def _lengths(macro, header):
    text = open(os.path.join(SRC, header)).read()
    m = re.search(r"#define %s\(X\)((?:\s*X\(\d+\))+)" % macro, text)
    return [int(v) for v in re.findall(r"X\((\d+)\)", m.group(1))] + [0]


def units():
    """(source, defines, object) of every translation unit."""
    out = [("cf_engine.cu", [], "cf_engine.o")]
    for p in _lengths("CF_COL_LENGTHS", "cf_dispatch.h"):
        out.append(("cf_inst_col.cu", [f"-DCF_INST_P={p}"], f"cf_col_{p}.o"))
    for n in _lengths("CF_STATIC_FFT_LENGTHS", "cf_fft.cuh"):
        out.append(("cf_inst_fft.cu", [f"-DCF_INST_L={n}"], f"cf_fft_{n}.o"))
    return out


def sources():
    return [os.path.join(SRC, f) for f in sorted(os.listdir(SRC))] + [os.path.join(PKG, "..", "include", "cfb200.h")]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in sources())


def _nvcc():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc]
    if os.path.exists("/usr/bin/g++"):
        cmd += ["-ccbin", "/usr/bin/g++"]
    return cmd


def build(force=False, verbose=False, jobs=None, extra=()):
    if not force and not needs_build():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    jobs = jobs or max(1, os.cpu_count() or 1)

    def compile_one(u):
        src, defs, obj = u
        cmd = _nvcc() + NVCC_FLAGS + list(extra) + defs + ["-c", "-o", os.path.join(OBJ, obj), os.path.join(SRC, src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return u, r

    # largest units first (the column kernels of the long lengths)
    todo = sorted(units(), key=lambda u: (u[0] != "cf_inst_col.cu", -int((u[1] or ["=0"])[0].split("=")[1])))
    failed = []
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        for (src, defs, obj), r in ex.map(compile_one, todo):
            if r.stdout or r.stderr:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(obj)
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    cmd = _nvcc() + ARCH + ["-shared", "-o", OUT + ".tmp"] + [os.path.join(OBJ, u[2]) for u in units()]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else ())
