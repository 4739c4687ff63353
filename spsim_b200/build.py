"""Build libspsim_b200.so in-tree (spsim_b200/_lib/) for sm_100a.

CUDA sources (kernels and the C ABI) go through nvcc with
``-gencode arch=compute_100a,code=sm_100a``; the reference-shaped C layer
(spsim_b200/csrc/host/*.c) through gcc.  The CUDA runtime is linked
statically and every symbol except the functions declared in include/*.h is
hidden by a linker version script, so the library neither exports nor binds
to another CUDA runtime loaded in the same process (PyTorch's, for example).

Also builds spsim_b200/_lib/spsim, the spsim command-line program on the
library (host/spsim_main.c).

Usage: python -m spsim_b200.build [--force] [--verbose]
"""
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(HERE, "_lib")
BUILD = os.path.join(ROOT, "_build", "spsim_b200")
LIBNAME = "libspsim_b200.so"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]
CC_FLAGS = ["-O2", "-fPIC", "-std=gnu11", "-Wall", "-Wno-unused-result", "-Werror=implicit-function-declaration",
            "-ffp-contract=off",
            "-I" + os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["sf_kernels.cu", "chain_kernels.cu", "adjoint_kernels.cu", "nufft_kernels.cu", "nufft_fft.cu", "capi.cu",
              "noalloc.cu"]
C_SOURCES = ["host/config.c", "host/legacy.c", "host/molecule.c", "host/crystal.c", "host/cxi.c"]


def lib_path():
    return os.path.join(LIBDIR, LIBNAME)


def exported_symbols():
    """Function names declared in include/*.h: the library's whole public surface."""
    names = set()
    for fn in sorted(os.listdir(INCLUDE)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
        for chunk in text.replace("{", ";").replace("}", ";").split(";"):
            m = re.search(r"\b([A-Za-z_]\w*)\s*\(", chunk)
            if m and "typedef" not in chunk and m.group(1) not in ("if", "while", "for", "return", "sizeof"):
                names.add(m.group(1))
    return sorted(names)


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: %s" % " ".join(cmd[:3]))
    return res


def build(force=False, verbose=False):
    """Compile and link the library; returns the path of the .so."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _newer(o, [s] + headers):
            _run([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _newer(o, [s] + headers):
            _run(["gcc"] + CC_FLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    vmap = os.path.join(BUILD, "exports.map")
    syms = exported_symbols()
    with open(vmap, "w") as f:
        f.write("{\n  global:\n")
        for s in syms:
            f.write("    %s;\n" % s)
        f.write("  local: *;\n};\n")
    out = lib_path()
    if force or _newer(out, objs + [vmap]):
        tmp = out + ".tmp"
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs +
             ["-Xlinker", "--version-script=" + vmap, "-Xlinker", "-Bsymbolic",
              "-lrt", "-ldl", "-lpthread"],
             verbose)
        shutil.move(tmp, out)
    cli = os.path.join(LIBDIR, "spsim")
    csrc = os.path.join(CSRC, "host", "spsim_main.c")
    if force or _newer(cli, [csrc, out]):
        _run(["gcc"] + CC_FLAGS + ["-o", cli, csrc, "-L" + LIBDIR, "-l:" + LIBNAME, "-Wl,-rpath,$ORIGIN"], verbose)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(lib_path())
