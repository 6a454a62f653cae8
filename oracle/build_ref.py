"""Build the two comparison libraries from the reference's own sources.

Test and benchmark infrastructure: nothing built here is part of the product.

The reference's per-pixel routines (lm_mils and everything it calls:
milosUtils.cu, mil_sinrf.cu, me_der.cu, lib.cu, convolution.cu, fgauss.cu,
svdcordic.cu, svdcmp.cu, create_cuantic.c) use CUDA dynamic parallelism:
each synthesis and derivative step launches a one-block child grid of nl
threads and waits for it with a device-side cudaDeviceSynchronize()
(mil_sinrf.cu:98-99, 112-113, 157-158; me_der.cu:44-45, 113-114, 140-150).
Device-side synchronisation is not available for sm_90 and later, so the
sources cannot be compiled for sm_100a as shipped, and they cannot be
compiled for a CPU at all.  This script copies them into a temporary
directory and applies one mechanical transformation, the same for both
builds:

  T1  every child launch `K<<<1, n...>>>(args);` becomes an in-thread loop
      `for (t = 0; t < n; ++t) K(args, t);`; the circular-convolution child
      `d_convCircular` becomes the reference's own serial `convCircular`
      (convolution.cu:251) with the scratch row the reference allocates for
      it (pM->resultConv);
  T2  the four child kernels (d_fvoigt, mil_sinrf_kernel,
      d_funcionComponentFor, me_der_kernel) become __device__ functions
      with the thread index as an extra argument; their index expression
      `blockIdx.x * blockDim.x + threadIdx.x` becomes that argument;
  T3  me_der_kernel's dynamic shared memory becomes a local array of the
      largest size it is launched with (MAX_LAMBDA * 7 * 7), and its
      __syncthreads() goes (each thread reads only the entries it zeroed);
  T4  the device-side cudaDeviceSynchronize() calls go;
  T5  me_der (me_der.cu:81-215), declared int, gets the `return 0;` it
      lacks (no caller reads the value; without it g++ miscompiles the
      stray-light branch, see add_missing_return).

Each substitution is counted and the build stops if a count differs from
what the sources above contain, so a changed reference fails loudly.  Then:

  oracle/_ref/libgmref_cpu.so  g++ with the host prelude (CUDA qualifiers
      removed, __fdividef -> '/', __sincosf -> sincosf, __ldg(p) -> *p),
      OpenMP driver oracle/ref_shim/gmref_cpu.cpp;
  oracle/_ref/libgmref_gpu.so  nvcc -gencode arch=compute_100a,code=sm_100a
      -O3 -rdc=true --ftz=true -lineinfo (the reference's own nvcc flags,
      makefile:154-155), device-heap guard prelude, harness
      oracle/ref_shim/gmref_gpu.cu.

Usage: python oracle/build_ref.py [--reference DIR] [--cpu-only]
The reference checkout is --reference, else the GM_REFERENCE_DIR environment
variable, else a directory named `reference` beside this repository's
directory when one exists (locate_reference); without it nothing is built.
Outputs only the two .so files.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "ref_shim")
OUT = os.path.join(HERE, "_ref")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

DEVICE_SOURCES = ["milosUtils.cu", "mil_sinrf.cu", "me_der.cu", "lib.cu", "convolution.cu",
                  "fgauss.cu", "svdcordic.cu", "svdcmp.cu"]
HOST_SOURCES = ["create_cuantic.c"]
HEADERS = ["defines.h", "definesCuda.cuh", "lib.cuh", "milosUtils.cuh", "convolution.cuh",
           "svdcmp.cuh", "readConfig.h"]
CHILD_KERNELS = ["d_fvoigt", "mil_sinrf_kernel", "d_funcionComponentFor", "me_der_kernel"]

# expected substitution counts per file: (launches, convCircular launches,
# child signatures, index expressions, device syncs)
EXPECTED = {
    "mil_sinrf.cu": dict(launch=2, conv=1, sig=4, index=2, sync=3),
    "me_der.cu": dict(launch=2, conv=2, sig=4, index=2, sync=4),
}


def locate_reference(explicit=None):
    """The reference checkout: `explicit`, else $GM_REFERENCE_DIR, else a
    directory named `reference` beside this repository; None when none of
    them holds the reference's sources."""
    repo = os.path.dirname(HERE)
    for cand in (explicit, os.environ.get("GM_REFERENCE_DIR"),
                 os.path.join(os.path.dirname(repo), "reference")):
        if cand and os.path.isfile(os.path.join(cand, "milosUtils.cu")):
            return cand
    return None


def _match_paren(text: str, open_pos: int) -> int:
    """Index of the ')' matching the '(' at open_pos."""
    depth = 0
    for i in range(open_pos, len(text)):
        c = text[i]
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
            if depth == 0:
                return i
    raise ValueError("unbalanced parentheses")


def _split_top(s: str) -> list[str]:
    """Split s on commas that are not inside parentheses."""
    out, depth, cur = [], 0, []
    for c in s:
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        if c == "," and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(c)
    out.append("".join(cur))
    return [x.strip() for x in out]


def transform_launches(text: str) -> tuple[str, int, int]:
    """T1: child launches -> in-thread loops (or the serial convCircular)."""
    n_loop = n_conv = 0
    pat = re.compile(r"(\w+)\s*<<<(.*?)>>>\s*\(", re.S)
    pos = 0
    out = []
    while True:
        m = pat.search(text, pos)
        if not m:
            out.append(text[pos:])
            break
        name, cfg = m.group(1), m.group(2)
        open_pos = m.end() - 1
        close = _match_paren(text, open_pos)
        semi = text.index(";", close)
        if text[close + 1:semi].strip():
            raise ValueError(f"unexpected text after launch of {name}")
        args = text[open_pos + 1:close]
        grid, block = _split_top(cfg)[:2]
        if grid != "1":
            raise ValueError(f"launch of {name} with grid {grid}")
        if name == "d_convCircular":
            repl = f"convCircular({args}, pM->resultConv);"
            n_conv += 1
        else:
            repl = (f"for (int gm_shim_t = 0; gm_shim_t < ({block}); ++gm_shim_t) "
                    f"{name}({args}, gm_shim_t);")
            n_loop += 1
        out.append(text[pos:m.start()])
        out.append(repl)
        pos = semi + 1
    return "".join(out), n_loop, n_conv


def transform_signatures(text: str) -> tuple[str, int]:
    """T2: child __global__ kernels -> __device__ functions taking the index."""
    n = 0
    for name in CHILD_KERNELS:
        pat = re.compile(r"__global__(\s+void\s+" + name + r"\s*)\(")
        pos = 0
        while True:
            m = pat.search(text, pos)
            if not m:
                break
            open_pos = m.end() - 1
            close = _match_paren(text, open_pos)
            text = (text[:m.start()] + "__device__" + m.group(1) + text[open_pos:close] +
                    ", int gm_shim_tid" + text[close:])
            n += 1
            pos = m.start() + 10
    return text, n


def add_missing_return(text: str, func: str) -> str:
    """T5: me_der is declared to return int but ends without a return
    statement and no caller reads its value.  Flowing off the end of a
    non-void function is undefined behaviour in C++, and g++ -O2 optimises
    on it (it assumes the branch that reaches the end is never taken); an
    explicit `return 0;` keeps the function's meaning and removes that."""
    for m in re.finditer(r"\bint\s+" + func + r"\s*\(", text):
        close = _match_paren(text, m.end() - 1)
        if not text[close + 1:].lstrip().startswith("{"):
            continue  # a declaration
        depth = 0
        for i in range(text.index("{", close), len(text)):
            if text[i] == "{":
                depth += 1
            elif text[i] == "}":
                depth -= 1
                if depth == 0:
                    return text[:i] + "\treturn 0;\n" + text[i:]
        raise ValueError(f"{func}: unbalanced braces")
    raise ValueError(f"{func}: definition not found")


def transform_file(name: str, text: str) -> str:
    if name not in EXPECTED:
        return text
    exp = EXPECTED[name]
    text, n_loop, n_conv = transform_launches(text)
    text, n_sig = transform_signatures(text)
    n_index = text.count("blockIdx.x * blockDim.x + threadIdx.x")
    text = text.replace("blockIdx.x * blockDim.x + threadIdx.x", "gm_shim_tid")
    n_sync = len(re.findall(r"\bcudaDeviceSynchronize\(\);", text))
    text = re.sub(r"\bcudaDeviceSynchronize\(\);", ";", text)
    if name == "me_der.cu":
        # T3
        before = text
        text = text.replace("extern __shared__ REAL d_ei[];", "REAL d_ei[MAX_LAMBDA * 7 * 7];")
        if text == before:
            raise ValueError("me_der.cu: shared-memory declaration not found")
        if text.count("__syncthreads();") != 1:
            raise ValueError("me_der.cu: expected one __syncthreads()")
        text = text.replace("__syncthreads();", ";")
        text = add_missing_return(text, "me_der")
    got = dict(launch=n_loop, conv=n_conv, sig=n_sig, index=n_index, sync=n_sync)
    if got != exp:
        raise ValueError(f"{name}: substitutions {got} differ from the expected {exp}")
    return text


def transform_cpu_extra(text: str) -> str:
    """Host build only: dynamic shared arrays of kernels that are compiled
    but never launched (the unused whole-grid convolution and matrix
    kernels) become local arrays, so the host object has no undefined
    symbols."""
    return re.sub(r"extern\s+__shared__\s+(\w+)\s+(\w+)\[\];", r"\1 \2[MAX_LAMBDA * 7 * 7];", text)


def stage(reference: str, dst: str, cpu: bool) -> None:
    for h in HEADERS:
        shutil.copy(os.path.join(reference, h), os.path.join(dst, h))
    for src in DEVICE_SOURCES + HOST_SOURCES:
        with open(os.path.join(reference, src), encoding="latin-1") as f:
            text = f.read()
        text = transform_file(src, text)
        if cpu and src in DEVICE_SOURCES:
            text = transform_cpu_extra(text)
        with open(os.path.join(dst, src), "w", encoding="latin-1") as f:
            f.write(text)


def run(cmd: list[str], cwd: str) -> None:
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {cmd[0]} ... {cmd[-1]}")


def build_cpu(reference: str) -> str:
    os.makedirs(OUT, exist_ok=True)
    out = os.path.join(OUT, "libgmref_cpu.so")
    with tempfile.TemporaryDirectory(prefix="gmref_cpu_") as tmp:
        stage(reference, tmp, cpu=True)
        inc = ["-I", tmp, "-I", SHIM, "-I", os.path.join(CUDA_HOME, "include")]
        flags = ["-O2", "-fPIC", "-fopenmp", "-std=c++17", "-w", "-include",
                 os.path.join(SHIM, "gm_shim_cpu.h")]
        objs = []
        for src in DEVICE_SOURCES + HOST_SOURCES:
            obj = os.path.join(tmp, src + ".o")
            run(["g++", "-x", "c++", *flags, *inc, "-c", os.path.join(tmp, src), "-o", obj], tmp)
            objs.append(obj)
        drv = os.path.join(tmp, "gmref_cpu.o")
        run(["g++", *flags, *inc, "-c", os.path.join(SHIM, "gmref_cpu.cpp"), "-o", drv], tmp)
        objs.append(drv)
        tmp_out = os.path.join(tmp, "libgmref_cpu.so")
        run(["g++", "-shared", "-fopenmp", *objs, "-o", tmp_out, "-Wl,--no-undefined"], tmp)
        shutil.copy(tmp_out, out)
    return out


def build_gpu(reference: str) -> str:
    os.makedirs(OUT, exist_ok=True)
    out = os.path.join(OUT, "libgmref_gpu.so")
    with tempfile.TemporaryDirectory(prefix="gmref_gpu_") as tmp:
        stage(reference, tmp, cpu=False)
        inc = ["-I", tmp, "-I", SHIM]
        nv = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-rdc=true",
              "--ftz=true", "-lineinfo", "-w", "-Xcompiler", "-fPIC"]
        objs = []
        for src in DEVICE_SOURCES:
            obj = os.path.join(tmp, src + ".o")
            run([*nv, *inc, "-include", os.path.join(SHIM, "gm_shim_gpu.h"), "-c",
                 os.path.join(tmp, src), "-o", obj], tmp)
            objs.append(obj)
        for src in HOST_SOURCES:
            obj = os.path.join(tmp, src + ".o")
            run(["g++", "-x", "c++", "-O2", "-fPIC", "-w", *inc, "-I",
                 os.path.join(CUDA_HOME, "include"), "-c", os.path.join(tmp, src), "-o", obj],
                tmp)
            objs.append(obj)
        hobj = os.path.join(tmp, "gmref_gpu.o")
        run([*nv, *inc, "-std=c++17", "-c", os.path.join(SHIM, "gmref_gpu.cu"), "-o", hobj], tmp)
        objs.append(hobj)
        tmp_out = os.path.join(tmp, "libgmref_gpu.so")
        run([*nv, "-shared", *objs, "-o", tmp_out], tmp)
        shutil.copy(tmp_out, out)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--reference", default=None)
    ap.add_argument("--cpu-only", action="store_true")
    a = ap.parse_args(argv)
    reference = locate_reference(a.reference)
    if reference is None:
        print("reference sources not found (--reference, GM_REFERENCE_DIR or ../reference); nothing built")
        return 0
    print(build_cpu(reference))
    if not a.cpu_only:
        print(build_gpu(reference))
    return 0


if __name__ == "__main__":
    sys.exit(main())
