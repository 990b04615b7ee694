"""Build the B200 library liblsmoke_gpu.so in-tree with nvcc (sm_100a).

The plain FP64 kernels, the output-field kernels and the property kernel are compiled with FMA
contraction off so their arithmetic rounds like the CPU reference; everything
else is compiled normally.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
OUT = os.path.join(PKG, "liblsmoke_gpu.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]

UNITS = [
    ("lsg_plain.cu", ["-fmad=false"]),
    ("lsg_batched.cu", []),
    ("lsg_rounds.cu", []),
    ("lsg_block.cu", []),
    ("lsg_outputs.cu", ["-fmad=false"]),
    ("lsg_properties.cu", ["-fmad=false"]),
    ("lsg_api.cu", []),
    ("lsg_mech_host.cpp", []),
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.exists(c) or c == "nvcc"):
            return c
    return "nvcc"


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    headers = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(PKG), "include", "lsmoke_gpu.h"))
    newest_header = max(os.path.getmtime(h) for h in headers if os.path.exists(h))
    for src, extra in UNITS:
        s = os.path.join(HERE, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if (not force and os.path.exists(o) and os.path.getmtime(o) >= os.path.getmtime(s)
                and os.path.getmtime(o) >= newest_header):
            continue
        cmd = [nvcc()] + ARCH + COMMON + extra + ["-c", s, "-o", o]
        if src.endswith(".cpp"):
            cmd = [nvcc()] + COMMON + ["-Wno-deprecated-gpu-targets", "-x", "c++", "-c", s, "-o", o]
        if verbose:
            cmd += ["-Xptxas", "-v"] if src.endswith(".cu") else []
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    if force or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
