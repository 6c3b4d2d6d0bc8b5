"""Builds libsqcuda.so in-tree for sm_100a with nvcc.

The traversal units are compiled with --fmad=false (the exactness contract:
no a*b+c contraction anywhere in the slab and narrow-phase arithmetic);
every unit targets sm_100a only.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsqcuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "--expt-relaxed-constexpr"]

# (source, extra flags)
UNITS = [
    ("sq_api.cu", ["--fmad=false"]),
    ("kernels_d2.cu", ["--fmad=false"]),
    ("kernels_d3.cu", ["--fmad=false"]),
    ("kernels_d4.cu", ["--fmad=false"]),
    ("kernels_d6.cu", ["--fmad=false"]),
    ("sq_tlas.cu", ["--fmad=false"]),
    ("tlas_kernels.cu", ["--fmad=false"]),
    ("guide.cu", []),
    ("tree_build_gpu.cu", ["--fmad=false"]),
    ("sq_f64.cu", ["--fmad=false"]),
    ("rtc.cu", ["-I", BUILD]),
    ("tree_build.cpp", []),
]


def _newer(src: list[str], dst: str) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in src)


def _deps() -> list[str]:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".hpp"))] + [
        os.path.join(HERE, "..", "include", "sq.h")]


def write_rtc_sources() -> None:
    """The traversal headers as string literals, for run-time compilation of
    consumer narrow phases (rtc.cu): _build/rtc_sources.h."""
    out = os.path.join(BUILD, "rtc_sources.h")
    parts = ["// generated by build.py from csrc/sq_math.cuh and csrc/traverse.cuh\n#pragma once\n"]
    for var, name in (("kRtcMath", "sq_math.cuh"), ("kRtcTraverse", "traverse.cuh")):
        text = open(os.path.join(CSRC, name)).read()
        assert ")SQRTC\"" not in text
        parts.append(f'static const char* const {var} = R"SQRTC({text})SQRTC";\n')
    new = "".join(parts)
    if not os.path.exists(out) or open(out).read() != new:
        with open(out, "w") as f:
            f.write(new)


def build(verbose: bool = False, ptxas_info: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    write_rtc_sources()
    deps = _deps()
    objs = []
    cmds = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer([s] + deps, o) or ptxas_info:
            cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if ptxas_info and src.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v")
            cmds.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for cmd, r in ex.map(run, cmds):
            if verbose or r.returncode != 0 or ptxas_info:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed: {cmd[-3]}")
    if cmds or not os.path.exists(LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread", "-lnvrtc",
               "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
