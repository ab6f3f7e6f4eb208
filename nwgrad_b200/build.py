"""Build the sm_100a shared library ``nwgrad_b200/_lib/libnwgrad_b200.so`` in place.

    python -m nwgrad_b200.build [--force] [--ptxas-v]

nvcc compiles each unit for sm_100a only (the kernels once per precision, in parallel) and
links them with the C ABI (csrc/nwg_capi.cu); the library depends on the CUDA runtime alone
(no torch), so any FFI can load it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libnwgrad_b200.so")
INCLUDE = os.path.join(HERE, "..", "include")
# (object name, source, extra defines)
UNITS = [
    (f"soft_{t}_am{am}", "nwg_soft_inst.cu", [f"-DNWG_T={ty}", f"-DNWG_SOFT_AM={am}", f"-DNWG_SOFT_FN=soft_fn_{t}_am{am}"])
    for t, ty in (("f32", "float"), ("f64", "double")) for am in (0, 1, 2)
] + [
    ("hard_f32", "nwg_hard_inst.cu", ["-DNWG_T=float", "-DNWG_HARD_FN=hard_fn_f32"]),
    ("hard_f64", "nwg_hard_inst.cu", ["-DNWG_T=double", "-DNWG_HARD_FN=hard_fn_f64"]),
    ("capi", "nwg_capi.cu", []),
    ("noalloc", "nwg_noalloc.cu", []),
    ("server", "nwg_server.cu", []),
    ("hb", "nwg_hb.cu", []),
]
DEPS = ["nwg_capi.cu", "nwg_common.cuh", "nwg_hard.cuh", "nwg_walk.cuh", "nwg_soft.cuh", "nwg_kernels.h",
        "nwg_hard_inst.cu", "nwg_soft_inst.cu", "nwg_noalloc.cu", "nwg_server.cu", "nwg_hb.cu", "nwg_hb.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cflags() -> list[str]:
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                   "-I", INCLUDE]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS] + [os.path.join(INCLUDE, "nwgrad_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(unit, verbose, ptxas_v):
    name, src, defs = unit
    obj = os.path.join(OUT_DIR, f"{name}.o")
    cmd = [nvcc_path()] + cflags() + defs + (["-Xptxas", "-v"] if ptxas_v else []) + \
        ["-c", "-o", obj, os.path.join(CSRC, src)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + r.stdout + r.stderr)
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        res = list(ex.map(lambda u: _compile(u, verbose, ptxas_v), UNITS))
    if ptxas_v:
        with open(os.path.join(OUT_DIR, "ptxas.txt"), "w") as f:
            for _, log in res:
                f.write(log)
    tmp = LIB + ".tmp"
    cmd = [nvcc_path()] + ARCH + ["-shared", "-o", tmp] + [o for o, _ in res]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_v="--ptxas-v" in sys.argv))
