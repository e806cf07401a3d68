"""Build libdpkem.so in-tree: every CUDA source compiled for sm_100a with nvcc.

    python -m dpcrypto_b200.build          # or dpcrypto_b200.build.build()

The shared library lands next to this file (dpcrypto_b200/libdpkem.so) so it travels
with the working tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdpkem.so")
SOURCES = ["frodo.cu", "saber.cu", "coins.cu", "peak.cu", "keccak_lanes.cu", "abi.cu", "noalloc.cu", "mixed.cu",
           "frames.cu", "serve.cu"]
# The persistent mixed-batch and service kernels read data other CTAs (and the host's
# copies) wrote during the launch: their global loads bypass the (non-coherent) L1.
EXTRA = {"mixed.cu": ["-Xptxas", "-dlcm=cg"], "serve.cu": ["-Xptxas", "-dlcm=cg"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    inc = os.path.join(HERE, "..", "include")
    deps += [os.path.join(inc, h) for h in os.listdir(inc) if h.endswith(".h")]
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


TUNING = os.path.join(HERE, "tuning.json")


def tuning_defines() -> list:
    """Compile-time knobs chosen by the autotuner (dpcrypto_b200/tuning.json)."""
    import json

    if not os.path.exists(TUNING):
        return []
    with open(TUNING) as f:
        chosen = json.load(f).get("chosen", {})
    defs = []
    for key, macro in (("keccak_unroll", "DPKEM_KECCAK_UNROLL"), ("keccak_unroll_rows", "DPKEM_KECCAK_UNROLL_ROWS")):
        if key in chosen:
            defs.append(f"-D{macro}={int(chosen[key])}")
    return defs


def build(verbose: bool = False, out: str | None = None, defines: list | None = None) -> str:
    lib = out or LIB
    defs = tuning_defines() if defines is None else defines
    obj_dir = OBJ if out is None else os.path.join(os.path.dirname(os.path.abspath(out)), "_obj")
    os.makedirs(obj_dir, exist_ok=True)
    stamp = os.path.join(obj_dir, "defines.txt")
    stale_defs = not os.path.exists(stamp) or open(stamp).read() != " ".join(defs)
    cc = nvcc()
    jobs = []
    for s in SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(obj_dir, s + ".o")
        if stale_defs or _stale(src, obj):
            jobs.append([cc, *FLAGS, *defs, *EXTRA.get(s, []), *ARCH, "-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)

    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        list(ex.map(run, jobs))
    with open(stamp, "w") as f:
        f.write(" ".join(defs))
    objs = [os.path.join(obj_dir, s + ".o") for s in SOURCES]
    if jobs or not os.path.exists(lib):
        link = [cc, *ARCH, "-shared", "-o", lib, *objs, "-lcudart"]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
