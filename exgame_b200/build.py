"""Builds libexg.so (the CUDA path, sm_100a) in-tree with nvcc.

Run as `python -m exgame_b200.build`; `__graft_entry__.build()` calls `build()`.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libexg.so")
OBJ_DIR = os.path.join(HERE, "_build")
SOURCES = ["exg_api.cu", "gravity.cu", "joints.cu", "bodies.cu", "newton.cu", "newton_wave.cu", "server.cu",
           "storage.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose=False, force=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    # the traced joint laws first: csrc/user_laws.cuh (rewritten only when its text changes)
    sys.path.insert(0, os.path.dirname(HERE))
    from exgame_b200 import viete
    viete.generate()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(HERE, "..", "include", "exg.h"))
    newest_header = max(os.path.getmtime(h) for h in headers)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ_DIR, src.replace(".cu", ".o"))
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= newest_header):
            continue
        cmd = [_nvcc(), *NVCC_FLAGS, "-c", path, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT, *objs, "-lcudart"]
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
