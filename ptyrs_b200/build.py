"""Builds `libptyb200.so` in-tree for sm_100a with nvcc (no GPU needed): every translation unit
compiled on its own process (in parallel), then one shared-library link.

    python -m ptyrs_b200.build [--force] [-v]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libptyb200.so")
# the per-side kernel units first: they take longest
SOURCES = ["kernels_256.cu", "kernels_192.cu", "kernels_128.cu", "kernels_96.cu",
           "kernels_64.cu", "engine.cu", "rpie.cu", "lsqml.cu", "ml.cu", "carried.cu",
           "bh.cu", "batch.cu", "forward.cu", "live.cu", "scan.cpp", "h5.cpp", "io.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    for name in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, name)) > t:
            return True
    header = os.path.join(os.path.dirname(HERE), "include", "ptyb200.h")
    return os.path.exists(header) and os.path.getmtime(header) > t


def _headers_mtime():
    names = [os.path.join(CSRC, n) for n in os.listdir(CSRC) if n.endswith((".cuh", ".h"))]
    names.append(os.path.join(os.path.dirname(HERE), "include", "ptyb200.h"))
    return max(os.path.getmtime(n) for n in names if os.path.exists(n))


def _compile(nvcc, src, verbose, force):
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    if not force and os.path.exists(obj):
        t = os.path.getmtime(obj)
        if t > os.path.getmtime(os.path.join(CSRC, src)) and t > _headers_mtime():
            return obj
    cmd = [nvcc] + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + res.stderr[-6000:])
    if verbose:
        sys.stderr.write(res.stderr)
    return obj


def build(force=False, verbose=False, jobs=None):
    """Compiles the library when a source is newer than it; returns its path."""
    if not force and not _stale():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    jobs = jobs or min(len(SOURCES), os.cpu_count() or 4)
    with ThreadPoolExecutor(jobs) as pool:
        objs = list(pool.map(lambda s: _compile(nvcc, s, verbose, force), SOURCES))
    # only the C ABI (ptyb_*) is exported
    exports = "--version-script=" + os.path.join(CSRC, "exports.map")
    # zlib inflates the deflate-compressed chunks of HDF5 files (io.cpp)
    cmd = [nvcc] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-Xlinker", exports] + objs + [
        "-lz", "-o", OUT + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stderr[-4000:])
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
