"""Build the native libraries in-tree.

    lib/libkfb200.so   -- the CUDA pipeline behind include/kf_api.h (sm_100a only)
    lib/libkfsynth.so  -- the synthetic depth-sequence generator (host only)

Run ``python build.py`` from anywhere; nvcc cross-compiles for sm_100a without a GPU.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "_build")
REPO = os.path.dirname(HERE)

CU_SOURCES = ["k_preprocess.cu", "k_raycast.cu", "k_tsdf.cu", "k_icp.cu", "k_display.cu", "k_probe.cu", "api.cu"]
CXX_SOURCES = ["dataset.cpp"]   # host-only parts of the library (zlib for 16-bit PNG)
# The depth pyramid is computed with the float semantics of the reference's Release build
# (FastMath, project/project.vcxproj:139): denormals flushed, division and square root to the
# fast forms.  With the same operations in the same order, the converted, filtered and
# down-sampled depth and the vertex maps are then bit-identical to the reference's kernels.
FILE_FLAGS = {"k_preprocess.cu": ["-ftz=true", "-prec-div=false", "-prec-sqrt=false", "-fmad=true"]}
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-I", os.path.join(REPO, "include"),
]


def _nvcc():
    for cand in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), "nvcc"):
        if shutil.which(cand) or os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, h) for h in ("kf_device.cuh", "kf_host.h")] + \
        [os.path.join(REPO, "include", "kf_api.h")]
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    objs = []
    jobs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if ptxas_info or _stale(o, [s] + headers + [os.path.abspath(__file__)]):
            jobs.append([nvcc] + NVCC_FLAGS + FILE_FLAGS.get(src, []) + extra + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cpp", ".o"))
        objs.append(o)
        if _stale(o, [s, os.path.join(REPO, "include", "kf_api.h")]):
            jobs.append([_cxx(), "-O2", "-std=c++17", "-fPIC", "-I", os.path.join(REPO, "include"), "-c", s, "-o", o])
    logs = []
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(lambda c: _run(c, verbose), jobs):
            logs.append(out)
    so = os.path.join(LIB, "libkfb200.so")
    if jobs or not os.path.exists(so):
        _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", so] + objs + ["-lz"], verbose)
    synth = os.path.join(LIB, "libkfsynth.so")
    ssrc = os.path.join(CSRC, "synth.cpp")
    if _stale(synth, [ssrc]):
        _run([_cxx(), "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-o", synth, ssrc], verbose)
    return "\n".join(logs)


if __name__ == "__main__":
    info = "-v" in sys.argv
    out = build(verbose=True, ptxas_info=info)
    if info:
        print(out)
