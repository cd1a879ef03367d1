"""Builds the sm_100a CUDA library npme_b200/libnpme_gpu.so in-tree.

    python -m npme_b200.build [--force]

nvcc compiles each translation unit of npme_b200/csrc for
`-gencode arch=compute_100a,code=sm_100a` (cross-compiles without a GPU) and
links them with cuFFT into one shared library exporting the C ABI declared in
include/npme_gpu.h.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnpme_gpu.so")
SOURCES = ["npme_gpu.cu", "setup.cu", "recsum.cu", "direct.cu", "noalloc.cu", "batch.cu", "fft.cu",
           "server.cu", "choose.cu"]
APPS = os.path.join(HERE, "apps")
BIN = os.path.join(HERE, "bin")
APPS_SRC = ["npme", "compareV", "makeRandomBox"]
HEADERS = ["common.cuh", "bodies.cuh", "internal.h",
           os.path.join("..", "..", "include", "npme_gpu.h")]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
         "-gencode", "arch=compute_100a,code=sm_100a",
         "--expt-relaxed-constexpr", "-Xptxas", "-v"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    cc = nvcc()
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            jobs.append([cc] + FLAGS + ["-c", src, "-o", obj])

    def run(cmd):
        p = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, p

    with cf.ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        for cmd, p in ex.map(run, jobs):
            log = os.path.join(OBJ, os.path.basename(cmd[-1]) + ".ptxas.txt")
            with open(log, "w") as f:
                f.write(p.stdout + p.stderr)
            if p.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + p.stderr[-6000:])
            if verbose:
                print(p.stderr)
    if force or jobs or _stale(LIB, objs):
        cmd = [cc, "-shared", "-o", LIB] + objs + [
            "-gencode", "arch=compute_100a,code=sm_100a", "-lcufft", "-lcudart"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + " ".join(cmd) + "\n" + p.stderr[-4000:])
    build_peak(force)
    build_apps(force)
    return LIB


PEAK = os.path.join(HERE, "libnpme_peak.so")


def build_peak(force=False):
    """The FP32 FMA throughput probe bench.py reports as the direct sum's
    roofline peak (npme_b200/libnpme_peak.so, C entry npme_peak_fp32)."""
    src = os.path.join(CSRC, "peak.cu")
    if not force and not _stale(PEAK, [src]):
        return
    cmd = [nvcc()] + FLAGS + ["-shared", "-o", PEAK, src]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + p.stderr[-4000:])


def build_apps(force=False):
    """Command-line tools of the reference (npme, compareV, makeRandomBox)
    over the C ABI, into npme_b200/bin/ (rpath to the library)."""
    os.makedirs(BIN, exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    hdrs = [os.path.join(APPS, "npme_io.h"), os.path.join(HERE, "..", "include", "npme_gpu.h")]
    for app in APPS_SRC:
        src = os.path.join(APPS, app + ".cpp")
        exe = os.path.join(BIN, app)
        if not force and not _stale(exe, [src, LIB] + hdrs):
            continue
        cmd = [cxx, "-std=c++17", "-O2", "-o", exe, src, "-L" + HERE, "-lnpme_gpu",
               "-Wl,-rpath,$ORIGIN/.."]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("app build failed:\n" + " ".join(cmd) + "\n" + p.stderr[-4000:])


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
