"""Build the native libraries of the Myers B200 package, in place.

    libmyers_b200.so   CUDA kernels (sm_100a) + host runtime + C ABI
    libmyers_synth.so  seeded synthetic workload generator (host C, OpenMP)

Run as a script or call build(). nvcc cross-compiles for sm_100a without a
GPU. Rebuilds only when a source is newer than its library.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["myers_kernels.cu", "myers_api.cu", "myers_serve.cu", "myers_traceback.cu"]
CUDA_HEADERS = ["myers_internal.h", "myers_device.cuh", os.path.join("..", "..", "include", "myers-interface.h")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_cuda(verbose_ptxas=False):
    """Compile each CUDA source to an object in parallel (the kernels' file
    takes most of the time), then link the shared library."""
    out = os.path.join(HERE, "libmyers_b200.so")
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    headers = [os.path.join(CSRC, h) for h in CUDA_HEADERS] + [__file__]
    extra = os.environ.get("MYERS_NVCC_FLAGS", "").split()  # e.g. -DMYERS_SHIFT_MODE=2
    stamp = out + ".flags"
    if os.path.exists(stamp) and open(stamp).read() != " ".join(extra):
        os.remove(out)  # rebuild when the build options change
        os.remove(stamp)
    if not _newer(out, srcs + headers) and not verbose_ptxas:
        return out
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", *extra,
              "-I", os.path.join(ROOT, "include")]
    if verbose_ptxas:
        common.insert(1, "-Xptxas=-v")
    objs, procs = [], []
    for src in srcs:
        obj = os.path.join(objdir, os.path.splitext(os.path.basename(src))[0] + ".o")
        objs.append(obj)
        if verbose_ptxas or not os.path.exists(stamp) or _newer(obj, [src, stamp] + headers):
            cmd = common + ["-c", "-o", obj, src]
            print(" ".join(cmd), flush=True)
            procs.append((cmd, subprocess.Popen(cmd)))
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs])
    with open(stamp, "w") as f:
        f.write(" ".join(extra))
    return out


def build_synth():
    out = os.path.join(HERE, "libmyers_synth.so")
    src = os.path.join(CSRC, "synth.c")
    if not _newer(out, [src, __file__]):
        return out
    _run(["gcc", "-O3", "-fPIC", "-fopenmp", "-shared", "-o", out, src, "-lm"])
    return out


def build(verbose_ptxas=False):
    return build_cuda(verbose_ptxas), build_synth()


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
