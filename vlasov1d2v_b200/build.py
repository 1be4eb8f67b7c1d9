"""Build the sm_100a shared library ``libvlasov1d2v.so`` in-tree with nvcc.

    python -m vlasov1d2v_b200.build          # or: python vlasov1d2v_b200/build.py

The library is a plain C ABI (``include/vlasov1d2v.h``) with the CUDA runtime linked
statically, so it loads with ctypes next to any PyTorch build.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libvlasov1d2v.so")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-fvisibility=hidden"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(INCLUDE, "vlasov1d2v.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    """Compile every translation unit in parallel (one nvcc per file), then link the library."""
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(objdir, os.path.basename(f)[:-3] + ".o") for f in srcs]

    def compile_one(src_obj):
        src, obj = src_obj
        cmd = [nvcc(), *ARCH_FLAGS, *COMMON, "-I", INCLUDE, "-I", CSRC, "-c", "-o", obj, src, *extra]
        if verbose:
            print(" ".join(cmd))
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, zip(srcs, objs)))
    for src, r in zip(srcs, results):
        if r.stdout or r.stderr:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, f"nvcc {os.path.basename(src)}")
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH_FLAGS, "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    args = sys.argv[1:]
    build(force=True, verbose=True, extra=[a for a in args if a != "-v"])
