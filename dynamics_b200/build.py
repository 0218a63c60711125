"""Build libdynb200.so (all CUDA sources, sm_100a) in-tree.

    python -m dynamics_b200.build          # build if sources are newer
    python -m dynamics_b200.build --force  # always rebuild

The library is a plain shared object with a C ABI (include/dynb200.h); the
CUDA runtime is linked statically and cuFFT dynamically (rpath to the CUDA
toolkit's lib64), so the same .so loads from ctypes, C++ or a Rust FFI.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdynb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = ["errors.cu", "nb_compat.cu", "nblist.cu", "pair.cu", "pme.cu", "integrate.cu",
           "bonded.cu", "system.cu", "batch.cu", "nb_static.cu", "minimize.cu", "list_export.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def cuda_home():
    return os.environ.get("CUDA_HOME", "/usr/local/cuda")


def nvcc():
    return os.path.join(cuda_home(), "bin", "nvcc")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "dynb200.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False):
    """Compile every source into dynamics_b200/libdynb200.so: one object per
    source, compiled in parallel under _build/, then linked."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    lib64 = os.path.join(cuda_home(), "lib64")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", *ARCH,
             "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=default", "-I" + INCLUDE]

    def compile_one(src):
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc(), "-c", *flags, os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}{r.stderr}")
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    cmd = [nvcc(), "-shared", *ARCH, "-cudart", "static", *objs,
           "-L" + lib64, "-lcufft", "-Xlinker", "-rpath=" + lib64, "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, verbose=True)
    print(path)
