"""Build cufe_b200/libcufe_b200.so: the sm_100a CUDA kernels and the C ABI (in-tree)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcufe_b200.so")
SOURCES = ["ipfe.cu", "sampler.cu", "batch.cu", "svm.cu", "serial.cu", "staging.cpp", "capi.cpp"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "cufe_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False):
    """compile every source (in parallel, one nvcc per file) and link the shared library;
    without force only when a source or the public header is newer than the library"""
    from concurrent.futures import ThreadPoolExecutor
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose else []

    def compile_one(src):
        obj = os.path.join(objdir, src + ".o")
        cmd = [NVCC, "-c", os.path.join(CSRC, src), "-o", obj] + FLAGS + extra
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, "-shared", "-o", tmp] + objs + ["-gencode", "arch=compute_100a,code=sm_100a"],
                   check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
