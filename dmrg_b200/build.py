"""Build recipe for the in-tree CUDA library dmrg_b200/libheff_b200.so (sm_100a only).

Each ``csrc/*.cu`` / ``csrc/*.cpp`` is compiled separately (in parallel) with nvcc
into ``_build/`` and linked into one shared library with the CUDA runtime
linked statically, so the library needs nothing but the NVIDIA driver at run time.
"""
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libheff_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_digest():
    hs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h")))
    hs.append(os.path.join(HERE, "..", "include", "heff.h"))
    h = hashlib.sha1()
    for p in hs:
        if os.path.exists(p):
            with open(p, "rb") as f:
                h.update(f.read())
    return h.hexdigest()


def _compile(src, verbose_ptxas=False):
    """Compile one source unless its object was built from identical source, headers and flags (content hash:
    file times can miss an edit made within the same timestamp tick)."""
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    h = hashlib.sha1()
    with open(src, "rb") as f:
        h.update(f.read())
    h.update(_headers_digest().encode())
    h.update(" ".join(ARCH + COMMON).encode())
    digest = h.hexdigest()
    stamp = obj + ".sha1"
    if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == digest:
        return obj, None  # up to date
    cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + COMMON + ["-x", "cu"] + ARCH + ["-c", src, "-o", obj]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    with open(stamp, "w") as f:
        f.write(digest)
    return obj, r.stderr


def build(verbose=False, jobs=None):
    """Compile and link; returns the path of the shared library."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(8, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    if not os.path.exists(LIB) or any(log is not None for _, log in results):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lcuda"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
