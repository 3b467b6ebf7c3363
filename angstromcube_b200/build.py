"""Build of the sm_100a shared library libangstromcube_b200.so (in-tree, next to this file).

    python -m angstromcube_b200.build            # incremental
    python -m angstromcube_b200.build --force    # rebuild

nvcc cross-compiles for sm_100a without a GPU; the library links the CUDA runtime statically.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libangstromcube_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3", "-I" + INCLUDE, "-I" + CSRC]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _compile(src, obj, verbose):
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc()] + NVCC_FLAGS + ["-x", "cu"] + ARCH + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    return subprocess.Popen(cmd)


def build(force=False, verbose=False):
    """Compile every source that changed and link the shared library; returns its path."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    newest_header = max((os.path.getmtime(h) for h in headers()), default=0)
    procs, objs = [], []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), newest_header)
        if stale:
            procs.append((src, _compile(src, obj, verbose)))
    failed = [s for s, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    if force or procs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
