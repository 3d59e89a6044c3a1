"""Build the CUDA library libfluidb200.so in-tree for sm_100a.

    python -m fluid_simulator_backup_b200.build [--force]

Each .cu file under csrc/ is compiled by nvcc (-gencode
arch=compute_100a,code=sm_100a, -O3, -lineinfo) into _build/, then linked
with the CUDA runtime into fluid_simulator_backup_b200/libfluidb200.so.
The CUDA runtime is linked statically, so the library does not depend on
which libcudart a host process (for instance PyTorch's) has loaded.  Objects
are rebuilt only when a source or header is newer.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfluidb200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    paths.append(os.path.join(ROOT, "include", "fluid_b200.h"))
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, force, hdr_mtime, extra):
    obj = os.path.join(BUILD, src[:-3] + ".o")
    s = os.path.join(CSRC, src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(s), hdr_mtime):
        return obj, None
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", s, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{p.stdout}{p.stderr}"
    return obj, None


def build(force=False, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    hdr = _headers_mtime()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force, hdr, list(extra)), srcs))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{p.stdout}{p.stderr}")
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
