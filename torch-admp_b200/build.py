"""Build libadmp_b200.so (all CUDA sources, sm_100a) into the package directory.

    python torch-admp_b200/build.py [--force] [--debug]

The library is a plain C-ABI shared object (no torch dependency); the Python
package loads it with ctypes.  Sources are compiled in parallel, one object
per translation unit, then linked with nvcc.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
OUT_DIR = os.path.join(HERE, "admp_b200")
LIB = os.path.join(OUT_DIR, "libadmp_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _digest(extra):
    h = hashlib.sha256()
    for f in sorted(os.listdir(CSRC)) + [os.path.join(INCLUDE, x) for x in sorted(os.listdir(INCLUDE))]:
        p = f if os.path.isabs(f) else os.path.join(CSRC, f)
        if os.path.isfile(p):
            h.update(p.encode())
            h.update(open(p, "rb").read())
    h.update(" ".join(ARCH + FLAGS + extra).encode())
    return h.hexdigest()


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    extra = ["-DADMP_DEBUG=1"] if debug else []
    stamp = os.path.join(OUT_DIR, ".libadmp_b200.sha256")
    dig = _digest(extra)
    if not force and os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read().strip() == dig:
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(OBJ_DIR, os.path.basename(s)[:-3] + ".o") for s in srcs]

    def compile_one(args):
        src, obj = args
        cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(compile_one, zip(srcs, objs)))
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


TORCH_OPS_SRC = os.path.join(CSRC, "torch_ops.cpp")
TORCH_OPS = os.path.join(OUT_DIR, "_torch_ops.so")


def build_torch_ops(force: bool = False, verbose: bool = False) -> str:
    """TorchScript-visible operators (torch.ops.admp_b200.*, csrc/torch_ops.cpp):
    a C++ torch extension linked against libadmp_b200.so (rpath $ORIGIN)."""
    import torch
    from torch.utils import cpp_extension as ce
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    incs = ce.include_paths(device_type="cuda") if "device_type" in ce.include_paths.__code__.co_varnames \
        else ce.include_paths(cuda=True)
    libs = ce.library_paths(device_type="cuda") if "device_type" in ce.library_paths.__code__.co_varnames \
        else ce.library_paths(cuda=True)
    flags = ["-O2", "-std=c++17", "-shared", "-fPIC", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
             "-DTORCH_EXTENSION_NAME=_torch_ops", f"-I{INCLUDE}"] + [f"-I{d}" for d in incs]
    h = hashlib.sha256()
    for f in (TORCH_OPS_SRC, os.path.join(INCLUDE, "admp_b200.h")):
        h.update(open(f, "rb").read())
    h.update((" ".join(flags) + torch.__version__).encode())
    dig = h.hexdigest()
    stamp = os.path.join(OUT_DIR, ".torch_ops.sha256")
    if not force and os.path.exists(TORCH_OPS) and os.path.exists(stamp) and open(stamp).read().strip() == dig:
        return TORCH_OPS
    tmp = TORCH_OPS + ".tmp"
    cmd = (["g++"] + flags + [TORCH_OPS_SRC, "-o", tmp] + [f"-L{d}" for d in libs] +
           ["-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", f"-L{OUT_DIR}", "-ladmp_b200",
            "-Wl,-rpath,$ORIGIN"] + [f"-Wl,-rpath,{d}" for d in libs])
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"torch ops build failed:\n{r.stdout}\n{r.stderr[-6000:]}")
    os.replace(tmp, TORCH_OPS)
    with open(stamp, "w") as f:
        f.write(dig)
    return TORCH_OPS


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, debug=a.debug, verbose=a.verbose))
    print(build_torch_ops(force=a.force, verbose=a.verbose))
    sys.exit(0)
