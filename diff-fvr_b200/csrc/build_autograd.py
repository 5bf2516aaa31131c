"""Build the native autograd binding ``fvr/_fvr_autograd.so`` from
``fvr_autograd.cpp`` against the installed PyTorch (host C++ only: it calls
the CUDA library through its C ABI and holds no kernels).

    python build_autograd.py [--force]

Rebuilds only when the source or this script is newer than the library.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "fvr_autograd.cpp"
OUT = HERE.parent / "fvr" / "_fvr_autograd.so"


def _command():
    import torch

    torch_dir = Path(torch.__file__).resolve().parent
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    incs = [torch_dir / "include", torch_dir / "include" / "torch" / "csrc" / "api" / "include",
            Path(cuda_home) / "include", Path(sysconfig.get_paths()["include"])]
    abi = int(bool(torch._C._GLIBCXX_USE_CXX11_ABI))
    lib = torch_dir / "lib"
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           f"-D_GLIBCXX_USE_CXX11_ABI={abi}", "-DTORCH_API_INCLUDE_EXTENSION_H",
           "-DTORCH_EXTENSION_NAME=_fvr_autograd"]
    cmd += [f"-I{p}" for p in incs]
    cmd += [str(SRC), "-o", str(OUT), f"-L{lib}", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu",
            "-ltorch_python", f"-Wl,-rpath,{lib}"]
    return cmd


def build(force: bool = False) -> Path:
    stamp = max(SRC.stat().st_mtime, Path(__file__).stat().st_mtime)
    if not force and OUT.exists() and OUT.stat().st_mtime >= stamp:
        return OUT
    subprocess.run(_command(), check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv[1:]))
