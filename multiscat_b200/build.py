"""Build the native CUDA library in-tree (sm_100a).

``python -m multiscat_b200.build`` compiles ``csrc/*.cu`` into
``multiscat_b200/libmultiscat_b200.so`` with nvcc.  Nothing is JIT-compiled
at import time: the built library travels with the source tree.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libmultiscat_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(cand).exists():
        raise RuntimeError("nvcc not found; set PATH to include the CUDA toolkit")
    return cand


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[pathlib.Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) +
                  list((PKG.parent / "include").glob("*.h")))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    if not force and up_to_date():
        return LIB
    cuda_home = pathlib.Path(nvcc_path()).resolve().parent.parent
    cmd = [
        nvcc_path(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--use_fast_math=false",
        "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-shared", "-cudart", "shared",
        f"-I{PKG.parent / 'include'}",
        "-o", str(LIB), *[str(s) for s in sources()],
        f"-L{cuda_home / 'lib64'}", f"-Xlinker", f"-rpath,{cuda_home / 'lib64'}",
    ]
    cmd = [c for c in cmd if c != "--use_fast_math=false"]
    if verbose:
        print(" ".join(cmd))
    env = dict(os.environ)
    subprocess.run(cmd, check=True, env=env)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
