"""Build liblcmx.so in-tree with nvcc for sm_100a.

``python -m pylcm_b200.build`` (also called by ``__graft_entry__.build()``).
The library links NVRTC (to compile generated model code at run time), the
CUDA driver API (module loading / launches) and the runtime.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "liblcmx.so"
SOURCES = ["lcmx.cu", "fues.cu", "envelopes.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def cuda_home() -> Path:
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and Path(cand, "bin", "nvcc").exists():
            return Path(cand)
    nvcc = shutil.which("nvcc")
    if nvcc:
        return Path(nvcc).resolve().parent.parent
    raise RuntimeError("nvcc not found (set CUDA_HOME)")


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES if (CSRC / s).exists()]


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + [PKG.parent / "include" / "lcmx.h"] + list((CSRC / "kernels").glob("*"))
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    home = cuda_home()
    OUT_DIR.mkdir(exist_ok=True)
    cmd = [
        str(home / "bin" / "nvcc"),
        *ARCH,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-shared",
        "-Xcompiler",
        "-fPIC",
        "-Xptxas",
        "-v" if verbose else "-O3",
        *map(str, sources()),
        "-o",
        str(LIB) + ".tmp",
        f"-L{home / 'lib64'}",
        "-lnvrtc",
        "-lcudart",
        f"-Xlinker=-rpath,{home / 'lib64'}",
    ]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
