"""Build recipe of the CUDA library ``glide_b200/libglide_b200.so``.

All kernels are compiled for sm_100a only (B200) with nvcc, into one shared
library that exports the C ABI declared in ``include/glide_b200.h``:

    python -m glide_b200.build            # or glide_b200.build.build()

``-fmad=false`` keeps a*b+c rounded twice, matching the reference's float32
torch CPU arithmetic; the kernels request fused multiply-adds explicitly
where torch's CPU kernels use them.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB_NAME = "libglide_b200.so"
LIB_PATH = PKG / LIB_NAME

SOURCES = ("abi.cu", "window_pack.cu", "step_kernel.cu", "footprint.cu", "convection.cu", "reorder.cu",
           "primitives.cu", "regrid.cu", "compact.cu")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the glide_b200 CUDA library cannot be built")


def _stale() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False, out: Path | None = None,
          extra_flags: list[str] | None = None) -> Path:
    """Compile the library in place (next to this file) if a source is newer than it.
    ``out`` / ``extra_flags`` build a variant elsewhere (always rebuilt)."""
    lib_path = Path(out) if out is not None else LIB_PATH
    if out is None and not force and not ptxas_info and not extra_flags and not _stale():
        return LIB_PATH
    nvcc = nvcc_path()
    out_dir = (lib_path.parent / (lib_path.stem + "_build")) if out is not None else PKG / "_build"
    out_dir.mkdir(exist_ok=True)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in SOURCES:
        obj = out_dir / (Path(src).stem + ".o")
        flags = list(NVCC_FLAGS)
        for f in extra_flags or []:
            if f.startswith("-fmad="):
                flags = [x for x in flags if not x.startswith("-fmad=")]
            flags.append(f)
        cmd = [nvcc, *ARCH_FLAGS, *flags, *extra, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(CSRC / src),
               "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = lib_path.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-cudart", "static", "-o", str(tmp), *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print("built", LIB_PATH)
