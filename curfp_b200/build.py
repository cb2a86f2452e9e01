"""Build libcurfp_b200.so in-tree with nvcc for sm_100a.

    python -m curfp_b200.build          # incremental
    python -m curfp_b200.build --force  # rebuild everything

Objects go to curfp_b200/_build/, the shared library to
curfp_b200/libcurfp_b200.so (next to the Python package that loads it).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcurfp_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) +
                  list((ROOT / "include").glob("*.h")))


def _compile(src: Path, extra: list[str]) -> Path:
    obj = BUILD / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in headers()])
    if obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [nvcc(), "-x", "cu"] + NVCC_FLAGS + extra + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    extra = extra or []
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as pool:
        objs = list(pool.map(lambda s: _compile(s, extra), sources()))
    if LIB.exists() and not force and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ([nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] +
           ["-lcuda", "-Xlinker", "--no-undefined"])  # an unresolved symbol fails the build
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


TORCH_SRC = PKG / "csrc_torch" / "torch_ops.cpp"
TORCH_BUILD = PKG / "_torch_build"
TORCH_EXT = TORCH_BUILD / "curfp_torch_ops.so"


def build_torch_ext(verbose: bool = False) -> Path:
    """The torch extension (torch.ops.curfp_b200.*) over the C ABI, built
    in-tree next to the library it links (rpath $ORIGIN/..)."""
    from torch.utils import cpp_extension
    build()
    TORCH_BUILD.mkdir(exist_ok=True)
    cpp_extension.load(
        name="curfp_torch_ops", sources=[str(TORCH_SRC)],
        extra_include_paths=[str(ROOT / "include")],
        extra_cflags=["-O2"],
        extra_ldflags=[f"-L{PKG}", "-lcurfp_b200", "-Wl,-rpath,'$$ORIGIN/..'"],
        build_directory=str(TORCH_BUILD), with_cuda=True, is_python_module=False,
        verbose=verbose)
    return TORCH_EXT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill info")
    a = ap.parse_args()
    build(force=a.force or a.ptxas_v, verbose=True,
          extra=["-Xptxas", "-v"] if a.ptxas_v else None)
    build_torch_ext()
    sys.exit(0)
