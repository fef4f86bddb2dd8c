"""Build recipe for the CUDA library libconductor_rigid.so (sm_100a).

Compiles every source under csrc/ with nvcc for ``sm_100a`` and links the shared
library in-tree next to this file, so it travels with the repository to the GPU
machine.  Incremental: an object is rebuilt when its source or any header changed.

    python -m conductorrigid_b200.build [--force] [-j N]
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
OBJ = PKG / "_build"
LIB = PKG / "libconductor_rigid.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("CUDA_HOME", ""), "/usr/local/cuda"):
        p = Path(cand) / "bin" / "nvcc"
        if cand and p.exists():
            return str(p)
    found = shutil.which("nvcc")
    if not found:
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libconductor_rigid.so")
    return found


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cc")))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h")))


def _compile_cmd(nvcc: str, src: Path, obj: Path) -> list[str]:
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"), "-ccbin", "g++"]
    if src.suffix == ".cu":
        return [nvcc, *ARCH, "-lineinfo", "--expt-relaxed-constexpr", "--extended-lambda", *common,
                "-c", str(src), "-o", str(obj)]
    return [nvcc, *common, "-x", "c++", "-c", str(src), "-o", str(obj)]


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    nvcc = _nvcc()
    OBJ.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    todo = []
    objs = []
    for src in _sources():
        obj = OBJ / (src.name + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            todo.append((src, obj))

    def run(item):
        src, obj = item
        cmd = _compile_cmd(nvcc, src, obj)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, file=sys.stderr)
        return src.name

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
            for name in ex.map(run, todo):
                if verbose:
                    print("compiled", name)
    if force or todo or not LIB.exists():
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcufft", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def build_module(force: bool = False) -> Path:
    """The pybind11 module _ConductorRigid (C++ force compute, reference surface)."""
    import sysconfig

    import pybind11

    src = PKG / "pybind" / "_ConductorRigid.cc"
    out = PKG / ("_ConductorRigid" + sysconfig.get_config_var("EXT_SUFFIX"))
    deps = [src, LIB, ROOT / "include" / "ConductorRigid.hpp"]
    if not force and out.exists() and out.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return out
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(ROOT / "include"), "-I", pybind11.get_include(),
           "-I", sysconfig.get_paths()["include"], str(src), "-L", str(PKG), "-lconductor_rigid",
           "-Wl,-rpath,$ORIGIN", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"pybind11 module build failed:\n{r.stdout}\n{r.stderr}")
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.j, verbose=a.v))
    print(build_module(force=a.force))


if __name__ == "__main__":
    main()
