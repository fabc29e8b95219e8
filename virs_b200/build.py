"""Build libvirs_b200.so in place (sm_100a only).

    python -m virs_b200.build            # incremental
    python -m virs_b200.build --force    # rebuild everything

The library goes next to this file so that it travels with the source tree;
nothing is installed into site-packages.
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
LIB = PKG / "libvirs_b200.so"
CLI_SRC = PKG / "cli" / "virs_simulate.cpp"
CLI = PKG / "virs_simulate"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = shutil.which("g++", path="/usr/bin") or "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = [f"-I{ROOT / 'include'}", f"-I{CSRC}"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-Xptxas", "-warn-spills", *INC]
# per-file extra flags: the step kernels flush subnormals like the reference
# build (--use_fast_math implies -ftz=true) and keep every rounding explicit
PER_FILE = {"kernels_step.cu": ["-ftz=true"], "kernels_step_tma.cu": ["-ftz=true"], "kernels_misc.cu": ["-ftz=true"],
            "kernels_ir.cu": ["-ftz=true"], "kernels_voxelize.cu": ["-fmad=false", "-ftz=false"]}
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off", "-Wall",
             f"-I{CUDA_HOME / 'include'}", *INC]


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _needs(src: Path, obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in [src, *deps])


def _compile(src: Path) -> Path:
    obj = OBJ / (src.name + ".o")
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, *PER_FILE.get(src.name, []), "-c", str(src), "-o", str(obj)]
    else:
        cmd = [CXX, *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        print(r.stderr.strip(), file=sys.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    deps = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    srcs = sources()
    todo = [s for s in srcs if force or _needs(s, OBJ / (s.name + ".o"), deps)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj in ex.map(_compile, todo):
                if verbose:
                    print("built", obj.name)
    objs = [OBJ / (s.name + ".o") for s in srcs]
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, "-shared", *ARCH, "-cudart", "static", "-o", str(LIB), *map(str, objs), "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    build_cli(force)
    return LIB


def build_cli(force: bool = False) -> Path:
    """The command-line program over the library (next to it, found through
    its rpath)."""
    deps = [CLI_SRC, LIB, ROOT / "include" / "virs.h", ROOT / "include" / "virs.hpp"]
    if force or not CLI.exists() or any(d.stat().st_mtime > CLI.stat().st_mtime for d in deps):
        cmd = [CXX, "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(CLI_SRC), f"-L{PKG}",
               "-lvirs_b200", "-Wl,-rpath,$ORIGIN", "-o", str(CLI)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return CLI


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
