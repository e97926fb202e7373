"""Build recipe of the native library libvfb200.so (sm_100a).

Every CUDA and C++ source under csrc/ is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared library
next to this file, so the library travels with the source tree.  Objects are
rebuilt when a source or any header under csrc/ or include/ is newer.

    python -m virtualfluids_b200.build [--force] [--verbose]
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
OBJ = ROOT / "_build" / "obj"
LIB = PKG / "libvfb200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    # the image's default CC wrapper lacks OpenMP specs; use the system g++
    gxx = shutil.which("g++", path="/usr/bin") or shutil.which("g++")
    return ["-ccbin", gxx] if gxx else []


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def compile_one(src: Path, force: bool, verbose: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, headers_mtime()):
        return obj
    obj.parent.mkdir(parents=True, exist_ok=True)
    cmd = [nvcc(), *host_compiler(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


GEN = PKG / "gen" / "adjoint_gen.cpp"
GEN_OUT = CSRC / "adjoint_ops.gen.cuh"


def cuda_include() -> str:
    return str(Path(nvcc()).resolve().parent.parent / "include")


def generate_adjoint(out: Path = GEN_OUT, verbose: bool = False) -> Path:
    """Compile and run the adjoint generator (host C++), writing the reverse
    sweep of the K17 operator to `out` (the header is rewritten only when its
    content changes, so an unchanged operator does not trigger a rebuild)."""
    exe = ROOT / "_build" / "gen" / "adjoint_gen"
    exe.parent.mkdir(parents=True, exist_ok=True)
    gxx = shutil.which("g++", path="/usr/bin") or shutil.which("g++") or "g++"
    cmd = [gxx, "-std=c++17", "-O1", "-I", cuda_include(), str(GEN), "-o", str(exe)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"adjoint generator failed to compile:\n{r.stdout}\n{r.stderr}")
    tmp = exe.parent / "adjoint_ops.gen.cuh.new"
    r = subprocess.run([str(exe), str(tmp)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"adjoint generator failed:\n{r.stdout}\n{r.stderr}")
    if not out.exists() or out.read_bytes() != tmp.read_bytes():
        shutil.copyfile(tmp, out)
    tmp.unlink()
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    # the generated reverse sweep follows the operator it is traced from
    op = CSRC / "collision_math.cuh"
    if force or not GEN_OUT.exists() or GEN_OUT.stat().st_mtime < max(GEN.stat().st_mtime, op.stat().st_mtime):
        generate_adjoint(verbose=verbose)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), *host_compiler(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
