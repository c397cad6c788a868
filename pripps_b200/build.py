"""Build the CUDA library in-tree: pripps_b200/libpripps_debye.so (sm_100a).

    python -m pripps_b200.build [--force] [--verbose]

Compiles pripps_b200/csrc/*.cu and *.cpp with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) and links the CUDA runtime
statically, so the library depends on nothing but the driver. The object
files go to pripps_b200/_build/ (git-ignored); the .so lands next to this
file, where pripps_b200._lib loads it.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libpripps_debye.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
              "--expt-relaxed-constexpr", "-Xptxas", "-v"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build pripps_b200")


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    nvcc = nvcc_path()
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    objs = []
    ptxas_log = []
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src, *headers]):
            continue
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src),
               "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd[cmd.index("-c"):cmd.index("-c")] = ["-x", "cu"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed on {src.name}")
        ptxas_log.append(res.stderr)
        if verbose:
            sys.stderr.write(res.stderr)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static",
               "-Xcompiler", "-fPIC", "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("nvcc link failed")
    if ptxas_log:
        (BUILD / "ptxas.log").write_text("\n".join(ptxas_log))
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()
