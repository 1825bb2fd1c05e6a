#!/usr/bin/env python3
"""Builds libanqi.so (CUDA, sm_100a) and the three command-line drivers in-tree.

    python anqi-implementation_b200/build.py [--clean] [--jobs N]

Objects go to anqi-implementation_b200/_build/; the library and the CLIs land
next to this file (lib/libanqi.so, bin/build_aknn_source, bin/rknn_query,
bin/dataset_gt) so they travel with the repository snapshot.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
CSRC = HERE / "csrc"
CLI = HERE / "cli"
BUILD = HERE / "_build"
LIB = HERE / "lib" / "libanqi.so"
BIN = HERE / "bin"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-Xptxas", "-warn-spills", f"-I{REPO / 'include'}", f"-I{CSRC}"]
CXX = "g++"
CXXFLAGS = ["-O2", "-std=c++17", "-Wall", "-Wextra", f"-I{REPO / 'include'}", f"-I{CLI}"]


def run(cmd: list[str]) -> None:
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + p.stdout + p.stderr)
        raise SystemExit(f"build failed: {cmd[-1]}")
    for line in (p.stdout + p.stderr).splitlines():
        if "spill" in line.lower() and "0 bytes spill" not in line:
            print(line)


def newer(src: list[Path], dst: Path) -> bool:
    if not dst.exists():
        return True
    t = dst.stat().st_mtime
    return any(s.stat().st_mtime > t for s in src)


def build(clean: bool = False, jobs: int = 8, verbose: bool = False) -> Path:
    if clean and BUILD.exists():
        shutil.rmtree(BUILD)
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [REPO / "include" / "anqi.h"]
    sources = sorted(CSRC.glob("*.cu"))
    objs = []
    todo = []
    for s in sources:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if newer([s] + headers, o):
            todo.append([NVCC, *ARCH, *NVFLAGS, "-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        list(ex.map(run, todo))
    if todo or newer(objs, LIB):
        run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)])
    # CLIs: C++17 host code over the C ABI
    cli_common = sorted(CLI.glob("*.h"))
    for name in ("build_aknn_source", "rknn_query", "dataset_gt"):
        src = CLI / f"{name}.cpp"
        if not src.exists():
            continue
        out = BIN / name
        extra = [p for p in sorted(CLI.glob("*_lib.cpp"))]
        if newer([src, LIB, *cli_common, *extra], out):
            run([CXX, *CXXFLAGS, str(src), *map(str, extra), "-o", str(out), f"-L{LIB.parent}", "-lanqi",
                 "-Wl,-rpath,$ORIGIN/../lib", "-lpthread"])
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    a = ap.parse_args()
    lib = build(a.clean, a.jobs)
    print(f"built {lib}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
