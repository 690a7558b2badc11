"""In-tree build of libgft.so and the reference-style CLI binaries.

Compiles every CUDA source for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a -lineinfo``) and the host sources with g++,
then links ``galoisgpu_b200/libgft.so`` (CUDA runtime linked statically) and
``galoisgpu_b200/bin/{bfs,sssp,cc,pr,mis}``.  Objects go to ``galoisgpu_b200/_build``;
unchanged sources are not recompiled.

    python -m galoisgpu_b200.build [--force] [--verbose]
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
INCLUDE = ROOT / "include"
LIB = PKG / "libgft.so"
BIN = PKG / "bin"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIB_SOURCES = [
    "graph_io.cpp",
    "ingest.cpp",
    "output.cpp",
    "gen_host.cpp",
    "engine.cu",
    "traversal.cu",
    "gen_device.cu",
    "batch.cu",
    "msbfs.cu",
    "serve.cpp",
    "resident.cu",
    "cc.cu",
    "pr.cu",
    "mis.cu",
]
HEADERS = ["gft_internal.h", "gen_common.h", "traverse.cuh", "frontier.cuh", "job.cuh"]
CLI_SOURCE = "cli_main.cpp"

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    *ARCH,
    "-lineinfo",
    "--extended-lambda",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    f"-I{INCLUDE}",
    f"-I{CSRC}",
]
CXX_FLAGS = [
    "-std=c++17",
    "-O3",
    "-fPIC",
    "-fvisibility=hidden",
    "-pthread",
    f"-I{INCLUDE}",
    f"-I{CSRC}",
    f"-I{CUDA_HOME / 'include'}",
]


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout.strip() or r.stderr.strip()):
        print(r.stdout, r.stderr, sep="\n", flush=True)


def _compile(src: Path, obj: Path, verbose: bool, ptxas_verbose: bool) -> None:
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    _run(cmd, verbose or ptxas_verbose)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False, jobs: int | None = None) -> Path:
    """Builds libgft.so and the CLI binaries; returns the library path."""
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "gft.h"]
    objs = []
    todo = []
    for name in LIB_SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if force or _newer(obj, [src, *headers]):
            todo.append((src, obj))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        futs = [ex.submit(_compile, s, o, verbose, ptxas_verbose) for s, o in todo]
        for f in futs:
            f.result()
    if force or todo or _newer(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs), "-lpthread", "-lz"], verbose)
        os.replace(tmp, LIB)
    cli_src = CSRC / CLI_SOURCE
    if cli_src.exists():
        for app_id, app in enumerate(("bfs", "sssp", "cc", "pr", "mis")):
            cli_obj = BUILD / f"cli_{app}.o"
            if force or _newer(cli_obj, [cli_src, INCLUDE / "gft.h"]):
                _run(["g++", *CXX_FLAGS, f"-DGFT_CLI_APP={app_id}", "-c", str(cli_src), "-o",
                      str(cli_obj)], verbose)
            exe = BIN / app
            if force or _newer(exe, [cli_obj, LIB]):
                _run(
                    [
                        "g++",
                        "-o",
                        str(exe),
                        str(cli_obj),
                        f"-L{PKG}",
                        "-lgft",
                        "-Wl,-rpath,$ORIGIN/..",
                        "-pthread",
                    ],
                    verbose,
                )
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/smem usage")
    a = ap.parse_args(argv)
    lib = build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
