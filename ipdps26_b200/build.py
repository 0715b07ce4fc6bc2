"""Build recipe for the engine's shared library (in-tree, sm_100a only).

Compiles every ``csrc/*.cu`` and ``csrc/*.cpp`` with nvcc for
``arch=compute_100a,code=sm_100a`` and links ``ipdps26_b200/libhmotif.so``
(static cudart, so the library only needs the driver at run time). The
library is built in place so that it travels with the source tree.

    python -m ipdps26_b200.build [--force] [--jobs N]
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
LIB = PKG / "libhmotif.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC,-O3,-Wall",
    "--expt-relaxed-constexpr",
    f"-I{ROOT / 'include'}",
    f"-I{CSRC}",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build the engine")


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    """Compile and link libhmotif.so if any source or header is newer."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = _headers()
    objs, todo = [], []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        cmd = [nvcc] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)
        return src.name

    if todo:
        n = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            for name in ex.map(compile_one, todo):
                if verbose:
                    print(f"compiled {name}", file=sys.stderr)
    if force or todo or _stale(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    build_cli(force)
    build_hmgen(force)
    return LIB


CLI_SRC = PKG / "cli" / "hmotif_cli.cpp"
CLI = PKG / "hmotif"
HMGEN_SRCS = [PKG / "cli" / "hmgen.cpp", CSRC / "hm_gen.cpp", CSRC / "hm_io.cpp", CSRC / "hm_error.cpp"]
HMGEN = PKG / "hmgen"


def build_hmgen(force: bool = False) -> Path:
    """The workload writer: the generator and file-format sources compiled
    with g++ alone (no CUDA, no libhmotif.so), so that a process timing the
    reference's own counters can produce the engine's exact inputs without
    mapping the engine."""
    deps = HMGEN_SRCS + [CSRC / "hm_internal.h", ROOT / "include" / "hmotif.h"]
    if not force and not _stale(HMGEN, deps):
        return HMGEN
    cxx = shutil.which("g++") or "g++"
    tmp = HMGEN.with_suffix(".tmp")
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", f"-I{ROOT / 'include'}", f"-I{CSRC}"] + [str(s) for s in HMGEN_SRCS] + \
          ["-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed on hmgen:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, HMGEN)
    return HMGEN


def build_cli(force: bool = False) -> Path:
    """The command-line driver: host C++ over the C ABI, linked against
    libhmotif.so next to it."""
    if not force and not _stale(CLI, [CLI_SRC, LIB, ROOT / "include" / "hmotif.h"]):
        return CLI
    cxx = shutil.which("g++") or "g++"
    tmp = CLI.with_suffix(".tmp")
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", f"-I{ROOT / 'include'}", str(CLI_SRC), "-o", str(tmp),
           f"-L{PKG}", "-lhmotif", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed on {CLI_SRC.name}:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, CLI)
    return CLI


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))


if __name__ == "__main__":
    main()
