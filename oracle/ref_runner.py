"""Runs the reference's own compiled counters (oracle/_ref, built by
build_ref.sh from the reference sources). TEST INFRASTRUCTURE ONLY.

Inputs are written in each program's own text format: MoCHy reads 0-based
comma-separated node lists, one hyperedge per line
(MoCHy-master/read_data.cpp:8-45); THyMe reads "n1,n2,...<TAB>time" lines
(THyMe-main/code/read_data.cpp:22-58).
"""
from __future__ import annotations

import os
import re
import subprocess
import tempfile
import time
from pathlib import Path

import numpy as np

REF = Path(__file__).resolve().parent / "_ref"


def available(name: str) -> bool:
    return (REF / name).exists()


def write_mochy(path, offsets, members) -> None:
    with open(path, "w") as f:
        for e in range(len(offsets) - 1):
            f.write(",".join(map(str, members[offsets[e] : offsets[e + 1]].tolist())) + "\n")


def write_thyme(path, offsets, members, times) -> None:
    with open(path, "w") as f:
        for e in range(len(offsets) - 1):
            f.write(",".join(map(str, members[offsets[e] : offsets[e + 1]].tolist())) + f"\t{int(times[e])}\n")


_MOTIF = re.compile(r"^motif (\d+): (\d+)$", re.M)
_RT = re.compile(r"TOTAL_RUNTIME_SECONDS\s+([0-9.eE+-]+)")


def run_mochy_file(path, threads: int | None = None, timeout: float | None = None):
    """MoCHy main_exact (threads=None) or main_exact_par on a file in its own
    format. Returns (26 counts, wall seconds of the child process including
    its file parse, self-reported seconds excluding the parse)."""
    if threads is None:
        cmd = [str(REF / "mochy_exact"), str(path)]
    else:
        cmd = [str(REF / "mochy_exact_par"), str(threads), str(path)]
    t0 = time.perf_counter()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, check=True)
    wall = time.perf_counter() - t0
    counts = np.zeros(26, np.uint64)
    for m in _MOTIF.finditer(r.stdout):
        counts[int(m.group(1)) - 1] = int(m.group(2))
    rt = _RT.search(r.stdout)
    return counts, wall, float(rt.group(1)) if rt else None


def run_mochy(offsets, members, threads: int | None = None, timeout: float | None = None):
    """Returns (26 counts, wall seconds, self-reported seconds)."""
    with tempfile.TemporaryDirectory() as d:
        g = os.path.join(d, "graph.txt")
        write_mochy(g, offsets, members)
        return run_mochy_file(g, threads, timeout)


def run_thymeP_file(path, delta: int, threads: int, timeout: float | None = None):
    """THyMe+ (main_thymeP.cpp:117-137: name, delta, threads, graph, result)
    on a file in THyMe's format. Returns (96 counts, wall seconds of the child
    process, its self-reported TOTAL_RUNTIME_SECONDS: clock() summed over its
    threads, i.e. CPU time, not wall time)."""
    with tempfile.TemporaryDirectory() as d:
        res = os.path.join(d, "result.txt")
        cmd = [str(REF / "thymeP"), "x", str(int(delta)), str(threads), str(path), res]
        t0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=d)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"{cmd[0]} failed: {r.stderr[-500:]}")
        lines = Path(res).read_text().split("\n")
    counts = np.zeros(96, np.uint64)
    for ln in lines[1:]:
        if ln.strip():
            i, c = ln.split("\t")
            counts[int(i) - 1] = int(c)
    return counts, wall, float(lines[0])


def run_thyme(offsets, members, times, delta: int, threads: int | None = None, timeout: float | None = None):
    """Returns (96 counts, wall seconds, self-reported CPU seconds).

    threads=None runs the sequential THyMe (main_thyme.cpp), which only takes
    a dataset name and reads ../data/<name>/<name>.txt, writing
    ../results/<name>_<delta>_thyme.txt; otherwise THyMe+ (main_thymeP.cpp)
    with explicit paths.
    """
    with tempfile.TemporaryDirectory() as d:
        work = os.path.join(d, "work")
        os.makedirs(os.path.join(d, "data", "x"))
        os.makedirs(os.path.join(d, "results"))
        os.makedirs(work)
        g = os.path.join(d, "data", "x", "x.txt")
        write_thyme(g, offsets, members, times)
        if threads is None:
            cmd = [str(REF / "thyme"), "x", str(int(delta))]
            res = os.path.join(d, "results", f"x_{float(delta):.6f}_thyme.txt")
        else:
            res = os.path.join(d, "result.txt")
            cmd = [str(REF / "thymeP"), "x", str(int(delta)), str(threads), g, res]
        t0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=work)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"{cmd[0]} failed: {r.stderr[-500:]}")
        lines = Path(res).read_text().split("\n")
    rt = float(lines[0])
    counts = np.zeros(96, np.uint64)
    for ln in lines[1:]:
        if ln.strip():
            i, c = ln.split("\t")
            counts[int(i) - 1] = int(c)
    return counts, wall, rt
