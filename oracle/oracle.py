"""ctypes wrapper of liboracle.so (TEST INFRASTRUCTURE ONLY: the checker).

Builds liboracle.so from hm_oracle.c on first use if it is missing (gcc).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


def build() -> Path:
    src = HERE / "hm_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        u32p, u64p, i64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_int64)
        L.hmo_static30.argtypes = [C.c_uint32, u64p, u32p, C.c_uint32, u64p]
        L.hmo_static30_shard.argtypes = [C.c_uint32, u64p, u32p, C.c_uint32, C.c_uint32, C.c_uint32, u64p]
        L.hmo_strictinc30.argtypes = [u64p, u32p, C.c_uint32] * 3 + [u64p]
        L.hmo_vertex_triads.argtypes = [C.c_uint32, u64p, u32p, u64p]
        L.hmo_static30_brute.argtypes = [C.c_uint32, u64p, u32p, u64p]
        L.hmo_temporal96.argtypes = [C.c_uint32, u64p, u32p, i64p, C.c_int64, u64p]
        L.hmo_temporal96_brute.argtypes = [C.c_uint32, u64p, u32p, i64p, C.c_int64, u64p]
        L.hmo_static_class_bits.argtypes = [C.c_int]
        L.hmo_temporal_class_bits.argtypes = [C.c_int]
        L.hmo_static_class.argtypes = [C.c_int] * 7
        L.hmo_temporal_class.argtypes = [C.c_int] * 7
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _csr(offsets, members):
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    mem = np.ascontiguousarray(members, dtype=np.uint32)
    if len(mem) == 0:
        mem = np.zeros(1, np.uint32)
    return off, mem


SKIPPED = (0, 1, 4, 6)  # classes only repeated hyperedges produce (main_exact.cpp:135)


def to26(c30) -> np.ndarray:
    return np.array([c30[k] for k in range(30) if k not in SKIPPED], dtype=np.uint64)


def static30(offsets, members, n_nodes: int) -> np.ndarray:
    off, mem = _csr(offsets, members)
    out = np.zeros(30, np.uint64)
    rc = lib().hmo_static30(len(off) - 1, _p(off, C.c_uint64), _p(mem, C.c_uint32), n_nodes, _p(out, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"hmo_static30 failed: {rc}")
    return out


def static30_shard(offsets, members, n_nodes: int, shard: int, n_shards: int) -> np.ndarray:
    """Triples owned by centres a = shard (mod n_shards)."""
    off, mem = _csr(offsets, members)
    out = np.zeros(30, np.uint64)
    rc = lib().hmo_static30_shard(len(off) - 1, _p(off, C.c_uint64), _p(mem, C.c_uint32), n_nodes, shard, n_shards,
                                  _p(out, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"hmo_static30_shard failed: {rc}")
    return out


def strictinc30(layers) -> np.ndarray:
    """Three-layer strictly increasing count; layers = [(offsets, members)] * 3
    in the order older, middle, newest."""
    args = []
    keep = []
    for off, mem in layers:
        o, m = _csr(off, mem)
        keep.append((o, m))
        args += [_p(o, C.c_uint64), _p(m, C.c_uint32), len(o) - 1]
    out = np.zeros(30, np.uint64)
    rc = lib().hmo_strictinc30(*args, _p(out, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"hmo_strictinc30 failed: {rc}")
    return out


def vertex_triads(offsets, members) -> np.ndarray:
    """(type1, type2, type3) vertex-triad counts."""
    off, mem = _csr(offsets, members)
    out = np.zeros(3, np.uint64)
    rc = lib().hmo_vertex_triads(len(off) - 1, _p(off, C.c_uint64), _p(mem, C.c_uint32), _p(out, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"hmo_vertex_triads failed: {rc}")
    return out


def static30_brute(offsets, members) -> np.ndarray:
    off, mem = _csr(offsets, members)
    out = np.zeros(30, np.uint64)
    rc = lib().hmo_static30_brute(len(off) - 1, _p(off, C.c_uint64), _p(mem, C.c_uint32), _p(out, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"hmo_static30_brute failed: {rc}")
    return out


def temporal96(offsets, members, times, delta: int) -> np.ndarray:
    off, mem = _csr(offsets, members)
    t = np.ascontiguousarray(times, dtype=np.int64)
    out = np.zeros(96, np.uint64)
    rc = lib().hmo_temporal96(len(off) - 1, _p(off, C.c_uint64), _p(mem, C.c_uint32), _p(t, C.c_int64),
                              int(delta), _p(out, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"hmo_temporal96 failed: {rc}")
    return out


def temporal96_brute(offsets, members, times, delta: int) -> np.ndarray:
    off, mem = _csr(offsets, members)
    t = np.ascontiguousarray(times, dtype=np.int64)
    out = np.zeros(96, np.uint64)
    rc = lib().hmo_temporal96_brute(len(off) - 1, _p(off, C.c_uint64), _p(mem, C.c_uint32), _p(t, C.c_int64),
                                    int(delta), _p(out, C.c_uint64))
    if rc != 0:
        raise RuntimeError(f"hmo_temporal96_brute failed: {rc}")
    return out
