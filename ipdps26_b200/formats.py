"""Hypergraph files in the reference programs' formats (hm_hostgraph_read /
hm_hostgraph_write of the C ABI).

    ESCHER  space-separated vertex ids >= 1 per line, '#' comments
            (dynamicHyperGraph/utils/utils.cpp:88-130); vertex v is node v - 1
    MOCHY   comma-separated node ids >= 0 per line (MoCHy-master/read_data.cpp)
    THYME   "n1,n2,...<TAB>time" per line (THyMe-main/code/read_data.cpp)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib, ptr, u32p, u64p, i64p, vp
from .gen import Hypergraph, _take

ESCHER, MOCHY, THYME = 0, 1, 2
_NAMES = {"escher": ESCHER, "mochy": MOCHY, "thyme": THYME}

_lib.bind({
    "hm_hostgraph_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(vp)]),
    "hm_hostgraph_write": (C.c_int, [vp, C.c_char_p, C.c_int]),
    "hm_hostgraph_from_csr": (C.c_int, [u64p, u32p, C.c_uint32, C.c_uint32, i64p, C.POINTER(vp)]),
})


def _fmt(fmt) -> int:
    return _NAMES[fmt] if isinstance(fmt, str) else int(fmt)


def read(path, fmt="escher") -> Hypergraph:
    h = vp()
    check(lib.hm_hostgraph_read(str(path).encode(), _fmt(fmt), C.byref(h)), "hm_hostgraph_read")
    return _take(h)


def write(h: Hypergraph, path, fmt="escher") -> None:
    off = np.ascontiguousarray(h.offsets, np.uint64)
    mem = np.ascontiguousarray(h.members, np.uint32)
    ts = None if h.timestamps is None else np.ascontiguousarray(h.timestamps, np.int64)
    hg = vp()
    check(lib.hm_hostgraph_from_csr(ptr(off, C.c_uint64), ptr(mem if len(mem) else np.zeros(1, np.uint32), C.c_uint32),
                                    len(off) - 1, int(h.n_nodes), ptr(ts, C.c_int64), C.byref(hg)),
          "hm_hostgraph_from_csr")
    try:
        check(lib.hm_hostgraph_write(hg, str(path).encode(), _fmt(fmt)), "hm_hostgraph_write")
    finally:
        lib.hm_hostgraph_free(hg)
