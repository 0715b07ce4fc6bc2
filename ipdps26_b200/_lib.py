"""ctypes binding of libhmotif.so (the engine's C ABI, include/hmotif.h).

The library is loaded from the package directory. There is no fallback: if
it is missing, importing the package fails with the build command to run.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libhmotif.so"

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
i64p = C.POINTER(C.c_int64)
vp = C.c_void_p


# status codes of include/hmotif.h
HM_OK = 0
HM_ERR_INVALID = -1
HM_ERR_CUDA = -2
HM_ERR_NOMEM = -3
HM_ERR_CAPACITY = -4
HM_ERR_NOT_LIVE = -5
HM_ERR_TIMEOUT = -6
HM_ERR_STATE = -7
HM_ERR_LIMIT = -8


class HmError(RuntimeError):
    """A negative status returned by the engine."""

    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: status {status}: {message}")
        self.status = status


class GenParams(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("n_nodes", C.c_uint32),
        ("n_edges", C.c_uint32),
        ("k_min", C.c_uint32),
        ("k_max", C.c_uint32),
        ("size_exp", C.c_double),
        ("pop_exp", C.c_double),
        ("pop_offset", C.c_double),
        ("dedupe", C.c_int32),
        ("permute_nodes", C.c_int32),
    ]


class BurstParams(C.Structure):
    _fields_ = [
        ("burst_rate", C.c_double),
        ("events_per_burst", C.c_uint32),
        ("gap_mean", C.c_double),
        ("span", C.c_int64),
    ]


class HostGraphInfo(C.Structure):
    _fields_ = [
        ("n_edges", C.c_uint32),
        ("n_nodes", C.c_uint32),
        ("n_members", C.c_uint64),
        ("offsets", u64p),
        ("members", u32p),
        ("timestamps", i64p),
        ("redraws", C.c_uint64),
    ]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: the CUDA engine is not built. "
            "Run `python -m ipdps26_b200.build` (nvcc, sm_100a)."
        )
    return C.CDLL(str(LIB_PATH))


lib = _load()

_SIGS = {
    "hm_last_error": (C.c_char_p, []),
    "hm_status_string": (C.c_char_p, [C.c_int]),
    "hm_gen_static": (C.c_int, [C.POINTER(GenParams), C.POINTER(vp)]),
    "hm_gen_temporal": (C.c_int, [C.POINTER(GenParams), C.POINTER(BurstParams), C.POINTER(vp)]),
    "hm_gen_batch": (
        C.c_int,
        [C.POINTER(GenParams), C.c_uint64, u32p, C.c_uint32, C.c_uint32, C.c_double, u32p, u32p, C.POINTER(vp)],
    ),
    "hm_hostgraph_view": (C.c_int, [vp, C.POINTER(HostGraphInfo)]),
    "hm_hostgraph_free": (None, [vp]),
}


def bind(sigs: dict) -> None:
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


bind(_SIGS)


def check(status: int, where: str) -> int:
    if status < 0:
        msg = lib.hm_last_error().decode(errors="replace")
        raise HmError(status, where, msg or lib.hm_status_string(status).decode())
    return status


def ptr(arr, ctype):
    """Pointer to a contiguous numpy array's data (or NULL for None)."""
    if arr is None:
        return None
    return arr.ctypes.data_as(C.POINTER(ctype))
