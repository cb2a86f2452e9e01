"""ctypes binding of libcurfp_b200.so (the C ABI of include/curfp.h).

Tensors cross as raw device pointers and streams as cudaStream_t integers,
as in the reference's pybind11 shim (curfp/_ext.cpp:1-9).  The library must be
built in-tree (``python -m curfp_b200.build``); there is no fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcurfp_b200.so"

_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_p = ctypes.c_void_p
_h = ctypes.c_void_p

# name -> argtypes (restype is always int = curfpStatus_t)
SIGNATURES = {
    "curfpCreate": [ctypes.POINTER(_h)],
    "curfpDestroy": [_h],
    "curfpSetStream": [_h, _p],
    "curfpGetStream": [_h, ctypes.POINTER(_p)],
    "curfpSsfrk": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_f), _p, _i,
                   ctypes.POINTER(_f), _p],
    "curfpSpftrf": [_h, _i, _i, _i, _p, ctypes.POINTER(_i)],
    "curfpSpftrs": [_h, _i, _i, _i, _i, _p, _p, _i],
    "curfpSstrttf": [_h, _i, _i, _i, _p, _i, _p],
    "curfpSpftri": [_h, _i, _i, _i, _p],
    "curfpSstfttr": [_h, _i, _i, _i, _p, _p, _i],
    "curfpSsfr2k": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_f), _p, _i, _p,
                    _i, ctypes.POINTER(_f), _p],
    "curfpRfpDiagIndices": [_h, _i, _i, _i, _p],
    "curfpSaddToDiagonal": [_h, _i, _i, _i, _f, _p],
    "curfpDaddToDiagonal": [_h, _i, _i, _i, _d, _p],
    "curfpSsfrkEx": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_f), _p, _i,
                     ctypes.POINTER(_f), _p, _i],
    "curfpSpftrfEx": [_h, _i, _i, _i, _p, ctypes.POINTER(_i), _i],
    "curfpSpftrfFromHost": [_h, _i, _i, _i, _p, _p, _p, ctypes.POINTER(_i), _i],
    "curfpSetMathMode": [_h, _i],
    "curfpGetMathMode": [_h, ctypes.POINTER(_i)],
    "curfpSpftrsRefine": [_h, _i, _i, _i, _i, _p, _p, _p, _i, _i, ctypes.POINTER(_i)],
    "curfpSsfmmAcc64": [_h, _i, _i, _i, _i, ctypes.POINTER(_f), _p, _p, _i,
                        ctypes.POINTER(_f), _p, _i],
    "curfpGetKernelLaunchCount": [_h, ctypes.POINTER(ctypes.c_longlong)],
    "curfpReleaseWorkspace": [_h],
    "curfpDiagWaitTimeout": [_h, ctypes.POINTER(ctypes.c_int)],
    "curfpDsfrk": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_d), _p, _i, ctypes.POINTER(_d), _p],
    "curfpDsfr2k": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_d), _p, _i, _p, _i,
                    ctypes.POINTER(_d), _p],
    "curfpDpftrf": [_h, _i, _i, _i, _p, ctypes.POINTER(_i)],
    "curfpDpftrs": [_h, _i, _i, _i, _i, _p, _p, _i],
    "curfpDpftri": [_h, _i, _i, _i, _p],
    "curfpDstrttf": [_h, _i, _i, _i, _p, _i, _p],
    "curfpDstfttr": [_h, _i, _i, _i, _p, _p, _i],
    "curfpDsfmm": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_d), _p, _p, _i, ctypes.POINTER(_d),
                   _p, _i],
    "curfpDsfmv": [_h, _i, _i, _i, ctypes.POINTER(_d), _p, _p, _i, ctypes.POINTER(_d), _p, _i],
    "curfpDsfr": [_h, _i, _i, _i, ctypes.POINTER(_d), _p, _i, _p],
    "curfpDsfr2": [_h, _i, _i, _i, ctypes.POINTER(_d), _p, _i, _p, _i, _p],
    "curfpDlansf": [_h, _i, _i, _i, _i, _p, ctypes.POINTER(_d)],
    "curfpDpfcon": [_h, _i, _i, _i, _p, _d, ctypes.POINTER(_d)],
    "curfpSlansf": [_h, _i, _i, _i, _i, _p, ctypes.POINTER(_f)],
    "curfpSsfmm": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_f), _p, _p, _i,
                   ctypes.POINTER(_f), _p, _i],
    "curfpSsfr": [_h, _i, _i, _i, ctypes.POINTER(_f), _p, _i, _p],
    "curfpSsfr2": [_h, _i, _i, _i, ctypes.POINTER(_f), _p, _i, _p, _i, _p],
    "curfpSsfmv": [_h, _i, _i, _i, ctypes.POINTER(_f), _p, _p, _i, ctypes.POINTER(_f), _p, _i],
    "curfpSpfcon": [_h, _i, _i, _i, _p, _f, ctypes.POINTER(_f)],
    "curfpSpftrsNoAlloc": [_h, _i, _i, _i, _i, _p, _p, _i],
    "curfpSsfrkBackward": [_h, _i, _i, _i, _i, _i, ctypes.POINTER(_f), _p, _i, _p, _p, _i],
    "curfpSpftrfBackward": [_h, _i, _i, _i, _p, _p, _p, _i],
    "curfpSpftrsBackward": [_h, _i, _i, _i, _i, _p, _p, _i, _p, _i, _p, _i, _p],
    "curfpSgpnllBackward": [_h, _i, _i, _i, _i, _f, _p, _p, _i, _p, _p, _p, _i, _p, _i],
    "curfpProfileEnable": [_h, _i],
    "curfpProfileRecords": [_h, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong), _p],
    "curfpProfileRead": [_h, _i, ctypes.POINTER(_d), ctypes.POINTER(_d), ctypes.POINTER(_d),
                         ctypes.POINTER(ctypes.c_longlong)],
}

_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m curfp_b200.build` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _i
    _lib = lib
    return lib


class CurfpError(RuntimeError):
    pass


def check(status: int) -> None:
    """Raise on a non-success status (reference curfp/_ext.cpp:21-25)."""
    if status != 0:
        raise CurfpError(f"curfp error: status={int(status)}")
