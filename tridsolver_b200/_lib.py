"""Loader of the in-tree C-ABI library (tridsolver_b200/lib/libtridsolver_b200.so).

The library is the product; this module only binds its exported symbols with
ctypes. There is no CPU or PyTorch fallback: if the library is missing the
import fails loudly and says how to build it.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libtridsolver_b200.so")

# (name, restype, argtypes); c_void_p stands for device pointers
_P = ctypes.c_void_p
_I = ctypes.c_int
_IP = ctypes.POINTER(ctypes.c_int)
_L = ctypes.c_longlong

SYMBOLS = {
    # reference ABI, scalar/include/tridsolver.h:39-69
    "tridDmtsvStridedBatch": (_I, [_P, _P, _P, _P, _P, _I, _I, _IP, _IP]),
    "tridSmtsvStridedBatch": (_I, [_P, _P, _P, _P, _P, _I, _I, _IP, _IP]),
    "tridDmtsvStridedBatchInc": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _IP, _IP]),
    "tridSmtsvStridedBatchInc": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _IP, _IP]),
    # extensions, include/tridsolver_b200.h
    "tridDsolveBatchedTrid": (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "tridSsolveBatchedTrid": (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "tridDsolveBatchedTridInc": (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "tridSsolveBatchedTridInc": (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P]),
    "tridSetStream": (_I, [_P]),
    "tridGetStream": (_P, []),
    "tridSetBlocking": (_I, [_I]),
    "tridGetBlocking": (_I, []),
    "tridGetPivotStatus": (_I, []),
    "tridGetLaunchCount": (ctypes.c_ulonglong, []),
    "tridReleaseScratch": (_I, []),
    "tridSetTracing": (_I, [_I]),
    "tridForcePlan": (_I, [_I, _I]),
    "tridForceSystemsPerBlock": (_I, [_I]),
    "tridForceTma": (_I, [_I]),
    "tridForceStream": (_I, [_I]),
    "tridDescribePlan": (_I, [_I, _I, _I, _IP, _IP, ctypes.c_char_p, _I]),
    "tridDescribePlanInc": (_I, [_I, _I, _I, _IP, _IP, _I, ctypes.c_char_p, _I]),
    "tridDmtsvRaggedBatch": (_I, [_P] * 6 + [ctypes.c_longlong]),
    "tridSmtsvRaggedBatch": (_I, [_P] * 6 + [ctypes.c_longlong]),
    "tridDmtsvRaggedBatchSized": (_I, [_P] * 6 + [ctypes.c_longlong] * 2),
    "tridSmtsvRaggedBatchSized": (_I, [_P] * 6 + [ctypes.c_longlong] * 2),
    "tridRaggedAutotune": (_I, [_I]),
    "tridRaggedTable": (_I, [_I, _IP, _I]),
    "tridRaggedSetWaitBound": (_I, [ctypes.c_ulonglong, _I]),
    "tridAutotune": (_I, [_I, _I, _I, _IP, _IP, _I, ctypes.POINTER(ctypes.c_float), ctypes.c_char_p,
                          _I]),
    "tridAutotuneReset": (_I, []),
    "tridDADIStepAdjoint": (_I, [_P, _P, _P, _P, _P, ctypes.c_double, _I, _I, _I]),
    "tridSADIStepAdjoint": (_I, [_P, _P, _P, _P, _P, ctypes.c_float, _I, _I, _I]),
    "tridDADIStep": (_I, [_P] * 7 + [ctypes.c_double, _I, _I, _I]),
    "tridSADIStep": (_I, [_P] * 7 + [ctypes.c_float, _I, _I, _I]),
    "tridDmtsvStridedBatchAdjoint": (_I, [_P] * 10 + [_I, _I, _IP, _IP]),
    "tridSmtsvStridedBatchAdjoint": (_I, [_P] * 10 + [_I, _I, _IP, _IP]),
    "tridDmtsvStridedBatchMixed": (_I, [_P, _P, _P, _P, _P, _I, _I, _IP, _IP, _I, ctypes.c_double,
                                        _IP, ctypes.POINTER(ctypes.c_double)]),
    "tridDmtsvStridedBatchRefine": (_I, [_P, _P, _P, _P, _P, _I, _I, _IP, _IP, _I, ctypes.c_double,
                                        _IP, ctypes.POINTER(ctypes.c_double)]),
    "tridSetMixedMode": (_I, [_I]),
    "tridDistInit": (_I, [_P, _I, _I, _I, _P, _P]),
    "tridDistFinalize": (_I, [_P]),
    "tridDistExchangeBytes": (_L, [_I, _I, _I, _IP]),
}

_lib = None


class LibraryMissing(RuntimeError):
    pass


def load():
    """Load and bind the library once; raises LibraryMissing if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryMissing(
            f"{LIB_PATH} is not built; run `python -m tridsolver_b200.build` "
            "(or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SYMBOLS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def header_symbols():
    """Every function name declared with EXTERN_C in include/*.h."""
    import re
    inc = os.path.join(os.path.dirname(HERE), "include")
    names = []
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"EXTERN_C\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.append(m.group(1))
    return names
