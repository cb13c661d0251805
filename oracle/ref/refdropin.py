"""ctypes front end of the host build of the reference drop-in (TEST INFRASTRUCTURE ONLY).

oracle/_ref/libuwref_dropin.so is src/physics/bxcompute_uwshcu_inv.cpp of the reference compiled
unchanged for the CPU through the shim in oracle/ref/shim (built by oracle/ref/Makefile when the
reference tree is present).  Its compile-time shape is mix = 1024, mkx = 30, ncnst = 25
(bxcompute_uwshcu_inv.cpp:11-13); it indexes the caller's arrays as k*ncol + i, so calls use
pcols = ncol, and it launches ncol/32 blocks of 32, so ncol must be a multiple of 32.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "_ref", "libuwref_dropin.so")
MKX, NCNST, MIX = 30, 25, 1024
_D = ctypes.POINTER(ctypes.c_double)
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def init(consts22, estbl, qmin25, wet25):
    c = np.ascontiguousarray(consts22, dtype=np.float64)
    t = np.ascontiguousarray(estbl, dtype=np.float64)
    q = np.ascontiguousarray(qmin25, dtype=np.float64)
    w = np.ascontiguousarray(wet25, dtype=np.int32)
    lib().uwref_init(c.ctypes.data_as(_D), t.ctypes.data_as(_D), q.ctypes.data_as(_D),
                     w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))


def compute_inv(si):
    """Run bxcompute_uwshcu_inv_ on a top-down sounding dict with ncol % 32 == 0, ncol <= 1024,
    mkx = 30, ncnst = 25.  Returns the output dict (top-down, as the entry writes it)."""
    n, mkx, nc = si["ncol"], si["mkx"], si["ncnst"]
    assert mkx == MKX and nc == NCNST and n % 32 == 0 and n <= MIX
    P = lambda a: a.ctypes.data_as(_D)
    o = {k: np.zeros((mkx + 1, n)) for k in ("umf", "slflx", "qtflx", "flxprc1", "flxsnow1", "wu")}
    o.update({k: np.zeros((mkx, n)) for k in ("qvten", "qlten", "qiten", "sten", "uten", "vten",
                                               "qrten", "qsten", "evapc", "cufrc", "qcu", "qlu",
                                               "qiu", "qc")})
    o["trten"] = np.zeros((nc, mkx, n))
    o.update({k: np.zeros(n) for k in ("precip", "snow", "cbmf", "rliq", "cnt", "cnb")})
    o["cush"] = np.array(si["cush"], dtype=np.float64)
    ci = lambda v: ctypes.byref(ctypes.c_int(v))
    lib().bxcompute_uwshcu_inv_(
        ci(n), ci(mkx), ci(n), ci(nc), ctypes.byref(ctypes.c_double(si["dt"])),
        P(si["ps0"]), P(si["zs0"]), P(si["p0"]), P(si["z0"]), P(si["dp0"]), P(si["u0"]),
        P(si["v0"]), P(si["qv0"]), P(si["ql0"]), P(si["qi0"]), P(si["t0"]), P(si["s0"]),
        P(si["tr0"]), P(si["tke"]), P(si["cldfrct"]), P(si["concldfrct"]), P(si["pblh"]),
        P(o["cush"]), P(o["umf"]), P(o["slflx"]), P(o["qtflx"]), P(o["flxprc1"]),
        P(o["flxsnow1"]), P(o["qvten"]), P(o["qlten"]), P(o["qiten"]), P(o["sten"]),
        P(o["uten"]), P(o["vten"]), P(o["trten"]), P(o["qrten"]), P(o["qsten"]),
        P(o["precip"]), P(o["snow"]), P(o["evapc"]), P(o["cufrc"]), P(o["qcu"]), P(o["qlu"]),
        P(o["qiu"]), P(o["cbmf"]), P(o["qc"]), P(o["rliq"]), P(o["cnt"]), P(o["cnb"]), ci(0),
        P(si["dpdry0"]), P(o["wu"]))
    return o
