"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/_build/libuwshcu_oracle.so (built by oracle/Makefile) and exposes
compute_uwshcu / compute_uwshcu_inv on the sounding dicts produced by
hpc-and-climate-model_b200/soundings.py.  Only tests, the smoke check and the CPU-baseline leg of
bench.py use this module; it is the checker, not the product.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATHS = {"glibc": os.path.join(HERE, "_build", "libuwshcu_oracle.so"),
             "portable": os.path.join(HERE, "_build", "libuwshcu_oracle_pm.so"),
             # glibc exp/log/pow with CALERF erfc: the functions a Fortran build of the scheme calls
             "fortran": os.path.join(HERE, "_build", "libuwshcu_oracle_ftn.so"),
             # operation-counting build (opcount.hpp): same results as "glibc", plus uwo_opcount
             "ops": os.path.join(HERE, "_build", "libuwshcu_oracle_ops.so")}
LIB_PATH = LIB_PATHS["glibc"]

OUT_IFACE = ("umf", "slflx", "qtflx", "flxprc1", "flxsnow1", "wu")
OUT_LAYER = ("qvten", "qlten", "qiten", "sten", "uten", "vten", "qrten", "qsten", "evapc",
             "cufrc", "qcu", "qlu", "qiu", "qc")
OUT_COL = ("precip", "snow", "cbmf", "rliq", "cnt", "cnb", "cush")
NDI, NDR = 8, 8
# per-level diagnostic rows: ufrc qtu thlu thvu uu vu uemf flxrain flxsnow (interfaces), fer fdr dwten
# diten (layers, rows 1..mkx); array (NDL, mkx + 1, ncol), levels bottom-up
NDL = 13
DL_NAMES = ("ufrc", "qtu", "thlu", "thvu", "uu", "vu", "uemf", "flxrain", "flxsnow", "fer", "fdr",
            "dwten", "diten")

_lib = None
_libs = {}
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def set_variant(variant):
    """Select the oracle build: 'glibc' (transcendentals from glibc; pinned bit for bit to the
    reference's drop-in), 'fortran' (glibc exp/log/pow and CAM's CALERF erfc, the functions a
    Fortran build of uwshcu.F90 calls) or 'portable' (the host/device-identical routines of
    uw_math.h that the CUDA path uses).  Each build keeps its own constants; the selected one is initialised with the
    default constants on first use."""
    global _lib, LIB_PATH
    LIB_PATH = LIB_PATHS[variant]
    _lib = _libs.get(variant)
    return lib()


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _libs[[k for k, v in LIB_PATHS.items() if v == LIB_PATH][0] if LIB_PATH in LIB_PATHS.values() else LIB_PATH] = _lib
        _lib.uwo_init_default.restype = ctypes.c_int
        _lib.uwo_compute_uwshcu.restype = ctypes.c_int
        _lib.uwo_compute_uwshcu_inv.restype = ctypes.c_int
        _lib.uwo_compute_zwshcu.restype = ctypes.c_int
        for name in ("uwo_exnf", "uwo_estblf", "uwo_qsinvert", "uwo_compute_alpha",
                     "uwo_compute_mumin2", "uwo_compute_ppen", "uwo_single_cin"):
            getattr(_lib, name).restype = ctypes.c_double
        rc = _lib.uwo_init_default()
        if rc != 0:
            raise RuntimeError("uwo_init_default failed: %d" % rc)
    return _lib


def init(xlv, cp, xlf, zvir, r, g, ep2, rpen, tmn, tmx, trice, icephs, epsqs, rgasv, tmelt,
         qmin, cnst_wet, ixnumliq, ixnumice):
    L = lib()
    qmin = np.ascontiguousarray(qmin, dtype=np.float64)
    wet = np.ascontiguousarray(cnst_wet, dtype=np.int32)
    f = ctypes.c_double
    rc = L.uwo_init(f(xlv), f(cp), f(xlf), f(zvir), f(r), f(g), f(ep2), f(rpen), f(tmn), f(tmx),
                    f(trice), ctypes.c_int(icephs), f(epsqs), f(rgasv), f(tmelt),
                    ctypes.c_int(len(qmin)), _p(qmin), wet.ctypes.data_as(_I),
                    ctypes.c_int(ixnumliq), ctypes.c_int(ixnumice))
    if rc != 0:
        raise RuntimeError("uwo_init failed: %d" % rc)


def set_params(rpen, rle, rkm, criqc):
    f = ctypes.c_double
    return lib().uwo_set_params(f(rpen), f(rle), f(rkm), f(criqc))


def init_default():
    rc = lib().uwo_init_default()
    if rc != 0:
        raise RuntimeError("uwo_init_default failed: %d" % rc)


def _p(a):
    return a.ctypes.data_as(_D)


def alloc_outputs(mkx, ncnst, mix, cush_in):
    out = {k: np.zeros((mkx + 1, mix)) for k in OUT_IFACE}
    out.update({k: np.zeros((mkx, mix)) for k in OUT_LAYER})
    out["trten"] = np.zeros((ncnst, mkx, mix))
    out.update({k: np.zeros(mix) for k in OUT_COL})
    out["cush"][:] = cush_in
    return out


def set_zw_options(lf=1, fwcrit=1.0, ent=0, ent0=0.015, cloud_sh=0, ufrcd=2.0, ufrc0=2.0, ufrcz=2.0):
    """Options of compute_zwshcu (zmh_shallow_lf, zmh_shallow_fwcrit, zmh_shallow_ent, zmh_ent0,
    zmh_cloud_sh, zmh_ufrcd, zmh_ufrc0, zmh_ufrcz); the defaults are the reference's."""
    d = ctypes.c_double
    return lib().uwo_set_zw_options(ctypes.c_int(lf), d(fwcrit), ctypes.c_int(ent), d(ent0),
                                    ctypes.c_int(cloud_sh), d(ufrcd), d(ufrc0), d(ufrcz))


def compute(s, nthreads=0, diag=True, inv=False, omega=None):
    """Run the oracle on a sounding dict (all columns, mix = iend = ncol).  Returns the output
    dict; with diag=True also 'diag_int' (8, ncol), 'diag_real' (8, ncol) and 'diag_level'
    (13, mkx + 1, ncol).  With omega (a (mkx, ncol) array of pressure velocity, bottom-up) it runs
    compute_zwshcu (zwshcu.F90) instead of compute_uwshcu."""
    L = lib()
    mkx, ncnst, n = s["mkx"], s["ncnst"], s["ncol"]
    o = alloc_outputs(mkx, ncnst, n, s["cush"])
    di = np.zeros((NDI, n), dtype=np.int32)
    dr = np.zeros((NDR, n))
    dl = np.zeros((NDL, mkx + 1, n))
    ci, cd = ctypes.c_int, ctypes.c_double
    if omega is not None:
        assert not inv
        om = np.ascontiguousarray(omega, dtype=np.float64)
        z = np.zeros(n)
        rc = L.uwo_compute_zwshcu(
            ci(n), ci(mkx), ci(n), ci(ncnst), cd(s["dt"]),
            _p(s["ps0"]), _p(s["zs0"]), _p(s["p0"]), _p(s["z0"]), _p(s["dp0"]), _p(s["u0"]),
            _p(s["v0"]), _p(s["qv0"]), _p(s["ql0"]), _p(s["qi0"]), _p(s["t0"]), _p(s["s0"]),
            _p(s["tr0"]), _p(s["tke"]), _p(s["cldfrct"]), _p(s["concldfrct"]), _p(s["pblh"]),
            _p(o["cush"]), _p(o["umf"]), _p(o["slflx"]), _p(o["qtflx"]), _p(o["flxprc1"]),
            _p(o["flxsnow1"]), _p(o["qvten"]), _p(o["qlten"]), _p(o["qiten"]), _p(o["sten"]),
            _p(o["uten"]), _p(o["vten"]), _p(o["trten"]), _p(o["qrten"]), _p(o["qsten"]),
            _p(o["precip"]), _p(o["snow"]), _p(o["evapc"]), _p(o["cufrc"]), _p(o["qcu"]),
            _p(o["qlu"]), _p(o["qiu"]), _p(o["cbmf"]), _p(o["qc"]), _p(o["rliq"]), _p(om),
            _p(s["massflx_sh"]), _p(z), _p(o["cnt"]), _p(o["cnb"]), _p(s["dpdry0"]), _p(o["wu"]),
            di.ctypes.data_as(_I) if diag else None, _p(dr) if diag else None,
            _p(dl) if diag else None, ci(nthreads))
    elif not inv:
        rc = L.uwo_compute_uwshcu(
            ci(n), ci(mkx), ci(n), ci(ncnst), cd(s["dt"]),
            _p(s["ps0"]), _p(s["zs0"]), _p(s["p0"]), _p(s["z0"]), _p(s["dp0"]), _p(s["u0"]),
            _p(s["v0"]), _p(s["qv0"]), _p(s["ql0"]), _p(s["qi0"]), _p(s["t0"]), _p(s["s0"]),
            _p(s["tr0"]), _p(s["tke"]), _p(s["cldfrct"]), _p(s["concldfrct"]), _p(s["pblh"]),
            _p(o["cush"]), _p(o["umf"]), _p(o["slflx"]), _p(o["qtflx"]), _p(o["flxprc1"]),
            _p(o["flxsnow1"]), _p(o["qvten"]), _p(o["qlten"]), _p(o["qiten"]), _p(o["sten"]),
            _p(o["uten"]), _p(o["vten"]), _p(o["trten"]), _p(o["qrten"]), _p(o["qsten"]),
            _p(o["precip"]), _p(o["snow"]), _p(o["evapc"]), _p(o["cufrc"]), _p(o["qcu"]),
            _p(o["qlu"]), _p(o["qiu"]), _p(o["cbmf"]), _p(o["qc"]), _p(o["rliq"]),
            _p(s["massflx_sh"]), _p(o["cnt"]), _p(o["cnb"]), _p(s["dpdry0"]), _p(o["wu"]),
            di.ctypes.data_as(_I) if diag else None, _p(dr) if diag else None,
            _p(dl) if diag else None, ci(nthreads))
    else:
        z = np.zeros(n)
        rc = L.uwo_compute_uwshcu_inv(
            ci(n), ci(mkx), ci(n), ci(ncnst), cd(s["dt"]),
            _p(s["ps0"]), _p(s["zs0"]), _p(s["p0"]), _p(s["z0"]), _p(s["dp0"]), _p(s["u0"]),
            _p(s["v0"]), _p(s["qv0"]), _p(s["ql0"]), _p(s["qi0"]), _p(s["t0"]), _p(s["s0"]),
            _p(s["tr0"]), _p(s["tke"]), _p(s["cldfrct"]), _p(s["concldfrct"]), _p(s["pblh"]),
            _p(o["cush"]), _p(z), _p(z), _p(s["massflx_sh"]),
            _p(o["umf"]), _p(o["slflx"]), _p(o["qtflx"]), _p(o["flxprc1"]), _p(o["flxsnow1"]),
            _p(o["qvten"]), _p(o["qlten"]), _p(o["qiten"]), _p(o["sten"]), _p(o["uten"]),
            _p(o["vten"]), _p(o["trten"]), _p(o["qrten"]), _p(o["qsten"]), _p(o["precip"]),
            _p(o["snow"]), _p(o["evapc"]), _p(o["cufrc"]), _p(o["qcu"]), _p(o["qlu"]),
            _p(o["qiu"]), _p(o["cbmf"]), _p(o["qc"]), _p(o["rliq"]), _p(o["cnt"]), _p(o["cnb"]),
            _p(s["dpdry0"]), _p(o["wu"]), ci(nthreads))
        diag = False
    o["status"] = rc
    if diag:
        o["diag_int"] = di
        o["diag_real"] = dr
        o["diag_level"] = dl
    return o


def estbl():
    t = np.zeros(250)
    lib().uwo_get_estbl(_p(t))
    return t


def consts():
    c = np.zeros(22)
    lib().uwo_get_consts(_p(c))
    return c


def uwmath(fn, x, y=None):
    """Host evaluation of uw_math.h: fn 0 exp, 1 log, 2 pow, 3 erfc."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y if y is not None else np.zeros_like(x), dtype=np.float64)
    out = np.zeros_like(x)
    lib().uwo_uwmath(ctypes.c_int(fn), _p(x), _p(y), _p(out), ctypes.c_int(x.size))
    return out
