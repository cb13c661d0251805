"""Python binding of libuwshcu_b200.so (ctypes over the C ABI of include/uwshcu.h).

This is the interface tests and the benchmark use.  It adds nothing to the computation: every call
goes to a C entry point with the Fortran argument list (compute_uwshcu_, compute_uwshcu_inv_,
bxcompute_uwshcu_inv_) or to the device-resident entry uwshcu_compute_device.  If the shared
library is missing, importing this module raises: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libuwshcu_b200.so")

OUT_IFACE = ("umf", "slflx", "qtflx", "flxprc1", "flxsnow1", "wu")
OUT_LAYER = ("qvten", "qlten", "qiten", "sten", "uten", "vten", "qrten", "qsten", "evapc",
             "cufrc", "qcu", "qlu", "qiu", "qc")
OUT_COL = ("precip", "snow", "cbmf", "rliq", "cnt", "cnb", "cush")
IN_IFACE = ("ps0", "zs0", "tke")
IN_LAYER = ("p0", "z0", "dp0", "u0", "v0", "qv0", "ql0", "qi0", "t0", "s0", "cldfrct",
            "concldfrct", "dpdry0")

OK = 0
ERR_MU_INCONSISTENT = 1
ERR_FINDSP_NONCONVERGED = 2
ERR_FINDSP_ENTHALPY = 3
ERR_BAD_ARGS = -1
ERR_NOT_INITIALIZED = -2
ERR_CUDA = -3
ERR_NO_DEVICE = -4
ERR_ALLOC = -5
ERR_TOO_LARGE = -6
NOALLOC_MAX_COLUMNS = 1048576
# per-level diagnostic rows of uwshcu_member.diag_level, array (NDL, mkx + 1, mix), levels bottom-up
DL_NAMES = ("ufrc", "qtu", "thlu", "thvu", "uu", "vu", "uemf", "flxrain", "flxsnow", "fer", "fdr",
            "dwten", "diten")
NDL = len(DL_NAMES)

EXPORTS = ("uwshcu_init", "uwshcu_set_rpen", "uwshcu_init_default", "uwshcu_set_precision",
           "uwshcu_set_block", "uwshcu_set_schedule", "uwshcu_set_profiling",
           "uwshcu_profile_read", "uwshcu_get_estbl", "uwshcu_finalize", "uwshcu_last_cuda_error",
           "compute_uwshcu_", "compute_uwshcu_inv_", "bxcompute_uwshcu_inv_",
           "uwshcu_compute_device", "uwshcu_device_status", "uwshcu_eval_math",
           "uwshcu_compute_device_noalloc", "uwshcu_batch_create", "uwshcu_batch_run",
           "uwshcu_batch_capture", "uwshcu_batch_autotune", "uwshcu_batch_status",
           "uwshcu_batch_destroy", "uwshcu_set_pipeline", "uwshcu_set_params",
           "uwshcu_budget_device", "uwshcu_tangent_device", "uwshcu_compute_member",
           "uwshcu_set_hand_slots", "uwshcu_adjoint_device", "uwshcu_adjoint_device_checked", "uwshcu_fp64_peak",
           "uwshcu_set_depth_order",
           "uwshcu_adjoint_last_records",
           "uwshcu_adjoint_release", "uwshcu_set_adjoint_rows", "compute_zwshcu_",
           "compute_zwshcu_inv_", "compute_zwshcu_device", "uwshcu_set_zw_options")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libuwshcu_b200.so is not built (%s); run build.py" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name in EXPORTS:
            getattr(L, name).restype = ctypes.c_int
        L.uwshcu_last_cuda_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def init_default():
    return lib().uwshcu_init_default()


def init(xlv, cp, xlf, zvir, r, g, ep2, tmin, tmax, ttrice, icephs, epsqs, rgasv, tmelt, qmin,
         cnst_wet, ixnumliq, ixnumice):
    qmin = np.ascontiguousarray(qmin, dtype=np.float64)
    wet = np.ascontiguousarray(cnst_wet, dtype=np.int32)
    f = ctypes.c_double
    return lib().uwshcu_init(f(xlv), f(cp), f(xlf), f(zvir), f(r), f(g), f(ep2), f(tmin), f(tmax),
                             f(ttrice), ctypes.c_int(icephs), f(epsqs), f(rgasv), f(tmelt),
                             ctypes.c_int(len(qmin)), qmin.ctypes.data_as(_D),
                             wet.ctypes.data_as(_I), ctypes.c_int(ixnumliq),
                             ctypes.c_int(ixnumice))


def set_rpen(rpen):
    return lib().uwshcu_set_rpen(ctypes.c_double(rpen))


PREC_FP64 = 0
PREC_MIXED = 1
PREC_FAST = 2


def set_params(rpen, rle, rkm, criqc):
    d = ctypes.c_double
    return lib().uwshcu_set_params(d(rpen), d(rle), d(rkm), d(criqc))


def set_zw_options(lf=1, fwcrit=1.0, ent=0, ent0=0.015, cloud_sh=0, ufrcd=2.0, ufrc0=2.0, ufrcz=2.0):
    """uwshcu_set_zw_options: the options of the compute_zwshcu entries (defaults: the reference's)."""
    d = ctypes.c_double
    return lib().uwshcu_set_zw_options(ctypes.c_int(lf), d(fwcrit), ctypes.c_int(ent), d(ent0),
                                       ctypes.c_int(cloud_sh), d(ufrcd), d(ufrc0), d(ufrcz))


def set_precision(mode):
    return lib().uwshcu_set_precision(ctypes.c_int(mode))


SCHED_SINGLE_PASS = 0
SCHED_TWO_PHASE = 1
SCHED_SORTED = 2
SCHED_DEFAULT = SCHED_SORTED


def set_schedule(schedule):
    return lib().uwshcu_set_schedule(ctypes.c_int(schedule))


def set_profiling(on):
    return lib().uwshcu_set_profiling(ctypes.c_int(1 if on else 0))


def profile_read():
    """(calls, trigger_ms, list_ms, worklist length of the last call) since the previous read."""
    n, a, b, c = ctypes.c_int(), ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    rc = lib().uwshcu_profile_read(ctypes.byref(n), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    if rc != 0:
        raise RuntimeError("uwshcu_profile_read: %d" % rc)
    return n.value, a.value, b.value, c.value


def set_pipeline(chunk_columns, streams):
    return lib().uwshcu_set_pipeline(ctypes.c_int(chunk_columns), ctypes.c_int(streams))


def set_depth_order(on):
    return lib().uwshcu_set_depth_order(ctypes.c_int(1 if on else 0))


def set_hand_slots(slots):
    return lib().uwshcu_set_hand_slots(ctypes.c_int(slots))


def set_block(threads):
    return lib().uwshcu_set_block(ctypes.c_int(threads))


def estbl():
    t = np.zeros(250)
    rc = lib().uwshcu_get_estbl(t.ctypes.data_as(_D))
    if rc != 0:
        raise RuntimeError("uwshcu_get_estbl: %d" % rc)
    return t


def last_cuda_error():
    return lib().uwshcu_last_cuda_error().decode()


def _p(a):
    return a.ctypes.data_as(_D)


def alloc_outputs(mkx, ncnst, mix, cush_in):
    out = {k: np.zeros((mkx + 1, mix)) for k in OUT_IFACE}
    out.update({k: np.zeros((mkx, mix)) for k in OUT_LAYER})
    out["trten"] = np.zeros((ncnst, mkx, mix))
    out.update({k: np.zeros(mix) for k in OUT_COL})
    out["cush"][:] = cush_in
    return out


def compute_host(s, entry="compute_uwshcu_", out=None, iend=None, omega=None):
    """Call a host entry point on a sounding dict (numpy arrays in the Fortran layout; mix = ncol).
    entry: 'compute_uwshcu_' or 'compute_zwshcu_' (bottom-up arrays), 'compute_uwshcu_inv_',
    'compute_zwshcu_inv_' or 'bxcompute_uwshcu_inv_' (CAM top-down arrays, e.g.
    soundings.to_inv(s)); the compute_zwshcu entries take omega (mkx, ncol) in the same level order.
    Returns (status, outputs)."""
    L = lib()
    mkx, ncnst, n = s["mkx"], s["ncnst"], s["ncol"]
    if out is None:
        out = alloc_outputs(mkx, ncnst, n, s["cush"])
    o = out
    ci = lambda v: ctypes.byref(ctypes.c_int(int(v)))
    cd = lambda v: ctypes.byref(ctypes.c_double(float(v)))
    ie = n if iend is None else iend
    common_in = (_p(s["ps0"]), _p(s["zs0"]), _p(s["p0"]), _p(s["z0"]), _p(s["dp0"]), _p(s["u0"]),
                 _p(s["v0"]), _p(s["qv0"]), _p(s["ql0"]), _p(s["qi0"]), _p(s["t0"]), _p(s["s0"]),
                 _p(s["tr0"]), _p(s["tke"]), _p(s["cldfrct"]), _p(s["concldfrct"]), _p(s["pblh"]),
                 _p(o["cush"]))
    outs1 = (_p(o["umf"]), _p(o["slflx"]), _p(o["qtflx"]), _p(o["flxprc1"]), _p(o["flxsnow1"]),
             _p(o["qvten"]), _p(o["qlten"]), _p(o["qiten"]), _p(o["sten"]), _p(o["uten"]),
             _p(o["vten"]), _p(o["trten"]), _p(o["qrten"]), _p(o["qsten"]), _p(o["precip"]),
             _p(o["snow"]), _p(o["evapc"]), _p(o["cufrc"]), _p(o["qcu"]), _p(o["qlu"]),
             _p(o["qiu"]), _p(o["cbmf"]), _p(o["qc"]), _p(o["rliq"]))
    lchnk = ci(0)
    if entry == "compute_uwshcu_":
        rc = L.compute_uwshcu_(ci(n), ci(mkx), ci(ie), ci(ncnst), cd(s["dt"]), *common_in, *outs1,
                               _p(s["massflx_sh"]), _p(o["cnt"]), _p(o["cnb"]), None, lchnk,
                               _p(s["dpdry0"]), _p(o["wu"]))
    elif entry == "compute_uwshcu_inv_":
        z = np.zeros(n)
        rc = L.compute_uwshcu_inv_(ci(n), ci(mkx), ci(ie), ci(ncnst), cd(s["dt"]), *common_in,
                                   _p(z), _p(z), _p(s["massflx_sh"]), *outs1, _p(o["cnt"]),
                                   _p(o["cnb"]), None, lchnk, _p(s["dpdry0"]), _p(o["wu"]))
    elif entry == "compute_zwshcu_":
        om = np.ascontiguousarray(omega, dtype=np.float64)
        z = np.zeros(n)
        rc = L.compute_zwshcu_(ci(n), ci(mkx), ci(ie), ci(ncnst), cd(s["dt"]), *common_in, *outs1,
                               _p(om), _p(s["massflx_sh"]), _p(z), _p(o["cnt"]), _p(o["cnb"]), None,
                               lchnk, _p(s["dpdry0"]), _p(o["wu"]))
    elif entry == "compute_zwshcu_inv_":
        om = np.ascontiguousarray(omega, dtype=np.float64)
        z = np.zeros(n)
        rc = L.compute_zwshcu_inv_(ci(n), ci(mkx), ci(ie), ci(ncnst), cd(s["dt"]), *common_in,
                                   _p(om), _p(z), _p(z), _p(z), _p(z), _p(z), _p(z), _p(z),
                                   _p(s["massflx_sh"]), *outs1, _p(o["cnt"]), _p(o["cnb"]), None, lchnk,
                                   _p(s["dpdry0"]), _p(o["wu"]))
    elif entry == "bxcompute_uwshcu_inv_":
        rc = L.bxcompute_uwshcu_inv_(ci(n), ci(mkx), ci(ie), ci(ncnst), cd(s["dt"]), *common_in,
                                     *outs1, _p(o["cnt"]), _p(o["cnb"]), lchnk, _p(s["dpdry0"]),
                                     _p(o["wu"]))
    else:
        raise ValueError(entry)
    return rc, o


class DeviceCase:
    """Inputs and outputs of one workload resident in device memory (torch tensors used only as
    allocations), for uwshcu_compute_device."""

    def __init__(self, s, device="cuda", diag=False, inputs=None):
        import torch
        self.torch = torch
        self.mkx, self.ncnst, self.n = s["mkx"], s["ncnst"], s["ncol"]
        self.dt = s["dt"]
        self.inp = inputs if inputs is not None else {
            k: torch.from_numpy(np.ascontiguousarray(s[k])).to(device)
            for k in IN_IFACE + IN_LAYER + ("tr0", "pblh")}
        self.cush0 = torch.from_numpy(np.ascontiguousarray(s["cush"])).to(device)
        n, mkx, nc = self.n, self.mkx, self.ncnst
        self.out = {k: torch.zeros((mkx + 1, n), dtype=torch.float64, device=device) for k in OUT_IFACE}
        self.out.update({k: torch.zeros((mkx, n), dtype=torch.float64, device=device) for k in OUT_LAYER})
        self.out["trten"] = torch.zeros((nc, mkx, n), dtype=torch.float64, device=device)
        self.out.update({k: torch.zeros(n, dtype=torch.float64, device=device) for k in OUT_COL})
        self.out["cush"].copy_(self.cush0)
        self.diag_int = torch.zeros((8, n), dtype=torch.int32, device=device) if diag else None
        self.diag_real = torch.zeros((8, n), dtype=torch.float64, device=device) if diag else None
        self.diag_level = (torch.zeros((NDL, mkx + 1, n), dtype=torch.float64, device=device)
                           if diag else None)

    def reset_cush(self):
        self.out["cush"].copy_(self.cush0)

    def launch(self, inv=0, stream=None, omega=None):
        """Enqueue one call on `stream` (torch stream or None for the current stream); with omega (a
        device tensor (mkx, n) of pressure velocity) one compute_zwshcu_device call instead."""
        torch = self.torch
        st = stream if stream is not None else torch.cuda.current_stream()
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        i, o = self.inp, self.out
        if omega is not None:
            return lib().compute_zwshcu_device(
                ctypes.c_int(self.n), ctypes.c_int(self.mkx), ctypes.c_int(self.n),
                ctypes.c_int(self.ncnst), ctypes.c_double(self.dt), ctypes.c_int(inv),
                P(i["ps0"]), P(i["zs0"]), P(i["p0"]), P(i["z0"]), P(i["dp0"]), P(i["u0"]), P(i["v0"]),
                P(i["qv0"]), P(i["ql0"]), P(i["qi0"]), P(i["t0"]), P(i["s0"]), P(i["tr0"]),
                P(i["tke"]), P(i["pblh"]), P(omega), P(o["cush"]), P(o["umf"]), P(o["slflx"]),
                P(o["qtflx"]), P(o["flxprc1"]), P(o["flxsnow1"]), P(o["qvten"]), P(o["qlten"]),
                P(o["qiten"]), P(o["sten"]), P(o["uten"]), P(o["vten"]), P(o["trten"]), P(o["qrten"]),
                P(o["qsten"]), P(o["precip"]), P(o["snow"]), P(o["evapc"]), P(o["cufrc"]),
                P(o["qcu"]), P(o["qlu"]), P(o["qiu"]), P(o["cbmf"]), P(o["qc"]), P(o["rliq"]),
                P(o["cnt"]), P(o["cnb"]), P(i["dpdry0"]), P(o["wu"]),
                P(self.diag_int) if self.diag_int is not None else None,
                P(self.diag_real) if self.diag_real is not None else None,
                ctypes.c_void_p(st.cuda_stream))
        return lib().uwshcu_compute_device(
            ctypes.c_int(self.n), ctypes.c_int(self.mkx), ctypes.c_int(self.n),
            ctypes.c_int(self.ncnst), ctypes.c_double(self.dt), ctypes.c_int(inv),
            P(i["ps0"]), P(i["zs0"]), P(i["p0"]), P(i["z0"]), P(i["dp0"]), P(i["u0"]), P(i["v0"]),
            P(i["qv0"]), P(i["ql0"]), P(i["qi0"]), P(i["t0"]), P(i["s0"]), P(i["tr0"]),
            P(i["tke"]), P(i["pblh"]), P(o["cush"]), P(o["umf"]), P(o["slflx"]), P(o["qtflx"]),
            P(o["flxprc1"]), P(o["flxsnow1"]), P(o["qvten"]), P(o["qlten"]), P(o["qiten"]),
            P(o["sten"]), P(o["uten"]), P(o["vten"]), P(o["trten"]), P(o["qrten"]),
            P(o["qsten"]), P(o["precip"]), P(o["snow"]), P(o["evapc"]), P(o["cufrc"]),
            P(o["qcu"]), P(o["qlu"]), P(o["qiu"]), P(o["cbmf"]), P(o["qc"]), P(o["rliq"]),
            P(o["cnt"]), P(o["cnb"]), P(i["dpdry0"]), P(o["wu"]),
            P(self.diag_int) if self.diag_int is not None else None,
            P(self.diag_real) if self.diag_real is not None else None,
            ctypes.c_void_p(st.cuda_stream))

    def launch_member(self, inv=0, stream=None):
        """Enqueue one call of uwshcu_compute_member (which also fills diag_level) on `stream`."""
        st = stream if stream is not None else self.torch.cuda.current_stream()
        m = member_of(self, inv)
        return lib().uwshcu_compute_member(ctypes.byref(m), ctypes.c_void_p(st.cuda_stream))

    def launch_noalloc(self, inv=0, stream=None, status_bits=None):
        """Enqueue one call of uwshcu_compute_device_noalloc on `stream`; status_bits is None or a
        one-element torch.int32 device tensor that receives the call's endrun bits."""
        torch = self.torch
        st = stream if stream is not None else torch.cuda.current_stream()
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        i, o = self.inp, self.out
        return lib().uwshcu_compute_device_noalloc(
            ctypes.c_int(self.n), ctypes.c_int(self.mkx), ctypes.c_int(self.n),
            ctypes.c_int(self.ncnst), ctypes.c_double(self.dt), ctypes.c_int(inv),
            P(i["ps0"]), P(i["zs0"]), P(i["p0"]), P(i["z0"]), P(i["dp0"]), P(i["u0"]), P(i["v0"]),
            P(i["qv0"]), P(i["ql0"]), P(i["qi0"]), P(i["t0"]), P(i["s0"]), P(i["tr0"]),
            P(i["tke"]), P(i["pblh"]), P(o["cush"]), P(o["umf"]), P(o["slflx"]), P(o["qtflx"]),
            P(o["flxprc1"]), P(o["flxsnow1"]), P(o["qvten"]), P(o["qlten"]), P(o["qiten"]),
            P(o["sten"]), P(o["uten"]), P(o["vten"]), P(o["trten"]), P(o["qrten"]),
            P(o["qsten"]), P(o["precip"]), P(o["snow"]), P(o["evapc"]), P(o["cufrc"]),
            P(o["qcu"]), P(o["qlu"]), P(o["qiu"]), P(o["cbmf"]), P(o["qc"]), P(o["rliq"]),
            P(o["cnt"]), P(o["cnb"]), P(i["dpdry0"]), P(o["wu"]),
            P(self.diag_int) if self.diag_int is not None else None,
            P(self.diag_real) if self.diag_real is not None else None,
            P(status_bits) if status_bits is not None else None,
            ctypes.c_void_p(st.cuda_stream))

    def status(self, stream=None):
        torch = self.torch
        st = stream if stream is not None else torch.cuda.current_stream()
        return lib().uwshcu_device_status(ctypes.c_void_p(st.cuda_stream))

    def budgets(self, inv=0, stream=None):
        """CAM's energy and water budget relative errors of the last call (uwshcu_budget_device),
        as two numpy arrays."""
        torch = self.torch
        st = stream if stream is not None else torch.cuda.current_stream()
        P = lambda t: ctypes.c_void_p(t.data_ptr())
        i, o = self.inp, self.out
        te = torch.empty(self.n, dtype=torch.float64, device=o["sten"].device)
        tw = torch.empty_like(te)
        rc = lib().uwshcu_budget_device(
            ctypes.c_int(self.n), ctypes.c_int(self.mkx), ctypes.c_int(self.n), ctypes.c_int(inv),
            ctypes.c_double(self.dt), P(i["s0"]), P(i["qv0"]), P(i["ql0"]), P(i["qi0"]), P(i["u0"]),
            P(i["v0"]), P(i["dp0"]), P(o["sten"]), P(o["qvten"]), P(o["qlten"]), P(o["qiten"]),
            P(o["uten"]), P(o["vten"]), P(o["precip"]), P(o["snow"]), P(o["rliq"]), P(te), P(tw),
            ctypes.c_void_p(st.cuda_stream))
        if rc != 0:
            raise RuntimeError("uwshcu_budget_device: %d %s" % (rc, last_cuda_error()))
        st.synchronize()
        return te.cpu().numpy(), tw.cpu().numpy()

    def outputs_numpy(self):
        o = {k: v.cpu().numpy() for k, v in self.out.items()}
        if self.diag_int is not None:
            o["diag_int"] = self.diag_int.cpu().numpy()
            o["diag_real"] = self.diag_real.cpu().numpy()
            o["diag_level"] = self.diag_level.cpu().numpy()
        return o


def eval_math_device(fn, x, y=None):
    """Evaluate the library's exp/log/pow/erfc (fn 0..3) on the GPU for numpy inputs."""
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
    yd = torch.from_numpy(np.ascontiguousarray(y if y is not None else x, dtype=np.float64)).cuda()
    od = torch.empty_like(xd)
    st = torch.cuda.current_stream()
    rc = lib().uwshcu_eval_math(ctypes.c_int(fn), ctypes.c_void_p(xd.data_ptr()),
                                ctypes.c_void_p(yd.data_ptr()), ctypes.c_void_p(od.data_ptr()),
                                ctypes.c_int(xd.numel()), ctypes.c_void_p(st.cuda_stream))
    if rc != 0:
        raise RuntimeError("uwshcu_eval_math: %d" % rc)
    st.synchronize()
    return od.cpu().numpy()


# ---- batched uneven launches -----------------------------------------------------------------------
MAX_MEMBERS = 8
_MEMBER_PTRS = ("ps0 zs0 p0 z0 dp0 u0 v0 qv0 ql0 qi0 t0 s0 tr0 tke pblh cush umf slflx qtflx flxprc1 "
                "flxsnow1 qvten qlten qiten sten uten vten trten qrten qsten precip snow evapc cufrc qcu "
                "qlu qiu cbmf qc rliq cnt cnb dpdry0 wu diag_int diag_real diag_level").split()


class Member(ctypes.Structure):
    """uwshcu_member of include/uwshcu.h."""
    _fields_ = ([("mix", ctypes.c_int), ("mkx", ctypes.c_int), ("iend", ctypes.c_int), ("inv", ctypes.c_int),
                 ("dt", ctypes.c_double)] + [(n, ctypes.c_void_p) for n in _MEMBER_PTRS])


def member_of(case, inv=0):
    """The uwshcu_member of a DeviceCase."""
    m = Member()
    m.mix = m.iend = case.n
    m.mkx = case.mkx
    m.inv = inv
    m.dt = case.dt
    for name in _MEMBER_PTRS:
        if name in ("diag_int", "diag_real", "diag_level"):
            t = getattr(case, name)
        elif name in case.out:
            t = case.out[name]
        else:
            t = case.inp[name]
        setattr(m, name, t.data_ptr() if t is not None else None)
    return m


class BatchPlan:
    """uwshcu_batch_* over a list of DeviceCase objects (one member each)."""

    def __init__(self, cases, inv=0):
        self.cases = list(cases)
        arr = (Member * len(self.cases))(*[member_of(c, inv) for c in self.cases])
        self._members = arr
        self.handle = ctypes.c_void_p()
        rc = lib().uwshcu_batch_create(ctypes.c_int(len(self.cases)), arr, ctypes.byref(self.handle))
        if rc != 0:
            raise RuntimeError("uwshcu_batch_create: %d %s" % (rc, last_cuda_error()))

    @staticmethod
    def _st(stream):
        import torch
        st = stream if stream is not None else torch.cuda.current_stream()
        return ctypes.c_void_p(st.cuda_stream)

    def run(self, stream=None):
        return lib().uwshcu_batch_run(self.handle, self._st(stream))

    def capture(self, stream):
        return lib().uwshcu_batch_capture(self.handle, self._st(stream))

    def autotune(self, stream=None):
        b, m, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        rc = lib().uwshcu_batch_autotune(self.handle, self._st(stream), ctypes.byref(b), ctypes.byref(m),
                                         ctypes.byref(c))
        if rc != 0:
            raise RuntimeError("uwshcu_batch_autotune: %d %s" % (rc, last_cuda_error()))
        return b.value, m.value, c.value

    def status(self, stream=None):
        return lib().uwshcu_batch_status(self.handle, self._st(stream))

    def close(self):
        if self.handle:
            lib().uwshcu_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()


# ---- tangent-linear model ----------------------------------------------------------------------------
_TANGENT_OUT = ("cush umf slflx qtflx flxprc1 flxsnow1 qvten qlten qiten sten uten vten trten qrten qsten "
                "precip snow evapc cufrc qcu qlu qiu cbmf qc rliq wu").split()


class Tangent(ctypes.Structure):
    """uwshcu_tangent of include/uwshcu.h."""
    _fields_ = ([(n, ctypes.c_void_p) for n in ("dt0", "dqv0", "dtke", "dpblh")] +
                [(n, ctypes.c_double) for n in ("drpen", "drle", "drkm", "dcriqc")] +
                [(n, ctypes.c_void_p) for n in _TANGENT_OUT])


def tangent_launch(case, dirs=None, dparams=(0.0, 0.0, 0.0, 0.0), inv=0, stream=None):
    """One uwshcu_tangent_device call on a DeviceCase: `dirs` maps t0/qv0/tke/pblh to device tensors
    (the direction), dparams = (drpen, drle, drkm, dcriqc).  Returns the tangent outputs (torch
    tensors shaped like case.out); the case's own outputs get the FP64 values."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    dirs = dirs or {}
    tout = {k: torch.zeros_like(case.out[k]) for k in _TANGENT_OUT}
    t = Tangent()
    for k in ("t0", "qv0", "tke", "pblh"):
        d = dirs.get(k)
        setattr(t, "d" + k, d.data_ptr() if d is not None else None)
    t.drpen, t.drle, t.drkm, t.dcriqc = [float(x) for x in dparams]
    for k in _TANGENT_OUT:
        setattr(t, k, tout[k].data_ptr())
    m = member_of(case, inv)
    rc = lib().uwshcu_tangent_device(ctypes.byref(m), ctypes.byref(t), ctypes.c_void_p(st.cuda_stream))
    if rc != 0:
        raise RuntimeError("uwshcu_tangent_device: %d %s" % (rc, last_cuda_error()))
    return tout


# ---- adjoint model -----------------------------------------------------------------------------------
_ADJ_GRAD = ("t0", "qv0", "tke", "pblh", "rpen", "rle", "rkm", "criqc")
# outputs that take a cotangent in adjoint_launch
ADJ_OUTPUTS = tuple(_TANGENT_OUT)


class Adjoint(ctypes.Structure):
    """uwshcu_adjoint of include/uwshcu.h."""
    _fields_ = [(n, ctypes.c_void_p) for n in _TANGENT_OUT] + [(n, ctypes.c_void_p) for n in _ADJ_GRAD]


def adjoint_launch(case, cot, inv=0, stream=None, defect=False):
    """One uwshcu_adjoint_device call on a DeviceCase: `cot` maps output names to device tensors
    shaped like case.out (the cotangents; missing ones are zero).  Returns (status, gradients): t0,
    qv0 (mkx, n), tke (mkx + 1, n), pblh (n) and the per-column parameter gradients rpen, rle, rkm,
    criqc (n), as torch tensors; the case's own outputs get the FP64 values.  defect=True calls
    uwshcu_adjoint_device_checked instead and adds the per-column defect of linearity (n) to the
    gradients as "defect"."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    dev = case.out["umf"].device
    n, mkx = case.n, case.mkx
    grads = {"t0": torch.zeros((mkx, n), dtype=torch.float64, device=dev),
             "qv0": torch.zeros((mkx, n), dtype=torch.float64, device=dev),
             "tke": torch.zeros((mkx + 1, n), dtype=torch.float64, device=dev)}
    grads.update({k: torch.zeros(n, dtype=torch.float64, device=dev) for k in _ADJ_GRAD[3:]})
    a = Adjoint()
    for k in _TANGENT_OUT:
        c = cot.get(k)
        setattr(a, k, c.data_ptr() if c is not None else None)
    for k in _ADJ_GRAD:
        setattr(a, k, grads[k].data_ptr())
    m = member_of(case, inv)
    if defect:
        grads["defect"] = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
        rc = lib().uwshcu_adjoint_device_checked(ctypes.byref(m), ctypes.byref(a),
                                                 ctypes.c_void_p(grads["defect"].data_ptr()),
                                                 ctypes.c_void_p(st.cuda_stream))
    else:
        rc = lib().uwshcu_adjoint_device(ctypes.byref(m), ctypes.byref(a), ctypes.c_void_p(st.cuda_stream))
    return rc, grads


def fp64_peak(stream=None):
    """Measured FP64 throughput of the current device in TFLOP/s (uwshcu_fp64_peak)."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    v = ctypes.c_double(0.0)
    rc = lib().uwshcu_fp64_peak(ctypes.byref(v), ctypes.c_void_p(st.cuda_stream))
    return rc, v.value


def adjoint_last_records():
    return lib().uwshcu_adjoint_last_records()


def adjoint_release():
    return lib().uwshcu_adjoint_release()


def set_adjoint_rows(rows):
    return lib().uwshcu_set_adjoint_rows(ctypes.c_int(rows))
