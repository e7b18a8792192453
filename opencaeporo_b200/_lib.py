"""ctypes declarations of the C ABI in ``include/ocp_flash.h`` and the loader
of ``opencaeporo_b200/libocpflash.so``.

The library is built in-tree (``python -m opencaeporo_b200.build``). There is
no fallback: if the library is missing or cannot be loaded, :func:`lib`
raises.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libocpflash.so")
MAX_NC = 16
NPH = 3

OCPF_OK, OCPF_EINVAL, OCPF_ECUDA, OCPF_ENOMEM, OCPF_EUNSUPPORTED, OCPF_ERANGE = 0, 1, 2, 3, 4, 5
NOALLOC_MAX_CELLS = 4096  # OCPF_NOALLOC_MAX_CELLS
FORM_PLAIN, FORM_BATCHED, FORM_MIXED, FORM_FAST = 0, 1, 2, 3

CELL_SSMSTA_CAP = 0x01
CELL_NRSTA_FAIL = 0x02
CELL_SSMSP_FAIL = 0x04
CELL_NRSP_FAIL = 0x08
CELL_COLLAPSED = 0x10
CELL_SINGULAR = 0x20
CELL_NONFINITE = 0x40
CELL_SPLIT_CAP = 0x80
CELL_GUARD = 0x100

# Every function the header declares (checked by the CPU test suite).
EXPORTS = ("ocpf_version", "ocpf_status_string", "ocpf_create", "ocpf_destroy",
           "ocpf_flash_fim", "ocpf_flash_fim_host", "ocpf_last_kernel_ms",
           "ocpf_measure_fma_peak", "ocpf_reserve", "ocpf_flash_fim_noalloc",
           "ocpf_mlp_param_count", "ocpf_mlp_forward", "ocpf_mlp_grad", "ocpf_mlp_adam",
           "ocpf_set_initializer", "ocpf_flash_fim_regions", "ocpf_measure_fp64_latency",
           "ocpf_flash_impec", "ocpf_init_flash_fim", "ocpf_init_flash_impec",
           "ocpf_flash_fimn", "ocpf_init_flash_fimn", "ocpf_flash_fim_subset", "ocpf_flash_impec_subset",
           "ocpf_krpc_create", "ocpf_krpc_destroy", "ocpf_cal_krpc", "ocpf_last_launch_count",
           "ocpf_conn_create", "ocpf_conn_destroy", "ocpf_fim_upwind", "ocpf_fim_jacobian",
           "ocpf_get_tuning", "ocpf_set_tuning", "ocpf_autotune", "ocpf_last_phase_ms",
           "ocpf_set_part_timing", "ocpf_update_last_step", "ocpf_reset_to_last_step", "ocpf_copy_arrays",
           "ocpf_krpc_create_sof3")

COPY_MAX = 64  # OCPF_COPY_MAX

SCHED_ONE_LAUNCH, SCHED_STREAMS = 0, 1  # OCPF_SCHED_*

_vp = C.c_void_p


class Fluid(C.Structure):
    _fields_ = [
        ("nc", C.c_int32), ("rr_maxit", C.c_int32), ("ssmsta_maxit", C.c_int32),
        ("nrsta_maxit", C.c_int32), ("ssmsp_maxit", C.c_int32), ("nrsp_maxit", C.c_int32),
        ("use_skip", C.c_int32), ("pad0", C.c_int32),
        ("rr_tol", C.c_double), ("ssmsta_tol", C.c_double), ("ssmsta_eyt", C.c_double),
        ("nrsta_tol", C.c_double), ("ssmsp_tol", C.c_double), ("nrsp_tol", C.c_double),
        ("Tc", C.c_double * MAX_NC), ("Pc", C.c_double * MAX_NC), ("Vc", C.c_double * MAX_NC),
        ("MW", C.c_double * MAX_NC), ("Acf", C.c_double * MAX_NC),
        ("OmegaA", C.c_double * MAX_NC), ("OmegaB", C.c_double * MAX_NC),
        ("Vshift", C.c_double * MAX_NC), ("BIC", C.c_double * (MAX_NC * MAX_NC)),
        ("LBCcoef", C.c_double * 5), ("pvtw", C.c_double * 5), ("std_rho_w", C.c_double),
    ]


IN_FIELDS = ("P", "T", "Ni", "S", "lastNP", "xij")
SKIP_FIELDS = ("flag", "minEig", "P", "T", "z")
OUT_FIELDS = ("phaseNum", "phaseExist", "S", "Nt", "vf", "vfP", "vfi", "rho", "xi", "mu",
              "rhoP", "xiP", "muP", "xij", "rhox", "xix", "mux", "dSec_dPri", "bRowSizedSdP",
              "pSderExist", "pVnumCom", "nj", "ePEC", "ftype", "iters", "status")
OPTIONAL_OUT = ("nj", "ePEC", "ftype", "iters", "status")


class FimIn(C.Structure):
    _fields_ = [(f, _vp) for f in IN_FIELDS]


class Skip(C.Structure):
    _fields_ = [(f, _vp) for f in SKIP_FIELDS]


class FimOut(C.Structure):
    _fields_ = [(f, _vp) for f in OUT_FIELDS]


IMPEC_IN_FIELDS = ("P", "T", "Ni", "lastNP", "xij")
IMPEC_OUT_FIELDS = ("phaseNum", "phaseExist", "S", "Nt", "vf", "vfP", "vfi", "vj", "rho", "xi", "mu", "xij",
                    "ePEC", "ftype", "iters", "status")


class ImpecIn(C.Structure):
    _fields_ = [(f, _vp) for f in IMPEC_IN_FIELDS]


class ImpecOut(C.Structure):
    _fields_ = [(f, _vp) for f in IMPEC_OUT_FIELDS]


INIT_IN_FIELDS = ("P", "T", "S", "Vpore", "zi")
KRPC_OUT_FIELDS = ("kr", "Pc", "Pj", "dKr_dS", "dPcj_dS")


class Satfunc(C.Structure):
    _fields_ = [("nrow_swof", C.c_int32), ("nrow_sgof", C.c_int32), ("swof", _vp), ("sgof", _vp)]


class Satfunc3(C.Structure):
    """ocpf_satfunc3 (SWFN, SGFN, SOF3)"""
    _fields_ = [("nrow_swfn", C.c_int32), ("nrow_sgfn", C.c_int32), ("nrow_sof3", C.c_int32), ("pad", C.c_int32),
                ("swfn", _vp), ("sgfn", _vp), ("sof3", _vp)]


class KrpcIn(C.Structure):
    _fields_ = [("P", _vp), ("S", _vp), ("satnum", _vp)]


class KrpcOut(C.Structure):
    _fields_ = [(f, _vp) for f in KRPC_OUT_FIELDS]


JAC_BULK_FIELDS = ("phaseExist", "pSderExist", "pVnumCom", "S", "rho", "xi", "mu", "muP", "xiP", "rhoP", "xij",
                   "rhox", "xix", "mux", "dSec_dPri", "vfP", "vfi", "kr", "Pj", "dKr_dS", "dPcj_dS", "v", "poroP",
                   "depth")
JAC_OUT_FIELDS = ("diag", "offEB", "offBE")


class JacBulk(C.Structure):
    _fields_ = [(f, _vp) for f in JAC_BULK_FIELDS]


class JacOut(C.Structure):
    _fields_ = [(f, _vp) for f in JAC_OUT_FIELDS]


class InitIn(C.Structure):
    _fields_ = [(f, _vp) for f in INIT_IN_FIELDS]


def out_shapes(nc: int) -> dict:
    """(number of SoA fields, element type) of every output array."""
    ncom = nc + 1
    ncol = ncom + 1
    return {
        "phaseNum": (1, "u32"), "phaseExist": (NPH, "u32"), "S": (NPH, "f64"), "Nt": (1, "f64"),
        "vf": (1, "f64"), "vfP": (1, "f64"), "vfi": (ncom, "f64"), "rho": (NPH, "f64"),
        "xi": (NPH, "f64"), "mu": (NPH, "f64"), "rhoP": (NPH, "f64"), "xiP": (NPH, "f64"),
        "muP": (NPH, "f64"), "xij": (NPH * ncom, "f64"), "rhox": (NPH * ncom, "f64"),
        "xix": (NPH * ncom, "f64"), "mux": (NPH * ncom, "f64"),
        "dSec_dPri": (NPH * ncol * ncol, "f64"), "bRowSizedSdP": (1, "u32"),
        "pSderExist": (NPH, "u32"), "pVnumCom": (NPH, "u32"), "nj": (NPH, "f64"),
        "ePEC": (1, "f64"), "ftype": (1, "u8"), "iters": (5, "i32"), "status": (1, "u16"),
    }


def in_shapes(nc: int) -> dict:
    ncom = nc + 1
    return {"P": (1, "f64"), "T": (1, "f64"), "Ni": (ncom, "f64"), "S": (NPH, "f64"),
            "lastNP": (1, "u32"), "xij": (NPH * ncom, "f64")}


def skip_shapes(nc: int) -> dict:
    return {"flag": (1, "u32"), "minEig": (1, "f64"), "P": (1, "f64"), "T": (1, "f64"),
            "z": (nc, "f64")}


class Tuning(C.Structure):
    """ocpf_tuning"""
    _fields_ = [("block", C.c_int32), ("persist_pct", C.c_int32), ("slow_threads", C.c_int32),
                ("schedule", C.c_int32), ("ms", C.c_float), ("pad", C.c_int32)]


_LIB = None


def lib():
    """Loads libocpflash.so (raises if it is missing: there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m opencaeporo_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.ocpf_version.restype = C.c_char_p
    L.ocpf_status_string.restype = C.c_char_p
    L.ocpf_status_string.argtypes = [C.c_int]
    L.ocpf_create.argtypes = [C.POINTER(Fluid), C.c_int, C.POINTER(_vp)]
    L.ocpf_create.restype = C.c_int
    L.ocpf_destroy.argtypes = [_vp]
    L.ocpf_destroy.restype = C.c_int
    L.ocpf_flash_fim.argtypes = [_vp, C.c_int64, C.POINTER(FimIn), C.POINTER(Skip),
                                 C.POINTER(FimOut), C.c_int, _vp]
    L.ocpf_flash_fim.restype = C.c_int
    L.ocpf_flash_fim_host.argtypes = [_vp, C.c_int64, C.POINTER(FimIn), C.POINTER(Skip),
                                      C.POINTER(FimOut), C.c_int]
    L.ocpf_flash_fim_host.restype = C.c_int
    L.ocpf_last_kernel_ms.argtypes = [_vp, C.POINTER(C.c_float)]
    L.ocpf_last_kernel_ms.restype = C.c_int
    L.ocpf_measure_fma_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.ocpf_measure_fma_peak.restype = C.c_int
    L.ocpf_reserve.argtypes = [_vp, C.c_int64]
    L.ocpf_reserve.restype = C.c_int
    L.ocpf_flash_fim_noalloc.argtypes = [_vp, C.c_int64, C.POINTER(FimIn), C.POINTER(Skip),
                                         C.POINTER(FimOut), _vp]
    L.ocpf_flash_fim_noalloc.restype = C.c_int
    L.ocpf_mlp_param_count.restype = C.c_int
    L.ocpf_mlp_forward.argtypes = [C.c_int, C.c_int, C.c_int64, _vp, _vp, _vp, _vp]
    L.ocpf_mlp_forward.restype = C.c_int
    L.ocpf_mlp_grad.argtypes = [C.c_int, C.c_int, C.c_int64, _vp, _vp, _vp, _vp, C.c_float, _vp, _vp, _vp]
    L.ocpf_mlp_grad.restype = C.c_int
    L.ocpf_mlp_adam.argtypes = [_vp, _vp, _vp, _vp, C.c_int, C.c_float, _vp]
    L.ocpf_mlp_adam.restype = C.c_int
    L.ocpf_set_initializer.argtypes = [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                       C.c_float]
    L.ocpf_set_initializer.restype = C.c_int
    L.ocpf_flash_fim_regions.argtypes = [C.c_int, C.POINTER(_vp), C.POINTER(C.c_int64), C.POINTER(FimIn),
                                         C.POINTER(Skip), C.POINTER(FimOut), C.c_int, _vp]
    L.ocpf_flash_fim_regions.restype = C.c_int
    L.ocpf_set_part_timing.argtypes = [_vp, C.c_int]
    L.ocpf_set_part_timing.restype = C.c_int
    L.ocpf_last_phase_ms.argtypes = [_vp, C.POINTER(C.c_float)]
    L.ocpf_last_phase_ms.restype = C.c_int
    for name in ("ocpf_update_last_step", "ocpf_reset_to_last_step"):
        getattr(L, name).argtypes = [C.c_int, C.c_int64, C.POINTER(FimOut), C.POINTER(Skip), C.POINTER(FimOut),
                                     C.POINTER(Skip), _vp]
        getattr(L, name).restype = C.c_int
    L.ocpf_copy_arrays.argtypes = [C.c_int, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.c_int64), _vp]
    L.ocpf_copy_arrays.restype = C.c_int
    L.ocpf_get_tuning.argtypes = [_vp, C.POINTER(Tuning)]
    L.ocpf_get_tuning.restype = C.c_int
    L.ocpf_set_tuning.argtypes = [_vp, C.POINTER(Tuning)]
    L.ocpf_set_tuning.restype = C.c_int
    L.ocpf_autotune.argtypes = [C.c_int, C.POINTER(_vp), C.POINTER(C.c_int64), C.POINTER(FimIn), C.POINTER(Skip),
                                C.c_int, C.c_int, _vp, C.POINTER(Tuning)]
    L.ocpf_autotune.restype = C.c_int
    L.ocpf_measure_fp64_latency.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.ocpf_measure_fp64_latency.restype = C.c_int
    L.ocpf_flash_impec.argtypes = [_vp, C.c_int64, C.POINTER(ImpecIn), C.POINTER(Skip), C.POINTER(ImpecOut),
                                   C.c_int, _vp]
    L.ocpf_flash_impec.restype = C.c_int
    L.ocpf_init_flash_fim.argtypes = [_vp, C.c_int64, C.POINTER(InitIn), C.POINTER(Skip), _vp, C.POINTER(FimOut),
                                      C.c_int, _vp]
    L.ocpf_init_flash_fim.restype = C.c_int
    L.ocpf_init_flash_impec.argtypes = [_vp, C.c_int64, C.POINTER(InitIn), C.POINTER(Skip), _vp,
                                        C.POINTER(ImpecOut), C.c_int, _vp]
    L.ocpf_init_flash_impec.restype = C.c_int
    L.ocpf_flash_fimn.argtypes = [_vp, C.c_int64, C.POINTER(FimIn), C.POINTER(Skip), C.POINTER(FimOut), _vp, _vp,
                                  C.c_int, _vp]
    L.ocpf_flash_fimn.restype = C.c_int
    L.ocpf_init_flash_fimn.argtypes = [_vp, C.c_int64, C.POINTER(InitIn), C.POINTER(Skip), _vp, C.POINTER(FimOut),
                                       _vp, _vp, C.c_int, _vp]
    L.ocpf_init_flash_fimn.restype = C.c_int
    L.ocpf_flash_fim_subset.argtypes = [_vp, C.c_int64, _vp, C.c_int64, C.POINTER(FimIn), C.POINTER(Skip),
                                        C.POINTER(FimOut), C.c_int, _vp]
    L.ocpf_flash_fim_subset.restype = C.c_int
    L.ocpf_flash_impec_subset.argtypes = [_vp, C.c_int64, _vp, C.c_int64, C.POINTER(ImpecIn), C.POINTER(Skip),
                                          C.POINTER(ImpecOut), C.c_int, _vp]
    L.ocpf_flash_impec_subset.restype = C.c_int
    L.ocpf_conn_create.argtypes = [C.c_int64, C.c_int64, _vp, _vp, _vp, C.c_int, C.POINTER(_vp)]
    L.ocpf_conn_create.restype = C.c_int
    L.ocpf_conn_destroy.argtypes = [_vp]
    L.ocpf_conn_destroy.restype = C.c_int
    L.ocpf_fim_upwind.argtypes = [_vp, C.POINTER(JacBulk), _vp, _vp, _vp]
    L.ocpf_fim_upwind.restype = C.c_int
    L.ocpf_fim_jacobian.argtypes = [_vp, C.c_int, C.c_double, C.POINTER(JacBulk), _vp, _vp, C.POINTER(JacOut), _vp]
    L.ocpf_fim_jacobian.restype = C.c_int
    L.ocpf_last_launch_count.argtypes = [_vp, C.POINTER(C.c_int)]
    L.ocpf_last_launch_count.restype = C.c_int
    L.ocpf_krpc_create.argtypes = [C.POINTER(Satfunc), C.c_int, C.c_int, C.POINTER(_vp)]
    L.ocpf_krpc_create_sof3.argtypes = [C.POINTER(Satfunc3), C.c_int, C.c_int, C.POINTER(_vp)]
    L.ocpf_krpc_create_sof3.restype = C.c_int
    L.ocpf_krpc_create.restype = C.c_int
    L.ocpf_krpc_destroy.argtypes = [_vp]
    L.ocpf_krpc_destroy.restype = C.c_int
    L.ocpf_cal_krpc.argtypes = [_vp, C.c_int64, C.POINTER(KrpcIn), C.POINTER(KrpcOut), _vp]
    L.ocpf_cal_krpc.restype = C.c_int
    _LIB = L
    return L


def make_fluid(fl) -> Fluid:
    """C-ABI fluid block from an :class:`opencaeporo_b200.fluid.Fluid`."""
    f = Fluid()
    nc = fl.nc
    c = fl.controls
    f.nc = nc
    f.rr_maxit, f.rr_tol = c.rr_maxit, c.rr_tol
    f.ssmsta_maxit, f.ssmsta_tol, f.ssmsta_eyt = c.ssmsta_maxit, c.ssmsta_tol, c.ssmsta_eyt
    f.nrsta_maxit, f.nrsta_tol = c.nrsta_maxit, c.nrsta_tol
    f.ssmsp_maxit, f.ssmsp_tol = c.ssmsp_maxit, c.ssmsp_tol
    f.nrsp_maxit, f.nrsp_tol = c.nrsp_maxit, c.nrsp_tol
    f.use_skip = 1 if c.use_skip else 0
    for name in ("Tc", "Pc", "Vc", "MW", "Acf", "OmegaA", "OmegaB", "Vshift"):
        arr = getattr(f, name)
        for i, v in enumerate(getattr(fl, name)):
            arr[i] = float(v)
    for i in range(nc):
        for k in range(nc):
            f.BIC[i * nc + k] = float(fl.BIC[i, k])
    for k in range(5):
        f.LBCcoef[k] = float(fl.LBCcoef[k])
        f.pvtw[k] = float(fl.pvtw[k])
    f.std_rho_w = float(fl.std_rho_w)
    return f


def check(rc: int, what: str):
    if rc != OCPF_OK:
        msg = lib().ocpf_status_string(rc).decode()
        raise RuntimeError(f"{what} failed: {msg} ({rc})")


def fp64_latency_cycles(device: int = 0) -> dict:
    """One-thread latencies (cycles) of FP64 division, division issued twelve
    at a time (per division), FMA, exp, log and acos + cos."""
    v = (C.c_double * 6)()
    check(lib().ocpf_measure_fp64_latency(int(device), v), "ocpf_measure_fp64_latency")
    return dict(zip(("div", "div_x12_each", "fma", "exp", "log", "acos_cos"), list(v)))


def fma_peak_tflops(device: int = 0, bits: int = 64) -> float:
    """Measured FMA throughput of the device (TFLOP/s)."""
    v = C.c_double(0)
    check(lib().ocpf_measure_fma_peak(int(device), int(bits), C.byref(v)), "ocpf_measure_fma_peak")
    return float(v.value)
