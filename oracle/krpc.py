"""TEST INFRASTRUCTURE ONLY: the relative permeabilities and capillary
pressures of a cell after the flash, as IsoT_FIM::CalKrPc computes them
(src/OCPFluidMethod.cpp:1189-1199) with the compositional model's default
flow unit FlowUnit_ODGW01 (src/FlowUnit.cpp:183-349) and, for the SWFN /
SGFN / SOF3 family (``*_sof3``), FlowUnit_ODGW02 (src/FlowUnit.cpp:522-671).

Two implementations:
  * ``reference`` -- the reference's own FlowUnit compiled into
    oracle/_ref/libocpref.so (orc_krpc and orc_krpc_sof3 in
    oracle/ref_harness.cpp);
  * ``restated`` -- a numpy restatement of the same arithmetic, kept bit for
    bit (no fused multiply-add anywhere), for checks where the compiled
    reference is absent.

Tables are given as the keywords list them: SWOF / SGOF rows of
(Sw, krw, krow, Pcow) and (Sg, krg, krog, Pcgo); SWFN / SGFN / SOF3 rows of
(Sw, krw, Pcow), (Sg, krg, Pcgo) and (So, krow, krog). Outputs are cell-major:
kr, Pc, Pj [n, 3] and dKr_dS, dPcj_dS [n, 9] (entry 3 j + k: d/dS_k of
phase j; phases oil, gas, water).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import oracle as O

_dp = C.POINTER(C.c_double)


class OrcSatfunc(C.Structure):
    _fields_ = [("nrow_swof", C.c_int32), ("nrow_sgof", C.c_int32), ("swof", _dp), ("sgof", _dp)]


class OrcKrpcBatch(C.Structure):
    _fields_ = [("n", C.c_int64), ("deriv", C.c_int32), ("P", _dp), ("S", _dp),
                ("satnum", C.POINTER(C.c_int32)), ("kr", _dp), ("Pc", _dp), ("Pj", _dp),
                ("dKr_dS", _dp), ("dPcj_dS", _dp)]


class OrcSatfunc3(C.Structure):
    _fields_ = [("nrow_swfn", C.c_int32), ("nrow_sgfn", C.c_int32), ("nrow_sof3", C.c_int32), ("pad", C.c_int32),
                ("swfn", _dp), ("sgfn", _dp), ("sof3", _dp)]


def _outputs(n):
    return {"kr": np.full((n, 3), np.nan), "Pc": np.full((n, 3), np.nan), "Pj": np.full((n, 3), np.nan),
            "dKr_dS": np.full((n, 9), np.nan), "dPcj_dS": np.full((n, 9), np.nan)}


def reference(regions, P, S, satnum=None, deriv=True, nthreads=0):
    """orc_krpc: the compiled reference. ``regions``: list of (swof, sgof)
    row arrays."""
    lib = O.load("reference")
    lib.orc_krpc.argtypes = [C.c_int, C.POINTER(OrcSatfunc), C.POINTER(OrcKrpcBatch), C.c_int,
                             C.POINTER(C.c_double)]
    lib.orc_krpc.restype = C.c_int
    tabs = [(np.ascontiguousarray(w, dtype=np.float64), np.ascontiguousarray(g, dtype=np.float64))
            for w, g in regions]
    regs = (OrcSatfunc * len(tabs))()
    for i, (w, g) in enumerate(tabs):
        regs[i] = OrcSatfunc(len(w), len(g), w.ctypes.data_as(_dp), g.ctypes.data_as(_dp))
    return _run(lib.orc_krpc, regs, len(tabs), P, S, satnum, deriv, nthreads)


def reference_sof3(regions, P, S, satnum=None, deriv=True, nthreads=0):
    """orc_krpc_sof3: the compiled reference's FlowUnit_ODGW02.
    ``regions``: list of (swfn, sgfn, sof3) row arrays."""
    lib = O.load("reference")
    lib.orc_krpc_sof3.argtypes = [C.c_int, C.POINTER(OrcSatfunc3), C.POINTER(OrcKrpcBatch), C.c_int,
                                  C.POINTER(C.c_double)]
    lib.orc_krpc_sof3.restype = C.c_int
    tabs = [tuple(np.ascontiguousarray(t, dtype=np.float64) for t in r) for r in regions]
    regs = (OrcSatfunc3 * len(tabs))()
    for i, (w, g, o) in enumerate(tabs):
        regs[i] = OrcSatfunc3(len(w), len(g), len(o), 0, w.ctypes.data_as(_dp), g.ctypes.data_as(_dp),
                              o.ctypes.data_as(_dp))
    return _run(lib.orc_krpc_sof3, regs, len(tabs), P, S, satnum, deriv, nthreads)


def _run(fn, regs, nreg, P, S, satnum, deriv, nthreads):
    n = len(P)
    P = np.ascontiguousarray(P, dtype=np.float64)
    S = np.ascontiguousarray(S, dtype=np.float64).reshape(n, 3)
    sn = None if satnum is None else np.ascontiguousarray(satnum, dtype=np.int32)
    out = _outputs(n)
    b = OrcKrpcBatch(n, 1 if deriv else 0, P.ctypes.data_as(_dp), S.ctypes.data_as(_dp),
                     None if sn is None else sn.ctypes.data_as(C.POINTER(C.c_int32)),
                     *[out[k].ctypes.data_as(_dp) for k in ("kr", "Pc", "Pj", "dKr_dS", "dPcj_dS")])
    secs = C.c_double(0)
    rc = fn(nreg, regs, C.byref(b), int(nthreads or os.cpu_count() or 1), C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"{fn.__name__} failed with {rc}")
    if not deriv:
        del out["dKr_dS"], out["dPcj_dS"]
    out["seconds"] = secs.value
    return out


def _eval_all(tab, val):
    """OCPTable::Eval_All on column 0 (src/OCPTable.cpp:47-87): the interval
    is the last node <= val (the reference's search from its remembered
    position finds the same one for any non-decreasing column); flat outside
    the table. Returns (values, slopes) of the table's columns."""
    x = tab[:, 0]
    ncol = tab.shape[1]
    if not val >= x[0]:
        return tab[0].copy(), np.zeros(ncol)
    if val >= x[-1]:
        return tab[-1].copy(), np.zeros(ncol)
    b = int(np.searchsorted(x, val, side="right")) - 1
    slope = (tab[b + 1] - tab[b]) / (x[b + 1] - x[b])
    return tab[b] + slope * (val - x[b]), slope


def restated(regions, P, S, satnum=None, deriv=True):
    n = len(P)
    out = _outputs(n)
    S = np.asarray(S, dtype=np.float64).reshape(n, 3)
    for c in range(n):
        swof, sgof = regions[0 if satnum is None else int(satnum[c])]
        swof = np.asarray(swof, dtype=np.float64)
        sgof = np.asarray(sgof, dtype=np.float64)
        kro_max = swof[0, 2]
        d, cd = _eval_all(swof, S[c, 2])
        krw, dkrw, krow, dkrow, pcwo, dpcw = d[1], cd[1], d[2], cd[2], -d[3], -cd[3]
        d, cd = _eval_all(sgof, S[c, 1])
        krg, dkrg, krog, dkrog, pcgo, dpcg = d[1], cd[1], d[2], cd[2], d[3], cd[3]
        # CalKro_Stone2Der, src/FlowUnit.cpp:301-328
        kro = kro_max * ((krow / kro_max + krw) * (krog / kro_max + krg) - (krw + krg))
        dkro_w = kro_max * ((dkrow / kro_max + dkrw) * (krog / kro_max + krg) - dkrw)
        dkro_g = kro_max * ((krow / kro_max + krw) * (dkrog / kro_max + dkrg) - dkrg)
        if kro < 0:
            kro, dkro_g, dkro_w = 0.0, 0.0, 0.0
        out["kr"][c] = (kro, krg, krw)
        out["Pc"][c] = (0.0, pcgo, pcwo)
        out["dKr_dS"][c] = (0, dkro_g, dkro_w, 0, dkrg, 0, 0, 0, dkrw)
        out["dPcj_dS"][c] = (0, 0, 0, 0, dpcg, 0, 0, 0, dpcw)
        out["Pj"][c] = P[c] + out["Pc"][c]
    if not deriv:
        del out["dKr_dS"], out["dPcj_dS"]
    return out


def restated_sof3(regions, P, S, satnum=None, deriv=True):
    """FlowUnit_ODGW02 (src/FlowUnit.cpp:537-652): SWFN at S_w, SGFN at S_g,
    SOF3 at S_o; with ``deriv`` (CalKrPcDeriv) Stone II with kroMax = SOF3's
    last krow and dKro/dS_o, without (CalKrPc) the default model
    (CalKro_Default, :166-177, TINY = 1e-8 from include/OCPConst.hpp)."""
    n = len(P)
    out = _outputs(n)
    S = np.asarray(S, dtype=np.float64).reshape(n, 3)
    for c in range(n):
        reg = regions[0 if satnum is None else int(satnum[c])]
        swfn, sgfn, sof3 = (np.asarray(t, dtype=np.float64) for t in reg)
        kro_max, swco = sof3[-1, 1], swfn[0, 0]
        So, Sg, Sw = S[c]
        d, cd = _eval_all(swfn, Sw)
        krw, dkrw, pcwo, dpcw = d[1], cd[1], -d[2], -cd[2]
        d, cd = _eval_all(sgfn, Sg)
        krg, dkrg, pcgo, dpcg = d[1], cd[1], d[2], cd[2]
        d, cd = _eval_all(sof3, So)
        krow, dkrow, krog, dkrog = d[1], cd[1], d[2], cd[2]
        if deriv:
            kro = kro_max * ((krow / kro_max + krw) * (krog / kro_max + krg) - (krw + krg))
            dkro = dkrow * (krog / kro_max + krg) + dkrog * (krow / kro_max + krw)
            if kro < 0:
                kro, dkro = 0.0, 0.0
        else:
            with np.errstate(invalid="ignore"):  # NaN and infinite saturations pass through
                tmp = Sg + Sw - swco
                kro = kro_max if tmp <= 1e-8 else (Sg * krog + (Sw - swco) * krow) / tmp
            dkro = 0.0
        out["kr"][c] = (kro, krg, krw)
        out["Pc"][c] = (0.0, pcgo, pcwo)
        out["dKr_dS"][c] = (dkro, 0, 0, 0, dkrg, 0, 0, 0, dkrw)
        out["dPcj_dS"][c] = (0, 0, 0, 0, dpcg, 0, 0, 0, dpcw)
        out["Pj"][c] = P[c] + out["Pc"][c]
    if not deriv:
        del out["dKr_dS"], out["dPcj_dS"]
    return out
