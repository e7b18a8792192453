"""Relative permeability and capillary pressure after the flash: the host
mirror of ``ocpf_cal_krpc``, the batched IsoT_FIM::CalKrPc /
IsoT_IMPEC::CalKrPc (src/OCPFluidMethod.cpp:1189-1199, 311-319) for the
compositional model's flow units: the default FlowUnit_ODGW01
(src/FlowUnit.cpp:183-349) and FlowUnit_ODGW02 (:522-671), which the
reference selects when SOF3 is given (src/Bulk.cpp:271-279).

Tables are given as the keywords list them, one tuple per saturation
region: (SWOF, SGOF) with rows (Sw, krw, krow, Pcow) and (Sg, krg, krog,
Pcgo), or (SWFN, SGFN, SOF3) with rows (Sw, krw, Pcow), (Sg, krg, Pcgo) and
(So, krow, krog). Device arrays are field-major like the flash's: P [n],
S [3, n] (the flash's ``out['S']``), kr / Pc / Pj [3, n], dKr_dS / dPcj_dS
[9, n].
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


def _torch():
    import torch
    return torch


class FlowUnitBatch:
    """The flow unit of every saturation region on one GPU: FlowUnit_ODGW01
    for (SWOF, SGOF) regions, FlowUnit_ODGW02 for (SWFN, SGFN, SOF3) ones
    (one family for all regions, as the reference's SATmode is)."""

    def __init__(self, regions, device: int = 0):
        self.device = device
        self._keep = []
        kinds = {len(r) for r in regions}
        if kinds == {2}:
            self.family = "swof"
            regs = (_lib.Satfunc * len(regions))()
            for i, (swof, sgof) in enumerate(regions):
                w = np.ascontiguousarray(swof, dtype=np.float64).reshape(-1, 4)
                g = np.ascontiguousarray(sgof, dtype=np.float64).reshape(-1, 4)
                self._keep += [w, g]
                regs[i] = _lib.Satfunc(len(w), len(g), w.ctypes.data, g.ctypes.data)
            create, name = lib().ocpf_krpc_create, "ocpf_krpc_create"
        elif kinds == {3}:
            self.family = "sof3"
            regs = (_lib.Satfunc3 * len(regions))()
            for i, tabs in enumerate(regions):
                t = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3) for x in tabs]
                self._keep += t
                regs[i] = _lib.Satfunc3(len(t[0]), len(t[1]), len(t[2]), 0, t[0].ctypes.data, t[1].ctypes.data,
                                        t[2].ctypes.data)
            create, name = lib().ocpf_krpc_create_sof3, "ocpf_krpc_create_sof3"
        else:
            raise ValueError("regions must all be (SWOF, SGOF) or all (SWFN, SGFN, SOF3)")
        h = C.c_void_p()
        check(create(regs, len(regions), int(device), C.byref(h)), name)
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ocpf_krpc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def new_outputs(self, ncell: int, deriv: bool = True) -> dict:
        torch = _torch()
        dev = f"cuda:{self.device}"
        out = {k: torch.empty((3, ncell), dtype=torch.float64, device=dev) for k in ("kr", "Pc", "Pj")}
        if deriv:
            for k in ("dKr_dS", "dPcj_dS"):
                out[k] = torch.empty((9, ncell), dtype=torch.float64, device=dev)
        return out

    def cal_krpc(self, P, S, satnum=None, out: dict | None = None, deriv: bool = True, stream=None) -> dict:
        """kr, Pc, Pj (and with ``deriv`` dKr_dS, dPcj_dS) of every cell from
        device P [n] and S [3, n]; ``satnum`` [n] int32 or None (region 0)."""
        torch = _torch()
        n = int(P.shape[0])
        if out is None:
            out = self.new_outputs(n, deriv)
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        fin = _lib.KrpcIn(P.data_ptr(), S.data_ptr(), None if satnum is None else satnum.data_ptr())
        fo = _lib.KrpcOut(*[(out[k].data_ptr() if (k in out and (deriv or k in ("kr", "Pc", "Pj"))) else None)
                            for k in _lib.KRPC_OUT_FIELDS])
        rc = lib().ocpf_cal_krpc(self._h, n, C.byref(fin), C.byref(fo), C.c_void_p(stream.cuda_stream))
        check(rc, "ocpf_cal_krpc")
        return out
