"""The consumer of the flash's derivatives: host mirror of
``ocpf_fim_upwind`` and ``ocpf_fim_jacobian``, the bulk part of the FIM
Jacobian that IsoT_FIM::AssembleMatBulksNew builds
(src/OCPFluidMethod.cpp:1569-1840) with the upstream choice of
src/BulkConn.cpp:170-215.

Bulk arrays are device tensors in the flash's field-major layout
(``[field, nbulk]``; the names of ``_lib.JAC_BULK_FIELDS``): the flash's
``CellState.out``, the KrPc outputs and the rock (v, poroP, depth).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


def _torch():
    import torch
    return torch


class ConnGraph:
    """The connections of a grid (begin bulk, end bulk, area) on one GPU."""

    def __init__(self, nbulk: int, bId, eId, area, device: int = 0):
        self.device = device
        self.nbulk = int(nbulk)
        b = np.ascontiguousarray(bId, dtype=np.int64)
        e = np.ascontiguousarray(eId, dtype=np.int64)
        a = np.ascontiguousarray(area, dtype=np.float64)
        self.nconn = len(b)
        h = C.c_void_p()
        check(lib().ocpf_conn_create(self.nbulk, self.nconn, b.ctypes.data, e.ctypes.data, a.ctypes.data,
                                     int(device), C.byref(h)), "ocpf_conn_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ocpf_conn_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @staticmethod
    def _bulk(bulk: dict):
        return _lib.JacBulk(*[(bulk[k].data_ptr() if k in bulk else None) for k in _lib.JAC_BULK_FIELDS])

    def upwind(self, bulk: dict, stream=None):
        """upblock [3, nconn] int32 and upblock_rho [3, nconn] (device)."""
        torch = _torch()
        dev = f"cuda:{self.device}"
        up = torch.empty((3, self.nconn), dtype=torch.int32, device=dev)
        rho = torch.empty((3, self.nconn), dtype=torch.float64, device=dev)
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        fb = self._bulk(bulk)
        check(lib().ocpf_fim_upwind(self._h, C.byref(fb), up.data_ptr(), rho.data_ptr(),
                                    C.c_void_p(stream.cuda_stream)), "ocpf_fim_upwind")
        return up, rho

    def jacobian(self, nc: int, dt: float, bulk: dict, up, uprho, out: dict | None = None, stream=None) -> dict:
        """diag [ncol^2, nbulk], offEB and offBE [ncol^2, nconn] (device),
        ncol = nc + 2."""
        torch = _torch()
        dev = f"cuda:{self.device}"
        ncol = nc + 2
        if out is None:
            out = {"diag": torch.empty((ncol * ncol, self.nbulk), dtype=torch.float64, device=dev),
                   "offEB": torch.empty((ncol * ncol, self.nconn), dtype=torch.float64, device=dev),
                   "offBE": torch.empty((ncol * ncol, self.nconn), dtype=torch.float64, device=dev)}
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        fb = self._bulk(bulk)
        fo = _lib.JacOut(*[out[k].data_ptr() for k in _lib.JAC_OUT_FIELDS])
        check(lib().ocpf_fim_jacobian(self._h, int(nc), float(dt), C.byref(fb), up.data_ptr(), uprho.data_ptr(),
                                      C.byref(fo), C.c_void_p(stream.cuda_stream)), "ocpf_fim_jacobian")
        return out
