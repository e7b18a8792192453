"""Batched compositional PR flash on the GPU: the host-side mirror of the
reference's ``MixtureComp`` interface for the FIM path.

The reference calls, for every bulk cell ``n`` (``src/OCPFluidMethod.cpp:1108-1187``)::

    flashCal[PVTNUM[n]]->FlashFIM(P[n], T[n], &Ni[n*nc], &S[n*np], phaseNum[n], &xij[n*np*nc], n)
    PassFlashValue(bk, n)

:class:`MixtureCompBatch` does the same for all cells in one call of the C ABI
(``include/ocp_flash.h``) on device-resident structure-of-arrays state:
``S``, ``phaseNum`` and ``xij`` are read as the previous step's values and
overwritten in place, exactly as the Bulk arrays are. PyTorch only supplies
device memory and streams; the flash itself is the CUDA library, which must
be present (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import FORM_BATCHED, FORM_FAST, FORM_MIXED, FORM_PLAIN, NPH, check, lib, make_fluid

_TORCH_DT = {"f64": "float64", "u32": "int32", "i32": "int32", "u16": "int16", "u8": "uint8"}
_NP_DT = {"f64": np.float64, "u32": np.uint32, "i32": np.int32, "u16": np.uint16, "u8": np.uint8}

FORMS = {"plain": FORM_PLAIN, "batched": FORM_BATCHED, "mixed": FORM_MIXED, "fast": FORM_FAST}


def _torch():
    import torch
    return torch


@dataclass
class CellState:
    """Device-resident cell arrays of one PVT region (SoA: ``[field, cell]``).

    ``P``, ``T`` and ``Ni`` are the flash inputs. ``out`` holds every output
    named as in ``Bulk``; ``out['S']``, ``out['phaseNum']`` and ``out['xij']``
    double as the warm-start inputs of the next call. ``skip`` is the
    SkipStaAnaly cache."""

    ncell: int
    nc: int
    P: object
    T: object
    Ni: object
    out: dict = field(default_factory=dict)
    skip: dict = field(default_factory=dict)

    def load(self, P, T, Ni):
        """Copies new P [n], T [n] and Ni [n, numCom] (host arrays, cell-major)
        into the device inputs."""
        torch = _torch()
        self.P.copy_(torch.as_tensor(np.ascontiguousarray(P, dtype=np.float64)))
        self.T.copy_(torch.as_tensor(np.ascontiguousarray(T, dtype=np.float64)))
        self.Ni.copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(Ni, dtype=np.float64).T)))

    def to_host(self) -> dict:
        """Outputs as numpy arrays in the cell-major layout of the oracle
        (``[cell, ...]``)."""
        ncom = self.nc + 1
        res = {}
        for k, t in self.out.items():
            a = t.cpu().numpy()
            if a.ndim == 2:
                a = a.T.copy()
            res[k] = a
        for k in ("phaseNum", "phaseExist", "bRowSizedSdP", "pSderExist", "pVnumCom"):
            res[k] = res[k].astype(np.int64)
        res["iters"] = res["iters"].astype(np.int64)
        res["status"] = res["status"].astype(np.uint16)
        for k in ("xij", "rhox", "xix", "mux"):
            res[k] = res[k].reshape(self.ncell, NPH, ncom)
        res["skip"] = {k: (v.cpu().numpy().T.copy() if v.ndim == 2 else v.cpu().numpy())
                       for k, v in self.skip.items()}
        return res


class MixtureCompBatch:
    """One PVT region's flash on one GPU (``MixtureComp`` + ``SkipStaAnaly``)."""

    def __init__(self, fluid, device: int = 0):
        self.fluid = fluid
        self.nc = fluid.nc
        self.device = device
        self._f = make_fluid(fluid)
        h = C.c_void_p()
        check(lib().ocpf_create(C.byref(self._f), int(device), C.byref(h)), "ocpf_create")
        self._h = h

    def tuning(self) -> dict:
        """This context's launch shape and regions schedule (ocpf_get_tuning)."""
        t = _lib.Tuning()
        check(lib().ocpf_get_tuning(self._h, C.byref(t)), "ocpf_get_tuning")
        return {k: getattr(t, k) for k in ("block", "persist_pct", "slow_threads", "schedule", "ms")}

    def set_tuning(self, block=128, persist_pct=100, slow_threads=0, schedule=0):
        """Sets the launch shape by hand (ocpf_set_tuning)."""
        t = _lib.Tuning(int(block), int(persist_pct), int(slow_threads), int(schedule), 0.0, 0)
        check(lib().ocpf_set_tuning(self._h, C.byref(t)), "ocpf_set_tuning")

    def close(self):
        if getattr(self, "_h", None):
            lib().ocpf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------------- device path
    def new_state(self, ncell: int) -> CellState:
        """Zero-initialised device state for ``ncell`` fresh cells (phaseNum 0:
        the first flash runs the strict stability test)."""
        torch = _torch()
        dev = torch.device("cuda", self.device)
        mk = lambda nf, dt: torch.zeros((nf, ncell) if nf > 1 else (ncell,),
                                        dtype=getattr(torch, _TORCH_DT[dt]), device=dev)
        st = CellState(ncell, self.nc, mk(1, "f64"), mk(1, "f64"), mk(self.nc + 1, "f64"))
        for k, (nf, dt) in _lib.out_shapes(self.nc).items():
            st.out[k] = mk(nf, dt)
        for k, (nf, dt) in _lib.skip_shapes(self.nc).items():
            st.skip[k] = mk(nf, dt)
        return st

    def _structs(self, st: CellState, optional=True, fresh=False):
        o = st.out
        if fresh:
            # warm-start inputs of a fresh cell (lastNP = 0), kept apart from
            # the outputs so that repeated calls do identical work
            if st.__dict__.get("_fresh") is None:
                torch = _torch()
                dev = st.P.device
                st.__dict__["_fresh"] = (
                    torch.zeros((NPH, st.ncell), dtype=torch.float64, device=dev),
                    torch.zeros(st.ncell, dtype=torch.int32, device=dev),
                    torch.zeros((NPH * (st.nc + 1), st.ncell), dtype=torch.float64, device=dev))
            S0, NP0, X0 = st.__dict__["_fresh"]
            fin = _lib.FimIn(st.P.data_ptr(), st.T.data_ptr(), st.Ni.data_ptr(), S0.data_ptr(),
                             NP0.data_ptr(), X0.data_ptr())
        else:
            fin = _lib.FimIn(st.P.data_ptr(), st.T.data_ptr(), st.Ni.data_ptr(), o["S"].data_ptr(),
                             o["phaseNum"].data_ptr(), o["xij"].data_ptr())
        sk = _lib.Skip(*[st.skip[k].data_ptr() for k in _lib.SKIP_FIELDS])
        vals = []
        for k in _lib.OUT_FIELDS:
            vals.append(o[k].data_ptr() if (optional or k not in _lib.OPTIONAL_OUT) else None)
        return fin, sk, _lib.FimOut(*vals)

    def flash_fim(self, st: CellState, form: str = "plain", stream=None, diagnostics: bool = True,
                  fresh: bool = False):
        """Batched FlashFIM + PassFlashValue on device state (asynchronous on
        ``stream``, default: torch's current stream). With ``fresh`` every
        cell is flashed as a new bulk (lastNP = 0) instead of warm-starting
        from the previous outputs."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        fin, sk, fo = self._structs(st, optional=diagnostics, fresh=fresh)
        rc = lib().ocpf_flash_fim(self._h, st.ncell, C.byref(fin), C.byref(sk), C.byref(fo),
                                  FORMS[form], C.c_void_p(stream.cuda_stream))
        check(rc, "ocpf_flash_fim")

    def flash_impec(self, st: CellState, form: str = "plain", stream=None, diagnostics: bool = True,
                    fresh: bool = False):
        """Batched FlashIMPEC + IsoT_IMPEC::PassFlashValue (``ocpf_flash_impec``)
        on device state: warm start from ``phaseNum`` and ``xij`` (or, with
        ``fresh``, as new bulks); writes the IMPEC outputs into ``st.out``
        and the phase volumes into ``st.out['vj']``."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        o = st.out
        if "vj" not in o:
            o["vj"] = torch.zeros((NPH, st.ncell), dtype=torch.float64, device=st.P.device)
        fin_fim, sk, _ = self._structs(st, optional=diagnostics, fresh=fresh)
        fin = _lib.ImpecIn(st.P.data_ptr(), st.T.data_ptr(), st.Ni.data_ptr(), fin_fim.lastNP, fin_fim.xij)
        vals = []
        for k in _lib.IMPEC_OUT_FIELDS:
            vals.append(o[k].data_ptr() if (diagnostics or k not in _lib.OPTIONAL_OUT) else None)
        rc = lib().ocpf_flash_impec(self._h, st.ncell, C.byref(fin), C.byref(sk), C.byref(_lib.ImpecOut(*vals)),
                                    FORMS[form], C.c_void_p(stream.cuda_stream))
        check(rc, "ocpf_flash_impec")

    def flash_subset(self, st: CellState, idx, impec: bool = False, form: str = "plain", stream=None,
                     diagnostics: bool = True, check_indices: bool = False):
        """IsoT_AIMc's flashes of a subset of the bulks
        (``ocpf_flash_fim_subset``, or with ``impec``
        ``ocpf_flash_impec_subset``): only the cells listed in ``idx`` (a
        tensor of distinct cell indices) of the full state ``st`` are read
        and written, each as the full call would, warm-started from their own
        outputs. An index outside [0, ncell) is skipped; a repeated index
        makes two slots scatter to one cell in no fixed order.
        ``check_indices`` raises ValueError on either before the call (one
        device synchronisation)."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        # the index copy is ordered on the call's stream, and the allocator
        # keeps its memory until the work queued there has read it
        with torch.cuda.stream(stream):
            idx = torch.as_tensor(idx).to(device=st.P.device, dtype=torch.int64).contiguous()
        idx.record_stream(stream)
        if check_indices and idx.numel():
            lo, hi = int(idx.min().item()), int(idx.max().item())
            if lo < 0 or hi >= st.ncell:
                raise ValueError(f"flash_subset: index outside [0, {st.ncell})")
            if int(torch.unique(idx).numel()) != int(idx.numel()):
                raise ValueError("flash_subset: repeated index")
        st.__dict__["_subset_idx"] = idx  # alive until the next call on this state
        fin, sk, fo = self._structs(st, optional=diagnostics)
        s = C.c_void_p(stream.cuda_stream)
        if impec:
            o = st.out
            if "vj" not in o:
                o["vj"] = torch.zeros((NPH, st.ncell), dtype=torch.float64, device=st.P.device)
            fi = _lib.ImpecIn(st.P.data_ptr(), st.T.data_ptr(), st.Ni.data_ptr(), fin.lastNP, fin.xij)
            vals = [o[k].data_ptr() if (diagnostics or k not in _lib.OPTIONAL_OUT) else None
                    for k in _lib.IMPEC_OUT_FIELDS]
            rc = lib().ocpf_flash_impec_subset(self._h, int(idx.numel()), idx.data_ptr(), st.ncell, C.byref(fi),
                                               C.byref(sk), C.byref(_lib.ImpecOut(*vals)), FORMS[form], s)
            check(rc, "ocpf_flash_impec_subset")
        else:
            rc = lib().ocpf_flash_fim_subset(self._h, int(idx.numel()), idx.data_ptr(), st.ncell, C.byref(fin),
                                             C.byref(sk), C.byref(fo), FORMS[form], s)
            check(rc, "ocpf_flash_fim_subset")

    def _fimn_outputs(self, st: CellState):
        torch = _torch()
        o, dev = st.out, st.P.device
        if "res" not in o:
            o["res"] = torch.zeros((NPH * (self.nc + 2), st.ncell), dtype=torch.float64, device=dev)
            o["resPc"] = torch.zeros(st.ncell, dtype=torch.float64, device=dev)
        return o["res"].data_ptr(), o["resPc"].data_ptr()

    def flash_fimn(self, st: CellState, form: str = "plain", stream=None, diagnostics: bool = True,
                   fresh: bool = False):
        """Batched FlashFIMn + IsoT_FIMn::PassFlashValue (``ocpf_flash_fimn``)
        on device state, warm-started like ``flash_fim``: ``st.out`` receives
        the FIMn outputs (dSec_dPri with the saturation and phase-mole rows,
        the per-n_ij partials, nj) and ``st.out['res']`` / ``st.out['resPc']``
        the residual terms (Bulk::res_n, Bulk::resPc)."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        fin, sk, fo = self._structs(st, optional=diagnostics, fresh=fresh)
        fo.nj = st.out["nj"].data_ptr()
        res, resPc = self._fimn_outputs(st)
        rc = lib().ocpf_flash_fimn(self._h, st.ncell, C.byref(fin), C.byref(sk), C.byref(fo), res, resPc,
                                   FORMS[form], C.c_void_p(stream.cuda_stream))
        check(rc, "ocpf_flash_fimn")

    def init_flash(self, st: CellState, Vpore, S=None, impec: bool = False, form: str = "plain", stream=None,
                   diagnostics: bool = True, fimn: bool = False):
        """IsoT_FIM::InitFlash (``ocpf_init_flash_fim``) or, with ``impec``,
        IsoT_IMPEC::InitFlash (``ocpf_init_flash_impec``) on device state.
        On entry ``st.Ni`` holds the initial mole fractions z and
        ``st.out['S']`` (or ``S`` [n, 3], copied in first) the initial
        saturations, of which S_w is read; ``Vpore`` [n] are the pore volumes
        in ft3. On return ``st.Ni`` holds the moles that fill the pore
        volume and ``st.out`` the FIM (or IMPEC, with ``vj``) outputs, as the
        reference leaves Bulk::Ni and the Bulk arrays. With ``fimn``,
        IsoT_FIMn::InitFlash (``ocpf_init_flash_fimn``) with the outputs of
        ``flash_fimn``."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        o = st.out
        dev = st.P.device
        if S is not None:
            o["S"].copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(S, dtype=np.float64).T)))
        vp = torch.as_tensor(Vpore, dtype=torch.float64).to(dev).reshape(st.ncell).contiguous()
        st.__dict__["_vpore"] = vp  # alive until the next call on this state
        sk = _lib.Skip(*[st.skip[k].data_ptr() for k in _lib.SKIP_FIELDS])
        fin = _lib.InitIn(st.P.data_ptr(), st.T.data_ptr(), o["S"].data_ptr(), vp.data_ptr(), st.Ni.data_ptr())
        h, s = self._h, C.c_void_p(stream.cuda_stream)
        if impec:
            if "vj" not in o:
                o["vj"] = torch.zeros((NPH, st.ncell), dtype=torch.float64, device=dev)
            vals = [o[k].data_ptr() if (diagnostics or k not in _lib.OPTIONAL_OUT) else None
                    for k in _lib.IMPEC_OUT_FIELDS]
            rc = lib().ocpf_init_flash_impec(h, st.ncell, C.byref(fin), C.byref(sk), st.Ni.data_ptr(),
                                             C.byref(_lib.ImpecOut(*vals)), FORMS[form], s)
            check(rc, "ocpf_init_flash_impec")
        elif fimn:
            vals = [o[k].data_ptr() if (diagnostics or k not in _lib.OPTIONAL_OUT or k == "nj") else None
                    for k in _lib.OUT_FIELDS]
            res, resPc = self._fimn_outputs(st)
            rc = lib().ocpf_init_flash_fimn(h, st.ncell, C.byref(fin), C.byref(sk), st.Ni.data_ptr(),
                                            C.byref(_lib.FimOut(*vals)), res, resPc, FORMS[form], s)
            check(rc, "ocpf_init_flash_fimn")
        else:
            vals = [o[k].data_ptr() if (diagnostics or k not in _lib.OPTIONAL_OUT) else None
                    for k in _lib.OUT_FIELDS]
            rc = lib().ocpf_init_flash_fim(h, st.ncell, C.byref(fin), C.byref(sk), st.Ni.data_ptr(),
                                           C.byref(_lib.FimOut(*vals)), FORMS[form], s)
            check(rc, "ocpf_init_flash_fim")

    def reserve(self, ncell: int):
        """Pre-allocates the batched forms' device scratch for ncell cells."""
        check(lib().ocpf_reserve(self._h, int(ncell)), "ocpf_reserve")

    def last_launch_count(self) -> int:
        """Kernels the last flash call launched (-1: unknown)."""
        k = C.c_int(0)
        check(lib().ocpf_last_launch_count(self._h, C.byref(k)), "ocpf_last_launch_count")
        return int(k.value)

    def set_part_timing(self, on: bool = True):
        """Records the batched sequence's part marks on later flash_fim calls
        (direct launches instead of graph replay; ocpf_set_part_timing)."""
        check(lib().ocpf_set_part_timing(self._h, 1 if on else 0), "ocpf_set_part_timing")

    def last_phase_ms(self) -> tuple:
        """(up to the restart path, restart path, finalize) device ms of the
        last batched-form flash_fim with part timing on (ocpf_last_phase_ms)."""
        ms = (C.c_float * 3)()
        check(lib().ocpf_last_phase_ms(self._h, ms), "ocpf_last_phase_ms")
        return tuple(float(v) for v in ms)

    def last_kernel_ms(self) -> float:
        ms = C.c_float(0)
        check(lib().ocpf_last_kernel_ms(self._h, C.byref(ms)), "ocpf_last_kernel_ms")
        return float(ms.value)

    # ------------------------------------------------------ last time step
    def new_last(self, st: CellState) -> CellState:
        """Device arrays for the last-time-step copy of ``st`` (Bulk's ``l*``
        arrays and SkipStaAnaly's ``l*`` cache), same shapes."""
        return self.new_state(st.ncell)

    def _step_copy(self, fn: str, st: CellState, last: CellState, inputs: bool, stream):
        torch = _torch()
        if last.ncell != st.ncell or last.nc != st.nc:
            raise ValueError("last-step state of another shape")
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        s = C.c_void_p(stream.cuda_stream)
        _, sk, out = self._structs(st)
        _, lsk, lout = self._structs(last)
        check(getattr(lib(), fn)(self.nc, st.ncell, C.byref(out), C.byref(sk), C.byref(lout), C.byref(lsk), s), fn)
        if inputs:
            pairs = [(last.P, st.P), (last.Ni, st.Ni)]
            copy_arrays(pairs if fn == "ocpf_update_last_step" else [(b, a) for a, b in pairs], stream)

    def update_last_step(self, st: CellState, last: CellState, inputs: bool = True, stream=None):
        """IsoT_FIM::UpdateLastTimeStep for the flash's arrays
        (``src/OCPFluidMethod.cpp:2915-2960``) and the skip cache
        (``src/AcceleratePVT.cpp:131-138``): ``last`` <- ``st``; with
        ``inputs`` also P and Ni (``lP``, ``lNi``). Asynchronous."""
        self._step_copy("ocpf_update_last_step", st, last, inputs, stream)

    def reset_to_last_step(self, st: CellState, last: CellState, inputs: bool = True, stream=None):
        """IsoT_FIM::ResetToLastTimeStep (``src/OCPFluidMethod.cpp:2859-2897``)
        and SkipStaAnaly::ResetToLastTimeStep (``src/AcceleratePVT.cpp:122-129``):
        ``st`` <- ``last``. Asynchronous."""
        self._step_copy("ocpf_reset_to_last_step", st, last, inputs, stream)

    # ------------------------------------------------------------- host path
    def new_host_state(self, ncell: int, pinned: bool = True) -> dict:
        """Host SoA buffers for :meth:`flash_fim_host` (pinned if requested)."""
        torch = _torch()

        def mk(nf, dt):
            shape = (nf, ncell) if nf > 1 else (ncell,)
            t = torch.zeros(shape, dtype=getattr(torch, _TORCH_DT[dt]), pin_memory=pinned)
            return t
        hs = {"P": mk(1, "f64"), "T": mk(1, "f64"), "Ni": mk(self.nc + 1, "f64"), "out": {}, "skip": {}}
        for k, (nf, dt) in _lib.out_shapes(self.nc).items():
            hs["out"][k] = mk(nf, dt)
        for k, (nf, dt) in _lib.skip_shapes(self.nc).items():
            hs["skip"][k] = mk(nf, dt)
        return hs

    def flash_fim_host(self, hs: dict, form: str = "plain", diagnostics: bool = True):
        """Same flash with every array in host memory (``new_host_state``);
        the library streams the cells through its device staging buffers and
        returns when the results are back on the host."""
        o = hs["out"]
        ncell = hs["P"].shape[0]
        fin = _lib.FimIn(hs["P"].data_ptr(), hs["T"].data_ptr(), hs["Ni"].data_ptr(),
                         o["S"].data_ptr(), o["phaseNum"].data_ptr(), o["xij"].data_ptr())
        sk = _lib.Skip(*[hs["skip"][k].data_ptr() for k in _lib.SKIP_FIELDS])
        fo = _lib.FimOut(*[(o[k].data_ptr() if (diagnostics or k not in _lib.OPTIONAL_OUT) else None)
                           for k in _lib.OUT_FIELDS])
        rc = lib().ocpf_flash_fim_host(self._h, ncell, C.byref(fin), C.byref(sk), C.byref(fo),
                                       FORMS[form])
        check(rc, "ocpf_flash_fim_host")


def _region_structs(regions, fresh, diagnostics):
    n = len(regions)
    ctx = (C.c_void_p * n)(*[m._h.value for m, _ in regions])
    cnt = (C.c_int64 * n)(*[st.ncell for _, st in regions])
    ins, sks, outs = (_lib.FimIn * n)(), (_lib.Skip * n)(), (_lib.FimOut * n)()
    for r, (m, st) in enumerate(regions):
        ins[r], sks[r], outs[r] = m._structs(st, optional=diagnostics, fresh=fresh)
    return ctx, cnt, ins, sks, outs


def flash_fim_regions(regions, form: str = "batched", stream=None, fresh: bool = False, diagnostics: bool = True):
    """Flashes several PVT regions in one call (``ocpf_flash_fim_regions``):
    ``regions`` is a list of (MixtureCompBatch, CellState) pairs, one per
    region, on one device; fluids may have different component counts. The
    batched forms run as one launch sequence over all regions, or as one
    sequence per region on the contexts' streams, as the first region's
    tuning says (``set_tuning`` / ``autotune``); the call is ordered on
    ``stream`` (default: torch's current stream)."""
    torch = _torch()
    n = len(regions)
    if n == 0:
        return
    dev = regions[0][0].device
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    ctx, cnt, ins, sks, outs = _region_structs(regions, fresh, diagnostics)
    rc = lib().ocpf_flash_fim_regions(n, ctx, cnt, ins, sks, outs, FORMS[form], C.c_void_p(stream.cuda_stream))
    check(rc, "ocpf_flash_fim_regions")


def copy_arrays(pairs, stream=None):
    """``ocpf_copy_arrays``: copies each (dst, src) pair of device tensors
    (same number of bytes) in one kernel launch, asynchronously."""
    torch = _torch()
    pairs = list(pairs)
    if not pairs:
        return
    if len(pairs) > _lib.COPY_MAX:
        raise ValueError(f"at most {_lib.COPY_MAX} pairs per launch")
    for d, s in pairs:
        if d.numel() * d.element_size() != s.numel() * s.element_size():
            raise ValueError("pair of different sizes")
        if not (d.is_contiguous() and s.is_contiguous()):
            raise ValueError("contiguous tensors only")
    if stream is None:
        stream = torch.cuda.current_stream(pairs[0][0].device)
    n = len(pairs)
    dst = (C.c_void_p * n)(*[d.data_ptr() for d, _ in pairs])
    src = (C.c_void_p * n)(*[s.data_ptr() for _, s in pairs])
    nb = (C.c_int64 * n)(*[s.numel() * s.element_size() for _, s in pairs])
    check(lib().ocpf_copy_arrays(n, dst, src, nb, C.c_void_p(stream.cuda_stream)), "ocpf_copy_arrays")


def autotune(regions, form: str = "fast", reps: int = 2, stream=None, fresh: bool = True) -> dict:
    """``ocpf_autotune`` over (MixtureCompBatch, CellState) pairs (one pair:
    that context's own launch shape): times every candidate launch shape on
    the states' inputs without changing them, keeps the fastest in every
    context and returns it."""
    torch = _torch()
    n = len(regions)
    dev = regions[0][0].device
    if stream is None:
        stream = torch.cuda.current_stream(dev)
    ctx, cnt, ins, sks, _ = _region_structs(regions, fresh, True)
    best = _lib.Tuning()
    rc = lib().ocpf_autotune(n, ctx, cnt, ins, sks, FORMS[form], int(reps), C.c_void_p(stream.cuda_stream),
                             C.byref(best))
    check(rc, "ocpf_autotune")
    return {k: getattr(best, k) for k in ("block", "persist_pct", "slow_threads", "schedule", "ms")}
