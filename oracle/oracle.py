"""TEST INFRASTRUCTURE ONLY: ctypes loader for the two CPU oracles.

``load("reference")`` opens ``oracle/_ref/libocpref.so`` -- the reference's own
``MixtureComp`` compiled from its sources by ``oracle/Makefile``.
``load("port")`` opens ``oracle/libflashport.so`` -- the plain-C restatement in
``oracle/flash_port.c`` (built on demand with gcc).

Both take and return arrays in the reference Bulk layout (cell-major), see
``oracle/oracle_api.h``. Only tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libocpref.so")
PORT_LIB = os.path.join(HERE, "libflashport.so")
MAX_NC = 16
NP = 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class OrcFluid(C.Structure):
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


_BATCH_FIELDS = [
    ("n", C.c_int64),
    ("P", _dp), ("T", _dp), ("Ni", _dp), ("S_in", _dp), ("lastNP", _ip), ("xij_in", _dp),
    ("skip_flag", _ip), ("skip_minEig", _dp), ("skip_P", _dp), ("skip_T", _dp), ("skip_z", _dp),
    ("phaseNum", _ip), ("phaseExist", _ip), ("S", _dp), ("Nt", _dp), ("vf", _dp),
    ("vfP", _dp), ("vfi", _dp), ("nj", _dp), ("rho", _dp), ("xi", _dp), ("mu", _dp),
    ("rhoP", _dp), ("xiP", _dp), ("muP", _dp), ("xij", _dp), ("rhox", _dp), ("xix", _dp),
    ("mux", _dp), ("dSec_dPri", _dp), ("bRowSizedSdP", _ip), ("pSderExist", _ip),
    ("pVnumCom", _ip), ("ePEC", _dp), ("ftype", _ip), ("NPhc", _ip), ("iters", _ip), ("restarts", _ip),
]


class OrcBatch(C.Structure):
    _fields_ = _BATCH_FIELDS


def make_orc_fluid(fl) -> OrcFluid:
    f = OrcFluid()
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


def build_port(force: bool = False) -> str:
    src = os.path.join(HERE, "flash_port.c")
    if force or not os.path.exists(PORT_LIB) or os.path.getmtime(PORT_LIB) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "oracle_api.h"))):
        subprocess.check_call(["make", "-s", "-C", HERE, "port"])
    return PORT_LIB


_LIBS = {}


def available(kind: str) -> bool:
    if kind == "port":
        return True
    return os.path.exists(REF_LIB)


def load(kind: str = "reference"):
    if kind in _LIBS:
        return _LIBS[kind]
    if kind == "reference":
        path = REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    elif kind == "port":
        path = build_port()
    else:
        raise ValueError(kind)
    lib = C.CDLL(path)
    lib.orc_flash_fim_batch.argtypes = [C.POINTER(OrcFluid), C.POINTER(OrcBatch), C.c_int,
                                        C.POINTER(C.c_double)]
    lib.orc_flash_fim_batch.restype = C.c_int
    lib.orc_kind.restype = C.c_char_p
    _LIBS[kind] = lib
    return lib


def flash_impec(fluid, P, T, Ni, lastNP=None, xij=None, skip=None, nthreads: int = 0):
    """Runs one FlashIMPEC per cell through the compiled reference
    (orc_flash_impec_batch; the restatement has no IMPEC entry). Arguments
    as flash_fim without S; returns the IMPEC outputs (Bulk layout, absent
    phases NaN) plus ``vj`` [n, 3]."""
    lib = load("reference")
    if not fluid.controls.use_skip:
        fluid = fluid.with_controls(use_skip=True)  # see flash_fim
        skip = None
    n = int(np.asarray(P).shape[0])
    vj = np.full((n, NP), np.nan)
    b, f, arrays, skip, _keep = _prepare(fluid, P, T, Ni, None, lastNP, xij, skip)
    secs = C.c_double(0.0)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    lib.orc_flash_impec_batch.argtypes = [C.POINTER(OrcFluid), C.POINTER(OrcBatch), _dp, C.c_int,
                                          C.POINTER(C.c_double)]
    lib.orc_flash_impec_batch.restype = C.c_int
    rc = lib.orc_flash_impec_batch(C.byref(f), C.byref(b), vj.ctypes.data_as(_dp), int(nthreads), C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"orc_flash_impec_batch failed with {rc}")
    arrays["vj"] = vj
    arrays["seconds"] = secs.value
    arrays["skip"] = skip
    return arrays


def init_flash(fluid, P, T, z, S, Vpore, impec: bool = False, skip=None, nthreads: int = 0):
    """Runs one InitFlashFIM (or, with ``impec``, InitFlashIMPEC) per cell
    through the compiled reference (orc_init_flash_batch; the restatement
    has no initialisation entry). z [n, numCom] are the initial mole
    fractions (water entry ignored), S [n, 3] the initial saturations (S_w
    read), Vpore [n] the pore volumes in ft3. Returns the FIM outputs (or
    the IMPEC ones plus ``vj``) and ``Ni`` [n, numCom], the moles the flash
    object holds afterwards."""
    lib = load("reference")
    if not fluid.controls.use_skip:
        fluid = fluid.with_controls(use_skip=True)  # see flash_fim
        skip = None
    n = int(np.asarray(P).shape[0])
    ncom = fluid.nc + 1
    vj = np.full((n, NP), np.nan)
    Niout = np.full((n, ncom), np.nan)
    Vp = np.ascontiguousarray(Vpore, dtype=np.float64).reshape(n)
    b, f, arrays, skip, _keep = _prepare(fluid, P, T, z, S, None, None, skip)
    secs = C.c_double(0.0)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    lib.orc_init_flash_batch.argtypes = [C.POINTER(OrcFluid), C.POINTER(OrcBatch), _dp, C.c_int, _dp, _dp,
                                         C.c_int, C.POINTER(C.c_double)]
    lib.orc_init_flash_batch.restype = C.c_int
    rc = lib.orc_init_flash_batch(C.byref(f), C.byref(b), Vp.ctypes.data_as(_dp), 1 if impec else 0,
                                  Niout.ctypes.data_as(_dp), vj.ctypes.data_as(_dp), int(nthreads),
                                  C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"orc_init_flash_batch failed with {rc}")
    if impec:
        arrays["vj"] = vj
    arrays["Ni"] = Niout
    arrays["seconds"] = secs.value
    arrays["skip"] = skip
    return arrays


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def new_skip(n: int, nc: int) -> dict:
    """An empty SkipStaAnaly cache (flag 0 everywhere)."""
    return {"flag": np.zeros(n, np.int32), "minEig": np.zeros(n), "P": np.zeros(n),
            "T": np.zeros(n), "z": np.zeros((n, nc))}


def _prepare(fluid, P, T, Ni, S, lastNP, xij, skip):
    """Batch struct, fluid struct, output arrays (NaN / -1 filled), skip cache
    and the input arrays the struct points into (kept alive by the caller)."""
    nc = fluid.nc
    ncom = nc + 1
    n = int(np.asarray(P).shape[0])
    P = np.ascontiguousarray(P, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    Ni = np.ascontiguousarray(np.asarray(Ni, dtype=np.float64).reshape(n, ncom))
    S = np.zeros((n, NP)) if S is None else np.ascontiguousarray(S, dtype=np.float64)
    lastNP = np.zeros(n, np.int32) if lastNP is None else np.ascontiguousarray(lastNP, np.int32)
    xij = np.zeros((n, NP, ncom)) if xij is None else np.ascontiguousarray(xij, dtype=np.float64)
    if skip is None:
        skip = new_skip(n, nc)
    for k in ("minEig", "P", "T", "z"):
        skip[k] = np.ascontiguousarray(skip[k], dtype=np.float64)
    skip["flag"] = np.ascontiguousarray(skip["flag"], dtype=np.int32)
    ncol = ncom + 1
    nan = lambda *s: np.full(s, np.nan)
    out = {
        "phaseNum": np.full(n, -1, np.int32), "phaseExist": np.full((n, NP), -1, np.int32),
        "S": nan(n, NP), "Nt": nan(n), "vf": nan(n), "vfP": nan(n), "vfi": nan(n, ncom),
        "nj": nan(n, NP), "rho": nan(n, NP), "xi": nan(n, NP), "mu": nan(n, NP),
        "rhoP": nan(n, NP), "xiP": nan(n, NP), "muP": nan(n, NP),
        "xij": nan(n, NP, ncom), "rhox": nan(n, NP, ncom), "xix": nan(n, NP, ncom),
        "mux": nan(n, NP, ncom), "dSec_dPri": nan(n, ncol * ncol * NP),
        "bRowSizedSdP": np.full(n, -1, np.int32), "pSderExist": np.full((n, NP), -1, np.int32),
        "pVnumCom": np.full((n, NP), -1, np.int32), "ePEC": nan(n),
        "ftype": np.full(n, -1, np.int32), "NPhc": np.full(n, -1, np.int32),
        "iters": np.full((n, 5), -1, np.int32), "restarts": np.full(n, -1, np.int32),
    }
    b = OrcBatch()
    b.n = n
    b.P, b.T, b.Ni, b.S_in = _ptr(P, C.c_double), _ptr(T, C.c_double), _ptr(Ni, C.c_double), _ptr(S, C.c_double)
    b.lastNP, b.xij_in = _ptr(lastNP, C.c_int32), _ptr(xij, C.c_double)
    b.skip_flag = _ptr(skip["flag"], C.c_int32)
    for k in ("minEig", "P", "T", "z"):
        setattr(b, "skip_" + k, _ptr(skip[k], C.c_double))
    for name, ct in _BATCH_FIELDS[12:]:
        arr = out[name]
        setattr(b, name, arr.ctypes.data_as(ct))
    return b, make_orc_fluid(fluid), out, skip, (P, T, Ni, S, lastNP, xij)


def flash_fim(kind: str, fluid, P, T, Ni, S=None, lastNP=None, xij=None, skip=None,
              nthreads: int = 0):
    """Runs one FlashFIM per cell through the chosen oracle.

    P [n] psia, T [n] degF, Ni [n, numCom]; S [n,3], lastNP [n] and
    xij [n,3,numCom] are the warm-start inputs (default: fresh cells,
    lastNP = 0). ``skip`` (dict of arrays, updated in place) is the
    SkipStaAnaly cache. Returns a dict of outputs in Bulk layout; entries of
    absent phases are NaN. ``out["seconds"]`` is the flash-loop wall time.
    """
    lib = load(kind)
    if kind == "reference" and not fluid.controls.use_skip:
        # The reference's FlashFIM sets SkipStaAnaly::flag[bulkId] after every
        # flash (CalSkipForNextStep, src/MixtureComp.cpp:5253 ->
        # include/AcceleratePVT.hpp:36) even when the skip option is off and
        # the array was never allocated (src/MixtureComp.cpp:5130-5131): a
        # write through an empty vector that crashes. Run it with the option
        # on and a fresh cache (flag 0: no cell skips, every cell takes the
        # full path), which gives the same flash; the cache it fills is
        # discarded.
        fluid = fluid.with_controls(use_skip=True)
        skip = None
    b, f, out, skip, _keep = _prepare(fluid, P, T, Ni, S, lastNP, xij, skip)
    secs = C.c_double(0.0)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    rc = lib.orc_flash_fim_batch(C.byref(f), C.byref(b), int(nthreads), C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"orc_flash_fim_batch failed with {rc}")
    out["seconds"] = secs.value
    out["skip"] = skip
    return out


def flash_fimn(fluid, P, T, Ni, S=None, lastNP=None, xij=None, skip=None, nthreads: int = 0):
    """Runs one FlashFIMn per cell through the compiled reference
    (orc_flash_fimn_batch; the restatement has no FIMn entry). Arguments as
    flash_fim; returns its outputs (FlashFIMn's dSec_dPri rows and per-n_ij
    partials) plus ``res`` [n, 3 (numCom + 1)] (the first bRowSizedSdP
    entries of each cell set, NaN beyond) and ``resPc`` [n]."""
    lib = load("reference")
    if not fluid.controls.use_skip:
        fluid = fluid.with_controls(use_skip=True)  # see flash_fim
        skip = None
    n = int(np.asarray(P).shape[0])
    res = np.full((n, NP * (fluid.nc + 2)), np.nan)
    resPc = np.full(n, np.nan)
    b, f, arrays, skip, _keep = _prepare(fluid, P, T, Ni, S, lastNP, xij, skip)
    secs = C.c_double(0.0)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    lib.orc_flash_fimn_batch.argtypes = [C.POINTER(OrcFluid), C.POINTER(OrcBatch), _dp, _dp, C.c_int,
                                         C.POINTER(C.c_double)]
    lib.orc_flash_fimn_batch.restype = C.c_int
    rc = lib.orc_flash_fimn_batch(C.byref(f), C.byref(b), res.ctypes.data_as(_dp), resPc.ctypes.data_as(_dp),
                                  int(nthreads), C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"orc_flash_fimn_batch failed with {rc}")
    arrays.update(res=res, resPc=resPc, seconds=secs.value, skip=skip)
    return arrays


def init_flash_fimn(fluid, P, T, z, S, Vpore, skip=None, nthreads: int = 0):
    """Runs one InitFlashFIMn per cell through the compiled reference
    (orc_init_flash_fimn_batch): inputs as init_flash, outputs as
    flash_fimn plus ``Ni``."""
    lib = load("reference")
    if not fluid.controls.use_skip:
        fluid = fluid.with_controls(use_skip=True)  # see flash_fim
        skip = None
    n = int(np.asarray(P).shape[0])
    ncom = fluid.nc + 1
    res = np.full((n, NP * (fluid.nc + 2)), np.nan)
    resPc = np.full(n, np.nan)
    Niout = np.full((n, ncom), np.nan)
    Vp = np.ascontiguousarray(Vpore, dtype=np.float64).reshape(n)
    b, f, arrays, skip, _keep = _prepare(fluid, P, T, z, S, None, None, skip)
    secs = C.c_double(0.0)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    lib.orc_init_flash_fimn_batch.argtypes = [C.POINTER(OrcFluid), C.POINTER(OrcBatch), _dp, _dp, _dp, _dp,
                                              C.c_int, C.POINTER(C.c_double)]
    lib.orc_init_flash_fimn_batch.restype = C.c_int
    rc = lib.orc_init_flash_fimn_batch(C.byref(f), C.byref(b), Vp.ctypes.data_as(_dp), Niout.ctypes.data_as(_dp),
                                       res.ctypes.data_as(_dp), resPc.ctypes.data_as(_dp), int(nthreads),
                                       C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"orc_init_flash_fimn_batch failed with {rc}")
    arrays.update(res=res, resPc=resPc, Ni=Niout, seconds=secs.value, skip=skip)
    return arrays
