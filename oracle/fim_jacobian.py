"""TEST INFRASTRUCTURE ONLY: the bulk part of the FIM Jacobian, as
IsoT_FIM::AssembleMatBulksNew builds it (src/OCPFluidMethod.cpp:1569-1840)
from the Bulk arrays the flash and CalKrPc leave: for every bulk the
accumulation block, and for every connection the flux derivatives of both
ends, dF/dXp + dF/dXs dSec_dPri (DaABpbC, src/DenseMat.cpp:75-94), scaled by
dt and scattered as the reference scatters them into the linear system
(diagonal blocks added in connection order, off-diagonal blocks inserted).

The reference's assembly cannot be compiled here (its LinearSystem includes
the FASP solver's headers, which are not present), so this restatement is
unpinned except for its dense product, which ``product_reference`` checks
against the reference's own DaABpbC (compiled into oracle/_ref). Every other
operation follows the reference's expressions in their left-to-right order
without fused multiply-adds, as the device kernel forms them.

Layout: cell-major (Bulk layout). numCom = nc + 1 (water last), numPhase 3,
ncol = numCom + 1; a block is ncol x ncol row-major. dSec_dPri of bulk n:
bRowSizedSdP[n] rows of ncol, row-major, in [n, 3 * ncol * ncol].
"""
from __future__ import annotations

import os

import numpy as np

CONV1 = 5.61458
CONV2 = 1.12712e-3
GRAVITY_FACTOR = 0.00694444
NP = 3


def upwind(bk, cn):
    """Upstream bulk and mean density of every connection and phase
    (BulkConn::CalUpwindFIM-style selection, src/BulkConn.cpp:170-215): the
    saturation-weighted density where both ends hold the phase, the existing
    end's otherwise; the begin bulk when the potential difference is >= 0.
    Returns (upblock [nconn, 3] int64, upblock_Rho [nconn, 3])."""
    nconn = len(cn["bId"])
    up = np.zeros((nconn, NP), np.int64)
    rho_u = np.zeros((nconn, NP))
    for c in range(nconn):
        b, e = int(cn["bId"][c]), int(cn["eId"][c])
        for j in range(NP):
            xb, xe = bool(bk["phaseExist"][b, j]), bool(bk["phaseExist"][e, j])
            if xb and xe:
                rho = (bk["rho"][b, j] * bk["S"][b, j] + bk["rho"][e, j] * bk["S"][e, j]) / \
                      (bk["S"][b, j] + bk["S"][e, j])
            elif xb:
                rho = bk["rho"][b, j]
            elif xe:
                rho = bk["rho"][e, j]
            else:
                up[c, j] = b
                rho_u[c, j] = 0.0
                continue
            dP = (bk["Pj"][b, j] - GRAVITY_FACTOR * rho * bk["depth"][b]) - \
                 (bk["Pj"][e, j] - GRAVITY_FACTOR * rho * bk["depth"][e])
            up[c, j] = e if dP < 0 else b
            rho_u[c, j] = rho
    return up, rho_u


def accumulation(bk, n, ncom):
    """The accumulation block of bulk n (src/OCPFluidMethod.cpp:1587-1596)."""
    ncol = ncom + 1
    b = np.zeros((ncol, ncol))
    for i in range(1, ncol):
        b[i, i] = 1.0
    b[0, 0] = bk["v"][n] * bk["poroP"][n] - bk["vfP"][n]
    for i in range(ncom):
        b[0, i + 1] = -bk["vfi"][n, i]
    return b


def conn_blocks(bk, cn, c, ncom, dt):
    """(bmatB, bmatE) of connection c before the scatter: dt (dFdXp +
    dFdXs dSec_dPri) of its begin and end bulks (src/OCPFluidMethod.cpp:
    1620-1822)."""
    ncol = ncom + 1
    bId, eId = int(cn["bId"][c]), int(cn["eId"][c])
    Akd = CONV1 * CONV2 * cn["area"][c]
    dFdXpB = np.zeros((ncol, ncol))
    dFdXpE = np.zeros((ncol, ncol))
    exB = bk["phaseExist"][bId].astype(bool)
    exE = bk["phaseExist"][eId].astype(bool)
    sB = bk["pSderExist"][bId].astype(bool)
    sE = bk["pSderExist"][eId].astype(bool)
    vB = bk["pVnumCom"][bId].astype(int)
    vE = bk["pVnumCom"][eId].astype(int)
    ncolB = int(vB.sum() + sB.sum())
    ncolE = int(vE.sum() + sE.sum())
    dFdXsB = np.zeros((ncol, max(ncolB, 1)))
    dFdXsE = np.zeros((ncol, max(ncolE, 1)))
    dGamma = GRAVITY_FACTOR * (bk["depth"][bId] - bk["depth"][eId])
    jxB, jxE = int(sB.sum()), int(sE.sum())
    for j in range(NP):
        uId = int(cn["upblock"][c, j])
        exU = exB[j] if uId == bId else exE[j]
        if not exU:
            jxB += vB[j]
            jxE += vE[j]
            continue
        dP = bk["Pj"][bId, j] - bk["Pj"][eId, j] - cn["upblock_Rho"][c, j] * dGamma
        xi, kr, mu = bk["xi"][uId, j], bk["kr"][uId, j], bk["mu"][uId, j]
        muP, xiP, rhoP = bk["muP"][uId, j], bk["xiP"][uId, j], bk["rhoP"][uId, j]
        transJ = Akd * kr / mu
        for i in range(ncom):
            xij = bk["xij"][uId, j, i]
            transIJ = xij * xi * transJ
            dFdXpB[i + 1, 0] += transIJ
            dFdXpE[i + 1, 0] -= transIJ
            tmp = xij * transJ * xiP * dP
            tmp += -transIJ * muP / mu * dP
            if not exE[j]:
                tmp += transIJ * (-rhoP * dGamma)
                dFdXpB[i + 1, 0] += tmp
            elif not exB[j]:
                tmp += transIJ * (-rhoP * dGamma)
                dFdXpE[i + 1, 0] += tmp
            else:
                dFdXpB[i + 1, 0] += transIJ * (-bk["rhoP"][bId, j] * dGamma) / 2
                dFdXpE[i + 1, 0] += transIJ * (-bk["rhoP"][eId, j] * dGamma) / 2
                if bId == uId:
                    dFdXpB[i + 1, 0] += tmp
                else:
                    dFdXpE[i + 1, 0] += tmp
            j1SB = j1SE = 0
            if bId == uId:
                for j1 in range(NP):
                    if sB[j1]:
                        dFdXsB[i + 1, j1SB] += transIJ * bk["dPcj_dS"][bId, j, j1]
                        tmp = Akd * xij * xi / mu * bk["dKr_dS"][uId, j, j1] * dP
                        dFdXsB[i + 1, j1SB] += tmp
                        j1SB += 1
                    if sE[j1]:
                        dFdXsE[i + 1, j1SE] -= transIJ * bk["dPcj_dS"][eId, j, j1]
                        j1SE += 1
                if not exE[j]:
                    for k in range(vB[j]):
                        rhox = bk["rhox"][uId, j, k]
                        xix = bk["xix"][uId, j, k]
                        mux = bk["mux"][uId, j, k]
                        tmp = -transIJ * rhox * dGamma
                        tmp += xij * transJ * xix * dP
                        tmp += -transIJ * mux / mu * dP
                        dFdXsB[i + 1, jxB + k] += tmp
                    if i < vB[j]:
                        dFdXsB[i + 1, jxB + i] += xi * transJ * dP
                else:
                    for k in range(vB[j]):
                        rhox = bk["rhox"][bId, j, k] / 2
                        xix = bk["xix"][uId, j, k]
                        mux = bk["mux"][uId, j, k]
                        tmp = -transIJ * rhox * dGamma
                        tmp += xij * transJ * xix * dP
                        tmp += -transIJ * mux / mu * dP
                        dFdXsB[i + 1, jxB + k] += tmp
                        dFdXsE[i + 1, jxE + k] += -transIJ * bk["rhox"][eId, j, k] / 2 * dGamma
                    if i < vB[j]:
                        dFdXsB[i + 1, jxB + i] += xi * transJ * dP
            else:
                for j1 in range(NP):
                    if sB[j1]:
                        dFdXsB[i + 1, j1SB] += transIJ * bk["dPcj_dS"][bId, j, j1]
                        j1SB += 1
                    if sE[j1]:
                        dFdXsE[i + 1, j1SE] -= transIJ * bk["dPcj_dS"][eId, j, j1]
                        tmp = Akd * xij * xi / mu * bk["dKr_dS"][uId, j, j1] * dP
                        dFdXsE[i + 1, j1SE] += tmp
                        j1SE += 1
                if not exB[j]:
                    for k in range(vE[j]):
                        rhox = bk["rhox"][uId, j, k]
                        xix = bk["xix"][uId, j, k]
                        mux = bk["mux"][uId, j, k]
                        tmp = -transIJ * rhox * dGamma
                        tmp += xij * transJ * xix * dP
                        tmp += -transIJ * mux / mu * dP
                        dFdXsE[i + 1, jxE + k] += tmp
                    if i < vE[j]:
                        dFdXsE[i + 1, jxE + i] += xi * transJ * dP
                else:
                    for k in range(vE[j]):
                        rhox = bk["rhox"][eId, j, k] / 2
                        xix = bk["xix"][uId, j, k]
                        mux = bk["mux"][uId, j, k]
                        tmp = -transIJ * rhox * dGamma
                        tmp += xij * transJ * xix * dP
                        tmp += -transIJ * mux / mu * dP
                        dFdXsE[i + 1, jxE + k] += tmp
                        dFdXsB[i + 1, jxB + k] += -transIJ * bk["rhox"][bId, j, k] / 2 * dGamma
                    if i < vE[j]:
                        dFdXsE[i + 1, jxE + i] += xi * transJ * dP
        jxB += vB[j]
        jxE += vE[j]
    secB = bk["dSec_dPri"][bId][: ncolB * ncol].reshape(ncolB, ncol)
    secE = bk["dSec_dPri"][eId][: ncolE * ncol].reshape(ncolE, ncol)
    return product(dFdXpB, dFdXsB, secB, dt), product(dFdXpE, dFdXsE, secE, dt)


def product(C, A, B, dt):
    """dt (A B + C) as DaABpbC(..., 1, A, B, 1, C) then Dscalar(dt) form it,
    with the sum over k taken in order and no fused multiply-add (the
    kernel's order; the reference's BLAS may round differently)."""
    s = np.zeros_like(C)
    for k in range(B.shape[0]):
        s = s + np.outer(A[:, k], B[k, :])
    return (s + C) * dt


def product_reference(A, B, C):
    """The reference's own DaABpbC (src/DenseMat.cpp:75-94) on row-major
    A (m x k), B (k x n), C (m x n): returns A B + C."""
    import ctypes as Cty
    from . import oracle as O
    lib = O.load("reference")
    dp = Cty.POINTER(Cty.c_double)
    lib.orc_daabpbc.argtypes = [Cty.c_int, Cty.c_int, Cty.c_int, dp, dp, dp]
    lib.orc_daabpbc.restype = None
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    out = np.ascontiguousarray(C, dtype=np.float64).copy()
    m, k = A.shape
    n = B.shape[1]
    lib.orc_daabpbc(m, n, k, A.ctypes.data_as(dp), B.ctypes.data_as(dp), out.ctypes.data_as(dp))
    return out


def assemble(bk, cn, ncom, dt):
    """Diagonal blocks [nb, ncol, ncol] (accumulation plus, in connection
    order, +bmatB at the begin bulk and -bmatE at the end bulk) and the
    off-diagonal blocks of every connection: (row eId, col bId) = -bmatB and
    (row bId, col eId) = bmatE, as [nconn, ncol, ncol] each."""
    nb = len(bk["vfP"])
    nconn = len(cn["bId"])
    ncol = ncom + 1
    diag = np.stack([accumulation(bk, n, ncom) for n in range(nb)])
    offEB = np.zeros((nconn, ncol, ncol))
    offBE = np.zeros((nconn, ncol, ncol))
    for c in range(nconn):
        bB, bE = conn_blocks(bk, cn, c, ncom, dt)
        diag[int(cn["bId"][c])] += bB
        offEB[c] = -bB
        offBE[c] = bE
        diag[int(cn["eId"][c])] += -bE
    return diag, offEB, offBE


# ------------------------------------------- the reference's own assembly
REF_JAC_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libocpjac.so")


def reference_available() -> bool:
    return os.path.exists(REF_JAC_LIB)


def assemble_reference(bk, cn, ncom, dt):
    """(diag, offEB, offBE) as the reference's own
    IsoT_FIM::AssembleMatBulksNew scatters them into its LinearSystem
    (compiled from the reference sources into oracle/_ref/libocpjac.so,
    ``make -C oracle jac``), on the same Bulk arrays and connections as
    ``assemble``."""
    import ctypes as C
    lib = C.CDLL(REF_JAC_LIB)
    dp, ip, lp = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64)

    class OrcJac(C.Structure):
        _fields_ = [("nb", C.c_int64), ("ncom", C.c_int32), ("lend", C.c_int32),
                    ("v", dp), ("poroP", dp), ("vfP", dp), ("vfi", dp),
                    ("phaseExist", ip), ("pSderExist", ip), ("pVnumCom", ip),
                    ("Pj", dp), ("depth", dp), ("xi", dp), ("kr", dp), ("mu", dp), ("muP", dp), ("xiP", dp),
                    ("rhoP", dp), ("xij", dp), ("rhox", dp), ("xix", dp), ("mux", dp), ("dPcj_dS", dp),
                    ("dKr_dS", dp), ("dSec_dPri", dp), ("nconn", C.c_int64), ("bId", lp), ("eId", lp),
                    ("area", dp), ("upblock", lp), ("upblock_Rho", dp), ("dt", C.c_double),
                    ("diag", dp), ("offEB", dp), ("offBE", dp)]

    nb = len(np.asarray(bk["vfP"]))
    ncol = ncom + 1
    nconn = len(cn["bId"])
    keep = []

    def d(a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        keep.append(a)
        return a.ctypes.data_as(dp)

    def i32(a):
        a = np.ascontiguousarray(np.asarray(a).astype(np.int32).reshape(-1))
        keep.append(a)
        return a.ctypes.data_as(ip)

    def i64(a):
        a = np.ascontiguousarray(np.asarray(a).astype(np.int64).reshape(-1))
        keep.append(a)
        return a.ctypes.data_as(lp)

    sec = np.asarray(bk["dSec_dPri"], dtype=np.float64).reshape(nb, -1)
    diag = np.zeros((nb, ncol, ncol))
    offEB = np.zeros((nconn, ncol, ncol))
    offBE = np.zeros((nconn, ncol, ncol))
    j = OrcJac(nb, ncom, sec.shape[1], d(bk["v"]), d(bk["poroP"]), d(bk["vfP"]), d(bk["vfi"]),
               i32(bk["phaseExist"]), i32(bk["pSderExist"]), i32(bk["pVnumCom"]), d(bk["Pj"]), d(bk["depth"]),
               d(bk["xi"]), d(bk["kr"]), d(bk["mu"]), d(bk["muP"]), d(bk["xiP"]), d(bk["rhoP"]), d(bk["xij"]),
               d(bk["rhox"]), d(bk["xix"]), d(bk["mux"]), d(bk["dPcj_dS"]), d(bk["dKr_dS"]), d(sec), nconn,
               i64(cn["bId"]), i64(cn["eId"]), d(cn["area"]), i64(cn["upblock"]), d(cn["upblock_Rho"]), float(dt),
               diag.ctypes.data_as(dp), offEB.ctypes.data_as(dp), offBE.ctypes.data_as(dp))
    lib.orc_assemble_bulks.argtypes = [C.POINTER(OrcJac)]
    lib.orc_assemble_bulks.restype = C.c_int
    rc = lib.orc_assemble_bulks(C.byref(j))
    if rc != 0:
        raise RuntimeError("reference assembly: unexpected row layout")
    return diag, offEB, offBE
