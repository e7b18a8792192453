"""Fluid descriptions for the compositional Peng-Robinson flash.

A :class:`Fluid` carries what one ``MixtureComp`` instance (one PVT region)
reads from its ``ComponentParam`` (``include/ParamReservoir.hpp:87-193``,
consumed in ``src/MixtureComp.cpp:28-165``) plus the water PVTW row
(``src/MixtureComp.cpp:155-167``) and the five solver-control keywords RR,
SSMSTA, NRSTA, SSMSP and NRSP (``include/MixtureComp.hpp:28-104``). Units are
the reference's FIELD units: degR for critical temperatures, psia, ft3/lbmol.

``synthetic_fluid`` draws a seeded fluid from SI property ranges and converts
it to FIELD units: Tc [K] x 1.8 -> degR, Pc [MPa] x 145.0377 -> psia,
Vc [m3/kmol] x 16.01846 -> ft3/lbmol; MW, acentric factor and BIPs unchanged.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np

GAS_CONSTANT = 10.73159  # include/OCPConst.hpp:37
RHOW_STD = 62.3664       # include/OCPConst.hpp:57
MPA_TO_PSIA = 145.0377
K_TO_R = 1.8
M3KMOL_TO_FT3LBMOL = 16.01846
MAX_NC = 16


@dataclass
class Controls:
    """Solver controls; defaults are the SPE5 deck values
    (``examples/spe5/EGOIL.in:65-92``)."""

    rr_maxit: int = 30
    rr_tol: float = 1e-12
    ssmsta_maxit: int = 100
    ssmsta_tol: float = 1e-12
    ssmsta_eyt: float = 1e-8
    nrsta_maxit: int = 55
    nrsta_tol: float = 1e-12
    ssmsp_maxit: int = 100
    ssmsp_tol: float = 1e-6
    nrsp_maxit: int = 55
    nrsp_tol: float = 1e-12
    use_skip: bool = True  # SkipStaAnaly::ifUseSkip default (include/AcceleratePVT.hpp:71)


@dataclass
class Fluid:
    nc: int
    Tc: np.ndarray      # degR
    Pc: np.ndarray      # psia
    Vc: np.ndarray      # ft3/lbmol
    MW: np.ndarray
    Acf: np.ndarray
    BIC: np.ndarray     # (nc, nc) symmetric, zero diagonal
    OmegaA: np.ndarray = None
    OmegaB: np.ndarray = None
    Vshift: np.ndarray = None  # dimensionless deck VSHIFT
    LBCcoef: np.ndarray = None  # deck LBCCOEF (before the x10 scaling)
    pvtw: np.ndarray = None     # Pref, Bw, Cw, muw, Cvw
    std_rho_w: float = RHOW_STD
    controls: Controls = field(default_factory=Controls)
    name: str = "fluid"

    def __post_init__(self):
        nc = self.nc
        if not 2 <= nc <= MAX_NC:
            raise ValueError(f"nc must be in [2, {MAX_NC}], got {nc}")
        as1 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(nc))
        self.Tc, self.Pc, self.Vc = as1(self.Tc), as1(self.Pc), as1(self.Vc)
        self.MW, self.Acf = as1(self.MW), as1(self.Acf)
        # defaults of src/MixtureComp.cpp:82-96 and src/ParamReservoir.cpp:931-938
        self.OmegaA = as1(np.full(nc, 0.457235529) if self.OmegaA is None else self.OmegaA)
        self.OmegaB = as1(np.full(nc, 0.077796074) if self.OmegaB is None else self.OmegaB)
        self.Vshift = as1(np.zeros(nc) if self.Vshift is None else self.Vshift)
        self.LBCcoef = np.ascontiguousarray(
            np.array([0.1023, 0.023364, 0.058533, -0.040758, 0.0093324])
            if self.LBCcoef is None else np.asarray(self.LBCcoef, dtype=np.float64).reshape(5))
        self.pvtw = np.ascontiguousarray(
            np.array([14.7, 1.0, 3.3e-6, 0.7, 0.0])
            if self.pvtw is None else np.asarray(self.pvtw, dtype=np.float64).reshape(5))
        self.BIC = np.ascontiguousarray(np.asarray(self.BIC, dtype=np.float64).reshape(nc, nc))
        if not np.allclose(self.BIC, self.BIC.T, rtol=0, atol=0):
            raise ValueError("BIC must be symmetric")

    @property
    def numCom(self) -> int:
        return self.nc + 1

    def with_controls(self, **kw) -> "Fluid":
        return replace(self, controls=replace(self.controls, **kw))


def spe5_fluid() -> Fluid:
    """The 6-component SPE5 fluid of ``examples/spe5/EGOIL.in`` (ZCRIT given,
    so Vc = 10.73159 Zc Tc / Pc as in ``src/MixtureComp.cpp:63-68``)."""
    Tc = np.array([343.0, 665.7, 913.4, 1111.8, 1270.0, 1380.0])
    Pc = np.array([667.8, 616.3, 436.9, 304.0, 200.0, 162.0])
    Zc = np.array([0.290, 0.277, 0.264, 0.257, 0.245, 0.235])
    MW = np.array([16.04, 44.10, 86.18, 149.29, 206.00, 282.00])
    Acf = np.array([0.013, 0.1524, 0.3007, 0.4885, 0.6500, 0.8500])
    Vc = 10.73159 * Zc * Tc / Pc
    bic = np.zeros((6, 6))
    low = {(3, 0): 0.05, (3, 1): 0.005, (4, 0): 0.05, (4, 1): 0.005}
    for (i, j), v in low.items():
        bic[i, j] = bic[j, i] = v
    return Fluid(nc=6, Tc=Tc, Pc=Pc, Vc=Vc, MW=MW, Acf=Acf, BIC=bic, name="spe5")


def synthetic_fluid(nc: int = 6, seed: int = 1234, bip_max: float = 0.15) -> Fluid:
    """Seeded Peng-Robinson fluid with SI property ranges Tc 190-900 K,
    Pc 4.6-1.0 MPa (falling), acentric factor 0.01-0.9, MW 16-280,
    Vc 0.1-1.0 m3/kmol and symmetric BIPs U(0, bip_max) with zero diagonal.
    Component index rises with MW: properties follow a sorted seeded grid
    t_0 = 0 < t_1 < ... < t_{nc-1} = 1."""
    rng = np.random.default_rng(seed)
    inner = np.sort(rng.uniform(0.0, 1.0, size=max(nc - 2, 0)))
    t = np.concatenate([[0.0], inner, [1.0]]) if nc >= 2 else np.zeros(nc)
    Tc_K = 190.0 + t * (900.0 - 190.0)
    Pc_MPa = 4.6 - t * (4.6 - 1.0)
    acf = 0.01 + t * (0.9 - 0.01)
    mw = 16.0 + t * (280.0 - 16.0)
    vc = 0.1 + t * (1.0 - 0.1)
    bic = np.zeros((nc, nc))
    iu = np.triu_indices(nc, 1)
    vals = rng.uniform(0.0, bip_max, size=len(iu[0]))
    bic[iu] = vals
    bic = bic + bic.T
    return Fluid(nc=nc, Tc=Tc_K * K_TO_R, Pc=Pc_MPa * MPA_TO_PSIA,
                 Vc=vc * M3KMOL_TO_FT3LBMOL, MW=mw, Acf=acf, BIC=bic,
                 name=f"synthetic-nc{nc}-seed{seed}")
