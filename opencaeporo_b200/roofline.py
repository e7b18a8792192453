"""Algorithmic work model of one FIM flash, used for roofline fractions.

FLOPs count +, -, *, / and sqrt as 1, FMA as 2, and each exp / log / pow /
acos / cos / cbrt call as 1. Per unit of work, for NC hydrocarbon components
(U_fug = one fugacity evaluation: mixing rule, cubic solve, ln phi):

    U_fug                 = 2 NC^2 + 10 NC + 40 + (NC + 4)
    stability SSM iter    = U_fug + 6 NC
    stability NR iter     = U_fug + 14 NC^2 + 2/3 NC^3
    Rachford-Rice iter    = 8 NC
    split SSM iter        = 2 U_fug + 6 NC
    split NR iter         = 2 U_fug + 26 NC^2 + 2/3 NC^3
    fixed, one phase      = U_fug + 12 NC^2 + 2 NC^3
    fixed, two phases     = 2 U_fug + 40 NC^2 + 2/3 NC^3 + 2 NC^2 (NC + 1) + 8 NC^2

The iteration counts are the per-cell counters the kernel writes (SSMSTA,
NRSTA, SSMSP, NRSP, RR: the reference's counters of
include/MixtureComp.hpp:134-146).

Algorithmic HBM bytes per cell are the bytes the flash must read and write:
P, T, Ni and the warm-start S / phase count; every output of the existing
phases (7 scalars + 4 rows of numCom per phase, water included), the
per-cell scalars and flags, the compact dSec_dPri rows, the diagnostics and
the skip cache.
"""
from __future__ import annotations

import numpy as np


def unit_flops(nc: int) -> dict:
    u = 2 * nc * nc + 10 * nc + 40 + (nc + 4)
    return {
        "ufug": u,
        "ssmsta": u + 6 * nc,
        "nrsta": u + 14 * nc * nc + (2.0 / 3.0) * nc ** 3,
        "rr": 8 * nc,
        "ssmsp": 2 * u + 6 * nc,
        "nrsp": 2 * u + 26 * nc * nc + (2.0 / 3.0) * nc ** 3,
        "fixed1": u + 12 * nc * nc + 2 * nc ** 3,
        "fixed2": 2 * u + 40 * nc * nc + (2.0 / 3.0) * nc ** 3 + 2 * nc * nc * (nc + 1) + 8 * nc * nc,
    }


def flops(nc: int, iters: np.ndarray, nphc: np.ndarray) -> float:
    """Total algorithmic FLOPs of a batch. iters: [n, 5] (SSMSTA, NRSTA,
    SSMSP, NRSP, RR); nphc: [n] hydrocarbon phase count (1 or 2)."""
    c = unit_flops(nc)
    it = np.asarray(iters, dtype=np.float64).reshape(-1, 5).sum(axis=0)
    n2 = float(np.count_nonzero(np.asarray(nphc) == 2))
    n1 = float(len(nphc)) - n2
    return (it[0] * c["ssmsta"] + it[1] * c["nrsta"] + it[2] * c["ssmsp"] + it[3] * c["nrsp"] +
            it[4] * c["rr"] + n1 * c["fixed1"] + n2 * c["fixed2"])


def bytes_per_cell(nc: int, nphc: int, skip_written: bool = True) -> int:
    ncom = nc + 1
    ncol = ncom + 1
    rd = 8 * (2 + ncom) + 8 * 2 + 4                 # P, T, Ni; S[0:2], lastNP
    per_phase = 8 * 7 + 8 * 4 * ncom                # rho xi mu rhoP xiP muP nj + 4 rows
    phases = (nphc + 1)                             # hydrocarbon phases + water
    scal = 8 * (3 + 3 + ncom) + 4 * (1 + 3 + 1 + 3 + 3)  # S, Nt vf vfP, vfi; flags
    rows = (nc + 2) if nphc == 1 else (3 + 2 * nc)
    dsec = 8 * rows * ncol
    diag = 8 + 1 + 4 * 5 + 2
    skip = 4 + 4 + (8 * (3 + nc) if skip_written else 0)
    return rd + phases * per_phase + scal + dsec + diag + skip


def batch_bytes(nc: int, nphc: np.ndarray, use_skip: bool = True) -> float:
    nphc = np.asarray(nphc)
    n2 = int(np.count_nonzero(nphc == 2))
    n1 = len(nphc) - n2
    return float(n1 * bytes_per_cell(nc, 1, use_skip) + n2 * bytes_per_cell(nc, 2, False))
