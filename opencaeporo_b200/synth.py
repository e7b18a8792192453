"""Seeded synthetic cell states for the flash workloads.

The reference publishes no flash dataset; every workload here is drawn from a
seeded generator (``numpy.random.default_rng(seed)``) with the distributions of
the benchmark configurations, converted from SI to the reference's FIELD
units (P [MPa] x 145.0377 -> psia; T [K] x 1.8 - 459.67 -> degF):

* ``uniform_states`` -- P ~ U(p_lo, p_hi) MPa, T ~ U(t_lo, t_hi) K,
  z ~ Dirichlet(alpha) (normalised Gamma draws), total hydrocarbon moles
  N_tot ~ U(1e3, 1e4) lbmol, Ni = z N_tot. Every cell also carries water,
  N_w = w N_tot with w ~ U(0.5, 2.0), so the water phase and its derivative
  rows are exercised (the reference treats water as a separate phase; it
  never enters the hydrocarbon flash).
* ``near_envelope_states`` -- for seeded (T, z) it bisects the upper
  saturation pressure P_sat on the phase count returned by a caller-supplied
  flash, then sets P = P_sat x U(0.95, 1.05).
* ``mixed_states`` -- a share of near-envelope states among uniform ones
  (1,048,576 states with 30 % near the envelope is the 1M-cell workload).
"""
from __future__ import annotations

import numpy as np

from .fluid import Fluid, K_TO_R, MPA_TO_PSIA

CONV5 = 459.67


def k_to_f(t_k):
    return np.asarray(t_k) * K_TO_R - CONV5


def mpa_to_psia(p_mpa):
    return np.asarray(p_mpa) * MPA_TO_PSIA


def _dirichlet(rng, n, nc, alpha):
    g = rng.gamma(alpha, 1.0, size=(n, nc))
    g = np.maximum(g, 1e-300)
    return g / g.sum(axis=1, keepdims=True)


def uniform_states(fluid: Fluid, n: int, seed: int, p_mpa=(5.0, 40.0), t_k=(340.0, 400.0),
                   alpha: float = 1.0, water=(0.5, 2.0)):
    """Returns dict(P [n] psia, T [n] degF, Ni [n, numCom] lbmol)."""
    rng = np.random.default_rng(seed)
    nc = fluid.nc
    P = mpa_to_psia(rng.uniform(p_mpa[0], p_mpa[1], size=n))
    T = k_to_f(rng.uniform(t_k[0], t_k[1], size=n))
    z = _dirichlet(rng, n, nc, alpha)
    ntot = rng.uniform(1e3, 1e4, size=n)
    Ni = np.empty((n, nc + 1))
    Ni[:, :nc] = z * ntot[:, None]
    Ni[:, nc] = rng.uniform(water[0], water[1], size=n) * ntot
    return {"P": P, "T": T, "Ni": Ni}


def saturation_pressure(phase_count, T, Ni, p_lo_mpa=0.5, p_hi_mpa=80.0, steps=40):
    """Upper saturation pressure (psia) of each (T, Ni) by bisection in ln P on
    ``phase_count(P, T, Ni) -> hydrocarbon phase count``. Returns (Psat, ok)
    with ok False where the state is not two-phase at p_lo and single-phase at
    p_hi."""
    n = len(T)
    lo = np.full(n, np.log(mpa_to_psia(p_lo_mpa)))
    hi = np.full(n, np.log(mpa_to_psia(p_hi_mpa)))
    np_lo = phase_count(np.exp(lo), T, Ni)
    np_hi = phase_count(np.exp(hi), T, Ni)
    ok = (np_lo >= 2) & (np_hi == 1)
    for _ in range(steps):
        mid = 0.5 * (lo + hi)
        two = phase_count(np.exp(mid), T, Ni) >= 2
        lo = np.where(two, mid, lo)
        hi = np.where(two, hi, mid)
    return np.exp(0.5 * (lo + hi)), ok


def near_envelope_states(fluid: Fluid, n: int, seed: int, phase_count, t_k=(340.0, 400.0),
                         alpha: float = 1.0, band=(0.95, 1.05), max_rounds: int = 20, steps: int = 40,
                         record=None, replay=None):
    """n states with P within ``band`` of the seeded state's saturation
    pressure. Candidates that have no upper saturation pressure in range are
    redrawn (deterministically, from the same generator stream).

    ``record``: a list that receives, per round, the accepted candidates'
    indices and saturation pressures; ``replay``: such a list, used instead
    of ``phase_count`` to rebuild the same states bit for bit without a
    flash (the bisection's outcome is the only part of a state that depends
    on a flash; everything else comes from the seeded generators)."""
    rng = np.random.default_rng(seed)
    nc = fluid.nc
    outT, outNi, outP = [], [], []
    have = 0
    rounds = 0
    while have < n and rounds < max_rounds:
        m = max(2 * (n - have), 64)
        cand = uniform_states(fluid, m, int(rng.integers(1 << 62)), t_k=t_k, alpha=alpha)
        if replay is not None:
            idx, psat = replay[rounds]
            idx = np.asarray(idx, np.int64)
            psat = np.asarray(psat, np.float64)
        else:
            psat, ok = saturation_pressure(phase_count, cand["T"], cand["Ni"], steps=steps)
            idx = np.nonzero(ok)[0][: n - have]
            psat = psat[idx]
            if record is not None:
                record.append((idx.astype(np.uint32), psat))
        outT.append(cand["T"][idx])
        outNi.append(cand["Ni"][idx])
        outP.append(psat * rng.uniform(band[0], band[1], size=len(idx)))
        have += len(idx)
        rounds += 1
    if have < n:
        raise RuntimeError(f"only {have} of {n} near-envelope states found")
    return {"P": np.concatenate(outP)[:n], "T": np.concatenate(outT)[:n],
            "Ni": np.concatenate(outNi)[:n].reshape(n, nc + 1)}


def mixed_states(fluid: Fluid, n: int, seed: int, phase_count, near_frac: float = 0.3, steps: int = 40,
                 record=None, replay=None):
    """Uniform states with ``near_frac`` of them replaced by near-envelope
    states at seeded positions (``record`` / ``replay``: see
    ``near_envelope_states``)."""
    base = uniform_states(fluid, n, seed)
    m = int(round(near_frac * n))
    if m == 0:
        return base
    rng = np.random.default_rng(seed + 1)
    pos = np.sort(rng.choice(n, size=m, replace=False))
    near = near_envelope_states(fluid, m, seed + 2, phase_count, steps=steps, record=record, replay=replay)
    for k in ("P", "T", "Ni"):
        base[k][pos] = near[k]
    base["near_mask"] = np.zeros(n, bool)
    base["near_mask"][pos] = True
    return base


def corey_tables(seed, swc=0.15, sorw=0.2, sgc=0.05, sorg=0.1, nrow=12, pc_scale=(4.0, 1.5)):
    """Seeded synthetic SWOF / SGOF rows (Corey-type curves with random
    exponents and end points; capillary pressures falling with saturation),
    the layout the keywords use: (Sw, krw, krow, Pcow), (Sg, krg, krog, Pcgo)."""
    rng = np.random.default_rng(seed)
    nw, now, ng, nog = rng.uniform(1.5, 4.0, 4)
    sw = np.linspace(swc, 1.0, nrow)
    swn = np.clip((sw - swc) / (1 - swc - sorw), 0, 1)
    krw = rng.uniform(0.3, 1.0) * swn ** nw
    krow = np.clip((1 - sw - sorw) / (1 - swc - sorw), 0, 1) ** now
    pcow = pc_scale[0] * (1 - swn) ** 2
    swof = np.stack([sw, krw, krow, pcow], axis=1)
    sg = np.linspace(0.0, 1 - swc - sorg, nrow)
    sgn = np.clip((sg - sgc) / (1 - swc - sgc - sorg), 0, 1)
    krg = rng.uniform(0.5, 1.0) * sgn ** ng
    krog = np.clip((1 - swc - sorg - sg) / (1 - swc - sorg), 0, 1) ** nog
    pcgo = pc_scale[1] * sg / sg[-1]
    sgof = np.stack([sg, krg, krog, pcgo], axis=1)
    return swof, sgof


def corey_fn_tables(seed, swc=0.15, sorw=0.2, sgc=0.05, sorg=0.1, nrow=12, pc_scale=(4.0, 1.5)):
    """Seeded synthetic SWFN / SGFN / SOF3 rows (the saturation-function
    family of keywords): (Sw, krw, Pcow), (Sg, krg, Pcgo) and (So, krow,
    krog), Corey-type curves with random exponents and an oil end point
    kroMax below one."""
    swof, sgof = corey_tables(seed, swc, sorw, sgc, sorg, nrow, pc_scale)
    rng = np.random.default_rng(seed + 7919)
    now, nog = rng.uniform(1.5, 4.0, 2)
    kmax = rng.uniform(0.6, 1.0)
    so = np.linspace(0.0, 1.0 - swc, nrow)
    krow = kmax * np.clip((so - sorw) / (1 - swc - sorw), 0, 1) ** now
    krog = kmax * np.clip((so - sorg) / (1 - swc - sorg), 0, 1) ** nog
    sof3 = np.stack([so, krow, krog], axis=1)
    return swof[:, [0, 1, 3]].copy(), sgof[:, [0, 1, 3]].copy(), sof3
