"""TEST INFRASTRUCTURE ONLY: field-by-field comparison of flash outputs.

Error metric, per output field over the cells whose phase counts agree and,
for per-phase fields, over existing phases only (absent phases keep stale
values in the reference, src/OCPFluidMethod.cpp:1141-1160):

    rel = |g - o| / max(|o|, 1e-12 * max_cells |o_field|, 1e-300)

dSec_dPri is compared on its compact rows only (the first
bRowSizedSdP * (numCom + 1) entries), each entry against
max(|entry|, 1e-4 x its column's largest entry) (see ``dsec_err``). ePEC, a
converged residual near rounding level, is not compared.

Conditioning-aware bar (``check``): a cell's field passes when its largest
element error is <= max(tol, factor * noise), where ``noise`` is the
reference's own largest relative change of that field in that cell when its
inputs are perturbed by a few units in the last place (recorded with the
golden fixtures). Outputs of well-conditioned cells are held to tol = 1e-8;
entries that the reference itself only determines to, say, 1e-6 (tiny
derivative entries behind an ill-conditioned dense solve) are held to ten
times that.
"""
from __future__ import annotations

import numpy as np

PHASE_FIELDS = ("rho", "xi", "mu", "rhoP", "xiP", "muP")
PHASE_COMP_FIELDS = ("xij", "rhox", "xix", "mux")
CELL_FIELDS = ("S", "Nt", "vf", "vfP", "vfi")
INT_FIELDS = ("phaseExist", "bRowSizedSdP", "pSderExist", "pVnumCom")


def _rel(g, o):
    g = np.asarray(g, dtype=np.float64)
    o = np.asarray(o, dtype=np.float64)
    if o.size == 0:
        return np.zeros(0)
    fin = np.isfinite(o)
    scale = np.max(np.abs(o[fin])) if fin.any() else 1.0
    den = np.maximum(np.maximum(np.abs(o), 1e-12 * scale), 1e-300)
    r = np.abs(g - o) / den
    r[~fin & ~np.isfinite(g)] = 0.0  # both non-finite: not an error here
    return r


def per_cell_errors(gpu: dict, ref: dict, nc: int) -> dict:
    """Per cell and field: the largest element-wise relative error (NaN where
    phase counts differ). Returns {field: [n] array} plus 'same' mask."""
    ncom = nc + 1
    ncol = ncom + 1
    n = len(ref["phaseNum"])
    same = np.asarray(gpu["phaseNum"]).astype(np.int64) == np.asarray(ref["phaseNum"]).astype(np.int64)
    same &= np.all(np.asarray(gpu["phaseExist"]).astype(np.int64) ==
                   np.asarray(ref["phaseExist"]).astype(np.int64), axis=1)
    exist = np.asarray(ref["phaseExist"]).astype(bool)
    out = {"same": same}

    def field_err(g, o, mask=None):
        g = np.asarray(g, dtype=np.float64).reshape(n, -1)
        o = np.asarray(o, dtype=np.float64).reshape(n, -1)
        m = np.ones_like(o, dtype=bool) if mask is None else mask
        fin = np.isfinite(o) & m
        scale = np.max(np.abs(o[fin])) if fin.any() else 1.0
        den = np.maximum(np.maximum(np.abs(o), 1e-12 * scale), 1e-300)
        r = np.abs(g - o) / den
        r[~np.isfinite(o) & ~np.isfinite(g)] = 0.0
        r[~m] = 0.0
        e = np.max(r, axis=1) if r.shape[1] else np.zeros(n)
        e[~same] = np.nan
        return e

    for k in CELL_FIELDS:
        out[k] = field_err(gpu[k], ref[k])
    for k in PHASE_FIELDS:
        out[k] = field_err(gpu[k], ref[k], exist)
    for k in PHASE_COMP_FIELDS:
        out[k] = field_err(gpu[k], ref[k], np.repeat(exist, ncom, axis=1))
    out["dSec_dPri"] = dsec_err(gpu["dSec_dPri"], ref["dSec_dPri"], ref["bRowSizedSdP"], ncol)
    out["dSec_dPri"][~same] = np.nan
    return out


def dsec_err(g, o, rows, ncol, col_floor=1e-4):
    """Per-cell error of the compact dSec_dPri rows. Each entry is judged
    relative to max(|entry|, col_floor * largest |entry| of its column): the
    matrix is the solution of a dense solve, and entries many orders below
    their column's scale carry the solve's normwise rounding, not a
    componentwise one (any LU with another operation order, OpenBLAS's
    included, moves them)."""
    n = len(rows)
    g = np.asarray(g, dtype=np.float64).reshape(n, -1)
    o = np.asarray(o, dtype=np.float64).reshape(n, -1)
    rows = np.asarray(rows).astype(np.int64)
    maxr = g.shape[1] // ncol
    g = g[:, :maxr * ncol].reshape(n, maxr, ncol)
    o = o[:, :maxr * ncol].reshape(n, maxr, ncol)
    m = np.broadcast_to(np.arange(maxr)[None, :, None] < rows[:, None, None], o.shape)
    oa = np.where(m & np.isfinite(o), np.abs(o), 0.0)
    colmax = oa.max(axis=1, keepdims=True)
    den = np.maximum(np.maximum(oa, col_floor * colmax), 1e-300)
    r = np.abs(g - o) / den
    r[~np.isfinite(o) & ~np.isfinite(g)] = 0.0
    r[~m] = 0.0
    return r.reshape(n, -1).max(axis=1)


def check(gpu: dict, ref: dict, nc: int, noise: dict = None, fragile=None, tol: float = 1e-8,
          factor: float = 10.0, errors=None, keys=None) -> dict:
    """Parity verdict. Returns {'ok': bool, 'np_mismatch': indices not
    excused by ``fragile``, 'worst': {field: (ratio, cell)}} where ratio =
    error / allowed (<= 1 passes). ``errors`` / ``keys``: the per-cell error
    function and its fields (default: the FIM outputs)."""
    errors = per_cell_errors if errors is None else errors
    keys = FLOAT_KEYS if keys is None else keys
    e = errors(gpu, ref, nc)
    n = len(e["same"])
    frag = np.zeros(n, bool) if fragile is None else np.asarray(fragile, bool)
    bad_np = np.nonzero(~e["same"] & ~frag)[0]
    worst = {}
    ok = len(bad_np) == 0
    for k in keys:
        allowed = np.full(n, tol)
        if noise is not None and k in noise:
            allowed = np.maximum(allowed, factor * np.nan_to_num(np.asarray(noise[k]), nan=0.0))
        ratio = np.where(e["same"], e[k] / allowed, 0.0)
        i = int(np.nanargmax(ratio)) if n else 0
        worst[k] = (float(ratio[i]) if n else 0.0, i)
        if n and ratio[i] > 1.0:
            ok = False
    return {"ok": ok, "np_mismatch": bad_np, "np_mismatch_all": np.nonzero(~e["same"])[0],
            "worst": worst, "errors": e}


def check_summary(res: dict) -> str:
    w = " ".join(f"{k}={v[0]:.2g}@{v[1]}" for k, v in res["worst"].items() if v[0] > 0.01)
    return (f"ok={res['ok']} np_mismatch={list(res['np_mismatch'])} "
            f"(all {len(res['np_mismatch_all'])}) ratios[{w}]")


def compare(gpu: dict, ref: dict, nc: int, cells=None) -> dict:
    """Returns {'n', 'np_mismatch' (indices), field: max rel error, ...}."""
    ncom = nc + 1
    ncol = ncom + 1
    n = len(ref["phaseNum"])
    idx = np.arange(n) if cells is None else np.asarray(cells)
    g_np = np.asarray(gpu["phaseNum"])[idx].astype(np.int64)
    r_np = np.asarray(ref["phaseNum"])[idx].astype(np.int64)
    same = g_np == r_np
    ex_g = np.asarray(gpu["phaseExist"])[idx].astype(np.int64)
    ex_r = np.asarray(ref["phaseExist"])[idx].astype(np.int64)
    same &= np.all(ex_g == ex_r, axis=1)
    res = {"n": len(idx), "np_mismatch": idx[~same]}
    ok = idx[same]
    exist = np.asarray(ref["phaseExist"])[ok].astype(bool)
    for k in CELL_FIELDS:
        res[k] = float(np.max(_rel(np.asarray(gpu[k])[ok], np.asarray(ref[k])[ok]), initial=0.0))
    for k in PHASE_FIELDS:
        g = np.asarray(gpu[k])[ok][exist]
        o = np.asarray(ref[k])[ok][exist]
        res[k] = float(np.max(_rel(g, o), initial=0.0))
    for k in PHASE_COMP_FIELDS:
        g = np.asarray(gpu[k]).reshape(n, 3, ncom)[ok][exist]
        o = np.asarray(ref[k]).reshape(n, 3, ncom)[ok][exist]
        res[k] = float(np.max(_rel(g, o), initial=0.0))
    res["dSec_dPri"] = float(np.max(dsec_err(np.asarray(gpu["dSec_dPri"]).reshape(n, -1)[ok],
                                             np.asarray(ref["dSec_dPri"]).reshape(n, -1)[ok],
                                             np.asarray(ref["bRowSizedSdP"])[ok], ncol), initial=0.0))
    for k in INT_FIELDS:
        a = np.asarray(gpu[k])[ok].astype(np.int64)
        b = np.asarray(ref[k])[ok].astype(np.int64)
        res[k + "_mismatch"] = int(np.count_nonzero(np.any((a != b).reshape(len(ok), -1), axis=1)))
    return res


FLOAT_KEYS = CELL_FIELDS + PHASE_FIELDS + PHASE_COMP_FIELDS + ("dSec_dPri",)


def max_rel(res: dict) -> float:
    return max(res[k] for k in FLOAT_KEYS)


def summary(res: dict) -> str:
    parts = [f"n={res['n']}", f"np_mismatch={len(res['np_mismatch'])}"]
    parts += [f"{k}={res[k]:.1e}" for k in FLOAT_KEYS]
    parts += [f"{k}={res[k]}" for k in res if k.endswith("_mismatch") and k != "np_mismatch" and res[k]]
    return " ".join(parts)


# ---------------------------------------------------------------- IMPEC flash
IMPEC_CELL_FIELDS = ("S", "Nt", "vf", "vfP", "vfi")
IMPEC_PHASE_FIELDS = ("rho", "xi", "mu", "vj")
IMPEC_FLOAT_KEYS = IMPEC_CELL_FIELDS + IMPEC_PHASE_FIELDS + ("xij",)


def impec_errors(gpu: dict, ref: dict, nc: int) -> dict:
    """per_cell_errors for the outputs of IsoT_IMPEC::PassFlashValue (no
    derivative blocks; the phase volumes vj)."""
    ncom = nc + 1
    n = len(ref["phaseNum"])
    same = np.asarray(gpu["phaseNum"]).astype(np.int64) == np.asarray(ref["phaseNum"]).astype(np.int64)
    same &= np.all(np.asarray(gpu["phaseExist"]).astype(np.int64) ==
                   np.asarray(ref["phaseExist"]).astype(np.int64), axis=1)
    exist = np.asarray(ref["phaseExist"]).astype(bool)
    out = {"same": same}

    def field_err(g, o, mask=None):
        g = np.asarray(g, dtype=np.float64).reshape(n, -1)
        o = np.asarray(o, dtype=np.float64).reshape(n, -1)
        m = np.ones_like(o, dtype=bool) if mask is None else mask
        fin = np.isfinite(o) & m
        scale = np.max(np.abs(o[fin])) if fin.any() else 1.0
        den = np.maximum(np.maximum(np.abs(o), 1e-12 * scale), 1e-300)
        r = np.abs(g - o) / den
        r[~np.isfinite(o) & ~np.isfinite(g)] = 0.0
        r[~m] = 0.0
        e = np.max(r, axis=1) if r.shape[1] else np.zeros(n)
        e[~same] = np.nan
        return e

    for k in IMPEC_CELL_FIELDS:
        out[k] = field_err(gpu[k], ref[k])
    for k in IMPEC_PHASE_FIELDS:
        out[k] = field_err(gpu[k], ref[k], exist)
    out["xij"] = field_err(gpu["xij"], ref["xij"], np.repeat(exist, ncom, axis=1))
    return out


def check_impec(gpu: dict, ref: dict, nc: int, noise: dict = None, fragile=None, tol: float = 1e-8,
                factor: float = 10.0) -> dict:
    """check() for the IMPEC outputs."""
    e = impec_errors(gpu, ref, nc)
    n = len(e["same"])
    frag = np.zeros(n, bool) if fragile is None else np.asarray(fragile, bool)
    bad_np = np.nonzero(~e["same"] & ~frag)[0]
    worst, ok = {}, len(bad_np) == 0
    for k in IMPEC_FLOAT_KEYS:
        allowed = np.full(n, tol)
        if noise is not None and k in noise:
            allowed = np.maximum(allowed, factor * np.nan_to_num(np.asarray(noise[k]), nan=0.0))
        ratio = np.where(e["same"], e[k] / allowed, 0.0)
        i = int(np.nanargmax(ratio)) if n else 0
        worst[k] = (float(ratio[i]) if n else 0.0, i)
        if n and ratio[i] > 1.0:
            ok = False
    return {"ok": ok, "np_mismatch": bad_np, "np_mismatch_all": np.nonzero(~e["same"])[0], "worst": worst,
            "errors": e}


# ------------------------------------------------- the reference's self-noise
NOISE_TRIALS = 32


def perturbed(P, T, X, trial, prng, eps=2.0 ** -50):
    """Inputs of noise trial `trial`: P, T or each entry of X (Ni or z)
    moved by a few units in the last place -- the first six trials one
    input at a time with both signs, the rest all together with random
    signs and sizes."""
    P, T, X = np.array(P, dtype=np.float64), np.array(T, dtype=np.float64), np.array(X, dtype=np.float64)
    sgn = 1 if trial % 2 == 0 else -1
    if trial < 2:
        P *= 1 + sgn * eps
    elif trial < 4:
        T = T + sgn * eps * np.maximum(np.abs(T), 1.0)
    elif trial < 6:
        X = X * (1 + eps * prng.choice([-1.0, 1.0], size=X.shape))
    else:
        P *= 1 + eps * prng.choice([-2.0, -1.0, 1.0, 2.0], size=P.shape)
        T = T * (1 + eps * prng.choice([-1.0, 1.0], size=T.shape))
        X = X * (1 + eps * prng.choice([-1.0, 1.0], size=X.shape))
    return P, T, X


def self_noise(run, P, T, X, base, nc, trials: int = NOISE_TRIALS, seed: int = 7, errors=None, keys=None):
    """(noise, moved): per FIM output field and cell, the largest relative
    change of ``run(P, T, X)`` (the reference on perturbed inputs) against
    ``base`` over ``trials`` perturbations; and the cells whose phase count
    moved. ``errors`` / ``keys`` as in ``check``."""
    errors = per_cell_errors if errors is None else errors
    keys = FLOAT_KEYS if keys is None else keys
    prng = np.random.default_rng(seed)
    n = len(P)
    noise = {k: np.zeros(n) for k in keys}
    moved = np.zeros(n, bool)
    for t in range(trials):
        r = run(*perturbed(P, T, X, t, prng))
        moved |= np.asarray(r["phaseNum"]) != np.asarray(base["phaseNum"])
        e = errors(r, base, nc)
        for k in keys:
            noise[k] = np.fmax(noise[k], np.nan_to_num(e[k], nan=0.0))
    return noise, moved


# ----------------------------------------------------------------- FIMn flash
FIMN_KEYS = FLOAT_KEYS + ("nj", "res", "resPc")


def fimn_errors(gpu: dict, ref: dict, nc: int, col_floor: float = 1e-4) -> dict:
    """per_cell_errors for the outputs of IsoT_FIMn::PassFlashValue, plus the
    phase moles nj of the existing phases, the residual terms ``res`` (the
    first bRowSizedSdP entries; each judged against max(|entry|, col_floor x
    the cell's largest entry), like dSec_dPri's columns: they are one
    column of the same dense solve) and ``resPc``."""
    e = per_cell_errors(gpu, ref, nc)
    n = len(e["same"])
    exist = np.asarray(ref["phaseExist"]).astype(bool)
    r = _rel(np.asarray(gpu["nj"], dtype=np.float64).reshape(n, -1), np.asarray(ref["nj"]).reshape(n, -1))
    r[~exist] = 0.0
    e["nj"] = np.where(e["same"], np.nan_to_num(r, nan=0.0).max(axis=1), np.nan)
    g = np.asarray(gpu["res"], dtype=np.float64).reshape(n, -1)
    o = np.asarray(ref["res"], dtype=np.float64).reshape(n, -1)
    rows = np.asarray(ref["bRowSizedSdP"]).astype(np.int64)
    m = np.arange(o.shape[1])[None, :] < rows[:, None]
    oa = np.where(m & np.isfinite(o), np.abs(o), 0.0)
    den = np.maximum(np.maximum(oa, col_floor * oa.max(axis=1, keepdims=True)), 1e-300)
    rr = np.abs(g - o) / den
    rr[~np.isfinite(o) & ~np.isfinite(g)] = 0.0
    rr[~m] = 0.0
    e["res"] = np.where(e["same"], rr.max(axis=1), np.nan)
    gp = np.asarray(gpu["resPc"], dtype=np.float64).reshape(n)
    op = np.asarray(ref["resPc"], dtype=np.float64).reshape(n)
    rp = np.abs(gp - op) / np.maximum(np.abs(op), 1e-300)
    rp[(gp == op) | (~np.isfinite(op) & ~np.isfinite(gp))] = 0.0
    e["resPc"] = np.where(e["same"], rp, np.nan)
    return e
