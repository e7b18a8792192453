"""Generates the golden flash fixtures in tests/golden/ from the reference's
own MixtureComp, compiled from the reference sources into
oracle/_ref/libocpref.so (``make -C oracle ref``).

Every fixture stores the fluid, the solver controls, the seeded inputs (with
the warm-start state where the case has one) and the reference's outputs in
the cell-major Bulk layout, plus a ``fragile`` mask: cells whose reference
phase count changes when the inputs are perturbed by a few units in the last
place (P, T and each Ni scaled by 1 +- 2^-50). Such cells sit on a knife
edge of an iteration cap or a stability threshold; any implementation whose
rounding differs from the reference's may legitimately land on either side.

    python tests/golden/make_golden.py            # writes tests/golden/*.npz
    python tests/golden/make_golden.py restart_nc6   # one case only (also impec_nc6, init_nc6, krpc, krpc_sof3,
                                                   # fimn_nc6, config1_nc6)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from opencaeporo_b200.fluid import Fluid, spe5_fluid, synthetic_fluid  # noqa: E402
from opencaeporo_b200 import synth  # noqa: E402

OUT_KEYS = ("phaseNum", "phaseExist", "S", "Nt", "vf", "vfP", "vfi", "nj", "rho", "xi", "mu",
            "rhoP", "xiP", "muP", "xij", "rhox", "xix", "mux", "dSec_dPri", "bRowSizedSdP",
            "pSderExist", "pVnumCom", "ePEC", "ftype", "NPhc", "iters")


def fluid_arrays(fl: Fluid) -> dict:
    c = fl.controls
    d = {f"fluid_{k}": getattr(fl, k) for k in ("Tc", "Pc", "Vc", "MW", "Acf", "OmegaA", "OmegaB",
                                                "Vshift", "BIC", "LBCcoef", "pvtw")}
    d["fluid_std_rho_w"] = np.float64(fl.std_rho_w)
    d["controls"] = np.array([c.rr_maxit, c.rr_tol, c.ssmsta_maxit, c.ssmsta_tol, c.ssmsta_eyt,
                              c.nrsta_maxit, c.nrsta_tol, c.ssmsp_maxit, c.ssmsp_tol, c.nrsp_maxit,
                              c.nrsp_tol, float(c.use_skip)])
    d["fluid_name"] = np.array(fl.name)
    return d


def fragile_mask(fl, inp, base, nthreads=8):
    """(fragile mask, per-field self-noise) of the reference on these cells."""
    from oracle import compare as CMP
    base_np = base["phaseNum"]
    n = len(inp["P"])
    frag = np.zeros(n, bool)
    noise = {k: np.zeros(n) for k in CMP.FLOAT_KEYS}
    eps = 2.0 ** -50
    rng = np.random.default_rng(7)
    for trial in range(6):
        P, T, Ni = inp["P"].copy(), inp["T"].copy(), inp["Ni"].copy()
        s = 1 if trial % 2 == 0 else -1
        if trial < 2:
            P *= 1 + s * eps
        elif trial < 4:
            T = T + s * eps * np.maximum(np.abs(T), 1.0)
        else:
            Ni = Ni * (1 + eps * rng.choice([-1.0, 1.0], size=Ni.shape))
        skip = {k: v.copy() for k, v in inp["skip"].items()} if "skip" in inp else None
        r = O.flash_fim("reference", fl, P, T, Ni, S=inp.get("S"), lastNP=inp.get("lastNP"),
                        xij=inp.get("xij"), skip=skip, nthreads=nthreads)
        frag |= r["phaseNum"] != base_np
        e = CMP.per_cell_errors(r, base, fl.nc)
        for k in CMP.FLOAT_KEYS:
            noise[k] = np.fmax(noise[k], np.nan_to_num(e[k], nan=0.0))
    return frag, noise


def run_case(name, fl, inp, keep=None, note=""):
    skip_in = {k: v.copy() for k, v in inp["skip"].items()} if "skip" in inp else O.new_skip(len(inp["P"]), fl.nc)
    skip_run = {k: v.copy() for k, v in skip_in.items()}
    r = O.flash_fim("reference", fl, inp["P"], inp["T"], inp["Ni"], S=inp.get("S"),
                    lastNP=inp.get("lastNP"), xij=inp.get("xij"), skip=skip_run, nthreads=8)
    inp2 = dict(inp)
    inp2["skip"] = skip_in
    frag, noise = fragile_mask(fl, inp2, r)
    n = len(inp["P"])
    sel = np.arange(n) if keep is None else np.asarray(keep)
    d = fluid_arrays(fl)
    d["note"] = np.array(note)
    d["index"] = sel
    d["in_P"], d["in_T"], d["in_Ni"] = inp["P"][sel], inp["T"][sel], inp["Ni"][sel]
    d["in_S"] = (inp["S"] if "S" in inp else np.zeros((n, 3)))[sel]
    d["in_lastNP"] = (inp["lastNP"] if "lastNP" in inp else np.zeros(n, np.int32))[sel]
    d["in_xij"] = (inp["xij"] if "xij" in inp else np.zeros((n, 3, fl.nc + 1)))[sel]
    for k, v in skip_in.items():
        d[f"skipin_{k}"] = v[sel]
    for k, v in skip_run.items():
        d[f"skipout_{k}"] = v[sel]
    for k in OUT_KEYS:
        d[f"out_{k}"] = r[k][sel]
    d["fragile"] = frag[sel]
    for k, v in noise.items():
        d[f"noise_{k}"] = v[sel].astype(np.float32)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **d)
    two = np.mean(r["NPhc"][sel] == 2)
    ft = np.bincount(r["ftype"][sel], minlength=3)
    nz = max(float(np.max(v[sel])) for v in noise.values())
    print(f"{name}: n={len(sel)} two-phase={two:.3f} ftype={ft.tolist()} fragile={frag[sel].sum()} "
          f"max self-noise={nz:.1e} "
          f"size={os.path.getsize(path) / 1e6:.2f} MB")
    return r


def restart_case():
    """Cells whose PhaseSplit keeps restarting: the 48 states of the 1M-state
    bench workload with the most split successive-substitution iterations
    (found on a GPU by find_restart_cells.py; each restart runs up to 2x or
    4x the iteration cap, and the batched form runs cells still restarting
    after three restarts on its warp-per-cell path), plus 16 ordinary ones."""
    fl = synthetic_fluid(6, 1234)
    d = np.load(os.path.join(HERE, "restart_nc6_cells.npz"))
    inp = {"P": d["P"], "T": d["T"], "Ni": d["Ni"]}
    run_case("restart_nc6", fl, inp, note="synthetic nc=6: bench-workload states with the most split restarts")


def impec_case():
    """FlashIMPEC on the 6-component fluid: a fresh step on 512 uniform states
    (the first 256) and near-envelope states (the rest), then a warm second
    step from the first step's phase counts, compositions and skip cache with
    P and Ni perturbed (skip hits, warm two-phase starts, relaxed stability);
    the fixture holds the second step, its warm-start inputs and the
    reference's IMPEC outputs, with the fragile mask and the self-noise over
    oracle.compare.NOISE_TRIALS perturbations (``perturbed``)."""
    from oracle import compare as CMP
    fl = synthetic_fluid(6, 1234)

    def pc(P, T, Ni):
        return O.flash_fim("reference", fl, P, T, Ni, nthreads=8)["NPhc"]

    a = synth.uniform_states(fl, 256, 77)
    b = synth.near_envelope_states(fl, 256, 78, pc)
    inp = {k: np.concatenate([a[k], b[k]]) for k in ("P", "T", "Ni")}
    n = 512
    skip = O.new_skip(n, fl.nc)
    s1 = O.flash_impec(fl, inp["P"], inp["T"], inp["Ni"], skip=skip, nthreads=8)
    rng = np.random.default_rng(11)
    scale = np.where(rng.uniform(size=n) < 0.5, 1e-4, 3e-2)
    P2 = inp["P"] * (1 + scale * rng.uniform(-1, 1, n))
    N2 = inp["Ni"] * (1 + scale[:, None] * rng.uniform(-1, 1, inp["Ni"].shape))
    lastNP = s1["phaseNum"].astype(np.int32)
    xij = np.nan_to_num(s1["xij"], nan=0.0)
    skip_in = {k: v.copy() for k, v in skip.items()}

    def run(P, T, Ni):
        sk = {k: v.copy() for k, v in skip_in.items()}
        return O.flash_impec(fl, P, T, Ni, lastNP=lastNP, xij=xij, skip=sk, nthreads=8), sk

    r, skip_out = run(P2, inp["T"], N2)
    frag = np.zeros(n, bool)
    noise = {k: np.zeros(n) for k in CMP.IMPEC_FLOAT_KEYS}
    prng = np.random.default_rng(7)
    for trial in range(CMP.NOISE_TRIALS):
        P, T, Ni = CMP.perturbed(P2, inp["T"], N2, trial, prng)
        rr, _ = run(P, T, Ni)
        frag |= rr["phaseNum"] != r["phaseNum"]
        e = CMP.impec_errors(rr, r, fl.nc)
        for k in CMP.IMPEC_FLOAT_KEYS:
            noise[k] = np.fmax(noise[k], np.nan_to_num(e[k], nan=0.0))
    d = fluid_arrays(fl)
    d["note"] = np.array("FlashIMPEC, second step: warm start from a first step, P and Ni perturbed")
    d["in_P"], d["in_T"], d["in_Ni"] = P2, inp["T"], N2
    d["in_lastNP"], d["in_xij"] = lastNP, xij
    for k, v in skip_in.items():
        d[f"skipin_{k}"] = v
    for k, v in skip_out.items():
        d[f"skipout_{k}"] = v
    for k in ("phaseNum", "phaseExist", "S", "Nt", "vf", "vfP", "vfi", "vj", "rho", "xi", "mu", "xij",
              "ePEC", "ftype", "NPhc", "iters"):
        d[f"out_{k}"] = r[k]
    d["fragile"] = frag
    for k, v in noise.items():
        d[f"noise_{k}"] = v.astype(np.float32)
    for k in OUT_KEYS:
        d[f"out2_{k}"] = s2[k]
    for k, v in noise2.items():
        d[f"noise2_{k}"] = v.astype(np.float32)
    d["fragile2"] = moved2
    path = os.path.join(HERE, "impec_nc6.npz")
    np.savez_compressed(path, **d)
    print(f"impec_nc6: n={n} two-phase={np.mean(r['NPhc'] == 2):.3f} ftype={np.bincount(r['ftype'], minlength=3)} "
          f"fragile={frag.sum()} size={os.path.getsize(path) / 1e6:.2f} MB")


def init_case():
    """InitFlashFIM and InitFlashIMPEC on the 6-component fluid: 512 initial
    states (256 uniform, 256 near the envelope) given as mole fractions z,
    with water saturations S_w ~ U(0.05, 0.5) and pore volumes
    Vpore ~ U(50, 5000) ft3. The fixture holds the inputs, the reference's
    FIM outputs (out_*) and IMPEC outputs (outi_*), each with the moles Ni
    the flash object holds afterwards, the fragile mask and the self-noise
    of both (``perturbed``); and the reference's next FlashFIM from the
    initialised state (out2_*, noise2_*, fragile2)."""
    from oracle import compare as CMP
    fl = synthetic_fluid(6, 1234)

    def pc(P, T, Ni):
        return O.flash_fim("reference", fl, P, T, Ni, nthreads=8)["NPhc"]

    a = synth.uniform_states(fl, 256, 91)
    # (seed 92's bisection reaches a state whose split restarts without end
    # in the reference)
    b = synth.near_envelope_states(fl, 256, 94, pc)
    P = np.concatenate([a["P"], b["P"]])
    T = np.concatenate([a["T"], b["T"]])
    Ni = np.concatenate([a["Ni"], b["Ni"]])
    n = len(P)
    z = Ni / Ni[:, :fl.nc].sum(axis=1, keepdims=True)
    z[:, fl.nc] = 0.0
    rng = np.random.default_rng(93)
    S = np.zeros((n, 3))
    S[:, 2] = rng.uniform(0.05, 0.5, n)
    S[:, 0] = 1 - S[:, 2]
    Vp = rng.uniform(50.0, 5000.0, n)

    def run(P, T, z, impec):
        return O.init_flash(fl, P, T, z, S, Vp, impec=impec, skip=O.new_skip(n, fl.nc), nthreads=8)

    r, ri = run(P, T, z, False), run(P, T, z, True)
    frag = np.zeros(n, bool)
    noise = {k: np.zeros(n) for k in CMP.FLOAT_KEYS + ("Ni", "nj")}
    noisei = {k: np.zeros(n) for k in CMP.IMPEC_FLOAT_KEYS + ("Ni",)}
    prng = np.random.default_rng(7)
    for trial in range(CMP.NOISE_TRIALS):
        Pp, Tp, zp = CMP.perturbed(P, T, z, trial, prng)
        rr, rri = run(Pp, Tp, zp, False), run(Pp, Tp, zp, True)
        frag |= (rr["phaseNum"] != r["phaseNum"]) | (rri["phaseNum"] != ri["phaseNum"])
        e, ei = CMP.per_cell_errors(rr, r, fl.nc), CMP.impec_errors(rri, ri, fl.nc)
        e["Ni"] = CMP._rel(rr["Ni"], r["Ni"]).max(axis=1)
        e["nj"] = np.nan_to_num(CMP._rel(rr["nj"][:, :2], r["nj"][:, :2]), nan=0.0).max(axis=1)
        ei["Ni"] = CMP._rel(rri["Ni"], ri["Ni"]).max(axis=1)
        for k in noise:
            noise[k] = np.fmax(noise[k], np.nan_to_num(e[k], nan=0.0))
        for k in noisei:
            noisei[k] = np.fmax(noisei[k], np.nan_to_num(ei[k], nan=0.0))
    # the next FlashFIM from the initialised state (IsoT_FIM's first Newton
    # iteration at unchanged P, T): warm start from the initialisation's
    # phase counts, saturations, compositions and skip cache
    xij0 = np.nan_to_num(r["xij"], nan=0.0)
    skip0 = {k: v.copy() for k, v in r["skip"].items()}

    def step2(P, T, Ni):
        return O.flash_fim("reference", fl, P, T, Ni, S=r["S"], lastNP=r["phaseNum"].astype(np.int32), xij=xij0,
                           skip={k: v.copy() for k, v in skip0.items()}, nthreads=8)

    s2 = step2(P, T, r["Ni"])

    # the sequence's own sensitivity: perturb the initial state and rerun
    # both calls (an ill-determined initialisation carries its noise into
    # the warm start of the next step)
    def both(Pp, Tp, zp):
        r1 = run(Pp, Tp, zp, False)
        return O.flash_fim("reference", fl, Pp, Tp, r1["Ni"], S=r1["S"], lastNP=r1["phaseNum"].astype(np.int32),
                           xij=np.nan_to_num(r1["xij"], nan=0.0), skip=r1["skip"], nthreads=8)

    noise2, moved2 = CMP.self_noise(both, P, T, z, s2, fl.nc)
    d = fluid_arrays(fl)
    d["note"] = np.array("InitFlashFIM / InitFlashIMPEC of initial states z, S_w, Vpore; then one warm FlashFIM")
    d["in_P"], d["in_T"], d["in_z"], d["in_S"], d["in_Vpore"] = P, T, z, S, Vp
    for k in OUT_KEYS + ("Ni",):
        d[f"out_{k}"] = r[k]
    for k in ("phaseNum", "phaseExist", "S", "Nt", "vf", "vfP", "vfi", "vj", "rho", "xi", "mu", "xij",
              "ePEC", "ftype", "NPhc", "iters", "Ni"):
        d[f"outi_{k}"] = ri[k]
    for k, v in r["skip"].items():
        d[f"skipout_{k}"] = v
    d["fragile"] = frag
    for k, v in noise.items():
        d[f"noise_{k}"] = v.astype(np.float32)
    for k in OUT_KEYS:
        d[f"out2_{k}"] = s2[k]
    for k, v in noise2.items():
        d[f"noise2_{k}"] = v.astype(np.float32)
    d["fragile2"] = moved2
    for k, v in noisei.items():
        d[f"noisei_{k}"] = v.astype(np.float32)
    path = os.path.join(HERE, "init_nc6.npz")
    np.savez_compressed(path, **d)
    print(f"init_nc6: n={n} two-phase={np.mean(r['NPhc'] == 2):.3f} fragile={frag.sum()} "
          f"step 2: phase changes={int(np.sum(s2['phaseNum'] != r['phaseNum']))} fragile={moved2.sum()} "
          f"size={os.path.getsize(path) / 1e6:.2f} MB")


FIMN_OUT_KEYS = OUT_KEYS + ("res", "resPc")


def fimn_case():
    """FlashFIMn and InitFlashFIMn (the FIM formulation with the phase moles
    as secondary variables, IsoT_FIMn) on the 6-component fluid, on inputs
    of the FIM fixtures (FlashFIMn's phase equilibrium is FlashFIM's): a
    fresh step on near_nc6's near-envelope states, a warm step on warm_nc6's
    warm-start state (skip hits, warm two-phase starts, relaxed stability)
    and InitFlashFIMn of init_nc6's initial states. (States drawn afresh near
    the envelope can hold one on which the reference's split restarts
    without end.) The fixture holds each call's inputs, the reference's
    outputs (res and resPc included), the cells whose phase count moved
    under perturbation and the self-noise over oracle.compare.NOISE_TRIALS
    perturbations (``perturbed``)."""
    from oracle import compare as CMP
    fl = synthetic_fluid(6, 1234)
    kw = dict(errors=CMP.fimn_errors, keys=CMP.FIMN_KEYS)
    g1 = np.load(os.path.join(HERE, "near_nc6.npz"))
    P1, T1, N1 = g1["in_P"], g1["in_T"], g1["in_Ni"]

    def step1(P, T, Ni):
        return O.flash_fimn(fl, P, T, Ni, skip=O.new_skip(len(P), fl.nc), nthreads=8)

    s1 = step1(P1, T1, N1)
    noise1, moved1 = CMP.self_noise(step1, P1, T1, N1, s1, fl.nc, **kw)
    g2 = np.load(os.path.join(HERE, "warm_nc6.npz"))
    P2, T2, N2 = g2["in_P"], g2["in_T"], g2["in_Ni"]
    S2, lastNP, xij = g2["in_S"], g2["in_lastNP"].astype(np.int32), g2["in_xij"]
    skip2 = {k: g2[f"skipin_{k}"] for k in ("flag", "minEig", "P", "T", "z")}

    def step2(P, T, Ni):
        return O.flash_fimn(fl, P, T, Ni, S=S2, lastNP=lastNP, xij=xij,
                            skip={k: v.copy() for k, v in skip2.items()}, nthreads=8)

    s2 = step2(P2, T2, N2)
    noise2, moved2 = CMP.self_noise(step2, P2, T2, N2, s2, fl.nc, **kw)
    gi = np.load(os.path.join(HERE, "init_nc6.npz"))
    Pi, Ti, zi, Si, Vp = gi["in_P"], gi["in_T"], gi["in_z"], gi["in_S"], gi["in_Vpore"]

    def init(P, T, z):
        return O.init_flash_fimn(fl, P, T, z, Si, Vp, skip=O.new_skip(len(P), fl.nc), nthreads=8)

    si = init(Pi, Ti, zi)
    noisei, movedi = CMP.self_noise(init, Pi, Ti, zi, si, fl.nc, **kw)
    d = fluid_arrays(fl)
    d["note"] = np.array("FlashFIMn fresh (near_nc6) and warm (warm_nc6) steps; InitFlashFIMn (init_nc6)")
    d["in1_P"], d["in1_T"], d["in1_Ni"] = P1, T1, N1
    d["in2_P"], d["in2_T"], d["in2_Ni"], d["in2_S"], d["in2_lastNP"], d["in2_xij"] = P2, T2, N2, S2, lastNP, xij
    for k, v in skip2.items():
        d[f"skipin2_{k}"] = v
    d["ini_P"], d["ini_T"], d["ini_z"], d["ini_S"], d["ini_Vpore"] = Pi, Ti, zi, Si, Vp
    for tag, r, noise, moved in (("1", s1, noise1, moved1), ("2", s2, noise2, moved2), ("i", si, noisei, movedi)):
        for k in FIMN_OUT_KEYS:
            d[f"out{tag}_{k}"] = r[k]
        for k, v in r["skip"].items():
            d[f"skipout{tag}_{k}"] = v
        for k, v in noise.items():
            d[f"noise{tag}_{k}"] = v.astype(np.float32)
        d[f"fragile{tag}"] = moved
    d["outi_Ni"] = si["Ni"]
    path = os.path.join(HERE, "fimn_nc6.npz")
    np.savez_compressed(path, **d)
    print(f"fimn_nc6: two-phase step1={np.mean(s1['NPhc'] == 2):.3f} step2 ftype="
          f"{np.bincount(s2['ftype'], minlength=3).tolist()} init two-phase={np.mean(si['NPhc'] == 2):.3f} "
          f"fragile={moved1.sum()}/{moved2.sum()}/{movedi.sum()} size={os.path.getsize(path) / 1e6:.2f} MB")


def krpc_case():
    """IsoT_FIM::CalKrPc with FlowUnit_ODGW01 on two saturation regions of
    synthetic tables (the second with a repeated saturation node), 4096
    cells: random saturations, every table node exactly, values outside the
    tables and NaN. Outputs of the compiled reference (derivatives
    included)."""
    from oracle import krpc as K
    r0 = synth.corey_tables(501)
    w1, g1 = synth.corey_tables(502, swc=0.2, sorw=0.15, nrow=9, pc_scale=(8.0, 3.0))
    w1 = np.insert(w1, 4, w1[4], axis=0)  # a repeated node
    regions = [r0, (w1, g1)]
    rng = np.random.default_rng(503)
    n = 4096
    S = np.zeros((n, 3))
    S[:, 2] = rng.uniform(-0.05, 1.05, n)
    S[:, 1] = rng.uniform(-0.05, 1.0, n)
    S[:, 0] = 1 - S[:, 1] - S[:, 2]
    satnum = rng.integers(0, 2, n).astype(np.int32)
    k = 0
    for r, (w, g) in enumerate(regions):
        for v in w[:, 0]:
            S[k, 2], satnum[k] = v, r
            k += 1
        for v in g[:, 0]:
            S[k, 1], satnum[k] = v, r
            k += 1
    S[k:k + 4, 1:] = [[np.nan, 0.3], [0.1, np.nan], [np.inf, -np.inf], [-np.inf, np.inf]]
    P = rng.uniform(500.0, 6000.0, n)
    out = K.reference(regions, P, S, satnum, deriv=True, nthreads=8)
    d = {"note": np.array("CalKrPc, FlowUnit_ODGW01, two synthetic regions"), "in_P": P, "in_S": S,
         "in_satnum": satnum}
    for i, (w, g) in enumerate(regions):
        d[f"swof{i}"], d[f"sgof{i}"] = w, g
    for key in ("kr", "Pc", "Pj", "dKr_dS", "dPcj_dS"):
        d[f"out_{key}"] = out[key]
    path = os.path.join(HERE, "krpc.npz")
    np.savez_compressed(path, **d)
    print(f"krpc: n={n} size={os.path.getsize(path) / 1e6:.2f} MB")


def krpc_sof3_case():
    """IsoT_FIM::CalKrPc (with derivatives) and IsoT_IMPEC::CalKrPc (without)
    with FlowUnit_ODGW02 on two saturation regions of synthetic SWFN / SGFN /
    SOF3 tables (the second with a repeated saturation node), 4096 cells:
    random saturations, every table node exactly, S_g + S_w at the connate
    water saturation (the default oil model's small-denominator branch),
    values outside the tables and NaN. Outputs of the compiled reference."""
    from oracle import krpc as K
    r0 = synth.corey_fn_tables(601)
    w1, g1, o1 = synth.corey_fn_tables(602, swc=0.2, sorw=0.15, nrow=9, pc_scale=(8.0, 3.0))
    o1 = np.insert(o1, 3, o1[3], axis=0)  # a repeated node
    regions = [r0, (w1, g1, o1)]
    rng = np.random.default_rng(603)
    n = 4096
    S = np.zeros((n, 3))
    S[:, 2] = rng.uniform(-0.05, 1.05, n)
    S[:, 1] = rng.uniform(-0.05, 1.0, n)
    S[:, 0] = 1 - S[:, 1] - S[:, 2]
    satnum = rng.integers(0, 2, n).astype(np.int32)
    k = 0
    for r, tabs in enumerate(regions):
        for col, t in zip((2, 1, 0), tabs):
            for v in t[:, 0]:
                S[k, col], satnum[k] = v, r
                k += 1
        swco = tabs[0][0, 0]
        for sg in (0.0, 1e-9, 5e-9, 1e-8, 2e-8):
            S[k], satnum[k] = (1 - swco - sg, sg, swco), r
            k += 1
    S[k:k + 4, 1:] = [[np.nan, 0.3], [0.1, np.nan], [np.inf, -np.inf], [-np.inf, np.inf]]
    S[k + 4, 0] = np.nan
    P = rng.uniform(500.0, 6000.0, n)
    out = K.reference_sof3(regions, P, S, satnum, deriv=True, nthreads=8)
    nod = K.reference_sof3(regions, P, S, satnum, deriv=False, nthreads=8)
    d = {"note": np.array("CalKrPc, FlowUnit_ODGW02, two synthetic regions"), "in_P": P, "in_S": S,
         "in_satnum": satnum}
    for i, (w, g, o) in enumerate(regions):
        d[f"swfn{i}"], d[f"sgfn{i}"], d[f"sof3{i}"] = w, g, o
    for key in ("kr", "Pc", "Pj", "dKr_dS", "dPcj_dS"):
        d[f"out_{key}"] = out[key]
    for key in ("kr", "Pc", "Pj"):
        d[f"impec_{key}"] = nod[key]
    path = os.path.join(HERE, "krpc_sof3.npz")
    np.savez_compressed(path, **d)
    print(f"krpc_sof3: n={n} size={os.path.getsize(path) / 1e6:.2f} MB")


def config1_case():
    """The CPU-runnable configuration in full: the 6-component fluid and 4096
    independent fresh states, P ~ U(5, 40) MPa, T ~ U(340, 400) K,
    z ~ Dirichlet(1), N_tot ~ U(1e3, 1e4) (synth.uniform_states, seed 1234;
    uniform_nc6 keeps 512 of the same states). Fragile mask and self-noise
    over oracle.compare.NOISE_TRIALS perturbations (``perturbed``)."""
    from oracle import compare as CMP
    fl = synthetic_fluid(6, 1234)
    inp = synth.uniform_states(fl, 4096, 1234)
    n = len(inp["P"])
    skip_in = O.new_skip(n, fl.nc)
    skip_run = {k: v.copy() for k, v in skip_in.items()}
    r = O.flash_fim("reference", fl, inp["P"], inp["T"], inp["Ni"], skip=skip_run, nthreads=8)

    def run(P, T, Ni):
        return O.flash_fim("reference", fl, P, T, Ni, nthreads=8)

    noise, moved = CMP.self_noise(run, inp["P"], inp["T"], inp["Ni"], r, fl.nc)
    d = fluid_arrays(fl)
    d["note"] = np.array("config 1: synthetic nc=6 seed 1234, 4096 uniform_states seed 1234, fresh cells")
    d["index"] = np.arange(n)
    d["in_P"], d["in_T"], d["in_Ni"] = inp["P"], inp["T"], inp["Ni"]
    d["in_S"] = np.zeros((n, 3))
    d["in_lastNP"] = np.zeros(n, np.int32)
    d["in_xij"] = np.zeros((n, 3, fl.nc + 1))
    for k, v in skip_in.items():
        d[f"skipin_{k}"] = v
    for k, v in skip_run.items():
        d[f"skipout_{k}"] = v
    for k in OUT_KEYS:
        d[f"out_{k}"] = r[k]
    d["fragile"] = moved
    for k, v in noise.items():
        d[f"noise_{k}"] = v.astype(np.float32)
    path = os.path.join(HERE, "config1_nc6.npz")
    np.savez_compressed(path, **d)
    print(f"config1_nc6: n={n} two-phase={np.mean(r['NPhc'] == 2):.3f} fragile={moved.sum()} "
          f"size={os.path.getsize(path) / 1e6:.2f} MB")


def main(only=()):
    if not O.available("reference"):
        raise SystemExit("oracle/_ref/libocpref.so missing: run `make -C oracle ref` first")
    if only:
        for name in only:
            {"restart_nc6": restart_case, "impec_nc6": impec_case, "init_nc6": init_case,
             "krpc": krpc_case, "krpc_sof3": krpc_sof3_case, "fimn_nc6": fimn_case,
             "config1_nc6": config1_case}[name]()
        return

    # 1) SPE5 fluid (examples/spe5/EGOIL.in) at 160 degF, the deck's initial composition
    fl = spe5_fluid()
    inp = {"P": np.array([1000.0, 2000.0, 3000.0, 4000.0]), "T": np.full(4, 160.0),
           "Ni": np.tile([500.0, 30, 70, 200, 150, 50, 100], (4, 1))}
    run_case("spe5", fl, inp, note="SPE5 fluid, fresh cells")

    # 2) 6-component synthetic fluid, uniform states (P 5-40 MPa, T 340-400 K,
    #    z ~ Dirichlet(1)); keep every two-phase cell of the first 1536 and
    #    single-phase cells up to 512 in total
    fl = synthetic_fluid(6, 1234)
    inp = synth.uniform_states(fl, 4096, 1234)
    r = O.flash_fim("reference", fl, inp["P"], inp["T"], inp["Ni"], nthreads=8)
    two = np.nonzero(r["NPhc"][:1536] == 2)[0]
    one = np.nonzero(r["NPhc"][:1536] == 1)[0][: max(512 - len(two), 0)]
    keep = np.sort(np.concatenate([two, one]))[:512]
    run_case("uniform_nc6", fl, inp, keep=keep, note="synthetic nc=6 seed 1234, uniform_states seed 1234")

    # 3) warm start: a second FIM step from the first step's state, with P and
    #    Ni perturbed (some cells inside the skip ranges -> ftype 1, two-phase
    #    cells -> ftype 2, the rest -> ftype 0 with the relaxed stability test)
    n = 512
    inp = synth.uniform_states(fl, n, 99)
    skip = O.new_skip(n, fl.nc)
    a = O.flash_fim("reference", fl, inp["P"], inp["T"], inp["Ni"], skip=skip, nthreads=8)
    rng = np.random.default_rng(5)
    scale = np.where(rng.uniform(size=n) < 0.5, 1e-4, 3e-2)
    inp2 = {"P": inp["P"] * (1 + scale * rng.uniform(-1, 1, n)), "T": inp["T"].copy(),
            "Ni": inp["Ni"] * (1 + scale[:, None] * rng.uniform(-1, 1, inp["Ni"].shape)),
            "S": a["S"], "lastNP": a["phaseNum"], "xij": np.nan_to_num(a["xij"], nan=0.0),
            "skip": skip}
    run_case("warm_nc6", fl, inp2, note="second FIM step: warm start, skip cache, perturbed P and Ni")

    # 4) config-3-style fluids: P 2-60 MPa, T 300-450 K, z ~ Dirichlet(0.5)
    for nc, seed in ((3, 31), (9, 91), (12, 121)):
        fl = synthetic_fluid(nc, seed)
        inp = synth.uniform_states(fl, 256, seed, p_mpa=(2.0, 60.0), t_k=(300.0, 450.0), alpha=0.5)
        run_case(f"uniform_nc{nc}", fl, inp, note=f"synthetic nc={nc} seed {seed}, Dirichlet(0.5)")

    # 5) near the phase envelope (P within 5 % of the saturation pressure)
    fl = synthetic_fluid(6, 1234)

    def pc(P, T, Ni):
        return O.flash_fim("reference", fl, P, T, Ni, nthreads=8)["NPhc"]

    inp = synth.near_envelope_states(fl, 256, 2024, pc)
    run_case("near_nc6", fl, inp, note="synthetic nc=6, P = Psat * U(0.95, 1.05)")

    # 6) cells with long split-restart chains
    restart_case()

    # 7) the IMPEC flash, warm-started
    impec_case()

    # 8) the initialisation flashes
    init_case()

    # 9) relative permeability and capillary pressure after the flash
    krpc_case()
    krpc_sof3_case()

    # 10) the FIMn formulation's flash and initialisation
    fimn_case()

    # 11) the CPU-runnable configuration in full (4096 fresh states)
    config1_case()


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
