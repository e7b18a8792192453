"""The flash inside a synthetic FIM loop: the 60 x 220 x 85 case.

A stand-in for the simulator around the flash (grid, wells, linear solver
and time stepping are outside this path). Per Newton iteration it produces
every cell's (P, T, Ni) the way a FIM iteration moves them -- fields that
change a little between iterations and more between time steps, a gas front
spreading from one injector and pressure drawn down at four producers --
and calls the flash on device-resident cell state with the previous
iteration's results as warm start (phase count, S, xij and the skip cache),
as ``IsoT_FIM::CalFlash`` does over the bulk (src/OCPFluidMethod.cpp:1108-1120).

Grid 60 x 220 x 85 = 1,122,000 cells; permeability log-normal (mean ln k = 3,
sigma 2, mD), porosity U(0.05, 0.35); 6-component fluid of the workload;
20 time steps x 4 Newton iterations.

    python -m opencaeporo_b200.fim_loop [--forms plain,fast] [--steps 20] [--newton 4]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def _torch():
    import torch
    return torch


class SyntheticFIM:
    """Seeded reservoir block and the per-iteration cell inputs it yields
    (device tensors: P [n] psia, T [n] degF, Ni [numCom, n] lbmol)."""

    def __init__(self, fluid, nx=60, ny=220, nz=85, seed=11, device=0):
        torch = _torch()
        self.dev = torch.device("cuda", device)
        self.shape = (nz, ny, nx)
        self.n = nx * ny * nz
        self.nc = fluid.nc
        rng = np.random.default_rng(seed)
        lnk = rng.normal(3.0, 2.0, self.shape)                    # ln(k / mD)
        poro = rng.uniform(0.05, 0.35, self.shape)
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        depth = 8000.0 + 2.0 * z                                  # ft, 2 ft layers
        self.P0 = 3000.0 + 0.35 * (depth - 8000.0)                # psia, hydrostatic
        self.T = np.full(self.shape, 160.0)                       # degF
        # wells: one injector, four producers (columns through all layers)
        inj = (ny // 2, 2)
        prods = [(5, nx - 3), (ny - 6, nx - 3), (5, nx // 2), (ny - 6, nx // 2)]
        # distance to a well, stretched by the local permeability (fast paths
        # feel the wells first)
        kfac = np.exp(0.25 * (lnk - 3.0))
        d_inj = np.hypot(y - inj[0], x - inj[1]) / kfac
        d_prod = np.min([np.hypot(y - py, x - px) for py, px in prods], axis=0) / kfac
        self.d_inj, self.d_prod = d_inj, d_prod
        # reservoir fluid and injected gas compositions (lightest components
        # are the first ones of the synthetic fluid: ordered by Tc)
        order = np.argsort(fluid.Tc)
        z0 = np.array([0.30, 0.10, 0.12, 0.15, 0.18, 0.15])[: self.nc]
        zi = np.array([0.80, 0.12, 0.05, 0.02, 0.005, 0.005])[: self.nc]
        self.z_res = np.empty(self.nc); self.z_res[order] = z0 / z0.sum()
        self.z_inj = np.empty(self.nc); self.z_inj[order] = zi / zi.sum()
        self.pv = poro * 1000.0                                   # ft3 of pore volume per cell
        self.noise = rng.normal(0.0, 1.0, self.shape)
        self.lnk, self.poro, self.depth = lnk, poro, depth

    def connections(self):
        """7-point connections (begin, end, area): x, y and z neighbours,
        area = harmonic mean permeability (mD) x 1 ft^2 face."""
        idx = np.arange(self.n, dtype=np.int64).reshape(self.shape)
        k = np.exp(self.lnk)
        b, e, a = [], [], []
        for axis in (2, 1, 0):
            lo = [slice(None)] * 3
            hi = [slice(None)] * 3
            lo[axis] = slice(0, self.shape[axis] - 1)
            hi[axis] = slice(1, self.shape[axis])
            lo, hi = tuple(lo), tuple(hi)
            b.append(idx[lo].ravel())
            e.append(idx[hi].ravel())
            a.append((2 * k[lo] * k[hi] / (k[lo] + k[hi])).ravel())
        return np.concatenate(b), np.concatenate(e), np.concatenate(a)

    def _fields(self, t):
        """(P, z) at time t (fractional time steps)."""
        P = self.P0 + 1500.0 * (1 - np.exp(-t / 6.0)) * np.exp(-self.d_inj / 25.0) \
            - 1200.0 * (1 - np.exp(-t / 4.0)) * np.exp(-self.d_prod / 18.0) + 3.0 * self.noise
        front = 8.0 * t
        phi = 1.0 / (1.0 + np.exp((self.d_inj - front) / 3.0))
        z = (1 - phi)[..., None] * self.z_res + phi[..., None] * self.z_inj
        return P, z

    def inputs(self, step, it, newton):
        """Cell inputs of Newton iteration `it` of time step `step`: the
        iterates approach the step's solution geometrically."""
        torch = _torch()
        Pa, za = self._fields(step)
        Pb, zb = self._fields(step + 1)
        w = 1.0 - 0.5 ** (it + 1)
        P = Pa + w * (Pb - Pa)
        z = za + w * (zb - za)
        nt = self.pv * P / (10.73 * (self.T + 459.67)) * 1.2     # lbmol hydrocarbon per cell
        Ni = np.empty(self.shape + (self.nc + 1,))
        Ni[..., : self.nc] = z * nt[..., None]
        Ni[..., self.nc] = 0.2 * self.pv * 3.4                   # water
        P_t = torch.as_tensor(P.reshape(-1), device=self.dev)
        T_t = torch.as_tensor(self.T.reshape(-1), device=self.dev)
        N_t = torch.as_tensor(np.ascontiguousarray(Ni.reshape(-1, self.nc + 1).T), device=self.dev)
        return P_t, T_t, N_t


def _gather(st, idx):
    """Host copies of a cell sample's inputs, warm-start state and outputs."""
    o = st.out
    return {"P": st.P[idx].cpu().numpy(), "T": st.T[idx].cpu().numpy(),
            "Ni": st.Ni[:, idx].cpu().numpy().T.copy(),
            "S": o["S"][:, idx].cpu().numpy().T.copy(), "lastNP": o["phaseNum"][idx].cpu().numpy().astype(np.int32),
            "xij": o["xij"][:, idx].cpu().numpy().T.copy(),
            "skip": {k: (v[idx] if v.dim() == 1 else v[:, idx].T).cpu().numpy().copy() for k, v in st.skip.items()},
            "out": {k: (v[idx] if v.dim() == 1 else v[:, idx].T).cpu().numpy().copy() for k, v in o.items()}}


def run(forms=("plain", "fast"), steps=20, newton=4, device=0, log=print, grid=(60, 220, 85), hook=None,
        sample=4096, seed=5, chain=True):
    """Runs the loop once per form in lockstep on identical inputs; returns
    per-iteration flash times and, for every form other than the first,
    phase-count differences and output errors against the first. With
    ``hook``, for a seeded sample of ``sample`` cells every iteration calls
    hook(form, step, it, before, after): the sample's inputs and warm-start
    state before the flash and its outputs after (host arrays, cell-major),
    e.g. to check them against an oracle. With ``chain``, after the last
    form's flash every iteration also runs what IsoT_FIM does next on the
    same device arrays -- KrPc (ocpf_cal_krpc), the upstream choice and the
    Jacobian's bulk part (ocpf_fim_upwind, ocpf_fim_jacobian) -- and their
    times are reported."""
    torch = _torch()
    from .flash import MixtureCompBatch
    from .workload import bench_fluid
    fl = bench_fluid()
    drv = SyntheticFIM(fl, nx=grid[0], ny=grid[1], nz=grid[2], device=device)
    ctx = []
    for form in forms:
        m = MixtureCompBatch(fl, device)
        if form == "fast":
            from .learn import DEFAULT_MODEL, Initializer
            Initializer.load(DEFAULT_MODEL).attach(m)
        st = m.new_state(drv.n)
        ctx.append((form, m, st))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in forms]
    idx = None
    if hook is not None:
        idx = torch.as_tensor(np.sort(np.random.default_rng(seed).choice(drv.n, min(sample, drv.n), replace=False)),
                              device=drv.dev)
    rec = {f: [] for f in forms}
    acc = {f: [] for f in forms[1:]}
    chain_ms = {"krpc": [], "upwind": [], "jacobian": []}
    if chain:
        from . import synth
        from .fim_jacobian import ConnGraph
        from .krpc import FlowUnitBatch
        cst = ctx[-1][2]
        fu = FlowUnitBatch([synth.corey_tables(501)], device)
        kout = fu.new_outputs(drv.n)
        cb, ce, ca = drv.connections()
        graph = ConnGraph(drv.n, cb, ce, ca, device)
        bulk = {k: cst.out[k] for k in ("phaseExist", "pSderExist", "pVnumCom", "S", "rho", "xi", "mu", "muP",
                                        "xiP", "rhoP", "xij", "rhox", "xix", "mux", "dSec_dPri", "vfP", "vfi")}
        bulk.update({"kr": kout["kr"], "Pj": kout["Pj"], "dKr_dS": kout["dKr_dS"], "dPcj_dS": kout["dPcj_dS"],
                     "v": torch.full((drv.n,), 1000.0, dtype=torch.float64, device=drv.dev),
                     "poroP": torch.as_tensor(3e-6 * drv.poro.reshape(-1), device=drv.dev),
                     "depth": torch.as_tensor(drv.depth.reshape(-1).astype(np.float64), device=drv.dev)})
        cev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        jout = None
    for step in range(steps):
        for it in range(newton):
            P, T, N = drv.inputs(step, it, newton)
            before = {}
            for k, (form, m, st) in enumerate(ctx):
                st.P.copy_(P); st.T.copy_(T); st.Ni.copy_(N)
                if hook is not None:
                    before[form] = _gather(st, idx)
                ev[k][0].record()
                m.flash_fim(st, form=form)
                ev[k][1].record()
            if chain:
                cev[0].record()
                fu.cal_krpc(cst.P, cst.out["S"], None, out=kout)
                cev[1].record()
                up, urho = graph.upwind(bulk)
                cev[2].record()
                jout = graph.jacobian(drv.nc, 1.0, bulk, up, urho, out=jout)
                cev[3].record()
            torch.cuda.synchronize()
            if chain:
                for key, a_, b_ in (("krpc", 0, 1), ("upwind", 1, 2), ("jacobian", 2, 3)):
                    chain_ms[key].append(cev[a_].elapsed_time(cev[b_]))
            if hook is not None:
                for form, m, st in ctx:
                    hook(form, step, it, before[form], _gather(st, idx)["out"])
            for k, (form, m, st) in enumerate(ctx):
                rec[form].append(ev[k][0].elapsed_time(ev[k][1]))
            base = ctx[0][2].out
            for form, m, st in ctx[1:]:
                o = st.out
                mism = int((o["phaseNum"] != base["phaseNum"]).sum())
                # outputs of phases present in both (absent phases' outputs
                # are left untouched by the flash, as in the reference)
                ex = (o["phaseExist"] == base["phaseExist"]).all(dim=0) & (o["phaseNum"] == base["phaseNum"])
                err = 0.0
                for key, per in (("S", 1), ("rho", 1), ("xi", 1), ("mu", 1), ("xij", fl.nc + 1)):
                    a, b = o[key], base[key]
                    for j in range(3):
                        msk = ex & (base["phaseExist"][j] > 0)
                        if not bool(msk.any()):
                            continue
                        rows = slice(j * per, (j + 1) * per)
                        aa, bb = a[rows][:, msk], b[rows][:, msk]
                        d = (aa - bb).abs() / bb.abs().clamp_min(1e-10)
                        err = max(err, float(torch.nan_to_num(d, nan=0.0).max()))
                acc[form].append({"phase_mismatch": mism, "max_rel_err": err})
        log(f"step {step}: " + ", ".join(f"{f} {np.mean(rec[f][-newton:]):.1f} ms" for f in forms))
    for _, m, _ in ctx:
        m.close()
    if chain:
        finite = bool(torch.isfinite(jout["diag"]).all().item())
        graph.close()
        fu.close()
    out = {"cells": drv.n, "steps": steps, "newton": newton,
           "ms_per_iteration": {f: float(np.mean(v)) for f, v in rec.items()},
           "ms_per_iteration_first": {f: float(v[0]) for f, v in rec.items()},
           "ms_per_iteration_after_first": {f: float(np.mean(v[1:])) for f, v in rec.items()}}
    if chain:
        out["after_flash_ms_per_iteration"] = {k: float(np.mean(v)) for k, v in chain_ms.items()}
        out["after_flash_form"] = forms[-1]
        out["jacobian_finite"] = finite
    for f, v in acc.items():
        out[f"{f}_vs_{forms[0]}"] = {"max_phase_mismatch": max(a["phase_mismatch"] for a in v),
                                     "max_rel_err": max(a["max_rel_err"] for a in v)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--forms", default="plain,batched,fast")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--newton", type=int, default=4)
    args = ap.parse_args()
    t0 = time.time()
    res = run(tuple(args.forms.split(",")), args.steps, args.newton)
    res["wall_s"] = time.time() - t0
    print(json.dumps(res))


if __name__ == "__main__":
    main()
