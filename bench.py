#!/usr/bin/env python
"""Flash throughput benchmark: states/s of the compositional PR FIM flash at
1M cells on B200.

Workload (one "step" = one FIM flash of every cell from a fresh state, i.e.
MixtureComp::FlashFIM with lastNP = 0 and an empty skip cache, plus the
PassFlashValue outputs): the 6-component seeded Peng-Robinson fluid, 1,048,576
states (a 128 x 128 x 64 cell block): 70 % with P ~ U(5, 40) MPa,
T ~ U(340, 400) K, z ~ Dirichlet(1); 30 % within 5 % of the seeded state's
saturation pressure. Synthetic, seeded data (the reference publishes no
dataset).

Output: one JSON line (rank 0). ``value`` is whole-job states/s with inputs
resident in HBM (device time, CUDA events, max over ranks); ``e2e`` is the
same metric through the host-buffer C-ABI call (host<->device copies inside
the timed region); ``roofline`` is the flash kernel against the measured FP64
FMA throughput (its binding pipe), with the HBM view beside it;
``cpu_baseline`` is the reference's own MixtureComp (compiled from its
sources) on a bounded sample on this host's cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--form fast|mixed|batched|plain]

The default form is ``fast``: FP32 successive substitution with FP64 cubic
roots near the discriminant, Rachford-Rice and Newton polish, batched phase
kernels, and the learned initialiser (opencaeporo_b200/models). The line
also carries the plain FP64 GPU form timed on the same states
(``plain_fp64_gpu``) and, on the CPU sample, every output's error against
the FP64 reference.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "flash states/s at 1M cells: mixed+learned vs plain FP64 GPU, err vs FP64 oracle"
NCELL = 1 << 20
from opencaeporo_b200.workload import BISECT_STEPS, SEED  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bench1m", choices=["bench1m", "regions4", "entries"],
                    help="bench1m: the headline 1M-cell workload; regions4: four fluids (3, 6, 9 and 12 "
                         "components, 524,288 states each) flashed together; entries: the initialisation "
                         "and IMPEC entry points on the 1M-cell workload")
    ap.add_argument("--form", default="fast", choices=["plain", "batched", "mixed", "fast"])
    ap.add_argument("--ncell", type=int, default=NCELL)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 form beside the form")
    ap.add_argument("--workload-cache", default=None,
                    help="npz file: load the workload from it if present, else generate and save it")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- workload
from opencaeporo_b200.workload import bench_fluid, gpu_phase_counter, make_workload  # noqa: E402


# ------------------------------------------------------------ reference arm
def bounded_states(O, fl, P, T, Ni, cores, max_steps=60000, max_restarts=150):
    """Indices of the states the reference's own flash is sure to finish on.
    Its PhaseSplit restart loop has no bound; the plain-C restatement bounds
    it at 200 restarts. A state is kept when the restatement needs fewer than
    ``max_steps`` split substitution steps and fewer than ``max_restarts``
    restarts (converging states of the workloads need at most 78)."""
    scr = O.flash_fim("port", fl, P, T, Ni, nthreads=cores)
    return np.nonzero((scr["iters"][:, 2] < max_steps) & (scr["restarts"] < max_restarts))[0]


def reference_arm(args):
    from oracle import oracle as O
    from opencaeporo_b200 import synth
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    fl = bench_fluid()
    kind = "reference" if O.available("reference") else "port"
    cores = os.cpu_count() or 1
    ns = int(min(args.ncell, max(8192, cores * 4000)))

    # The reference's split restart loop has no bound: some states near the
    # critical point (met by the saturation-pressure bisection, and possibly
    # in the sample) make it run without end. The bisection therefore counts
    # phases with the plain-C restatement, which bounds restarts at 200 as the
    # CUDA library does, and the sample leaves out the states it needs
    # >= 60,000 split substitution steps for (a bounded run ends near 80,000;
    # the slowest state of the 1M workload that converges takes ~31,000).
    def pc(P, T, Ni):
        return O.flash_fim("port", fl.with_controls(use_skip=False), P, T, Ni, nthreads=cores)["NPhc"]

    w = synth.mixed_states(fl, ns, SEED, pc, near_frac=0.3, steps=BISECT_STEPS)
    keep = bounded_states(O, fl, w["P"], w["T"], w["Ni"], cores)
    w = {k: w[k][keep] for k in ("P", "T", "Ni")}
    dropped = ns - len(keep)
    ns = len(keep)
    times = []
    for s in range(args.warmup + args.steps):
        r = O.flash_fim(kind, fl, w["P"], w["T"], w["Ni"], nthreads=cores)
        if s >= args.warmup:
            times.append(r["seconds"])
    t = float(np.mean(times))
    v = ns / t
    line = {"metric": METRIC, "value": v, "unit": "states/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": "FIM flash of fresh cells, 6-component PR fluid, 70 % uniform / "
                                   "30 % near-envelope states", "cells_per_step": ns,
                       "full_workload_cells": args.ncell},
            "cpu_baseline": {"value": v, "unit": "states/s", "cores": cores, "kind": kind,
                             "sample": f"{ns} states of the 1M-cell workload distribution per step "
                                       f"({dropped} left out: unbounded restart loop)"},
            "e2e": {"value": v, "unit": "states/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def host_bytes(nc, use_skip):
    from opencaeporo_b200 import _lib
    ins = sum(nf * (4 if dt == "u32" else 8) for nf, dt in _lib.in_shapes(nc).values())
    staged = sum(_lib.out_shapes(nc)[k][0] * 8 for k in
                 ("rho", "xi", "mu", "rhoP", "xiP", "muP", "xij", "rhox", "xix", "mux", "nj"))
    sk = sum(nf * (4 if dt == "u32" else 8) for nf, dt in _lib.skip_shapes(nc).values()) if use_skip else 0
    esz = {"f64": 8, "u32": 4, "i32": 4, "u16": 2, "u8": 1}
    outs = sum(nf * esz[dt] for nf, dt in _lib.out_shapes(nc).values())
    return ins + staged + sk, outs + sk


def our_arm(args):
    import torch
    from opencaeporo_b200 import _lib, roofline, shards
    from opencaeporo_b200.flash import MixtureCompBatch

    world, rank, local = shards.env()
    torch.cuda.set_device(local)
    shards.init("nccl")
    dev = local
    fl = bench_fluid()
    n = args.ncell
    cache = args.workload_cache
    if cache and world == 1 and os.path.exists(cache):
        d = np.load(cache)
        w = {"P": d["P"][:n], "T": d["T"][:n], "Ni": d["Ni"][:n]}
    else:
        w = make_workload(fl, n, shards.shard_seed(SEED, rank), dev)
        if cache and world == 1:
            np.savez(cache, P=w["P"], T=w["T"], Ni=w["Ni"])
    nc = fl.nc

    m = MixtureCompBatch(fl, dev)
    init_note = None
    if args.form == "fast":
        from opencaeporo_b200.learn import DEFAULT_MODEL, Initializer
        if os.path.exists(DEFAULT_MODEL):
            init = Initializer.load(DEFAULT_MODEL)
            init.attach(m)
            init_note = {"model": os.path.relpath(DEFAULT_MODEL, ROOT), "confidence": init.confidence,
                         "train_states": int(init.meta.get("train_states", 0))}
        else:
            init_note = "no trained initialiser found: the fast form ran as the mixed form"
    st = m.new_state(n)
    st.load(w["P"], w["T"], w["Ni"])
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step(ev=None):
        flush.zero_()                       # evict L2 (256 MiB > 126 MB) between steps
        st.skip["flag"].zero_()             # fresh cells: empty skip cache
        if ev is not None:
            ev[0].record(stream)
        m.flash_fim(st, form=args.form, fresh=True)
        if ev is not None:
            ev[1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    shards.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        t0.record(stream)
        for k in range(args.steps):
            step(evs[k])
        t1.record(stream)
        torch.cuda.synchronize()
    shards.barrier()
    ms_total = t0.elapsed_time(t1)
    kern_ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    per_call = m.last_launch_count()  # kernels of one flash call (the replayed sequence)
    res = st.to_host()

    # the plain FP64 GPU form on the same states, for the headline ratio
    plain, plain_res = None, None
    if args.form != "plain" and not args.no_plain:
        pe = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        times = []
        for s_ in range(3):
            flush.zero_()
            st.skip["flag"].zero_()
            pe[0].record(stream)
            m.flash_fim(st, form="plain", fresh=True)
            pe[1].record(stream)
            torch.cuda.synchronize()
            if s_ > 0:
                times.append(pe[0].elapsed_time(pe[1]))
        pms = shards.max_over_ranks([float(np.mean(times))], dev)[0]
        plain = {"value": n / (pms * 1e-3), "unit": "states/s", "ms_per_step": pms,
                 "form_speedup": pms / kern_ms}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            plain_res = st.to_host()
    # every batched form on the same states, split into its parts: the
    # sequence up to the split-restart path, the restart path (the few cells
    # whose split restarts: one dependent chain each), and finalize
    forms = {}
    if not args.no_plain:
        m.set_part_timing(True)
        for fm in ("batched", "mixed", "fast"):
            parts, tot = [], []
            for s_ in range(3):
                flush.zero_()
                st.skip["flag"].zero_()
                m.flash_fim(st, form=fm, fresh=True)
                torch.cuda.synchronize()
                if s_ > 0:
                    parts.append(m.last_phase_ms())
                    tot.append(m.last_kernel_ms())
            p = np.mean(np.array(parts), axis=0)
            forms[fm] = {"ms": float(np.mean(tot)), "to_restart_path_ms": float(p[0]), "restart_path_ms": float(p[1]),
                         "finalize_ms": float(p[2]), "excluding_restart_path_ms": float(p[0] + p[2]),
                         "launch": "direct launches on one stream (part marks); the headline call forks trials 1-3 splits and the learned round onto side streams"}
        m.set_part_timing(False)
    ms_total, kern_ms = shards.max_over_ranks([ms_total, kern_ms], dev)
    ms_step = ms_total / args.steps
    value = world * n / (ms_step * 1e-3)

    # roofline of the flash kernel (work model from the device's iteration counters)
    nphc = res["phaseNum"] - 1
    fl_launch = roofline.flops(nc, res["iters"], nphc)
    by_launch = roofline.batch_bytes(nc, nphc, fl.controls.use_skip)
    fp64_peak = _lib.fma_peak_tflops(dev, 64)
    hbm_peak, hbm_src = hbm_peak_gbs()
    ach_tf = fl_launch / (kern_ms * 1e-3) / 1e12
    ach_gbs = by_launch / (kern_ms * 1e-3) / 1e9
    # DRAM bytes of one flash call from an ncu capture (profiles/): the plain
    # kernel, or the batched sequence of the chosen form
    traffic = None
    tf = os.path.join(ROOT, "profiles", "flash_plain_nc6_traffic.json" if args.form == "plain"
                      else f"flash_phased_nc6_{args.form}_traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("bytes_per_launch_1M")
        except (OSError, ValueError):
            traffic = None

    line = {
        "metric": METRIC, "value": value, "unit": "states/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "FIM flash of fresh cells (lastNP=0, empty skip cache), 6-component PR "
                               "fluid, 1,048,576 states per GPU (128x128x64): 70 % uniform, 30 % within "
                               "5 % of the saturation pressure", "form": args.form, "cells_per_gpu": n,
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"independent shards x{world}",
                   "two_phase_share": float(np.mean(nphc == 2)), "near_envelope_share": 0.3},
        "gpu_launches": args.steps * per_call if per_call > 0 else None,
        "gpu_launches_per_step": per_call,
        "roofline": {"bound": "fp64", "achieved": ach_tf, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": ach_tf / fp64_peak, "traffic": traffic,
                     "peak_source": "FP64 FMA throughput measured in this run (ocpf_measure_fma_peak); "
                                    "MEASURED_PEAKS.json has no FP64 entry",
                     "flops_per_launch": fl_launch, "kernel_ms": kern_ms},
        "roofline_hbm": {"bound": "hbm", "achieved": ach_gbs, "peak": hbm_peak, "unit": "GB/s",
                         "frac": ach_gbs / hbm_peak, "bytes_per_launch": by_launch,
                         "peak_source": hbm_src},
        "plain_fp64_gpu": plain,
        "forms_by_part": forms or None,
        "initializer": init_note,
        "iters_per_cell": {k: float(v) for k, v in zip(("ssmsta", "nrsta", "ssmsp", "nrsp", "rr"),
                                                         res["iters"].mean(axis=0))},
        "status_cells": int(np.count_nonzero(res["status"] & 0xC0)),
    }
    line["clocks"] = clk.summary()

    # ------------------------------------------------ e2e through host buffers
    if not args.no_e2e:
        hs = m.new_host_state(n, pinned=True)
        hs["P"].copy_(torch.as_tensor(w["P"]))
        hs["T"].copy_(torch.as_tensor(w["T"]))
        hs["Ni"].copy_(torch.as_tensor(np.ascontiguousarray(w["Ni"].T)))
        times = []
        for s in range(args.warmup + args.steps):
            hs["skip"]["flag"].zero_()
            hs["out"]["phaseNum"].zero_()
            t_a = time.perf_counter()
            m.flash_fim_host(hs, form=args.form)
            t_b = time.perf_counter()
            if s >= args.warmup:
                times.append(t_b - t_a)
        te = float(np.mean(times))
        te = shards.max_over_ranks([te], dev)[0]
        h2d, d2h = host_bytes(nc, fl.controls.use_skip)
        line["e2e"] = {"value": world * n / te, "unit": "states/s", "h2d_bytes_per_step": h2d * n,
                       "d2h_bytes_per_step": d2h * n, "ms_per_step": te * 1e3,
                       "path": "ocpf_flash_fim_host, pinned host SoA buffers"}
        del hs

    # ------------------------------------------------ CPU baseline (rank 0, N=1)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        forms = {"measured": res}
        if plain_res is not None:
            forms["plain"] = plain_res
        line["cpu_baseline"] = cpu_baseline(fl, w, forms)

    m.close()
    shards.finalize()
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_baseline(fl, w, forms):
    """The reference's own MixtureComp on the first cells of the workload
    with every host thread, and, as a checker, each GPU form's outputs
    (``forms``: {name: host outputs}) against it on those cells.

    Phase counts: a cell whose phase count differs from the reference's is
    "knife-edge" when the reference's own phase count there changes under
    1-ulp input perturbations (oracle.compare.perturbed: 32 trials of P, T
    and Ni moved by 2^-50 relative); any other mismatch is unexplained.

    Other outputs: single-phase cells and two-phase cells whose split
    converged (the reference's ePEC <= 1e-9) are taken as well determined,
    except where the reference's own outputs move by more than 1e-9 relative
    under those perturbations -- measured on every such cell that misses
    1e-8 -- which are ill-determined by the reference's own sensitivity;
    there the bar is 10x that sensitivity."""
    from oracle import compare as CMP
    from oracle import oracle as O
    kind = "reference" if O.available("reference") else "port"
    cores = os.cpu_count() or 1
    ns = int(min(len(w["P"]), max(8192, cores * 4000)))
    # leave out the states the reference's unbounded restart loop may not end
    # on (see reference_arm)
    idx = bounded_states(O, fl, w["P"][:ns], w["T"][:ns], w["Ni"][:ns], cores)
    r = O.flash_fim(kind, fl, w["P"][idx], w["T"][idx], w["Ni"][idx], nthreads=cores)
    dropped = ns - len(idx)
    ns = len(idx)
    errs = {}
    for name, gres in forms.items():
        sub = {k: (v[idx] if isinstance(v, np.ndarray) else v) for k, v in gres.items() if k != "skip"}
        e = CMP.per_cell_errors(sub, r, fl.nc)
        worst = np.zeros(ns)
        for k in CMP.FLOAT_KEYS:
            worst = np.fmax(worst, np.nan_to_num(e[k], nan=0.0))
        errs[name] = (e, worst)
    conv = (r["NPhc"] == 1) | (r["ePEC"] <= 1e-9)
    # cells that need the reference's own sensitivity: every phase-count
    # mismatch, every cell whose split did not converge and every converged
    # cell above 1e-8, in any form
    need = ~conv
    for e, worst in errs.values():
        need = need | ~e["same"] | (e["same"] & conv & (worst > 1e-8))
    cand = np.nonzero(need)[0]
    noise = {k: np.zeros(ns) for k in CMP.FLOAT_KEYS}
    moved = np.zeros(ns, bool)
    if len(cand):
        base = {k: (v[cand] if isinstance(v, np.ndarray) and v.shape[:1] == (ns,) else v) for k, v in r.items()}

        def run_ref(P, T, Ni):
            return O.flash_fim(kind, fl, P, T, Ni, nthreads=min(cores, max(1, len(cand))))
        src = idx[cand]
        nz, mv = CMP.self_noise(run_ref, w["P"][src], w["T"][src], w["Ni"][src], base, fl.nc)
        for k in CMP.FLOAT_KEYS:
            noise[k][cand] = nz[k]
        moved[cand] = mv
    sens = np.zeros(ns)
    for k in CMP.FLOAT_KEYS:
        sens = np.fmax(sens, noise[k])
    out = {"value": ns / r["seconds"], "unit": "states/s", "cores": cores, "kind": kind,
           "sample": f"first {ns + dropped} states of the 1M-cell workload, one flash each, {cores} threads "
                     f"({dropped} left out: the reference's restart loop is unbounded, see bounded_states)"}
    for name, (e, worst) in errs.items():
        same = e["same"]
        mism = np.nonzero(~same)[0]
        unexplained = mism[~moved[mism]]
        det = same & conv & ~(need & (sens > 1e-9))
        ill = same & ~det
        within = np.ones(ns, bool)
        for k in CMP.FLOAT_KEYS:
            within &= np.nan_to_num(e[k], nan=0.0) <= np.maximum(1e-8, 10 * noise[k])
        recl = np.nonzero(same & conv & need & (sens > 1e-9))[0]
        per_output = {k: float(np.max(np.nan_to_num(e[k][det], nan=0.0), initial=0.0)) for k in CMP.FLOAT_KEYS}
        out["parity_on_sample" if name == "measured" else f"parity_on_sample_{name}"] = {
            "cells": ns,
            "phase_count_mismatches": int(len(mism)),
            "knife_edge_mismatches": int(len(mism) - len(unexplained)),
            "unexplained_phase_mismatches": int(len(unexplained)),
            "unexplained_cells": [int(idx[c]) for c in unexplained[:16]],
            "well_determined_cells": int(det.sum()),
            "max_rel_err_well_determined": float(np.max(worst[det], initial=0.0)),
            "well_determined_above_1e-8": int(np.count_nonzero(det & (worst > 1e-8))),
            "max_rel_err_per_output_well_determined": per_output,
            "ill_determined_cells": int(ill.sum()),
            "ill_determined_within_10x_reference_sensitivity": int(np.count_nonzero(ill & within)),
            "converged_cells_reclassified_by_sensitivity": [
                {"cell": int(idx[c]), "max_rel_err": float(worst[c]), "reference_1ulp_sensitivity": float(sens[c])}
                for c in recl[:12]],
            "converged_cells_reclassified_count": int(len(recl)),
            "metric": "max over outputs of |gpu-ref|/max(|ref|, 1e-12 field scale); dSec_dPri entries "
                      "against max(|ref|, 1e-4 column scale)"}
    return out


def regions_arm(args):
    """The batched uneven workload: four PVT regions of 3, 6, 9 and 12
    components, 524,288 seeded states each (P 2-60 MPa, T 300-450 K,
    z ~ Dirichlet(0.5): iteration counts from 2 to 200+), flashed by one
    ocpf_flash_fim_regions call -- one launch sequence over all four fluids,
    replayed from a CUDA graph, with the launch shape the autotuner picks --
    against the same call with one sequence per region on the regions'
    streams, one call per region in turn, and the plain FP64 form; on the
    first states of every fluid, each region's outputs against the
    reference's own MixtureComp. One JSON line; not the headline metric."""
    import torch
    from oracle import compare as CMP
    from oracle import oracle as O
    from opencaeporo_b200 import synth
    from opencaeporo_b200.flash import MixtureCompBatch, autotune, flash_fim_regions
    from opencaeporo_b200.fluid import synthetic_fluid
    per = args.ncell // 2
    t_start = time.time()

    def note(what):  # progress on stderr: the arm runs for minutes
        print(f"[regions4 {time.time() - t_start:7.1f} s] {what}", file=sys.stderr, flush=True)
    regs, wls = [], []
    for nc, seed in ((3, 31), (6, 61), (9, 91), (12, 121)):
        fl = synthetic_fluid(nc, seed)
        w = synth.uniform_states(fl, per, seed, p_mpa=(2.0, 60.0), t_k=(300.0, 450.0), alpha=0.5)
        m = MixtureCompBatch(fl, 0)
        st = m.new_state(per)
        st.load(w["P"], w["T"], w["Ni"])
        regs.append((m, st))
        wls.append((fl, w))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fn, steps=args.steps):
        ts = []
        for s_ in range(args.warmup + steps):
            flush.zero_()
            for _, st in regs:
                st.skip["flag"].zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            if s_ >= args.warmup:
                ts.append(a.elapsed_time(b))
        return float(np.mean(ts))

    note("states loaded")
    form = args.form
    lead = regs[0][0]
    lead.set_tuning(schedule=0)
    t_one_default = timed(lambda: flash_fim_regions(regs, form=form, fresh=True))
    note(f"one launch {t_one_default:.1f} ms")
    lead.set_tuning(schedule=1)
    t_streams_default = timed(lambda: flash_fim_regions(regs, form=form, fresh=True))
    note(f"streams {t_streams_default:.1f} ms")
    best = autotune(regs, form=form, reps=1)
    note(f"autotuned {best}")
    t_tuned = timed(lambda: flash_fim_regions(regs, form=form, fresh=True))
    note(f"tuned {t_tuned:.1f} ms")
    t_serial = timed(lambda: [m.flash_fim(st, form=form, fresh=True) for m, st in regs])
    note(f"one call per region {t_serial:.1f} ms")
    t_plain = timed(lambda: [m.flash_fim(st, form="plain", fresh=True) for m, st in regs], steps=1)
    note(f"plain {t_plain:.1f} ms")
    # outputs of the tuned call, and each fluid's first states against the reference
    flash_fim_regions(regs, form=form, fresh=True)
    torch.cuda.synchronize()
    total = per * len(regs)
    per_fluid = []
    cores = os.cpu_count() or 1
    ns = min(per, 4096)
    for (m, st), (fl, w) in zip(regs, wls):
        got = st.to_host()
        # leave out the states the reference's unbounded restart loop may not
        # end on: those the bounded restatement needs >= 60,000 split steps
        # for (see reference_arm)
        note(f"nc={fl.nc}: screening the reference sample")
        ix = bounded_states(O, fl, w["P"][:ns], w["T"][:ns], w["Ni"][:ns], cores)
        wv = {k: w[k][ix] for k in ("P", "T", "Ni")}
        sub = {k: v[ix] for k, v in got.items() if isinstance(v, np.ndarray)}
        note(f"nc={fl.nc}: reference on {len(ix)} states")
        ref = O.flash_fim("reference" if O.available("reference") else "port", fl, wv["P"], wv["T"], wv["Ni"],
                          nthreads=cores)
        left_out = ns - len(ix)
        ns_k = len(ix)
        e = CMP.per_cell_errors(sub, ref, fl.nc)
        worst = np.zeros(ns_k)
        for k in CMP.FLOAT_KEYS:
            worst = np.fmax(worst, np.nan_to_num(e[k], nan=0.0))
        conv = (ref["NPhc"] == 1) | (ref["ePEC"] <= 1e-9)
        mism = np.nonzero(~e["same"])[0]
        # knife-edge test of every phase-count mismatch and sensitivity of
        # the converged cells above 1e-8 (the bar of the headline line)
        need = np.nonzero(~e["same"] | (e["same"] & conv & (worst > 1e-8)))[0]
        moved = np.zeros(ns_k, bool)
        sens = np.zeros(ns_k)
        if len(need):
            base = {k: (v[need] if isinstance(v, np.ndarray) and v.shape[:1] == (ns_k,) else v)
                    for k, v in ref.items()}

            def run_ref(P, T, Ni):
                return O.flash_fim("reference" if O.available("reference") else "port", fl, P, T, Ni,
                                   nthreads=min(cores, len(need)))
            nz, mv = CMP.self_noise(run_ref, wv["P"][need], wv["T"][need], wv["Ni"][need], base, fl.nc)
            moved[need] = mv
            for k in CMP.FLOAT_KEYS:
                sens[need] = np.fmax(sens[need], nz[k])
        det = e["same"] & conv & ~(sens > 1e-9)
        per_fluid.append({"nc": fl.nc, "two_phase_share": float(np.mean(got["phaseNum"] == 3)),
                          "sample": int(ns_k), "left_out_unbounded_restarts": int(left_out),
                          "phase_count_mismatches": int(len(mism)),
                          "unexplained_phase_mismatches": int(np.count_nonzero(~moved[mism])),
                          "well_determined_cells": int(det.sum()),
                          "max_rel_err_well_determined": float(np.max(worst[det], initial=0.0)),
                          "max_iterations_ssmsp": int(got["iters"][:, 2].max())})
    for m, _ in regs:
        m.close()
    print(json.dumps({
        "metric": "flash states/s, four fluids (NC 3/6/9/12) in one call", "value": total / (t_tuned * 1e-3),
        "unit": "states/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_tuned,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded)", "form": form,
        "config": {"workload": "4 fluids x 524,288 states, P 2-60 MPa, T 300-450 K, z ~ Dirichlet(0.5)",
                   "l2": "flushed between steps (256 MiB write)"},
        "autotuned": best,
        "one_launch_default_shape": {"value": total / (t_one_default * 1e-3), "ms_per_step": t_one_default},
        "streams_default_shape": {"value": total / (t_streams_default * 1e-3), "ms_per_step": t_streams_default},
        "one_call_per_region_in_turn": {"value": total / (t_serial * 1e-3), "ms_per_step": t_serial},
        "plain_fp64_per_region": {"value": total / (t_plain * 1e-3), "ms_per_step": t_plain},
        "parity_per_fluid": per_fluid}), flush=True)


def hbm_peak_gbs():
    """(peak HBM GB/s, its source): the measured copy bandwidth of this
    pool's B200s from MEASURED_PEAKS.json, else the earlier pool measurement
    of 6650 GB/s, labelled as the fallback."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), \
            "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "6650 GB/s (of fallback: MEASURED_PEAKS.json absent)"


def entries_arm(args):
    """The other flash entry points on the bench workload (1,048,576 fresh
    states of the 6-component fluid): ocpf_init_flash_fim (InitFlashFIM:
    the initial mole fractions z = Ni / sum Ni, S_w ~ U(0.05, 0.5), pore
    volumes ~ U(50, 5000) ft3), ocpf_flash_impec (FlashIMPEC of fresh
    cells) and ocpf_flash_fimn (FlashFIMn of fresh cells), each in the
    chosen form and in the plain FP64 form, timed with CUDA events; the
    reference's own calls on the first states with every host thread, and
    the error of the chosen form against them. One JSON line; not the
    headline metric."""
    import torch
    from oracle import compare as CMP
    from oracle import oracle as O
    from opencaeporo_b200.flash import MixtureCompBatch
    fl = bench_fluid()
    n = args.ncell
    cache = args.workload_cache
    if cache and os.path.exists(cache):
        d = np.load(cache)
        w = {"P": d["P"][:n], "T": d["T"][:n], "Ni": d["Ni"][:n]}
    else:
        w = make_workload(fl, n, SEED, 0)
        if cache:
            np.savez(cache, P=w["P"], T=w["T"], Ni=w["Ni"])
    nc = fl.nc
    z = w["Ni"] / w["Ni"][:, :nc].sum(axis=1, keepdims=True)
    z[:, nc] = 0.0
    rng = np.random.default_rng(SEED + 1)
    S = np.zeros((n, 3))
    S[:, 2] = rng.uniform(0.05, 0.5, n)
    S[:, 0] = 1 - S[:, 2]
    Vp = rng.uniform(50.0, 5000.0, n)
    m = MixtureCompBatch(fl, 0)
    if args.form == "fast":
        from opencaeporo_b200.learn import DEFAULT_MODEL, Initializer
        Initializer.load(DEFAULT_MODEL).attach(m)
    st = m.new_state(n)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    Pt = torch.as_tensor(w["P"]).cuda()
    Tt = torch.as_tensor(w["T"]).cuda()
    Zt = torch.as_tensor(np.ascontiguousarray(z.T)).cuda()
    Nt = torch.as_tensor(np.ascontiguousarray(w["Ni"].T)).cuda()
    St = torch.as_tensor(np.ascontiguousarray(S.T)).cuda()
    Vt = torch.as_tensor(Vp).cuda()

    def timed(prep, call):
        ts = []
        for s_ in range(args.warmup + args.steps):
            flush.zero_()
            prep()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            call()
            b.record(stream)
            torch.cuda.synchronize()
            if s_ >= args.warmup:
                ts.append(a.elapsed_time(b))
        return float(np.mean(ts))

    def prep_init():
        st.P.copy_(Pt)
        st.T.copy_(Tt)
        st.Ni.copy_(Zt)
        st.out["S"].copy_(St)
        st.skip["flag"].zero_()

    def prep_impec():
        st.P.copy_(Pt)
        st.T.copy_(Tt)
        st.Ni.copy_(Nt)
        st.skip["flag"].zero_()

    res = {}
    for name, prep, call in (
            ("init_flash_fim", prep_init, lambda f: m.init_flash(st, Vt, form=f)),
            ("flash_impec", prep_impec, lambda f: m.flash_impec(st, form=f, fresh=True)),
            ("flash_fimn", prep_impec, lambda f: m.flash_fimn(st, form=f, fresh=True))):
        t_form = timed(prep, lambda: call(args.form))
        gpu = st.to_host()
        if name == "init_flash_fim":
            gpu["Ni"] = st.Ni.cpu().numpy().T.copy()
        t_plain = timed(prep, lambda: call("plain"))
        cores = os.cpu_count() or 1
        ns0 = int(min(n, max(8192, cores * 4000)))
        # states the reference's unbounded restart loop may not end on are
        # left out (see reference_arm)
        ix = bounded_states(O, fl, w["P"][:ns0], w["T"][:ns0], w["Ni"][:ns0], cores)
        ns = len(ix)
        if name == "init_flash_fim":
            ref = O.init_flash(fl, w["P"][ix], w["T"][ix], z[ix], S[ix], Vp[ix], nthreads=cores)
            sub = {k: v[ix] for k, v in gpu.items() if isinstance(v, np.ndarray)}
            e = CMP.per_cell_errors(sub, ref, nc)
            keys = CMP.FLOAT_KEYS
        elif name == "flash_fimn":
            ref = O.flash_fimn(fl, w["P"][ix], w["T"][ix], w["Ni"][ix], nthreads=cores)
            sub = {k: v[ix] for k, v in gpu.items() if isinstance(v, np.ndarray)}
            e = CMP.fimn_errors(sub, ref, nc)
            keys = CMP.FLOAT_KEYS + ("nj",)  # res, resPc: residuals, determined only to rounding
        else:
            ref = O.flash_impec(fl, w["P"][ix], w["T"][ix], w["Ni"][ix], nthreads=cores)
            sub = {k: v[ix] for k, v in gpu.items() if isinstance(v, np.ndarray)}
            e = CMP.impec_errors(sub, ref, nc)
            keys = CMP.IMPEC_FLOAT_KEYS
        worst = np.zeros(ns)
        for k in keys:
            worst = np.fmax(worst, np.nan_to_num(e[k], nan=0.0))
        det = e["same"] & ((ref["NPhc"] == 1) | (ref["ePEC"] <= 1e-9))
        res[name] = {
            "value": n / (t_form * 1e-3), "unit": "states/s", "ms_per_step": t_form, "form": args.form,
            "plain_fp64_gpu": {"value": n / (t_plain * 1e-3), "ms_per_step": t_plain},
            "reference_cpu": {"value": ns / ref["seconds"], "unit": "states/s", "cores": cores,
                              "sample": f"first {ns0} states, one call each ({ns0 - ns} left out: "
                                        f"unbounded restart loop)"},
            "parity_on_sample": {"cells": ns, "phase_count_mismatches": int(np.count_nonzero(~e["same"])),
                                 "well_determined_cells": int(det.sum()),
                                 "share_well_determined_le_1e-8": float(np.mean(worst[det] <= 1e-8))}}
    # relative permeability and capillary pressure of the flash's S in place
    # (ocpf_cal_krpc, FlowUnit_ODGW01 on two synthetic regions); HBM-bound
    from oracle import krpc as KO
    from opencaeporo_b200 import synth
    from opencaeporo_b200.krpc import FlowUnitBatch
    regions = [synth.corey_tables(501), synth.corey_tables(502, swc=0.2, sorw=0.15, nrow=9, pc_scale=(8.0, 3.0))]
    fu = FlowUnitBatch(regions)
    satnum = torch.as_tensor(np.random.default_rng(SEED + 2).integers(0, 2, n).astype(np.int32)).cuda()
    kout = fu.new_outputs(n)
    t_k = timed(lambda: None, lambda: fu.cal_krpc(st.P, st.out["S"], satnum, out=kout))
    ns = min(n, 65536)
    Sh = st.out["S"][:, :ns].cpu().numpy().T.copy()
    sh = satnum[:ns].cpu().numpy()
    want = KO.reference(regions, w["P"][:ns], Sh, sh, nthreads=os.cpu_count() or 1)
    exact = all(np.array_equal(kout[k][:, :ns].cpu().numpy().T, want[k])
                for k in ("kr", "Pc", "Pj", "dKr_dS", "dPcj_dS"))
    kbytes = n * (8 + 24 + 4 + 3 * 24 + 2 * 72)
    peak, peak_src = hbm_peak_gbs()
    res["cal_krpc"] = {
        "value": n / (t_k * 1e-3), "unit": "cells/s", "ms_per_step": t_k,
        "roofline": {"bound": "hbm", "achieved": kbytes / (t_k * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": (kbytes / (t_k * 1e-3) / 1e9 / peak) if peak else None,
                     "bytes_per_launch": kbytes, "peak_source": peak_src},
        "reference_cpu": {"value": ns / want["seconds"], "unit": "cells/s", "cores": os.cpu_count() or 1,
                          "sample": f"first {ns} cells"},
        "bit_identical_on_sample": bool(exact)}
    # the Jacobian's bulk part after a FIM flash and KrPc, on the bench grid
    # (128 x 128 x 64 bulks, 7-point connections): upwind and assembly
    from opencaeporo_b200.fim_jacobian import ConnGraph
    nx, ny, nz = 128, 128, 64
    if n == nx * ny * nz:
        st.P.copy_(Pt)
        st.T.copy_(Tt)
        st.Ni.copy_(Nt)
        st.skip["flag"].zero_()
        m.flash_fim(st, form=args.form, fresh=True)
        fu.cal_krpc(st.P, st.out["S"], satnum, out=kout)
        grid = np.arange(n, dtype=np.int64).reshape(nz, ny, nx)
        cb, ce = [], []
        for axis in (2, 1, 0):
            cb.append(np.take(grid, range(grid.shape[axis] - 1), axis=axis).ravel())
            ce.append(np.take(grid, range(1, grid.shape[axis]), axis=axis).ravel())
        cb, ce = np.concatenate(cb), np.concatenate(ce)
        rng2 = np.random.default_rng(SEED + 3)
        g = ConnGraph(n, cb, ce, rng2.uniform(100.0, 400.0, len(cb)))
        bulk = {k: st.out[k] for k in ("phaseExist", "pSderExist", "pVnumCom", "S", "rho", "xi", "mu", "muP", "xiP",
                                       "rhoP", "xij", "rhox", "xix", "mux", "dSec_dPri", "vfP", "vfi")}
        bulk.update({"kr": kout["kr"], "Pj": kout["Pj"], "dKr_dS": kout["dKr_dS"], "dPcj_dS": kout["dPcj_dS"],
                     "v": torch.as_tensor(rng2.uniform(5e3, 5e4, n)).cuda(),
                     "poroP": torch.as_tensor(rng2.uniform(1e-6, 1e-5, n)).cuda(),
                     "depth": torch.as_tensor(np.repeat(np.arange(nz) * 10.0 + 8000.0, nx * ny)).cuda()})
        up, urho = g.upwind(bulk)
        jout = g.jacobian(nc, 1.0, bulk, up, urho)
        t_up = timed(lambda: None, lambda: g.upwind(bulk))
        t_jac = timed(lambda: None, lambda: g.jacobian(nc, 1.0, bulk, up, urho, out=jout))
        torch.cuda.synchronize()
        finite = bool(torch.isfinite(jout["diag"]).all().item() and torch.isfinite(jout["offEB"]).all().item())
        ncol = nc + 2
        nconn = len(cb)
        # algorithmic bytes: each bulk's inputs once, each connection's ends,
        # area and upstream data, the two off-diagonal blocks and the diagonal
        rows = st.out["bRowSizedSdP"].double().sum().item()
        per_bulk_in = 4 * 9 + 8 * (7 * 3 + 4 * 3 * (nc + 1) + (nc + 1) + 1 + 3 * 2 + 9 * 2 + 3)
        jbytes = n * per_bulk_in + 8 * ncol * rows + nconn * (8 * 3 + 3 * 12) + 8 * ncol * ncol * (2 * nconn + n)
        res["fim_jacobian"] = {
            "value": nconn / (t_jac * 1e-3), "unit": "connections/s", "ms_per_step": t_jac,
            "connections": nconn, "bulks": n, "upwind_ms": t_up, "finite": finite,
            "roofline": {"bound": "hbm", "achieved": jbytes / (t_jac * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": (jbytes / (t_jac * 1e-3) / 1e9 / peak) if peak else None,
                         "bytes_per_launch": jbytes, "peak_source": peak_src},
            "parity": "bit-identical to the restatement on the 8x8x8 test grid (tests/test_fim_jacobian.py)"}
        g.close()
    # the last-time-step copies of the flash's arrays and the skip cache
    # (IsoT_FIM::UpdateLastTimeStep / ResetToLastTimeStep): one copy launch,
    # HBM-bound (each byte read once and written once)
    last = m.new_last(st)
    t_save = timed(lambda: None, lambda: m.update_last_step(st, last, inputs=False))
    t_reset = timed(lambda: None, lambda: m.reset_to_last_step(st, last, inputs=False))
    torch.cuda.synchronize()
    bits = lambda x, y: torch.equal(x.view(torch.uint8), y.view(torch.uint8))  # NaN-safe
    same = all(bits(st.out[k], last.out[k]) for k in st.out) and all(bits(st.skip[k], last.skip[k]) for k in st.skip)
    cbytes = sum(t.numel() * t.element_size() for t in list(st.out.values()) + list(st.skip.values()))
    res["update_last_step"] = {
        "value": n / (t_save * 1e-3), "unit": "cells/s", "ms_per_step": t_save, "reset_ms": t_reset,
        "identical_after_copy": bool(same),
        "roofline": {"bound": "hbm", "achieved": 2 * cbytes / (t_save * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": (2 * cbytes / (t_save * 1e-3) / 1e9 / peak) if peak else None,
                     "bytes_per_launch": 2 * cbytes, "peak_source": peak_src}}
    del last
    fu.close()
    m.close()
    print(json.dumps({
        "metric": "flash states/s of the initialisation and IMPEC entry points", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "1,048,576 states of the bench workload; init: z = Ni / sum Ni, "
                               "S_w ~ U(0.05, 0.5), Vpore ~ U(50, 5000) ft3; IMPEC: fresh cells",
                   "l2": "flushed between steps (256 MiB write)"},
        "entries": res}), flush=True)


def main():
    args = parse()
    if args.workload == "regions4":
        regions_arm(args)
        return
    if args.workload == "entries":
        entries_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args)
        return
    our_arm(args)


if __name__ == "__main__":
    main()
