"""The benchmark workload: the 6-component synthetic PR fluid and seeded
states of the 1,048,576-cell block (70 % uniform in P 5-40 MPa, T 340-400 K,
z ~ Dirichlet(1); 30 % within 5 % of the saturation pressure found by
bisection on the phase count of the batched GPU flash).

The bisection is the only part of a state that depends on a flash. For the
benchmark's own block (seed SEED, NCELL cells) its outcome is frozen in
``workloads/bench1m_near_envelope.npz`` -- the accepted candidates and their
saturation pressures, recorded once with ``record()`` -- and replayed, so
that the benchmark's states do not move when the flash kernels change (a
near-critical state's iteration count follows its last bits). Other seeds
and sizes bisect with the current library."""
from __future__ import annotations

import os

import numpy as np

SEED = 2025
NCELL = 1 << 20
# bisection steps in ln P over [0.5, 80] MPa for the saturation pressure of
# the near-envelope states: 2^-20 of ln(160) is 5e-6 relative, far inside the
# 5 % band the states are drawn from
BISECT_STEPS = 20
NEAR_FRAC = 0.3
FROZEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "workloads", "bench1m_near_envelope.npz")


def bench_fluid():
    from .fluid import synthetic_fluid
    return synthetic_fluid(6, 1234)


def gpu_phase_counter(fluid, device, chunk=1 << 20):
    """Hydrocarbon phase count of (P, T, Ni) batches with the batched GPU
    flash (used only to place the near-envelope states)."""
    from .flash import MixtureCompBatch
    fl = fluid.with_controls(use_skip=False)
    m = MixtureCompBatch(fl, device)
    st = m.new_state(chunk)

    def count(P, T, Ni):
        n = len(P)
        res = np.empty(n, np.int64)
        for c0 in range(0, n, chunk):
            c1 = min(n, c0 + chunk)
            k = c1 - c0
            P_ = np.full(chunk, 1000.0)
            T_ = np.full(chunk, 100.0)
            N_ = np.tile(Ni[c0:c0 + 1], (chunk, 1))
            P_[:k], T_[:k], N_[:k] = P[c0:c1], T[c0:c1], Ni[c0:c1]
            st.load(P_, T_, N_)
            st.out["phaseNum"].zero_()
            m.flash_fim(st, form="batched", diagnostics=False, fresh=True)
            res[c0:c1] = st.out["phaseNum"][:k].cpu().numpy() - 1
        return res

    return count, m


def frozen_rounds(n, seed):
    """The recorded bisection outcome for (n, seed), or None."""
    if not os.path.exists(FROZEN):
        return None
    d = np.load(FROZEN)
    if int(d["ncell"]) != n or int(d["seed"]) != seed:
        return None
    return [(d[f"idx{r}"], d[f"psat{r}"]) for r in range(int(d["rounds"]))]


def make_workload(fluid, n, seed, device):
    from . import synth
    rounds = frozen_rounds(n, seed)
    if rounds is not None:
        return synth.mixed_states(fluid, n, seed, None, near_frac=NEAR_FRAC, steps=BISECT_STEPS, replay=rounds)
    count, m = gpu_phase_counter(fluid, device)
    w = synth.mixed_states(fluid, n, seed, count, near_frac=NEAR_FRAC, steps=BISECT_STEPS)
    m.close()
    return w


def record(fluid, n, seed, count, path=FROZEN, note=""):
    """Bisects the near-envelope states with ``count`` (a phase counter such
    as gpu_phase_counter's) and writes the outcome to ``path``; returns the
    workload."""
    from . import synth
    rec = []
    w = synth.mixed_states(fluid, n, seed, count, near_frac=NEAR_FRAC, steps=BISECT_STEPS, record=rec)
    d = {"ncell": np.int64(n), "seed": np.int64(seed), "rounds": np.int64(len(rec)), "note": np.array(note)}
    for r, (idx, psat) in enumerate(rec):
        d[f"idx{r}"] = idx
        d[f"psat{r}"] = psat
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, **d)
    return w


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="record the benchmark block's near-envelope bisection")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=FROZEN)
    a = ap.parse_args()
    fl = bench_fluid()
    cnt, mm = gpu_phase_counter(fl, a.device)
    record(fl, NCELL, SEED, cnt, a.out, note="batched GPU flash of this library")
    mm.close()
