"""Several PVT regions in one call (ocpf_flash_fim_regions). The streams
schedule runs the one-region kernels and gives exactly one ocpf_flash_fim
per region; the one-launch schedule (every step of the batched sequence one
kernel over all regions) runs the same device code in other kernels, which
the compiler contracts into fused multiply-adds on its own, so it agrees to
rounding: identical phase counts and flash types, and outputs within 1e-9
wherever the iteration counts agree. In every batched form, fresh and
warm-started, directly and replayed from the captured graph. The regions'
golden fixtures pass the reference bar through the one call; the autotuner
leaves the caller's arrays alone."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import compare as CMP

pytestmark = pytest.mark.gpu

SCHEDS = {"one_launch": 0, "streams": 1}


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _regions(form, seeds=((3, 31), (6, 61), (9, 91), (12, 121)), n0=2000):
    from opencaeporo_b200 import synth
    from opencaeporo_b200.flash import MixtureCompBatch
    from opencaeporo_b200.fluid import synthetic_fluid
    from opencaeporo_b200.learn import DEFAULT_MODEL, Initializer
    out = []
    for nc, seed in seeds:
        fl = synthetic_fluid(nc, seed)
        w = synth.uniform_states(fl, n0 + 300 * nc, seed, p_mpa=(2.0, 60.0), t_k=(300.0, 450.0), alpha=0.5)
        m = MixtureCompBatch(fl)
        if form == "fast" and nc == 6:
            Initializer.load(DEFAULT_MODEL).attach(m)
        out.append((m, w))
    return out


def _gpu_self_noise(m, w, base, form, trials=6):
    """(noise, moved): per output field and cell, the largest relative change
    of the one-region flash of `form` (fresh cells) under 1-ulp input
    perturbations (oracle.compare.perturbed's first six trials) against
    ``base``, and the cells whose phase count those perturbations change."""
    import torch
    prng = np.random.default_rng(7)
    n = len(w["P"])
    noise = {k: np.zeros(n) for k in CMP.FLOAT_KEYS}
    moved = np.zeros(n, bool)
    st = m.new_state(n)
    for t in range(trials):
        P, T, Ni = CMP.perturbed(w["P"], w["T"], w["Ni"], t, prng)
        st.load(P, T, Ni)
        m.flash_fim(st, form=form, fresh=True)
        torch.cuda.synchronize()
        h = st.to_host()
        moved |= h["phaseNum"] != base["phaseNum"]
        e = CMP.per_cell_errors(h, base, m.nc)
        for k in CMP.FLOAT_KEYS:
            noise[k] = np.fmax(noise[k], np.nan_to_num(e[k], nan=0.0))
    return noise, moved


def _host(st):
    h = st.to_host()
    sk = h.pop("skip")
    h.update({f"skip_{k}": v for k, v in sk.items()})
    return h


@pytest.mark.parametrize("form", ["batched", "mixed", "fast"])
@pytest.mark.parametrize("sched", list(SCHEDS))
def test_regions_equal_one_call_per_region(form, sched):
    torch = _torch()
    from opencaeporo_b200 import roofline
    from opencaeporo_b200.flash import flash_fim_regions
    regs = _regions(form)
    alone, together = [], []
    for m, w in regs:
        a, b = m.new_state(len(w["P"])), m.new_state(len(w["P"]))
        for st in (a, b):
            st.load(w["P"], w["T"], w["Ni"])
        alone.append(a)
        together.append(b)
    regs[0][0].set_tuning(schedule=SCHEDS[sched])
    regs_w = {m.nc: w for m, w in regs}
    pairs = [(m, b) for (m, _), b in zip(regs, together)]
    # a fresh step (twice: the second replays the captured sequence), then a
    # warm step from the first step's state with P moved
    for step in range(3):
        fresh = step < 2
        if step == 2:
            for (m, w), a, b in zip(regs, alone, together):
                P2 = torch.as_tensor(w["P"] * 1.003).cuda()
                a.P.copy_(P2)
                b.P.copy_(P2)
        for (m, _), a in zip(regs, alone):
            m.flash_fim(a, form=form, fresh=fresh)
        flash_fim_regions(pairs, form=form, fresh=fresh)
        torch.cuda.synchronize()
        for (m, _), a, b in zip(regs, alone, together):
            ha, hb = _host(a), _host(b)
            if sched == "streams":
                for k, v in ha.items():
                    if isinstance(v, np.ndarray):
                        np.testing.assert_array_equal(v, hb[k], err_msg=f"step {step} nc={m.nc} {k}")
                continue
            # phase counts: identical but for knife-edge cells (at most 0.1 %,
            # and at step 0 only cells whose count the one-region flash
            # itself changes under 1-ulp input perturbations)
            diff = ha["phaseNum"] != hb["phaseNum"]
            assert np.mean(diff) <= 1e-3, (step, m.nc, np.nonzero(diff)[0][:8])
            # iteration counts that end on a convergence threshold (tol^2 =
            # 1e-24) move with rounding, as between the plain and batched
            # forms: the modelled work stays within 1 %
            same_it = np.all(ha["iters"] == hb["iters"], axis=1)
            assert np.mean(same_it) > 0.85, (step, m.nc, np.count_nonzero(~same_it))
            wa = roofline.flops(m.nc, ha["iters"], ha["phaseNum"] - 1)
            wb = roofline.flops(m.nc, hb["iters"], hb["phaseNum"] - 1)
            assert abs(wb / wa - 1) < 0.01, (step, m.nc, wa, wb)
            if step == 0:
                # outputs: within 1e-9, or 10x the one-region flash's own
                # change under 1-ulp input perturbations (Dirichlet(0.5)
                # states near their critical point are ill-conditioned)
                noise, moved = _gpu_self_noise(m, regs_w[m.nc], ha, form)
                chk = CMP.check(hb, ha, m.nc, noise=noise, fragile=moved, tol=1e-9)
                assert chk["ok"], f"step {step} nc={m.nc}: {CMP.check_summary(chk)}"
    for m, _ in regs:
        m.close()


@pytest.mark.parametrize("form", ["batched", "mixed"])
def test_regions_goldens_in_one_launch(form):
    """The 3-, 6-, 9- and 12-component golden fixtures flashed together in
    one call pass the bar of the one-region tests against the reference."""
    torch = _torch()
    from opencaeporo_b200.flash import MixtureCompBatch, flash_fim_regions
    cases = ("uniform_nc3", "config1_nc6", "uniform_nc9", "uniform_nc12")
    pairs, refs = [], []
    for case in cases:
        fl, inp, ref, fragile = load_golden(case)
        m = MixtureCompBatch(fl)
        st = m.new_state(len(inp["P"]))
        st.load(inp["P"], inp["T"], inp["Ni"])
        pairs.append((m, st))
        refs.append((fl, ref, fragile))
    pairs[0][0].set_tuning(schedule=SCHEDS["one_launch"])
    flash_fim_regions(pairs, form=form, fresh=True)
    torch.cuda.synchronize()
    for case, (m, st), (fl, ref, fragile) in zip(cases, pairs, refs):
        got = st.to_host()
        chk = CMP.check(got, ref, fl.nc, noise=ref["noise"], fragile=fragile)
        assert chk["ok"], f"{case}: {CMP.check_summary(chk)}"
        m.close()


def test_autotune_leaves_caller_arrays_and_sets_every_context():
    torch = _torch()
    from opencaeporo_b200.flash import autotune, flash_fim_regions
    regs = _regions("mixed", n0=1500)
    pairs = []
    for m, w in regs:
        st = m.new_state(len(w["P"]))
        st.load(w["P"], w["T"], w["Ni"])
        pairs.append((m, st))
    flash_fim_regions(pairs, form="mixed", fresh=True)  # outputs and skip cache to keep
    torch.cuda.synchronize()
    before = [(_host(st), st.P.cpu().numpy().copy(), st.Ni.cpu().numpy().copy()) for _, st in pairs]
    best = autotune(pairs, form="mixed", reps=1, fresh=False)
    torch.cuda.synchronize()
    assert best["block"] in (64, 128) and 1 <= best["persist_pct"] <= 100 and best["ms"] > 0
    assert best["schedule"] in (0, 1) and best["slow_threads"] in (0, 1)
    for (m, st), (h, P, Ni) in zip(pairs, before):
        assert m.tuning()["block"] == best["block"]
        assert m.tuning()["schedule"] == best["schedule"]
        np.testing.assert_array_equal(st.P.cpu().numpy(), P)
        np.testing.assert_array_equal(st.Ni.cpu().numpy(), Ni)
        h2 = _host(st)
        for k, v in h.items():
            if isinstance(v, np.ndarray):
                np.testing.assert_array_equal(v, h2[k], err_msg=k)
    for m, _ in pairs:
        m.close()


def test_set_tuning_rejects_invalid_shapes():
    _torch()
    from opencaeporo_b200.flash import MixtureCompBatch
    fl = load_golden("spe5")[0]
    m = MixtureCompBatch(fl)
    assert m.tuning()["block"] == 128 and m.tuning()["persist_pct"] == 100
    for bad in ({"block": 96}, {"persist_pct": 0}, {"persist_pct": 101}, {"slow_threads": 2}, {"schedule": 5}):
        with pytest.raises(RuntimeError):
            m.set_tuning(**bad)
    m.set_tuning(block=64, persist_pct=50, slow_threads=1, schedule=1)
    assert m.tuning() == {"block": 64, "persist_pct": 50, "slow_threads": 1, "schedule": 1, "ms": 0.0}
    m.close()


@pytest.mark.parametrize("slow_threads", [0, 1])
@pytest.mark.parametrize("block,pct", [(64, 50), (128, 100)])
def test_launch_shapes_pass_the_golden_bar(slow_threads, block, pct):
    """Every launch shape the autotuner may pick passes the reference bar on
    the restart-heaviest cells (split restarts on one warp or one thread per
    cell) and on the config-1 states; block size and persistent grid alone
    give the default shape's outputs bit for bit."""
    torch = _torch()
    from opencaeporo_b200.flash import MixtureCompBatch
    for case in ("restart_nc6", "config1_nc6"):
        fl, inp, ref, fragile = load_golden(case)
        res = []
        for shape in ((128, 100, slow_threads), (block, pct, slow_threads)):
            m = MixtureCompBatch(fl)
            m.set_tuning(block=shape[0], persist_pct=shape[1], slow_threads=shape[2])
            st = m.new_state(len(inp["P"]))
            st.load(inp["P"], inp["T"], inp["Ni"])
            m.flash_fim(st, form="batched", fresh=True)
            torch.cuda.synchronize()
            res.append(st.to_host())
            m.close()
        chk = CMP.check(res[1], ref, fl.nc, noise=ref["noise"], fragile=fragile)
        assert chk["ok"], f"{case}: {CMP.check_summary(chk)}"
        for k, v in res[0].items():
            if isinstance(v, np.ndarray):
                np.testing.assert_array_equal(v, res[1][k], err_msg=f"{case} {k}")
