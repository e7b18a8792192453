"""The learned initialiser: its network kernels against the NumPy oracle
(oracle/mlp.py), the oracle against finite differences, training, and the
fast form that uses a trained network (parity with the reference and what
the network saves)."""
import os

import numpy as np
import pytest

from oracle import mlp as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODEL = os.path.join(ROOT, "opencaeporo_b200", "models", "learned_init_nc6.npz")


def _problem(n=300, nin=8, nout=7, seed=3):
    rng = np.random.default_rng(seed)
    from opencaeporo_b200.learn import init_params
    p = init_params(nin, nout, seed).astype(np.float64)
    p[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.1, M.H)
    p[M.OFF_B2:M.OFF_W3] = rng.normal(0, 0.1, M.H)
    p[M.OFF_B3:M.OFF_B3 + nout] = rng.normal(0, 0.1, nout)
    x = rng.normal(0, 1, (nin, n))
    t = np.vstack([rng.integers(0, 2, n), rng.normal(0, 2, (nout - 1, n))])
    w = (rng.uniform(size=n) < 0.6).astype(np.float64)
    return p.astype(np.float32), x.astype(np.float32), t.astype(np.float32), w.astype(np.float32)


def test_oracle_gradient_matches_finite_differences():
    """The oracle's hand-derived backward pass (float64) is the derivative
    of its loss."""
    p, x, t, w = _problem(n=40)
    p = p.astype(np.float64)
    lam = 0.7
    _, g = M.loss_and_grad(p, x, t, w, lam, bf16=False)
    rng = np.random.default_rng(0)
    nin, nout = x.shape[0], t.shape[0]
    live = [i for i in range(M.NPARAM)
            if not (M.OFF_W1 <= i < M.OFF_B1 and (i - M.OFF_W1) % M.IO >= nin)
            and not (M.OFF_W3 <= i < M.OFF_B3 and (i - M.OFF_W3) // M.H >= nout)
            and not (M.OFF_B3 + nout <= i < M.NPARAM)]
    n = x.shape[1]

    def L(q):
        s, _ = M.loss_and_grad(q, x, t, w, lam, bf16=False)
        return (s[0] + lam * s[1]) / n

    for i in rng.choice(live, 60, replace=False):
        h = 1e-6
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        fd = (L(q1) - L(q2)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], np.float32)
    r = M.bf16_round(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] - (-3.140625)) < 1e-9 and r[4] == 0.0


@pytest.mark.gpu
def test_mlp_forward_matches_oracle():
    import torch
    from opencaeporo_b200 import learn
    p, x, t, w = _problem(n=1000)
    dev = torch.device("cuda", 0)
    y = learn.forward(torch.as_tensor(p, device=dev), torch.as_tensor(x, device=dev), 7).cpu().numpy()
    ref, _ = M.forward(p, x, bf16=True)
    err = np.abs(y - ref[:7])
    assert np.max(err) < 2e-2 * (1 + np.max(np.abs(ref[:7]))), np.max(err)
    assert np.mean(err) < 2e-3, np.mean(err)


@pytest.mark.gpu
def test_tcgen05_forward_over_many_tiles_and_a_ragged_end():
    """The evaluation forward pass (tcgen05, 128 samples per tile) on a batch
    with more tiles than its grid holds CTAs (each CTA loops over several
    tiles, reusing its tensor memory) and a partial last tile: against the
    oracle sample by sample, and against the training kernel's own
    forward pass through the loss both give for the same outputs."""
    import torch
    from opencaeporo_b200 import learn
    n = 128 * 148 * 8 * 2 + 77
    p, x, t, w = _problem(n=n, seed=11)
    dev = torch.device("cuda", 0)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    y = learn.forward(T(p), T(x), 7).cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(y))
    ref, _ = M.forward(p, x, bf16=True)
    err = np.abs(y - ref[:7])
    assert np.max(err) < 2e-2 * (1 + np.max(np.abs(ref[:7]))), np.max(err)
    assert np.mean(err) < 2e-3, np.mean(err)
    # the same loss from the tcgen05 outputs and from the training kernel's forward pass
    lam = 0.5
    g = torch.zeros(M.NPARAM, dtype=torch.float32, device=dev)
    loss = torch.zeros(2, dtype=torch.float32, device=dev)
    learn.grad(T(p), T(x), T(t), T(w), lam, g, loss)
    lk = loss.cpu().numpy().astype(np.float64)
    z = y[0]
    bce = np.sum(np.maximum(z, 0) + np.log1p(np.exp(-np.abs(z))) - t[0] * z)
    mse = np.sum(w * np.sum((y[1:] - t[1:]) ** 2, axis=0) / 6)
    np.testing.assert_allclose([bce, mse], lk, rtol=1e-3)


@pytest.mark.gpu
def test_mlp_gradient_matches_oracle():
    """Gradient of the BF16 tensor-core kernel against the CPU oracle with
    the same BF16 roundings; and against the exact float64 gradient to
    BF16 accuracy."""
    import torch
    from opencaeporo_b200 import learn
    p, x, t, w = _problem(n=777)
    dev = torch.device("cuda", 0)
    g = torch.zeros(M.NPARAM, dtype=torch.float32, device=dev)
    loss = torch.zeros(2, dtype=torch.float32, device=dev)
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    learn.grad(T(p), T(x), T(t), T(w), 0.5, g, loss)
    gk = g.cpu().numpy().astype(np.float64)
    lk = loss.cpu().numpy().astype(np.float64)
    lo, go = M.loss_and_grad(p, x, t, w, 0.5, bf16=True)
    np.testing.assert_allclose(lk, lo, rtol=2e-3)
    rel = np.linalg.norm(gk - go) / np.linalg.norm(go)
    assert rel < 1e-2, rel
    cos = gk @ go / (np.linalg.norm(gk) * np.linalg.norm(go))
    assert cos > 0.9999, cos
    _, gx = M.loss_and_grad(p, x, t, w, 0.5, bf16=False)
    assert np.linalg.norm(gk - gx) / np.linalg.norm(gx) < 5e-2


@pytest.mark.gpu
def test_training_fits_a_known_function():
    """The training kernels (grad + Adam) fit a smooth target: the logit
    classifies a half-space and the regression rows learn linear maps."""
    from opencaeporo_b200 import learn
    rng = np.random.default_rng(11)
    n, nin, nout = 65536, 8, 7
    x = rng.normal(0, 1, (nin, n)).astype(np.float32)
    t = np.zeros((nout, n), np.float32)
    t[0] = (x[0] + 0.5 * x[1] > 0)
    A = rng.normal(0, 0.5, (nout - 1, nin))
    t[1:] = A @ x
    w = np.ones(n, np.float32)
    logs = []
    params = learn.train(x, t, w, epochs=12, batch=4096, lr=3e-3, log=logs.append)
    import torch
    y = learn.forward(torch.as_tensor(params, device="cuda"), torch.as_tensor(x, device="cuda"), nout).cpu().numpy()
    acc = np.mean((y[0] > 0) == (t[0] > 0.5))
    mse = np.mean((y[1:] - t[1:]) ** 2)
    assert acc > 0.97, (acc, logs)
    assert mse < 0.02 * np.mean(t[1:] ** 2), (mse, logs)


def _model():
    from opencaeporo_b200.learn import Initializer
    if not os.path.exists(MODEL):
        pytest.fail(f"trained initialiser missing: {MODEL} (python -m opencaeporo_b200.learn)")
    return Initializer.load(MODEL)


def _sub(d, mask):
    n = len(mask)
    out = {}
    for k, v in d.items():
        if isinstance(v, dict):
            out[k] = _sub(v, mask)
        elif isinstance(v, np.ndarray) and v.ndim and v.shape[0] == n:
            out[k] = v[mask]
        else:
            out[k] = v
    return out


def _clean_equilibrium(res, nc):
    """Cells whose result is a converged equilibrium: residual at or below
    1e-9 and every present hydrocarbon phase's composition summing to one."""
    n = len(res["phaseNum"])
    x = np.nan_to_num(np.asarray(res["xij"]).reshape(n, 3, nc + 1)[:, :2, :nc])
    ex = np.asarray(res["phaseExist"])[:, :2].astype(bool)
    sums_ok = np.all(~ex | (np.abs(x.sum(axis=2) - 1) < 1e-9), axis=1)
    return (np.asarray(res["ePEC"]) <= 1e-9) & sums_ok


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["uniform_nc6", "near_nc6", "warm_nc6", "restart_nc6", "config1_nc6"])
def test_fast_matches_reference_goldens(case):
    """Fast form (mixed + trained initialiser) against the reference. Where
    the reference converged (ePEC <= 1e-9: its answer is an equilibrium),
    the bar of every other form: identical phase counts except knife-edge
    cells, outputs within 1e-8 relative or 10x the reference's own 1-ulp
    sensitivity. Where it did not -- SplitNR stopped on its small-step test
    short of its tolerance, with compositions no longer summing to one --
    the fast form may have found the converged equilibrium instead; every
    such cell it does not reproduce must be one."""
    from conftest import load_golden, run_gpu
    from oracle import compare as CMP
    fl, inp, ref, fragile = load_golden(case)
    got = run_gpu(fl, inp, form="fast", init=_model())
    det = np.asarray(ref["ePEC"]) <= 1e-9
    chk = CMP.check(_sub(got, det), _sub(ref, det), fl.nc, noise=_sub(ref["noise"], det), fragile=fragile[det])
    assert chk["ok"], f"{case}: {CMP.check_summary(chk)}"
    if (~det).any():
        c2 = CMP.check(_sub(got, ~det), _sub(ref, ~det), fl.nc, noise=_sub(ref["noise"], ~det),
                       fragile=fragile[~det])
        worst = np.zeros(int((~det).sum()))
        for k in CMP.FLOAT_KEYS:
            allowed = np.maximum(1e-8, 10 * np.nan_to_num(_sub(ref["noise"], ~det)[k], nan=0.0))
            worst = np.fmax(worst, np.nan_to_num(c2["errors"][k], nan=0.0) / allowed)
        differs = (worst > 1) | ~c2["errors"]["same"]
        clean = _clean_equilibrium(_sub(got, ~det), fl.nc)
        assert np.all(clean[differs]), np.nonzero(~det)[0][differs & ~clean]


@pytest.mark.gpu
def test_fast_init_flash_matches_reference_golden():
    """InitFlashFIM in the fast form (every initial state is a fresh cell,
    so every one goes through the trained initialiser) against the
    reference, with the bar of test_fast_matches_reference_goldens."""
    from conftest import load_golden_init, run_gpu_init
    from oracle import compare as CMP
    fl, inp, ref, _, fragile = load_golden_init()
    got = run_gpu_init(fl, inp, form="fast", init=_model())
    det = np.asarray(ref["ePEC"]) <= 1e-9
    chk = CMP.check(_sub(got, det), _sub(ref, det), fl.nc, noise=_sub(ref["noise"], det), fragile=fragile[det])
    assert chk["ok"], CMP.check_summary(chk)
    same = det & (got["phaseNum"] == ref["phaseNum"]) & ~fragile
    e = CMP._rel(got["Ni"], ref["Ni"]).max(axis=1)
    assert np.all(e[same] <= np.maximum(1e-8, 10 * ref["noise"]["Ni"][same]))
    if (~det).any():
        diff = (got["phaseNum"] != ref["phaseNum"]) & ~det
        assert np.all(_clean_equilibrium(_sub(got, diff), fl.nc))


@pytest.mark.gpu
def test_initialiser_gain_over_mixed():
    """What the trained network buys on 65,536 held-out states of the
    workload distribution (a seed it was not trained on): the fast form ends
    with the same phase counts as the mixed form (up to a handful of
    knife-edge cells) while doing less work -- the stability test is skipped
    for the cells the network is confident are two-phase, so fewer stability
    iterations and less modelled work. (The times of both forms are printed;
    at this size the learned round's extra kernels cost about what they
    save.)"""
    import torch
    from opencaeporo_b200 import roofline
    from opencaeporo_b200.flash import MixtureCompBatch
    from opencaeporo_b200.workload import bench_fluid, make_workload
    fl = bench_fluid()
    n = 1 << 16
    w = make_workload(fl, n, 424242, 0)
    res, ms = {}, {}
    for form in ("mixed", "fast"):
        m = MixtureCompBatch(fl)
        if form == "fast":
            _model().attach(m)
        st = m.new_state(n)
        best = 1e9
        for _ in range(3):
            st.load(w["P"], w["T"], w["Ni"])
            st.skip["flag"].zero_()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            m.flash_fim(st, form=form, fresh=True)
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        res[form], ms[form] = st.to_host(), best
        m.close()
    mix, fast = res["mixed"], res["fast"]
    # where the mixed form's answer is a converged equilibrium the fast form
    # ends with the same phase count (a few knife-edge cells aside); where it
    # is not, a differing fast answer must be one
    det = _clean_equilibrium(mix, fl.nc)
    diff = mix["phaseNum"] != fast["phaseNum"]
    mism = int(np.count_nonzero(diff & det))
    assert mism <= max(3, n // 20000), mism
    assert np.all(_clean_equilibrium(fast, fl.nc)[diff & ~det])
    it_m, it_f = mix["iters"].sum(axis=0), fast["iters"].sum(axis=0)
    work_m = roofline.flops(fl.nc, mix["iters"], mix["phaseNum"] - 1)
    work_f = roofline.flops(fl.nc, fast["iters"], fast["phaseNum"] - 1)
    print(f"mixed {ms['mixed']:.2f} ms iters {it_m.tolist()}  fast {ms['fast']:.2f} ms iters {it_f.tolist()}  "
          f"model work {work_f / work_m:.3f}x")
    assert it_f[0] < 0.95 * it_m[0], (it_m, it_f)
    assert it_f[1] < it_m[1], (it_m, it_f)
    assert work_f < 0.98 * work_m, (work_m, work_f)


@pytest.mark.gpu
def test_fast_form_config1_at_the_plain_bar():
    """The CPU-runnable configuration in full (4096 fresh states) in the fast
    form, held to the bar of the FP64 forms on every cell: identical phase
    counts except where the reference itself flips under 1-ulp input
    perturbations, every output within 1e-8 relative or 10x the reference's
    own 1-ulp sensitivity -- no exception for cells whose reference split
    did not converge."""
    from conftest import load_golden, run_gpu
    from oracle import compare as CMP
    fl, inp, ref, fragile = load_golden("config1_nc6")
    got = run_gpu(fl, inp, form="fast", init=_model())
    chk = CMP.check(got, ref, fl.nc, noise=ref["noise"], fragile=fragile)
    assert chk["ok"], CMP.check_summary(chk)
