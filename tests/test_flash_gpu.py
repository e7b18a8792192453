"""GPU parity tests: the CUDA flash through the C ABI against the reference's
golden fixtures and against the plain-C oracle on larger seeded sets.

Bar (oracle/compare.py): identical phase counts except on knife-edge cells
(where the reference itself flips under 1-ulp input perturbations), and per
output <= 1e-8 relative error, or <= 10x the reference's own 1-ulp
sensitivity in the cells where the reference is ill-conditioned."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden, run_gpu
from oracle import compare as CMP
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _run_gpu(fl, inp, form="plain"):
    return run_gpu(fl, inp, form)


@pytest.mark.parametrize("form", ["plain", "batched"])
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_matches_reference_goldens(case, form):
    fl, inp, ref, fragile = load_golden(case)
    got = _run_gpu(fl, inp, form=form)
    chk = CMP.check(got, ref, fl.nc, noise=ref["noise"], fragile=fragile)
    assert chk["ok"], f"{case}: {CMP.check_summary(chk)}"
    res = CMP.compare(got, ref, fl.nc)
    for k in ("phaseExist", "bRowSizedSdP", "pSderExist", "pVnumCom"):
        assert res[k + "_mismatch"] == 0, f"{case}: {k}"
    same = got["phaseNum"] == ref["phaseNum"]
    assert np.array_equal(got["ftype"][same], ref["ftype"][same])
    # the work done follows the reference's: iteration counts are noise-
    # sensitive near tol^2 = 1e-24, so the flop-weighted total over the
    # cells that are not knife-edge is held to 5 %
    from opencaeporo_b200 import roofline
    k = same & ~fragile
    wa = roofline.flops(fl.nc, got["iters"][k], got["phaseNum"][k] - 1)
    wb = roofline.flops(fl.nc, ref["iters"][k], ref["NPhc"][k])
    assert abs(wa - wb) <= 0.05 * wb, (got["iters"].sum(axis=0), ref["iters"].sum(axis=0))


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_mixed_matches_reference_goldens(case):
    """Mixed form (FP32 successive substitution; FP64 cubic roots near the
    discriminant, Rachford-Rice and Newton polish) against the reference:
    the same bar as the FP64 forms -- identical phase counts except on
    knife-edge cells, every output within 1e-8 relative or 10x the
    reference's own 1-ulp sensitivity where that is larger."""
    fl, inp, ref, fragile = load_golden(case)
    got = _run_gpu(fl, inp, form="mixed")
    chk = CMP.check(got, ref, fl.nc, noise=ref["noise"], fragile=fragile)
    assert chk["ok"], f"{case}: {CMP.check_summary(chk)}"
    res = CMP.compare(got, ref, fl.nc)
    for k in ("phaseExist", "bRowSizedSdP", "pSderExist", "pVnumCom"):
        assert res[k + "_mismatch"] == 0, f"{case}: {k}"
    same = got["phaseNum"] == ref["phaseNum"]
    assert np.array_equal(got["ftype"][same], ref["ftype"][same])


@pytest.mark.parametrize("form", ["plain", "batched", "mixed"])
def test_skip_cache_matches_reference(form):
    fl, inp, ref, fragile = load_golden("warm_nc6")
    got = _run_gpu(fl, inp, form=form)
    ok = (got["phaseNum"] == ref["phaseNum"]) & ~fragile
    sg, sr = got["skip"], ref["skip"]
    assert np.array_equal(sg["flag"][ok].astype(int), sr["flag"][ok].astype(int))
    f = sr["flag"].astype(bool) & ok
    np.testing.assert_allclose(sg["P"][f], sr["P"][f], rtol=0)
    np.testing.assert_allclose(sg["T"][f], sr["T"][f], rtol=0)
    np.testing.assert_allclose(sg["z"][f], sr["z"][f], rtol=1e-15)
    np.testing.assert_allclose(sg["minEig"][f], sr["minEig"][f], rtol=2e-5, atol=2e-6)


def test_host_path_equals_device_path():
    """ocpf_flash_fim_host (host buffers, chunked copies on two streams) gives
    bit-identical results to the device-buffer call."""
    from opencaeporo_b200.flash import MixtureCompBatch
    torch = _torch()
    fl, inp, ref, _ = load_golden("warm_nc6")
    dev = _run_gpu(fl, inp)
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    hs = m.new_host_state(n)
    hs["P"].copy_(torch.as_tensor(inp["P"]))
    hs["T"].copy_(torch.as_tensor(inp["T"]))
    hs["Ni"].copy_(torch.as_tensor(np.ascontiguousarray(inp["Ni"].T)))
    o = hs["out"]
    o["S"].copy_(torch.as_tensor(np.ascontiguousarray(inp["S"].T)))
    o["phaseNum"].copy_(torch.as_tensor(inp["lastNP"].astype(np.int32)))
    o["xij"].copy_(torch.as_tensor(np.ascontiguousarray(inp["xij"].reshape(n, -1).T)))
    sk = inp["skip"]
    hs["skip"]["flag"].copy_(torch.as_tensor(sk["flag"].astype(np.int32)))
    for k in ("minEig", "P", "T"):
        hs["skip"][k].copy_(torch.as_tensor(np.asarray(sk[k], dtype=np.float64)))
    hs["skip"]["z"].copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(sk["z"]).T)))
    m.flash_fim_host(hs)
    for k in ("phaseNum", "S", "vfi", "xij", "mux", "dSec_dPri", "status", "iters"):
        a = o[k].numpy()
        a = a.T if a.ndim == 2 else a
        b = dev[k].reshape(a.shape) if k in ("xij", "mux") else dev[k]
        np.testing.assert_array_equal(np.nan_to_num(a.reshape(b.shape).astype(np.float64)),
                                      np.nan_to_num(b.astype(np.float64)), err_msg=k)
    m.close()


def _port_noise(fl, inp, base, runs=4):
    """The port's own 1-ulp sensitivity (per cell and field) and knife-edge mask."""
    n = len(inp["P"])
    noise = {k: np.zeros(n) for k in CMP.FLOAT_KEYS}
    frag = np.zeros(n, bool)
    eps = 2.0 ** -50
    for t in range(runs):
        s = 1 if t % 2 == 0 else -1
        P = inp["P"] * (1 + s * eps) if t < 2 else inp["P"]
        Ni = inp["Ni"] * (1 + s * eps) if t >= 2 else inp["Ni"]
        r = O.flash_fim("port", fl, P, inp["T"], Ni, nthreads=0)
        frag |= r["phaseNum"] != base["phaseNum"]
        e = CMP.per_cell_errors(r, base, fl.nc)
        for k in CMP.FLOAT_KEYS:
            noise[k] = np.fmax(noise[k], np.nan_to_num(e[k], nan=0.0))
    return noise, frag


@pytest.mark.parametrize("form", ["plain", "batched", "mixed"])
@pytest.mark.parametrize("nc,seed", [(6, 1234), (12, 7)])
def test_matches_port_4096(nc, seed, form):
    """4096 seeded states (the 6-component workload distribution; and a
    12-component fluid) against the plain-C oracle."""
    from opencaeporo_b200.fluid import synthetic_fluid
    from opencaeporo_b200 import synth
    fl = synthetic_fluid(nc, seed)
    inp = synth.uniform_states(fl, 4096, seed)
    port = O.flash_fim("port", fl, inp["P"], inp["T"], inp["Ni"], nthreads=0)
    noise, frag = _port_noise(fl, inp, port)
    full = dict(inp, S=np.zeros((4096, 3)), lastNP=np.zeros(4096, np.int32),
                xij=np.zeros((4096, 3, nc + 1)), skip=O.new_skip(4096, nc))
    got = _run_gpu(fl, full, form=form)
    chk = CMP.check(got, port, nc, noise=noise, fragile=frag)
    assert chk["ok"], CMP.check_summary(chk)
    assert len(chk["np_mismatch_all"]) <= 4


def test_degenerate_inputs_do_not_hang_or_fault():
    """NaN pressure, zero and negative moles, a single cell: the kernel
    returns with every loop bounded and flags non-finite results."""
    fl = load_golden("spe5")[0]
    n = 4
    inp = {"P": np.array([np.nan, 2000.0, 3000.0, 1e-3]), "T": np.full(n, 160.0),
           "Ni": np.array([[500.0, 30, 70, 200, 150, 50, 100]] * n),
           "S": np.zeros((n, 3)), "lastNP": np.zeros(n, np.int32),
           "xij": np.zeros((n, 3, 7)), "skip": O.new_skip(n, 6)}
    inp["Ni"][1, :6] = 0.0
    inp["Ni"][2, 0] = -5.0
    got = _run_gpu(fl, inp)
    assert got["status"][0] & 0x40  # non-finite flagged
    assert set(got["phaseNum"].tolist()) <= {2, 3}


def test_zero_cells_is_a_noop():
    from opencaeporo_b200.flash import MixtureCompBatch
    _torch()
    m = MixtureCompBatch(load_golden("spe5")[0])
    st = m.new_state(0)
    m.flash_fim(st)
    m.close()


@pytest.mark.parametrize("case", ["uniform_nc6", "warm_nc6", "uniform_nc12"])
def test_batched_equals_plain(case):
    """The batched form takes the reference's steps in the same order with
    the same expressions as the plain form. The compiler fuses
    multiply-adds per kernel, so the two round alike only up to that: phase
    counts, flash types and status agree exactly, an iteration count that
    ends on a convergence threshold may move by a few steps (the total
    modelled work stays within 1 %), outputs agree to 1e-9 or 10x the
    reference's own 1-ulp sensitivity."""
    from opencaeporo_b200 import _lib, roofline
    fl, inp, ref, _ = load_golden(case)
    a = _run_gpu(fl, inp, form="plain")
    b = _run_gpu(fl, inp, form="batched")
    for k in ("phaseNum", "ftype"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    # status: the outcome bits agree everywhere; the bits that record an
    # intermediate event (an iteration that hit its cap or stopped short of
    # its tolerance, a singular dense solve on the way) agree wherever the
    # iteration counts do -- rounding moves such an event only together with
    # the counts of the iteration it ends
    event = (_lib.CELL_SSMSTA_CAP | _lib.CELL_NRSTA_FAIL | _lib.CELL_SSMSP_FAIL | _lib.CELL_NRSP_FAIL |
             _lib.CELL_SINGULAR)
    keep = np.uint16(0xFFFF & ~event)
    np.testing.assert_array_equal(a["status"] & keep, b["status"] & keep, err_msg="status")
    same_it = np.all(a["iters"] == b["iters"], axis=1)
    diff = np.nonzero(same_it & (a["status"] != b["status"]))[0]
    assert len(diff) == 0, [(int(c), int(a["status"][c]), int(b["status"][c]), a["iters"][c].tolist())
                            for c in diff[:8]]
    wa = roofline.flops(fl.nc, a["iters"], a["phaseNum"] - 1)
    wb = roofline.flops(fl.nc, b["iters"], b["phaseNum"] - 1)
    assert abs(wb / wa - 1) < 0.01, (wa, wb)
    moved = np.abs(a["iters"] - b["iters"]).max(axis=1)
    assert np.mean(moved == 0) > 0.9, np.nonzero(moved)[0]
    chk = CMP.check(b, a, fl.nc, noise=ref["noise"], tol=1e-9)
    assert chk["ok"], CMP.check_summary(chk)
    sa, sb = a["skip"], b["skip"]
    np.testing.assert_array_equal(sa["flag"], sb["flag"])
    np.testing.assert_allclose(sa["minEig"], sb["minEig"], rtol=1e-6, atol=1e-7)


def test_batched_host_path_and_reserve():
    """Host-buffer path of the batched form (two streams, separate scratch
    parts) equals its device path; ocpf_reserve pre-sizes the scratch."""
    from opencaeporo_b200.flash import MixtureCompBatch
    torch = _torch()
    fl, inp, ref, _ = load_golden("uniform_nc6")
    dev = _run_gpu(fl, inp, form="batched")
    m = MixtureCompBatch(fl)
    m.reserve(4096)
    n = len(inp["P"])
    hs = m.new_host_state(n)
    hs["P"].copy_(torch.as_tensor(inp["P"]))
    hs["T"].copy_(torch.as_tensor(inp["T"]))
    hs["Ni"].copy_(torch.as_tensor(np.ascontiguousarray(inp["Ni"].T)))
    m.flash_fim_host(hs, form="batched")
    for k in ("phaseNum", "S", "dSec_dPri", "iters"):
        a = hs["out"][k].numpy()
        a = a.T if a.ndim == 2 else a
        np.testing.assert_array_equal(np.nan_to_num(a.astype(np.float64)),
                                      np.nan_to_num(dev[k].astype(np.float64)), err_msg=k)
    m.close()


@pytest.mark.parametrize("case", ["restart_nc6", "config1_nc6"])
@pytest.mark.parametrize("form", ["batched", "fast"])
def test_side_stream_schedule_changes_no_output(case, form):
    """The default schedule of a device-buffer call runs some of the work on
    side streams:
    * the split and restarts of the cells that stability trials 1-3 find
      unstable;
    * in the fast form, the learned round and the strict test of its
      fallback cells.
    With the part marks on, the call keeps everything on its own stream in
    the plain order. Both give the same outputs bit for bit. The
    restart-heavy cells include trial-1 cells and long chains. The config-1
    states include learned splits that are kept and ones that fall back."""
    torch = _torch()
    from opencaeporo_b200.flash import MixtureCompBatch
    from opencaeporo_b200.learn import DEFAULT_MODEL, Initializer
    fl, inp, ref, _ = load_golden(case)
    outs = []
    for one_stream in (False, True):
        m = MixtureCompBatch(fl)
        if form == "fast":
            Initializer.load(DEFAULT_MODEL).attach(m)
        m.set_part_timing(one_stream)
        st = m.new_state(len(inp["P"]))
        st.load(inp["P"], inp["T"], inp["Ni"])
        for _ in range(2):  # the second call replays the captured sequence
            st.skip["flag"].zero_()
            m.flash_fim(st, form=form, fresh=True)
        torch.cuda.synchronize()
        outs.append(st.to_host())
        m.close()
    for k, v in outs[0].items():
        if isinstance(v, np.ndarray):
            np.testing.assert_array_equal(v, outs[1][k], err_msg=k)


def test_caller_stream_capture_equals_direct_call():
    """A caller captures its own stream around a batched call. The side
    streams of the per-trial split schedule join that capture through their
    fork and join events. The restart-heavy cells include ones that trials 1-3
    find unstable, and so ones whose split runs on a side stream. Replaying
    the caller's graph gives the direct call's outputs bit for bit."""
    torch = _torch()
    from opencaeporo_b200.flash import MixtureCompBatch
    fl, inp, ref, _ = load_golden("restart_nc6")
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    m.reserve(n)
    st = m.new_state(n)
    s = torch.cuda.Stream()

    def prefill():
        # outputs of absent phases are left as they were: start both runs alike
        for t in st.out.values():
            t.fill_(7 if t.dtype.is_floating_point else 1)
        st.skip["flag"].zero_()

    st.load(inp["P"], inp["T"], inp["Ni"])
    with torch.cuda.stream(s):
        prefill()
        m.flash_fim(st, form="batched", fresh=True, stream=s)
    torch.cuda.synchronize()
    direct = st.to_host()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        m.flash_fim(st, form="batched", fresh=True, stream=s)
    for _ in range(2):
        with torch.cuda.stream(s):
            prefill()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        got = st.to_host()
        for k, v in direct.items():
            if isinstance(v, np.ndarray):
                np.testing.assert_array_equal(v, got[k], err_msg=k)
    del g
    m.close()


def test_graph_replay_equals_direct_launch():
    """From the second call on, the batched sequence is replayed from a
    captured CUDA graph; replays (also after the arguments change, which
    re-captures) give exactly the direct launch's outputs."""
    torch = _torch()
    from opencaeporo_b200.flash import MixtureCompBatch
    fl, inp, ref, _ = load_golden("uniform_nc6")
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    sts = [m.new_state(n), m.new_state(n)]
    outs = []
    for call in range(4):
        st = sts[call % 2 if call > 1 else 0]
        st.load(inp["P"], inp["T"], inp["Ni"])
        st.skip["flag"].zero_()  # every call a fresh flash (no skip-cache hits)
        m.flash_fim(st, form="mixed", fresh=True)
        torch.cuda.synchronize()
        outs.append(st.to_host())
    m.close()
    for o in outs[1:]:
        for k, v in outs[0].items():
            if isinstance(v, np.ndarray):
                np.testing.assert_array_equal(v, o[k], err_msg=k)


@pytest.mark.parametrize("form", ["plain", "batched", "mixed"])
def test_impec_matches_reference_golden(form):
    """ocpf_flash_impec (FlashIMPEC + IsoT_IMPEC::PassFlashValue) on a
    warm-started second step against the reference's outputs: identical
    phase counts except knife-edge cells, flash types and skip cache, every
    output (S, Nt, vf, vfP, vfi, vj, rho, xi, mu, xij) within 1e-8 relative
    or 10x the reference's own 1-ulp sensitivity."""
    from conftest import load_golden_impec, run_gpu_impec
    fl, inp, ref, fragile = load_golden_impec()
    got = run_gpu_impec(fl, inp, form=form)
    chk = CMP.check_impec(got, ref, fl.nc, noise=ref["noise"], fragile=fragile)
    assert chk["ok"], f"{form}: np_mismatch={list(chk['np_mismatch'])} worst={chk['worst']}"
    same = (got["phaseNum"] == ref["phaseNum"]) & ~fragile
    assert np.array_equal(got["ftype"][same], ref["ftype"][same])
    assert set(np.unique(ref["ftype"])) == {0, 1}
    sg, sr = got["skip"], ref["skip"]
    assert np.array_equal(sg["flag"][same].astype(int), sr["flag"][same].astype(int))


def _ni_ok(got, ref, noise, same):
    """Ni of the cells with matching phase counts within 1e-8 relative or
    10x the reference's own 1-ulp sensitivity."""
    e = CMP._rel(got["Ni"], ref["Ni"]).max(axis=1)
    allowed = np.maximum(1e-8, 10 * np.nan_to_num(noise["Ni"], nan=0.0))
    bad = np.nonzero(same & (e > allowed))[0]
    return bad


@pytest.mark.parametrize("impec", [False, True], ids=["fim", "impec"])
@pytest.mark.parametrize("form", ["plain", "batched", "mixed"])
def test_init_flash_matches_reference_golden(form, impec):
    """ocpf_init_flash_fim / ocpf_init_flash_impec (InitFlashFIM /
    InitFlashIMPEC + PassFlashValue) on 512 initial states against the
    reference: identical phase counts except knife-edge cells, the moles Ni
    that fill the pore volume and every output within 1e-8 relative or 10x
    the reference's own 1-ulp sensitivity, flash type 0 everywhere, and the
    skip cache the reference leaves."""
    from conftest import load_golden_init, run_gpu_init
    fl, inp, ref, refi, fragile = load_golden_init()
    r = refi if impec else ref
    got = run_gpu_init(fl, inp, impec=impec, form=form)
    if impec:
        chk = CMP.check_impec(got, r, fl.nc, noise=r["noise"], fragile=fragile)
    else:
        chk = CMP.check(got, r, fl.nc, noise=r["noise"], fragile=fragile)
    assert chk["ok"], f"{form}: np_mismatch={list(chk['np_mismatch'])} worst={chk['worst']}"
    same = (got["phaseNum"] == r["phaseNum"]) & ~fragile
    bad = _ni_ok(got, r, r["noise"], same)
    assert len(bad) == 0, bad
    assert np.all(got["ftype"] == 0)
    if not impec:
        # hydrocarbon nj: the phase fractions, as the reference's CopyPhase leaves them
        ex = r["phaseExist"][:, :2].astype(bool) & same[:, None]
        allowed = np.maximum(1e-8, 10 * r["noise"]["nj"])[:, None] * np.ones((1, 2))
        e = CMP._rel(got["nj"][:, :2], r["nj"][:, :2])
        assert np.all(e[ex] <= allowed[ex]), np.nonzero(np.any(ex & (e > allowed), axis=1))[0]
        sg, sr = got["skip"], ref["skip"]
        assert np.array_equal(sg["flag"][same].astype(int), sr["flag"][same].astype(int))


def test_init_flash_then_fim_step_matches_reference():
    """IsoT_FIM's start: InitFlashFIM, then the first FlashFIM at unchanged
    P and T, warm-started from the initialisation's phase counts,
    saturations, compositions and skip cache, against the reference making
    the same two calls (the warm step changes a few phase counts in the
    reference too: relaxed stability and skip tests replace the strict
    test). The initialised state fills the pore volume."""
    import torch
    from conftest import load_golden_init
    from opencaeporo_b200.flash import MixtureCompBatch
    fl, inp, ref, _, fragile = load_golden_init()
    nxt = ref["next"]
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["z"])
    m.init_flash(st, inp["Vpore"], S=inp["S"], form="batched")
    torch.cuda.synchronize()
    a = st.to_host()
    np.testing.assert_allclose(a["vf"], inp["Vpore"], rtol=1e-12)
    m.flash_fim(st, form="batched")
    torch.cuda.synchronize()
    b = st.to_host()
    m.close()
    chk = CMP.check(b, nxt, fl.nc, noise=nxt["noise"], fragile=fragile | nxt["fragile"])
    assert chk["ok"], CMP.check_summary(chk)
    same = b["phaseNum"] == nxt["phaseNum"]
    assert np.array_equal(b["ftype"][same], nxt["ftype"][same])


def _state_from(fl, inp):
    """A device state holding a fixture's warm-start inputs and skip cache."""
    import torch
    from opencaeporo_b200.flash import MixtureCompBatch
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["Ni"])
    o = st.out
    if "S" in inp:
        o["S"].copy_(torch.as_tensor(np.ascontiguousarray(inp["S"].T)))
    o["phaseNum"].copy_(torch.as_tensor(inp["lastNP"].astype(np.int32)))
    ncom = fl.nc + 1
    o["xij"].copy_(torch.as_tensor(np.ascontiguousarray(inp["xij"].reshape(n, 3 * ncom).T)))
    sk = inp["skip"]
    st.skip["flag"].copy_(torch.as_tensor(sk["flag"].astype(np.int32)))
    for k in ("minEig", "P", "T"):
        st.skip[k].copy_(torch.as_tensor(np.asarray(sk[k], dtype=np.float64)))
    st.skip["z"].copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(sk["z"]).T)))
    return m, st


def _host_all(st):
    h = st.to_host()
    sk = h.pop("skip")
    h.update({f"skip_{k}": v for k, v in sk.items()})
    return h


@pytest.mark.parametrize("impec", [False, True], ids=["fim", "impec"])
@pytest.mark.parametrize("form", ["plain", "batched"])
def test_subset_call_equals_full_call_on_its_cells(form, impec):
    """ocpf_flash_fim_subset / ocpf_flash_impec_subset (IsoT_AIMc's flashes
    of the implicit or explicit bulks): on a warm-started state, the listed
    cells (every third, in shuffled order) get exactly the full call's
    outputs and skip cache; every other cell keeps its state bit for bit."""
    import torch
    from conftest import load_golden_impec
    if impec:
        fl, inp, _, _ = load_golden_impec()
    else:
        fl, inp, _, _ = load_golden("warm_nc6")
    n = len(inp["P"])
    idx = np.random.default_rng(5).permutation(np.arange(0, n, 3))
    m, full = _state_from(fl, inp)
    if impec:
        full.out["vj"] = torch.zeros((3, n), dtype=torch.float64, device="cuda")
    before = _host_all(full)
    if impec:
        m.flash_impec(full, form=form)
    else:
        m.flash_fim(full, form=form)
    torch.cuda.synchronize()
    want = _host_all(full)
    m.close()
    m, sub = _state_from(fl, inp)
    if impec:
        sub.out["vj"] = torch.zeros((3, n), dtype=torch.float64, device="cuda")
    m.flash_subset(sub, torch.as_tensor(idx), impec=impec, form=form)
    torch.cuda.synchronize()
    got = _host_all(sub)
    m.close()
    rest = np.setdiff1d(np.arange(n), idx)
    for k, v in got.items():
        a, w, b = np.asarray(v), np.asarray(want[k]), np.asarray(before[k])
        f = a.dtype.kind == "f"
        assert np.array_equal(a[idx], w[idx], equal_nan=f), k
        assert np.array_equal(a[rest], b[rest], equal_nan=f), k


def test_subset_rejects_bad_arguments():
    import ctypes as C
    import torch
    from opencaeporo_b200 import _lib
    from opencaeporo_b200.flash import MixtureCompBatch
    fl, inp, _, _ = load_golden("uniform_nc6")
    m = MixtureCompBatch(fl)
    st = m.new_state(16)
    fin, sk, fo = m._structs(st)
    idx = torch.arange(4, dtype=torch.int64, device="cuda")
    L = _lib.lib()
    assert L.ocpf_flash_fim_subset(m._h, 4, None, 16, C.byref(fin), C.byref(sk), C.byref(fo), 0, None) != 0
    assert L.ocpf_flash_fim_subset(m._h, 17, idx.data_ptr(), 16, C.byref(fin), C.byref(sk), C.byref(fo), 0,
                                   None) != 0
    assert L.ocpf_flash_fim_subset(m._h, 0, None, 16, C.byref(fin), C.byref(sk), C.byref(fo), 0, None) == 0
    m.close()


def test_subset_skips_indices_outside_the_arrays():
    """An index outside [0, ncell) in a subset call names no cell: the other
    listed cells get the full call's outputs, no cell outside the list
    changes, and the Python mirror's optional check rejects such a list (and
    a repeated index) before calling."""
    import torch
    fl, inp, _, _ = load_golden("warm_nc6")
    n = len(inp["P"])
    good = np.arange(1, n, 5)
    m, full = _state_from(fl, inp)
    before = _host_all(full)
    m.flash_fim(full, form="batched")
    torch.cuda.synchronize()
    want = _host_all(full)
    m.close()
    m, sub = _state_from(fl, inp)
    idx = np.concatenate([good[:7], [-3, n, n + 100], good[7:]])
    m.flash_subset(sub, torch.as_tensor(idx), form="batched")
    torch.cuda.synchronize()
    got = _host_all(sub)
    with pytest.raises(ValueError):
        m.flash_subset(sub, torch.as_tensor(idx), form="batched", check_indices=True)
    with pytest.raises(ValueError):
        m.flash_subset(sub, torch.as_tensor(np.array([0, 2, 2])), form="batched", check_indices=True)
    m.close()
    rest = np.setdiff1d(np.arange(n), good)
    for k, v in got.items():
        a, w, b = np.asarray(v), np.asarray(want[k]), np.asarray(before[k])
        f = a.dtype.kind == "f"
        assert np.array_equal(a[good], w[good], equal_nan=f), k
        assert np.array_equal(a[rest], b[rest], equal_nan=f), k
