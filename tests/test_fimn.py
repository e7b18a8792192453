"""MixtureComp::FlashFIMn and InitFlashFIMn with IsoT_FIMn::PassFlashValue
(src/MixtureComp.cpp:355-442, 575-695; src/OCPFluidMethod.cpp:3129-3196):
the FIM formulation whose secondary variables are the saturations and the
phase moles, through ocpf_flash_fimn / ocpf_init_flash_fimn.

The fixture tests/golden/fimn_nc6.npz holds the compiled reference's
outputs of a fresh step, a warm step and an initialisation with their
self-noise. CPU tests pin it (the compiled reference reproduces it; its
equilibrium equals the FIM fixtures'; the balances its derivative rows obey);
GPU tests hold the device's outputs to it, per form, with the bar of
oracle.compare.check and the same balances."""
import os

import numpy as np
import pytest

from conftest import FIMN_CALLS, load_golden_fimn
from oracle import compare as CMP
from oracle import oracle as O

KW = dict(errors=CMP.fimn_errors, keys=CMP.FIMN_KEYS)


def _reference_run(fl, call, inp):
    if call == "init":
        return O.init_flash_fimn(fl, inp["P"], inp["T"], inp["z"], inp["S"], inp["Vpore"],
                                 skip=O.new_skip(len(inp["P"]), fl.nc), nthreads=4)
    return O.flash_fimn(fl, inp["P"], inp["T"], inp["Ni"], S=inp["S"], lastNP=inp["lastNP"], xij=inp["xij"],
                        skip={k: np.array(v) for k, v in inp["skip"].items()}, nthreads=4)


def _same(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)],
                                                                                          b[~np.isnan(b)])


@pytest.mark.skipif(not O.available("reference"), reason="compiled reference not built")
@pytest.mark.parametrize("call", FIMN_CALLS)
def test_reference_reproduces_fixture(call):
    fl, calls = load_golden_fimn()
    inp, ref, _ = calls[call]
    r = _reference_run(fl, call, inp)
    for k in ("phaseNum", "S", "dSec_dPri", "bRowSizedSdP", "xix", "mux", "vfi", "nj", "res", "resPc"):
        assert _same(r[k], ref[k]), k


def test_fimn_equilibrium_is_fims():
    """FlashFIMn runs FlashFIM's flash type and phase equilibrium
    (src/MixtureComp.cpp:593-603 against :505-515): on warm_nc6's inputs the
    reference's FIMn phase counts, saturations, compositions and phase
    properties are FlashFIM's bit for bit, and its volume derivatives (from
    the phase-mole rows, CalVfiVfp_full03) agree with FlashFIM's to
    rounding."""
    from conftest import load_golden
    fl, calls = load_golden_fimn()
    _, ref, _ = calls["warm"]
    _, _, fim, _ = load_golden("warm_nc6")
    assert np.array_equal(ref["phaseNum"], fim["phaseNum"])
    ex = fim["phaseExist"].astype(bool)
    for k in ("S", "Nt", "vf"):
        assert np.array_equal(ref[k], fim[k]), k
    for k in ("rho", "xi", "mu"):
        assert np.array_equal(ref[k][ex], fim[k][ex]), k
    assert np.array_equal(ref["xij"][ex], fim["xij"][ex])
    # the pressure partials at fixed composition: the two tails form dZ/dP
    # with differently rounded expressions
    for k in ("xiP", "rhoP", "muP"):
        e = CMP._rel(ref[k][ex], fim[k][ex])
        assert np.max(e) < 1e-12, (k, np.max(e))
    for k in ("vfP", "vfi"):
        e = CMP._rel(ref[k], fim[k]).reshape(len(ref["phaseNum"]), -1).max(axis=1)
        allowed = np.maximum(1e-8, 10 * np.maximum(ref["noise"][k], fim["noise"][k]))
        assert np.all(e <= allowed), (k, np.max(e / allowed))


def test_fimn_init_moles_are_init_fims():
    """InitFlashFIMn fills the pore volume as InitFlashFIM does
    (src/MixtureComp.cpp:365-411 against :271-314): the same moles, bit for
    bit, on init_nc6's initial states."""
    fl, calls = load_golden_fimn()
    _, ref, _ = calls["init"]
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "init_nc6.npz"))
    assert np.array_equal(ref["Ni"], g["out_Ni"])


def _balances(out, nc):
    """Per cell: the largest violation of S_o + S_g + S_w = 1 and
    n_0i + n_1i = N_i differentiated (sum of the saturation rows = 0, sum of
    each component's phase-mole rows = e_i), relative to the rows' scale;
    and whether every single-phase cell's residual column is zero."""
    n = len(out["phaseNum"])
    ncol = nc + 2
    rows = out["bRowSizedSdP"].astype(int)
    D = np.asarray(out["dSec_dPri"], dtype=np.float64).reshape(n, -1)
    nph = out["phaseExist"][:, :2].sum(axis=1).astype(int)
    worst = np.zeros(n)
    for c in range(n):
        k = nph[c]
        assert rows[c] == k + 1 + k * nc
        M = D[c, :rows[c] * ncol].reshape(rows[c], ncol)
        sS = M[:k + 1].sum(axis=0)
        scale = np.max(np.abs(M[:k + 1]), initial=1e-300)
        v = np.max(np.abs(sS)) / scale
        nrow = M[k + 1:].reshape(k, nc, ncol).sum(axis=0)
        want = np.zeros((nc, ncol))
        want[np.arange(nc), 1 + np.arange(nc)] = 1.0
        v = max(v, np.max(np.abs(nrow - want)) / max(np.max(np.abs(M[k + 1:])), 1.0))
        worst[c] = v
    single = nph == 1
    res0 = np.all(np.asarray(out["res"])[single, :nc + 2] == 0) and np.all(np.asarray(out["resPc"])[single] == 0)
    return worst, res0


@pytest.mark.parametrize("call", FIMN_CALLS)
def test_fixture_balances(call):
    fl, calls = load_golden_fimn()
    _, ref, _ = calls[call]
    worst, res0 = _balances(ref, fl.nc)
    assert np.max(worst) < 1e-9, np.max(worst)
    assert res0


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plain", "batched", "mixed"])
@pytest.mark.parametrize("call", FIMN_CALLS)
def test_fimn_matches_reference_golden(call, form):
    """Identical phase counts except knife-edge cells, every FIM output,
    nj, res and resPc within 1e-8 relative or 10x the reference's own 1-ulp
    sensitivity (res and resPc are residuals at the convergence tolerance:
    the reference itself determines them only to that sensitivity, and to
    zero in single-phase cells), flash types, the skip cache, Ni of the
    initialisation, and the balances the derivative rows obey."""
    from conftest import run_gpu_fimn
    fl, calls = load_golden_fimn()
    inp, ref, fragile = calls[call]
    got = run_gpu_fimn(fl, call, inp, form=form)
    chk = CMP.check(got, ref, fl.nc, noise=ref["noise"], fragile=fragile, **KW)
    assert chk["ok"], f"{call}/{form}: np_mismatch={list(chk['np_mismatch'])} worst={chk['worst']}"
    same = (got["phaseNum"] == ref["phaseNum"]) & ~fragile
    assert np.array_equal(got["ftype"][same], ref["ftype"][same])
    assert np.array_equal(got["skip"]["flag"][same].astype(int), ref["skip"]["flag"][same].astype(int))
    if call == "init":
        # Ni is InitFlashFIM's (test_fimn_init_moles_are_init_fims): its bar is
        # the self-noise recorded with that fixture
        noise_ni = np.load(os.path.join(os.path.dirname(__file__), "golden", "init_nc6.npz"))["noise_Ni"]
        e = CMP._rel(got["Ni"], ref["Ni"]).max(axis=1)
        allowed = np.maximum(1e-8, 10 * noise_ni.astype(np.float64))
        assert np.all(e[same] <= allowed[same]), np.nonzero(same & (e > allowed))
    worst, res0 = _balances(got, fl.nc)
    assert np.max(worst) < 1e-9, np.max(worst)
    assert res0


@pytest.mark.gpu
def test_fimn_rejects_missing_outputs():
    """nj, res and resPc are required outputs of the FIMn entry points."""
    import ctypes as C
    import torch
    from opencaeporo_b200 import _lib
    from opencaeporo_b200.flash import MixtureCompBatch
    fl, calls = load_golden_fimn()
    m = MixtureCompBatch(fl)
    st = m.new_state(8)
    fin, sk, fo = m._structs(st)
    res = torch.zeros((3 * (fl.nc + 2), 8), dtype=torch.float64, device="cuda")
    rpc = torch.zeros(8, dtype=torch.float64, device="cuda")
    L = _lib.lib()
    assert L.ocpf_flash_fimn(m._h, 8, C.byref(fin), C.byref(sk), C.byref(fo), None, rpc.data_ptr(), 0, None) != 0
    assert L.ocpf_flash_fimn(m._h, 8, C.byref(fin), C.byref(sk), C.byref(fo), res.data_ptr(), None, 0, None) != 0
    fo.nj = None
    assert L.ocpf_flash_fimn(m._h, 8, C.byref(fin), C.byref(sk), C.byref(fo), res.data_ptr(), rpc.data_ptr(), 0,
                             None) != 0
    m.close()
