"""CPU tests of the oracles: the plain-C restatement (oracle/flash_port.c) and,
when it can be built here, the compiled reference (oracle/_ref) against the
golden fixtures that the reference produced."""
import os

import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden
from oracle import compare as CMP
from oracle import REF_ROOT
from oracle import oracle as O

REF_SRC = os.path.join(REF_ROOT, "src", "MixtureComp.cpp")


def _run(kind, fl, inp):
    skip = {k: np.array(v, copy=True) for k, v in inp["skip"].items()}
    return O.flash_fim(kind, fl, inp["P"], inp["T"], inp["Ni"], S=inp["S"], lastNP=inp["lastNP"],
                       xij=inp["xij"], skip=skip, nthreads=4)


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_port_matches_reference_goldens(case):
    """The port reproduces the reference's outputs: identical phase counts
    (except knife-edge cells) and <= 1e-8 relative error on every output, or
    10x the reference's own 1-ulp sensitivity where that is larger."""
    fl, inp, ref, fragile = load_golden(case)
    got = _run("port", fl, inp)
    chk = CMP.check(got, ref, fl.nc, noise=ref["noise"], fragile=fragile)
    assert chk["ok"], f"{case}: {CMP.check_summary(chk)}"
    res = CMP.compare(got, ref, fl.nc)
    for k in ("phaseExist", "bRowSizedSdP", "pSderExist", "pVnumCom"):
        assert res[k + "_mismatch"] == 0, f"{case}: {k}"


@pytest.mark.parametrize("case", ["warm_nc6"])
def test_port_skip_cache_and_flash_type(case):
    """Warm-started step: the flash type (0 full / 1 skip / 2 two-phase warm)
    and the SkipStaAnaly cache written back agree with the reference."""
    fl, inp, ref, fragile = load_golden(case)
    got = _run("port", fl, inp)
    ok = ~fragile
    assert np.array_equal(got["ftype"][ok], ref["ftype"][ok])
    assert set(np.unique(ref["ftype"])) == {0, 1, 2}
    sk_g, sk_r = got["skip"], ref["skip"]
    assert np.array_equal(sk_g["flag"][ok], sk_r["flag"][ok])
    np.testing.assert_allclose(sk_g["P"][ok], sk_r["P"][ok], rtol=0, atol=0)
    np.testing.assert_allclose(sk_g["z"][ok], sk_r["z"][ok], rtol=1e-15)
    # single-precision minimum eigenvalue (ssyevd in the reference)
    f = sk_r["flag"].astype(bool) & ok
    np.testing.assert_allclose(sk_g["minEig"][f], sk_r["minEig"][f], rtol=2e-5, atol=2e-6)


def test_port_iteration_counts_close():
    """Stability and split iteration counts of the port track the reference's
    (they are noise-sensitive at tol^2 = 1e-24, so only the totals are held
    to a few percent)."""
    fl, inp, ref, fragile = load_golden("uniform_nc6")
    got = _run("port", fl, inp)
    a = got["iters"].sum(axis=0).astype(float)
    b = ref["iters"].sum(axis=0).astype(float)
    assert np.all(np.abs(a - b) <= 0.05 * np.maximum(b, 1) + 5), (a, b)


def test_port_spe5_bitwise():
    """On the SPE5 deck fluid the restatement is bit-for-bit the reference."""
    fl, inp, ref, _ = load_golden("spe5")
    got = _run("port", fl, inp)
    assert np.array_equal(got["phaseNum"], ref["phaseNum"])
    ex = ref["phaseExist"].astype(bool)
    for k in ("S", "Nt", "vf"):
        np.testing.assert_allclose(got[k], ref[k], rtol=1e-15, atol=0)
    for k in ("rho", "xi", "mu"):
        np.testing.assert_allclose(got[k][ex], ref[k][ex], rtol=1e-15, atol=0)


@pytest.mark.skipif(not os.path.exists(REF_SRC), reason="reference sources not present")
def test_reference_reproduces_goldens():
    """The compiled reference, rebuilt here, still produces the committed
    fixtures (guards the fixtures and the harness)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", os.path.join(os.path.dirname(O.__file__)), "ref"])
    for case in GOLDEN_CASES:
        fl, inp, ref, _ = load_golden(case)
        got = _run("reference", fl, inp)
        res = CMP.compare(got, ref, fl.nc)
        assert len(res["np_mismatch"]) == 0, case
        assert CMP.max_rel(res) == 0.0, f"{case}: {CMP.summary(res)}"


def test_compare_flags_planted_error():
    """The comparison catches a planted error in oracle output."""
    fl, inp, ref, _ = load_golden("spe5")
    bad = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in ref.items()}
    bad["xi"][0, 0] *= 1 + 1e-6
    res = CMP.compare(bad, ref, fl.nc)
    assert res["xi"] > 5e-7
    bad["phaseNum"][1] = 2
    res = CMP.compare(bad, ref, fl.nc)
    assert list(res["np_mismatch"]) == [1]


@pytest.mark.skipif(not O.available("reference"), reason="oracle/_ref not built")
def test_reference_with_skip_option_off():
    """With the skip option off the reference's FlashFIM writes its skip flag
    through an unallocated array; the loader runs it with the option on and a
    fresh cache instead, which must give the same flash as the port with the
    option off."""
    fl, inp, _, _ = load_golden("uniform_nc6")
    fl = fl.with_controls(use_skip=False)
    P = np.full(64, 72.5)
    T, Ni = inp["T"][:64], inp["Ni"][:64]
    a = O.flash_fim("reference", fl, P, T, Ni, nthreads=2)
    b = O.flash_fim("port", fl, P, T, Ni, nthreads=2)
    assert np.array_equal(a["NPhc"], b["NPhc"])
    assert np.array_equal(a["ftype"], np.zeros(64, np.int32))


@pytest.mark.skipif(not os.path.exists(REF_SRC), reason="reference sources not present")
def test_reference_reproduces_impec_golden():
    """The compiled reference's FlashIMPEC, rebuilt here, reproduces the
    IMPEC fixture (guards the fixture and the IMPEC harness)."""
    import subprocess
    from conftest import load_golden_impec
    subprocess.check_call(["make", "-s", "-C", os.path.join(os.path.dirname(O.__file__)), "ref"])
    fl, inp, ref, _ = load_golden_impec()
    skip = {k: np.array(v, copy=True) for k, v in inp["skip"].items()}
    got = O.flash_impec(fl, inp["P"], inp["T"], inp["Ni"], lastNP=inp["lastNP"], xij=inp["xij"], skip=skip,
                        nthreads=4)
    e = CMP.impec_errors(got, ref, fl.nc)
    assert e["same"].all()
    for k in CMP.IMPEC_FLOAT_KEYS:
        assert np.nanmax(e[k]) == 0.0, k


@pytest.mark.skipif(not os.path.exists(REF_SRC), reason="reference sources not present")
@pytest.mark.parametrize("impec", [False, True], ids=["fim", "impec"])
def test_reference_reproduces_init_golden(impec):
    """The compiled reference's InitFlashFIM / InitFlashIMPEC, rebuilt here,
    reproduces the initialisation fixture bit for bit (guards the fixture
    and the harness's initialisation entry), and the initialised state
    fills the pore volume: vf = Vpore to rounding."""
    import subprocess
    from conftest import load_golden_init
    subprocess.check_call(["make", "-s", "-C", os.path.join(os.path.dirname(O.__file__)), "ref"])
    fl, inp, ref, refi, _ = load_golden_init()
    r = refi if impec else ref
    got = O.init_flash(fl, inp["P"], inp["T"], inp["z"], inp["S"], inp["Vpore"], impec=impec,
                       skip=O.new_skip(len(inp["P"]), fl.nc), nthreads=4)
    e = CMP.impec_errors(got, r, fl.nc) if impec else CMP.per_cell_errors(got, r, fl.nc)
    assert e["same"].all()
    for k in (CMP.IMPEC_FLOAT_KEYS if impec else CMP.FLOAT_KEYS):
        assert np.nanmax(e[k]) == 0.0, k
    assert np.array_equal(got["Ni"], r["Ni"])
    np.testing.assert_allclose(got["vf"], inp["Vpore"], rtol=1e-12)
    if not impec:
        # the fixture's next FlashFIM from the initialised state
        nxt = ref["next"]
        s2 = O.flash_fim("reference", fl, inp["P"], inp["T"], got["Ni"], S=got["S"],
                         lastNP=got["phaseNum"].astype(np.int32), xij=np.nan_to_num(got["xij"], nan=0.0),
                         skip=got["skip"], nthreads=4)
        e2 = CMP.per_cell_errors(s2, nxt, fl.nc)
        assert e2["same"].all()
        for k in CMP.FLOAT_KEYS:
            assert np.nanmax(e2[k]) == 0.0, k
