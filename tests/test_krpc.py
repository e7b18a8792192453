"""Relative permeability and capillary pressure after the flash
(IsoT_FIM::CalKrPc, src/OCPFluidMethod.cpp:1189-1199, with FlowUnit_ODGW01,
src/FlowUnit.cpp:183-349, and FlowUnit_ODGW02, :522-671): the oracle
against the golden fixtures made by the compiled reference, and
ocpf_cal_krpc against both, bit for bit (the kernel rounds every operation
as the reference does)."""
import os

import numpy as np
import pytest

from oracle import REF_ROOT
from oracle import krpc as K

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "krpc.npz")
REF_SRC = os.path.join(REF_ROOT, "src", "FlowUnit.cpp")
KEYS = ("kr", "Pc", "Pj", "dKr_dS", "dPcj_dS")


def _fixture():
    d = np.load(GOLDEN)
    regions = [(d["swof0"], d["sgof0"]), (d["swof1"], d["sgof1"])]
    return regions, d["in_P"], d["in_S"], d["in_satnum"], {k: d[f"out_{k}"] for k in KEYS}


def _fixture_sof3():
    """FlowUnit_ODGW02 (SWFN / SGFN / SOF3) fixture: regions, inputs, the
    FIM call's outputs and the IMPEC call's (kr, Pc, Pj: another oil model)."""
    d = np.load(os.path.join(HERE, "golden", "krpc_sof3.npz"))
    regions = [(d[f"swfn{i}"], d[f"sgfn{i}"], d[f"sof3{i}"]) for i in range(2)]
    return (regions, d["in_P"], d["in_S"], d["in_satnum"], {k: d[f"out_{k}"] for k in KEYS},
            {k: d[f"impec_{k}"] for k in ("kr", "Pc", "Pj")})


def test_restated_oracle_matches_fixture():
    regions, P, S, sn, ref = _fixture()
    got = K.restated(regions, P, S, sn)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


@pytest.mark.skipif(not os.path.exists(REF_SRC), reason="reference sources not present")
def test_reference_reproduces_fixture():
    import subprocess
    from oracle import oracle as O
    subprocess.check_call(["make", "-s", "-C", os.path.dirname(O.__file__), "ref"])
    regions, P, S, sn, ref = _fixture()
    got = K.reference(regions, P, S, sn, nthreads=4)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    # the IMPEC call (no derivatives) gives the same kr, Pc, Pj
    nod = K.reference(regions, P, S, sn, deriv=False, nthreads=4)
    for k in ("kr", "Pc", "Pj"):
        np.testing.assert_array_equal(nod[k], ref[k], err_msg=k)


def test_restated_sof3_oracle_matches_fixture():
    regions, P, S, sn, ref, impec = _fixture_sof3()
    got = K.restated_sof3(regions, P, S, sn)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    nod = K.restated_sof3(regions, P, S, sn, deriv=False)
    for k in ("kr", "Pc", "Pj"):
        np.testing.assert_array_equal(nod[k], impec[k], err_msg=k)
    # the two calls' oil models differ (Stone II vs the default model), the
    # rest agrees; the default model's small-denominator branch is covered
    assert not np.array_equal(ref["kr"][:, 0], impec["kr"][:, 0])
    np.testing.assert_array_equal(ref["kr"][:, 1:], impec["kr"][:, 1:])
    kmax = {r: regions[r][2][-1, 1] for r in range(2)}
    assert np.sum(impec["kr"][:, 0] == np.array([kmax[r] for r in sn])) > 10


@pytest.mark.skipif(not os.path.exists(REF_SRC), reason="reference sources not present")
def test_reference_reproduces_sof3_fixture():
    import subprocess
    from oracle import oracle as O
    subprocess.check_call(["make", "-s", "-C", os.path.dirname(O.__file__), "ref"])
    regions, P, S, sn, ref, impec = _fixture_sof3()
    got = K.reference_sof3(regions, P, S, sn, nthreads=4)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    nod = K.reference_sof3(regions, P, S, sn, deriv=False, nthreads=4)
    for k in ("kr", "Pc", "Pj"):
        np.testing.assert_array_equal(nod[k], impec[k], err_msg=k)


def test_table_search_is_state_independent():
    """The reference searches each table from the interval it found for the
    previous cell; for a non-decreasing first column that search always ends
    at the last node <= S, so the order of the cells does not matter (the
    device kernel bisects for that node directly)."""
    regions, P, S, sn, ref = _fixture()
    perm = np.random.default_rng(1).permutation(len(P))
    got = K.restated(regions, P[perm], S[perm], sn[perm])
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k][perm], err_msg=k)


def _dev(a, dtype=None):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


def _run_gpu(regions, P, S, sn, deriv=True):
    import torch
    from opencaeporo_b200.krpc import FlowUnitBatch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    fu = FlowUnitBatch(regions)
    out = fu.cal_krpc(_dev(P), _dev(S.T), None if sn is None else _dev(sn, torch.int32), deriv=deriv)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy().T.copy() for k, v in out.items()}
    fu.close()
    return res


@pytest.mark.gpu
def test_krpc_matches_reference_bit_for_bit():
    regions, P, S, sn, ref = _fixture()
    got = _run_gpu(regions, P, S, sn)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    nod = _run_gpu(regions, P, S, sn, deriv=False)
    assert set(nod) == {"kr", "Pc", "Pj"}
    for k in ("kr", "Pc", "Pj"):
        np.testing.assert_array_equal(nod[k], ref[k], err_msg=k)


@pytest.mark.gpu
def test_krpc_sof3_matches_reference_bit_for_bit():
    """FlowUnit_ODGW02 on the device: the FIM call (Stone II, dKro/dS_o) and
    the IMPEC call (the default oil model) equal the compiled reference's."""
    regions, P, S, sn, ref, impec = _fixture_sof3()
    got = _run_gpu(regions, P, S, sn)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    nod = _run_gpu(regions, P, S, sn, deriv=False)
    assert set(nod) == {"kr", "Pc", "Pj"}
    for k in ("kr", "Pc", "Pj"):
        np.testing.assert_array_equal(nod[k], impec[k], err_msg=k)


@pytest.mark.gpu
def test_krpc_unknown_region_gives_nan():
    regions, P, S, sn, ref = _fixture()
    bad = sn.copy()
    bad[:3] = [-1, 2, 1000]
    got = _run_gpu(regions, P, S, bad)
    assert np.all(np.isnan(got["kr"][:3])) and np.all(np.isnan(got["dKr_dS"][:3]))
    for k in KEYS:
        np.testing.assert_array_equal(got[k][3:], ref[k][3:], err_msg=k)


@pytest.mark.gpu
def test_krpc_after_the_flash():
    """The step after the flash on device: kr and Pc of the flash's own S
    (read in place), against the oracle on the same saturations."""
    import torch
    from conftest import load_golden, run_gpu
    from opencaeporo_b200.flash import MixtureCompBatch
    from opencaeporo_b200.krpc import FlowUnitBatch
    fl, inp, _, _ = load_golden("uniform_nc6")
    regions = _fixture()[0][:1]
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["Ni"])
    m.flash_fim(st, form="batched", fresh=True)
    fu = FlowUnitBatch(regions)
    out = fu.cal_krpc(st.P, st.out["S"])
    torch.cuda.synchronize()
    S = st.out["S"].cpu().numpy().T.copy()
    got = {k: v.cpu().numpy().T.copy() for k, v in out.items()}
    fu.close()
    m.close()
    want = K.restated(regions, inp["P"], S)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_krpc_rejects_bad_tables():
    """Argument checks need no GPU work: a table of one row or with a
    decreasing saturation column is refused at creation."""
    from opencaeporo_b200 import _lib
    import ctypes as C
    try:
        L = _lib.lib()
    except RuntimeError:
        pytest.skip("library not built")
    w = np.array([[0.2, 0, 1, 1], [0.1, 0.5, 0, 0]], dtype=np.float64)
    g = np.array([[0.0, 0, 1, 0], [0.8, 1, 0, 1]], dtype=np.float64)
    regs = (_lib.Satfunc * 1)()
    regs[0] = _lib.Satfunc(2, 2, w.ctypes.data, g.ctypes.data)
    h = C.c_void_p()
    assert L.ocpf_krpc_create(regs, 1, 0, C.byref(h)) == 1  # decreasing Sw
    regs[0] = _lib.Satfunc(1, 2, g.ctypes.data, g.ctypes.data)
    assert L.ocpf_krpc_create(regs, 1, 0, C.byref(h)) == 1  # one row
    assert L.ocpf_krpc_create(regs, 0, 0, C.byref(h)) == 1  # no region


def test_krpc_sof3_rejects_bad_tables():
    """The SWFN / SGFN / SOF3 creator refuses a table of one row, a
    decreasing saturation column or a missing table, before any GPU work."""
    from opencaeporo_b200 import _lib
    import ctypes as C
    L = _lib.lib()
    regions = _fixture_sof3()[0]
    w, g, o = (np.ascontiguousarray(t) for t in regions[0])
    bad = o[::-1].copy()  # decreasing So
    h = C.c_void_p()
    regs = (_lib.Satfunc3 * 1)()
    for args in ((len(w), len(g), len(bad), w, g, bad), (1, len(g), len(o), w, g, o),
                 (len(w), len(g), len(o), w, None, o)):
        nw, ng, no, a, b, c = args
        regs[0] = _lib.Satfunc3(nw, ng, no, 0, a.ctypes.data, None if b is None else b.ctypes.data, c.ctypes.data)
        assert L.ocpf_krpc_create_sof3(regs, 1, 0, C.byref(h)) == 1
    assert L.ocpf_krpc_create_sof3(regs, 0, 0, C.byref(h)) == 1
