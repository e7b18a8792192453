"""The consumer of the flash's derivatives: the FIM Jacobian's bulk part
(IsoT_FIM::AssembleMatBulksNew, src/OCPFluidMethod.cpp:1569-1840) and the
upstream choice before it (src/BulkConn.cpp:170-215), on the reference's
own flash outputs of the uniform_nc6 fixture laid out as an 8 x 8 x 8 grid.

The oracle is the reference's own AssembleMatBulksNew, compiled from its
sources with stand-ins for the absent FASP library's type names
(oracle/_ref/libocpjac.so, ``make -C oracle jac``), and the restatement
oracle/fim_jacobian.py. The device kernels round every operation as the
restatement does, in the same order, so those two agree bit for bit; both
agree with the compiled reference to rounding (its dense product is a BLAS
dgemm, which sums in its own order)."""
import os

import numpy as np
import pytest

from oracle import fim_jacobian as J
from oracle import krpc as K

REF_LIB = os.path.join(os.path.dirname(J.__file__), "_ref", "libocpref.so")
# agreement with the compiled reference: every block within 1e-14 of its
# largest entry (the reference's dgemm and the restatement's ordered sums
# differ by a few units in the last place of the block's scale)
BLOCK_TOL = 1e-14


def _problem(seed=5):
    """Bulk arrays (cell-major), connections and the KrPc tables of the
    test grid."""
    from conftest import load_golden
    from opencaeporo_b200 import synth
    fl, inp, ref, _ = load_golden("uniform_nc6")
    n = len(inp["P"])
    nx = ny = nz = 8
    assert n == nx * ny * nz
    rng = np.random.default_rng(seed)
    regions = [synth.corey_tables(501)]
    kp = K.restated(regions, inp["P"], np.nan_to_num(ref["S"], nan=0.0))
    idx = np.arange(n).reshape(nz, ny, nx)
    bId, eId, area = [], [], []
    for axis, a in ((2, 150.0), (1, 150.0), (0, 400.0)):
        lo = np.take(idx, range(idx.shape[axis] - 1), axis=axis).ravel()
        hi = np.take(idx, range(1, idx.shape[axis]), axis=axis).ravel()
        bId += lo.tolist()
        eId += hi.tolist()
        area += (a * rng.uniform(0.5, 1.5, len(lo))).tolist()
    cn = {"bId": np.array(bId, np.int64), "eId": np.array(eId, np.int64), "area": np.array(area)}
    depth = (np.repeat(np.arange(nz), nx * ny) * 10.0 + 8000.0) + rng.uniform(-1, 1, n)
    bk = {k: ref[k] for k in ("phaseExist", "pSderExist", "pVnumCom", "S", "rho", "xi", "mu", "muP", "xiP",
                              "rhoP", "xij", "rhox", "xix", "mux", "dSec_dPri", "vfP", "vfi")}
    bk.update({"kr": kp["kr"], "Pj": kp["Pj"], "dKr_dS": kp["dKr_dS"].reshape(n, 3, 3),
               "dPcj_dS": kp["dPcj_dS"].reshape(n, 3, 3), "v": rng.uniform(5e3, 5e4, n),
               "poroP": rng.uniform(1e-6, 1e-5, n), "depth": depth})
    return fl, bk, cn


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="compiled reference not built")
def test_product_matches_reference_daabpbc():
    """The dense product of the assembly has the reference's semantics (A B +
    C, row-major) and agrees with its BLAS to rounding."""
    rng = np.random.default_rng(3)
    for k in (8, 15):
        A, B, Cm = rng.normal(size=(8, k)), rng.normal(size=(k, 8)), rng.normal(size=(8, 8))
        got = J.product(Cm, A, B, 1.0)
        want = J.product_reference(A, B, Cm)
        assert np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want))


def test_restatement_blocks_are_finite_and_scatter_consistently():
    """On the test grid every block is finite; each off-diagonal pair is the
    negated begin contribution and the end contribution, and the diagonal
    equals accumulation plus the incident contributions in connection order."""
    fl, bk, cn = _problem()
    up, rho = J.upwind(bk, cn)
    cn.update(upblock=up, upblock_Rho=rho)
    ncom = fl.nc + 1
    diag, offEB, offBE = J.assemble(bk, cn, ncom, 0.5)
    assert np.all(np.isfinite(diag)) and np.all(np.isfinite(offEB)) and np.all(np.isfinite(offBE))
    b0 = int(cn["bId"][0])
    acc = J.accumulation(bk, b0, ncom)
    want = acc.copy()
    for c in range(len(cn["bId"])):
        if cn["bId"][c] == b0:
            want = want + (-offEB[c])
        elif cn["eId"][c] == b0:
            want = want + (-offBE[c])
    np.testing.assert_array_equal(diag[b0], want)


def _blocks_close(got, want, what):
    scale = np.max(np.abs(want), axis=(1, 2), keepdims=True)
    err = np.abs(got - want) / np.maximum(scale, 1e-300)
    assert np.all(np.isfinite(got) == np.isfinite(want)), what
    assert np.nanmax(err) <= BLOCK_TOL, (what, float(np.nanmax(err)))


@pytest.mark.skipif(not J.reference_available(), reason="compiled reference assembly not built")
def test_restatement_matches_compiled_reference_assembly():
    """The restatement against the reference's own AssembleMatBulksNew on the
    test grid: every diagonal and off-diagonal block, in the reference's
    scatter order, to rounding of the block's scale."""
    fl, bk, cn = _problem()
    up, rho = J.upwind(bk, cn)
    cn.update(upblock=up, upblock_Rho=rho)
    ncom = fl.nc + 1
    for dt in (0.25, 3.0):
        got = J.assemble(bk, cn, ncom, dt)
        want = J.assemble_reference(bk, cn, ncom, dt)
        for name, g, w in zip(("diag", "offEB", "offBE"), got, want):
            _blocks_close(g, w, name)


def _dev(a, dtype=None):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


def _soa(bk, n):
    import torch
    out = {}
    for k, v in bk.items():
        a = np.asarray(v)
        if a.ndim == 1:
            out[k] = _dev(a.astype(np.float64))
        else:
            a2 = a.reshape(n, -1).T
            if k in ("phaseExist", "pSderExist", "pVnumCom"):
                out[k] = _dev(a2.astype(np.int32))
            else:
                out[k] = _dev(np.nan_to_num(a2.astype(np.float64), nan=np.nan))
    return out


@pytest.mark.gpu
def test_upwind_and_jacobian_match_restatement_bit_for_bit():
    import torch
    from opencaeporo_b200.fim_jacobian import ConnGraph
    fl, bk, cn = _problem()
    n = len(bk["vfP"])
    ncom, ncol = fl.nc + 1, fl.nc + 2
    up_r, rho_r = J.upwind(bk, cn)
    g = ConnGraph(n, cn["bId"], cn["eId"], cn["area"])
    dbk = _soa(bk, n)
    up, rho = g.upwind(dbk)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(up.cpu().numpy().T, up_r)
    np.testing.assert_array_equal(rho.cpu().numpy().T, rho_r)
    cn.update(upblock=up_r, upblock_Rho=rho_r)
    dt = 0.25
    diag_r, offEB_r, offBE_r = J.assemble(bk, cn, ncom, dt)
    out = g.jacobian(fl.nc, dt, dbk, up, rho)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy().T.reshape(-1, ncol, ncol) for k, v in out.items()}
    g.close()
    np.testing.assert_array_equal(got["offEB"], offEB_r)
    np.testing.assert_array_equal(got["offBE"], offBE_r)
    np.testing.assert_array_equal(got["diag"], diag_r)
    if J.reference_available():
        want = J.assemble_reference(bk, cn, ncom, dt)
        for name, w in zip(("diag", "offEB", "offBE"), want):
            _blocks_close(got[name], w, name)


@pytest.mark.gpu
def test_jacobian_rejects_shapes_no_flash_writes():
    """A connection whose bulk reports more compositions than components gets
    NaN blocks (the kernel reads nothing outside the arrays)."""
    import torch
    from opencaeporo_b200.fim_jacobian import ConnGraph
    fl, bk, cn = _problem()
    n = len(bk["vfP"])
    bk = dict(bk)
    bk["pVnumCom"] = bk["pVnumCom"].copy()
    bad = int(cn["bId"][0])
    bk["pVnumCom"][bad, 0] = 99
    g = ConnGraph(n, cn["bId"], cn["eId"], cn["area"])
    dbk = _soa(bk, n)
    up, rho = g.upwind(dbk)
    out = g.jacobian(fl.nc, 1.0, dbk, up, rho)
    torch.cuda.synchronize()
    offEB = out["offEB"].cpu().numpy()
    g.close()
    touched = (cn["bId"] == bad) | (cn["eId"] == bad)
    assert np.all(np.isnan(offEB[:, touched]))
    assert np.all(np.isfinite(offEB[:, ~touched]))


def test_conn_graph_rejects_bad_connections():
    from opencaeporo_b200 import _lib
    import ctypes as C
    try:
        L = _lib.lib()
    except RuntimeError:
        pytest.skip("library not built")
    b = np.array([0, 1], np.int64)
    e = np.array([1, 1], np.int64)
    a = np.ones(2)
    h = C.c_void_p()
    assert L.ocpf_conn_create(2, 2, b.ctypes.data, e.ctypes.data, a.ctypes.data, 0, C.byref(h)) == 1  # self loop
    e2 = np.array([1, 5], np.int64)
    assert L.ocpf_conn_create(2, 2, b.ctypes.data, e2.ctypes.data, a.ctypes.data, 0, C.byref(h)) == 1  # out of range
