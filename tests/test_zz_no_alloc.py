"""GPU test of ocpf_flash_fim_noalloc, the batched flash for callers that
cannot allocate device memory (an application that owns the GPU's memory
through its own pool, runs under a fixed memory budget, or must not let a
flash call synchronise the device the way cudaMalloc/cudaFree can). Its
scratch is an array compiled into the library, shared by every call on a
device.

The entry point is called through the C ABI twice in a row, on two different
batches, and each result is checked against the existing batched entry point
(ocpf_flash_fim, OCPF_FORM_BATCHED) on the same inputs: the second call must
not see anything of the first one left in the shared array. This file is
collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from oracle import compare as CMP

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _state(m, fl, inp):
    """Device state of a golden case (inputs, warm start and skip cache)."""
    torch = _torch()
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["Ni"])
    o = st.out
    o["S"].copy_(torch.as_tensor(np.ascontiguousarray(inp["S"].T)))
    o["phaseNum"].copy_(torch.as_tensor(inp["lastNP"].astype(np.int32)))
    o["xij"].copy_(torch.as_tensor(np.ascontiguousarray(inp["xij"].reshape(n, 3 * (fl.nc + 1)).T)))
    sk = inp["skip"]
    st.skip["flag"].copy_(torch.as_tensor(sk["flag"].astype(np.int32)))
    for k in ("minEig", "P", "T"):
        st.skip[k].copy_(torch.as_tensor(np.asarray(sk[k], dtype=np.float64)))
    st.skip["z"].copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(sk["z"]).T)))
    return st


def _run_noalloc(m, st):
    from opencaeporo_b200 import _lib
    torch = _torch()
    fin, sk, fo = m._structs(st)
    stream = torch.cuda.current_stream(m.device)
    rc = _lib.lib().ocpf_flash_fim_noalloc(m._h, st.ncell, C.byref(fin), C.byref(sk), C.byref(fo),
                                           C.c_void_p(stream.cuda_stream))
    assert rc == _lib.OCPF_OK, _lib.lib().ocpf_status_string(rc)
    torch.cuda.synchronize()
    return st.to_host()


def _run_batched(m, st):
    torch = _torch()
    m.flash_fim(st, form="batched")
    torch.cuda.synchronize()
    return st.to_host()


def test_noalloc_matches_batched_on_two_calls_in_a_row():
    from opencaeporo_b200.flash import MixtureCompBatch
    _torch()
    fl, _, _, _ = load_golden("uniform_nc6")
    m = MixtureCompBatch(fl)
    try:
        for case in ("uniform_nc6", "warm_nc6"):  # same fluid, different batches
            fl_c, inp, ref, _ = load_golden(case)
            want = _run_batched(m, _state(m, fl_c, inp))
            got = _run_noalloc(m, _state(m, fl_c, inp))
            for k in ("phaseNum", "iters", "status", "ftype"):
                np.testing.assert_array_equal(got[k], want[k], err_msg=f"{case} {k}")
            chk = CMP.check(got, want, fl.nc, noise=ref["noise"], tol=1e-9)
            assert chk["ok"], f"{case}: {CMP.check_summary(chk)}"
            np.testing.assert_array_equal(got["skip"]["flag"], want["skip"]["flag"])
            np.testing.assert_allclose(got["skip"]["minEig"], want["skip"]["minEig"], rtol=1e-6, atol=1e-7)
    finally:
        m.close()


def test_noalloc_rejects_batches_beyond_its_scratch():
    from opencaeporo_b200 import _lib
    from opencaeporo_b200.flash import MixtureCompBatch
    _torch()
    fl = load_golden("spe5")[0]
    m = MixtureCompBatch(fl)
    try:
        st = m.new_state(4)
        fin, sk, fo = m._structs(st)
        rc = _lib.lib().ocpf_flash_fim_noalloc(m._h, _lib.NOALLOC_MAX_CELLS + 1, C.byref(fin), C.byref(sk),
                                               C.byref(fo), None)
        assert rc == _lib.OCPF_ERANGE
        assert b"OCPF_NOALLOC_MAX_CELLS" in _lib.lib().ocpf_status_string(rc)
    finally:
        m.close()
