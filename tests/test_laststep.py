"""The last-time-step copies (IsoT_FIM::UpdateLastTimeStep /
ResetToLastTimeStep, src/OCPFluidMethod.cpp:2915-2960 and 2859-2897, and
SkipStaAnaly's, src/AcceleratePVT.cpp:122-138): argument checks on the CPU
(they return before any device call), and on the GPU that the copies are
exact and that a flash after ResetToLastTimeStep is the flash the saved
state would have given (a cut time step repeated with a smaller step)."""
import ctypes as C

import numpy as np
import pytest

from opencaeporo_b200 import _lib

OK, EINVAL = 0, 1


def _fake_out(base, stride=1 << 20):
    """An ocpf_fim_out whose fields are distinct fake addresses (never
    dereferenced: the calls below fail their checks first)."""
    return _lib.FimOut(*[base + i * stride for i in range(len(_lib.OUT_FIELDS))])


def _fake_skip(base, stride=1 << 20):
    return _lib.Skip(*[base + i * stride for i in range(len(_lib.SKIP_FIELDS))])


def test_copy_arrays_rejects_bad_pairs():
    L = _lib.lib()

    def call(dst, src, nb):
        n = len(dst)
        return L.ocpf_copy_arrays(n, (C.c_void_p * n)(*dst), (C.c_void_p * n)(*src), (C.c_int64 * n)(*nb), None)

    assert L.ocpf_copy_arrays(0, None, None, None, None) == OK
    assert L.ocpf_copy_arrays(-1, None, None, None, None) == EINVAL
    assert L.ocpf_copy_arrays(_lib.COPY_MAX + 1, None, None, None, None) == EINVAL
    assert L.ocpf_copy_arrays(1, None, None, None, None) == EINVAL
    assert call([0x10000], [0x20000], [-8]) == EINVAL              # negative size
    assert call([0x10000], [None], [8]) == EINVAL                  # null source of a non-empty pair
    assert call([0x10000], [0x10008], [16]) == EINVAL              # overlap
    assert call([0x10008], [0x10000], [16]) == EINVAL
    # all pairs empty or in place: nothing to launch, no device touched
    assert call([0x10000, 0x30000], [0x20000, 0x30000], [0, 64]) == OK
    # a bad pair anywhere: nothing launched
    assert call([0x10000, 0x30000], [0x20000, 0x30004], [8, 8]) == EINVAL


def test_step_copies_reject_bad_arguments():
    L = _lib.lib()
    cur, last = _fake_out(0x100000000), _fake_out(0x900000000)
    sk, lsk = _fake_skip(0x500000000), _fake_skip(0xd00000000)
    for fn in (L.ocpf_update_last_step, L.ocpf_reset_to_last_step):
        assert fn(0, 16, C.byref(cur), C.byref(sk), C.byref(last), C.byref(lsk), None) == EINVAL  # nc
        assert fn(17, 16, C.byref(cur), C.byref(sk), C.byref(last), C.byref(lsk), None) == EINVAL
        assert fn(6, -1, C.byref(cur), C.byref(sk), C.byref(last), C.byref(lsk), None) == EINVAL  # ncell
        assert fn(6, 16, None, C.byref(sk), C.byref(last), C.byref(lsk), None) == EINVAL
        assert fn(6, 16, C.byref(cur), C.byref(sk), C.byref(last), None, None) == EINVAL       # one skip
        one_sided = _fake_out(0x900000000)
        one_sided.xij = None                                        # a field set on one side only
        assert fn(6, 16, C.byref(cur), None, C.byref(one_sided), None, None) == EINVAL
        overlap = _fake_out(0x100000000 + 8)                        # every field overlaps its pair
        assert fn(6, 16, C.byref(cur), None, C.byref(overlap), None, None) == EINVAL
        # nothing to copy (no cells, or every field in place): no launch
        assert fn(6, 0, C.byref(cur), C.byref(sk), C.byref(last), C.byref(lsk), None) == OK
        assert fn(6, 16, C.byref(cur), C.byref(sk), C.byref(cur), C.byref(sk), None) == OK


def _same_bits(x, y):
    """Bit-wise equality (NaN outputs such as ePEC of cells without a split
    compare equal to themselves)."""
    import torch
    return x.shape == y.shape and x.dtype == y.dtype and torch.equal(x.view(torch.uint8), y.view(torch.uint8))


def _state_equal(a, b):
    """Names of the arrays (outputs, skip cache) that differ bit-wise."""
    bad = [k for k in a.out if not _same_bits(a.out[k], b.out[k])]
    bad += ["skip." + k for k in a.skip if not _same_bits(a.skip[k], b.skip[k])]
    return bad


@pytest.mark.gpu
def test_update_and_reset_round_trip():
    """UpdateLastTimeStep copies every output and the skip cache exactly;
    after a second flash changed them, ResetToLastTimeStep restores them,
    P and Ni included."""
    import torch
    from conftest import load_golden
    from opencaeporo_b200.flash import MixtureCompBatch
    fl, inp, ref, fragile = load_golden("warm_nc6")
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["Ni"])
    m.flash_fim(st, form="batched", fresh=True)
    last = m.new_last(st)
    m.update_last_step(st, last)
    torch.cuda.synchronize()
    assert _state_equal(st, last) == []
    assert torch.equal(st.P, last.P) and torch.equal(st.Ni, last.Ni)
    saved = {k: v.clone() for k, v in st.out.items()}
    saved_skip = {k: v.clone() for k, v in st.skip.items()}
    P0, N0 = st.P.clone(), st.Ni.clone()
    # the next step moves pressure and composition; its flash overwrites
    # the outputs and the skip cache
    st.load(inp["P"] * 0.93, inp["T"], inp["Ni"] * np.linspace(0.9, 1.1, inp["Ni"].shape[1]))
    m.flash_fim(st, form="batched")
    torch.cuda.synchronize()
    assert not all(_same_bits(st.out[k], saved[k]) for k in ("S", "xij", "rho"))
    m.reset_to_last_step(st, last)
    torch.cuda.synchronize()
    for k in st.out:
        assert _same_bits(st.out[k], saved[k]), k
    for k in st.skip:
        assert _same_bits(st.skip[k], saved_skip[k]), k
    assert torch.equal(st.P, P0) and torch.equal(st.Ni, N0)
    m.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["batched", "fast"])
def test_cut_step_repeats_from_the_saved_state(form):
    """A time-step cut: flash step n, save, flash a step that is rejected,
    reset, flash a smaller step. The result equals that smaller step's flash
    from an untouched copy of step n's state, bit for bit (warm starts and
    the skip cache come from the restored arrays)."""
    import torch
    from conftest import load_golden
    from opencaeporo_b200.flash import MixtureCompBatch
    fl, inp, ref, fragile = load_golden("warm_nc6")
    m = MixtureCompBatch(fl)
    if form == "fast":
        from opencaeporo_b200.learn import DEFAULT_MODEL, Initializer
        Initializer.load(DEFAULT_MODEL).attach(m)
    n = len(inp["P"])
    a, b = m.new_state(n), m.new_state(n)
    for s in (a, b):
        s.load(inp["P"], inp["T"], inp["Ni"])
        m.flash_fim(s, form=form, fresh=True)
    last = m.new_last(a)
    m.update_last_step(a, last)
    a.load(inp["P"] * 0.8, inp["T"], inp["Ni"])          # the rejected step
    m.flash_fim(a, form=form)
    m.reset_to_last_step(a, last)
    for s in (a, b):                                      # the smaller step
        s.load(inp["P"] * 0.95, inp["T"], inp["Ni"])
        m.flash_fim(s, form=form)
    torch.cuda.synchronize()
    assert _state_equal(a, b) == []
    m.close()


@pytest.mark.gpu
def test_copy_arrays_any_alignment():
    """Pairs at every byte offset and odd sizes (the 1-, 2-, 4-, 8- and
    16-byte paths); bytes outside the ranges are left alone."""
    import torch
    from opencaeporo_b200.flash import copy_arrays
    g = torch.Generator(device="cuda").manual_seed(7)
    src = torch.randint(0, 256, (1 << 20,), dtype=torch.uint8, device="cuda", generator=g)
    dst = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    pairs, spans = [], []
    at = 0
    for off, size in [(0, 4096), (1, 4095), (2, 1002), (4, 4 * 1001), (8, 8 * 3001), (3, 70001),
                      (16, 16 * 20000), (5, 1), (0, 16 * 1024 * 3 + 16)]:
        s0, d0 = at + off, at + 2 * off + 7 * (off % 2)
        pairs.append((dst[d0:d0 + size], src[s0:s0 + size]))
        spans.append((d0, s0, size))
        at = d0 + size + 64
    assert at < (1 << 20)
    copy_arrays(pairs)
    torch.cuda.synchronize()
    want = torch.zeros_like(dst)
    for d0, s0, size in spans:
        want[d0:d0 + size] = src[s0:s0 + size]
    assert torch.equal(dst, want)
