"""The flash inside the synthetic FIM loop (warm starts across Newton
iterations and time steps: skip cache, two-phase warm starts, relaxed
stability), on a reduced grid: every form runs, the faster forms agree with
the plain FP64 form iteration by iteration, and KrPc, the upstream choice and
the Jacobian's bulk part run after the flash on its device arrays."""
import pytest


@pytest.mark.gpu
def test_fim_loop_forms_agree_with_plain():
    from opencaeporo_b200.fim_loop import run
    res = run(("plain", "batched", "mixed"), steps=3, newton=3, grid=(24, 40, 12), log=lambda *_: None)
    assert res["cells"] == 24 * 40 * 12
    b = res["batched_vs_plain"]
    assert b["max_phase_mismatch"] == 0, b
    assert b["max_rel_err"] < 1e-8, b
    m = res["mixed_vs_plain"]
    assert m["max_phase_mismatch"] <= 2, m
    # the steps after the flash ran on its arrays every iteration
    assert res["jacobian_finite"]
    assert set(res["after_flash_ms_per_iteration"]) == {"krpc", "upwind", "jacobian"}
