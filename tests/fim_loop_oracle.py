"""The synthetic FIM loop (opencaeporo_b200/fim_loop.py) at full size with
every iteration's flash checked against the compiled reference on a seeded
sample of 4096 cells: the sample's inputs and warm-start state (last phase
count, S, xij, skip cache) before the flash go to the reference's own
MixtureComp::FlashFIM on the host, its outputs are compared with the GPU's.
Needs a GPU and oracle/_ref (built from the reference sources by
`make -C oracle ref`; the plain-C restatement is used when it is absent).

    python tests/fim_loop_oracle.py [--forms plain,fast] [--steps 20] [--newton 4]
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import compare as CMP  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--forms", default="plain,fast")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--newton", type=int, default=4)
    args = ap.parse_args()
    from opencaeporo_b200.fim_loop import run
    from opencaeporo_b200.workload import bench_fluid
    fl = bench_fluid()
    kind = "reference" if O.available("reference") else "port"
    stats = {}

    def hook(form, step, it, before, after):
        skip = {k: np.ascontiguousarray(v) for k, v in before["skip"].items()}
        skip["flag"] = skip["flag"].astype(np.int32)
        n = len(before["P"])
        r = O.flash_fim(kind, fl, before["P"], before["T"], before["Ni"], S=before["S"], lastNP=before["lastNP"],
                        xij=before["xij"].reshape(n, 3, fl.nc + 1), skip=skip, nthreads=0)
        got = dict(after)
        got["xij"] = got["xij"].reshape(n, 3, fl.nc + 1)
        e = CMP.per_cell_errors(got, r, fl.nc)
        # well determined: single-phase cells, and two-phase cells whose
        # split the reference converged (ePEC <= 1e-9)
        det = e["same"] & ((r["NPhc"] == 1) | (r["ePEC"] <= 1e-9))
        worst = np.zeros(n)
        s = stats.setdefault(form, {"iterations": 0, "phase_mismatch_max": 0, "well_determined_min": n,
                                    "max_rel_err_well_determined": 0.0, "share_le_1e-8_min": 1.0,
                                    "max_rel_err_per_output": {}})
        for k in CMP.FLOAT_KEYS:
            ek = np.nan_to_num(e[k], nan=0.0)
            worst = np.fmax(worst, ek)
            s["max_rel_err_per_output"][k] = max(s["max_rel_err_per_output"].get(k, 0.0),
                                                 float(np.max(ek[det], initial=0.0)))
        s["iterations"] += 1
        s["phase_mismatch_max"] = max(s["phase_mismatch_max"], int((~e["same"]).sum()))
        s["well_determined_min"] = min(s["well_determined_min"], int(det.sum()))
        s["max_rel_err_well_determined"] = max(s["max_rel_err_well_determined"], float(np.max(worst[det], initial=0.0)))
        s["share_le_1e-8_min"] = min(s["share_le_1e-8_min"], float(np.mean(worst[det] <= 1e-8)) if det.any() else 1.0)

    res = run(tuple(args.forms.split(",")), args.steps, args.newton, hook=hook)
    res["oracle"] = {"kind": kind, "sample_cells_per_iteration": 4096, "per_form": stats}
    print(json.dumps(res))


if __name__ == "__main__":
    main()
