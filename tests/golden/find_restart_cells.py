"""Finds the inputs of the ``restart_nc6`` golden case (needs a GPU).

Cells whose PhaseSplit keeps restarting are rare -- a handful per million
states of the bench workload sit close enough to a critical point that the
split's successive substitution needs thousands of iterations -- too rare to
find with the CPU reference in reasonable time. This script generates the
1,048,576-state bench workload (``bench.make_workload``, the bench's seed),
flashes it with the plain GPU form and keeps the 48 states with the most
split successive-substitution iterations plus the first 16 states, in
``tests/golden/restart_nc6_cells.npz`` (inputs only). ``make_golden.py
restart_nc6`` then computes the reference's outputs for them on the CPU.

    python tests/golden/find_restart_cells.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main():
    import torch
    import bench
    from opencaeporo_b200.flash import MixtureCompBatch
    fl = bench.bench_fluid()
    n = bench.NCELL
    w = bench.make_workload(fl, n, bench.SEED, 0)
    m = MixtureCompBatch(fl, 0)
    st = m.new_state(n)
    st.load(w["P"], w["T"], w["Ni"])
    m.flash_fim(st, form="plain", fresh=True)
    torch.cuda.synchronize()
    it = st.to_host()["iters"]
    m.close()
    order = np.argsort(-it[:, 2], kind="stable")
    keep = np.unique(np.concatenate([order[:48], np.arange(16)]))
    out = os.path.join(HERE, "restart_nc6_cells.npz")
    np.savez_compressed(out, P=w["P"][keep], T=w["T"][keep], Ni=w["Ni"][keep], index=keep,
                        gpu_iters=it[keep])
    print(f"wrote {out}: split SSM iterations of the kept cells: {sorted(it[keep, 2].tolist())[-10:]}")


if __name__ == "__main__":
    main()
