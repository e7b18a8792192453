"""The learned initialiser of the fast form (``OCPF_FORM_FAST``): data,
training and attachment. No counterpart in the reference.

A small MLP maps a cell's (ln P, T, z_1..z_NC) to the logit of "the flash
ends with two hydrocarbon phases" and the ln K_i = ln(y_i / x_i) of that
split. Trained on states flashed by the plain GPU form, it lets the fast
form start a confidently two-phase fresh cell's split from the predicted K
and skip the stability test; the split's own checks (and the stability test
wherever the network is not confident, or its split fails) keep every
answer the converged one.

Forward, backward and the Adam step are the library's own kernels
(``ocpf_mlp_forward`` / ``ocpf_mlp_grad`` / ``ocpf_mlp_adam``: BF16 tensor-
core products with FP32 accumulation); this module only moves data.

    python -m opencaeporo_b200.learn --train 8388608 --out opencaeporo_b200/models/learned_init_nc6.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import time

import numpy as np

from . import _lib
from ._lib import check, lib

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "models", "learned_init_nc6.npz")
NPARAM = 6288          # ocpf_mlp_param_count()
HIDDEN = 64
IO = 16                # padded input / output width


def _torch():
    import torch
    return torch


def raw_features(P, T, Ni):
    """(ln P, T, z_1..z_NC) per cell, feature-major float64 [NC + 2, n]
    (Ni [n, NC + 1], water last)."""
    Ni = np.asarray(Ni, dtype=np.float64)
    nc = Ni.shape[1] - 1
    z = Ni[:, :nc] / np.sum(np.abs(Ni[:, :nc]), axis=1, keepdims=True)
    return np.ascontiguousarray(np.vstack([np.log(np.asarray(P, dtype=np.float64))[None, :],
                                           np.asarray(T, dtype=np.float64)[None, :], z.T]))


def targets_from_flash(out: dict, nc: int):
    """Labels from flash outputs (host arrays as MixtureCompBatch returns
    them): t0 = 1 for two hydrocarbon phases, t_i = ln(y_i / x_i) (gas over
    oil) for those cells, 0 elsewhere; and the ln K weight (1 where defined)."""
    nphc = np.asarray(out["phaseNum"]) - 1
    two = nphc == 2
    n = len(nphc)
    t = np.zeros((nc + 1, n))
    t[0] = two
    xij = np.asarray(out["xij"]).reshape(n, 3, nc + 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        lnk = np.log(xij[:, 1, :nc] / xij[:, 0, :nc]).T
    ok = two & np.all(np.isfinite(lnk), axis=0)
    t[1:, ok] = lnk[:, ok]
    return t, ok.astype(np.float64)


def init_params(nin: int, nout: int, seed: int = 0) -> np.ndarray:
    """Kaiming-uniform weights for SiLU layers, zero biases, zero padding."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    o = 0
    W1 = np.zeros((HIDDEN, IO), np.float32)
    W1[:, :nin] = rng.uniform(-1, 1, (HIDDEN, nin)) * np.sqrt(6.0 / nin)
    p[o:o + HIDDEN * IO] = W1.ravel(); o += HIDDEN * IO + HIDDEN
    W2 = rng.uniform(-1, 1, (HIDDEN, HIDDEN)) * np.sqrt(6.0 / HIDDEN)
    p[o:o + HIDDEN * HIDDEN] = W2.ravel(); o += HIDDEN * HIDDEN + HIDDEN
    W3 = np.zeros((IO, HIDDEN), np.float32)
    W3[:nout] = rng.uniform(-1, 1, (nout, HIDDEN)) * np.sqrt(3.0 / HIDDEN)
    p[o:o + IO * HIDDEN] = W3.ravel()
    return p


class Initializer:
    """Trained network plus its input normalisation and confidence."""

    def __init__(self, nc, params, in_mean, in_scale, confidence=0.95, meta=None):
        self.nc = int(nc)
        self.params = np.ascontiguousarray(params, dtype=np.float32)
        self.in_mean = np.ascontiguousarray(in_mean, dtype=np.float32)
        self.in_scale = np.ascontiguousarray(in_scale, dtype=np.float32)
        self.confidence = float(confidence)
        self.meta = meta or {}
        assert self.params.shape == (NPARAM,) and self.in_mean.shape == (self.nc + 2,)

    def save(self, path):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, nc=self.nc, params=self.params, in_mean=self.in_mean, in_scale=self.in_scale,
                 confidence=self.confidence, **{f"meta_{k}": np.asarray(v) for k, v in self.meta.items()})

    @classmethod
    def load(cls, path):
        d = np.load(path)
        meta = {k[5:]: d[k] for k in d.files if k.startswith("meta_")}
        return cls(int(d["nc"]), d["params"], d["in_mean"], d["in_scale"], float(d["confidence"]), meta)

    def attach(self, m):
        """Hands the network to a MixtureCompBatch (ocpf_set_initializer)."""
        fp = C.POINTER(C.c_float)
        check(lib().ocpf_set_initializer(m._h, self.params.ctypes.data_as(fp), self.in_mean.ctypes.data_as(fp),
                                         self.in_scale.ctypes.data_as(fp), C.c_float(self.confidence)),
              "ocpf_set_initializer")

    def normalise(self, raw):
        return np.ascontiguousarray((raw - self.in_mean[:, None]) / self.in_scale[:, None], dtype=np.float32)


def forward(params_dev, x_dev, nout):
    """Network outputs [nout, n] for normalised features x [nin, n] (device tensors)."""
    torch = _torch()
    x_dev = x_dev.contiguous()  # the kernel reads x[f * n + s]
    nin, n = x_dev.shape
    y = torch.empty((nout, n), dtype=torch.float32, device=x_dev.device)
    check(lib().ocpf_mlp_forward(nin, nout, n, params_dev.data_ptr(), x_dev.data_ptr(), y.data_ptr(), None),
          "ocpf_mlp_forward")
    return y


def grad(params_dev, x_dev, t_dev, w_dev, lnk_weight, grad_dev, loss_dev):
    x_dev, t_dev, w_dev = x_dev.contiguous(), t_dev.contiguous(), w_dev.contiguous()
    nin, n = x_dev.shape
    nout = t_dev.shape[0]
    check(lib().ocpf_mlp_grad(nin, nout, n, params_dev.data_ptr(), x_dev.data_ptr(), t_dev.data_ptr(),
                              w_dev.data_ptr(), C.c_float(lnk_weight), grad_dev.data_ptr(), loss_dev.data_ptr(),
                              None), "ocpf_mlp_grad")


def train(x, t, w, epochs=8, batch=8192, lr=2e-3, lnk_weight=1.0, seed=0, device=0, log=print):
    """Adam training with the library's kernels. x [nin, n] normalised float32,
    t [nout, n], w [n] (host arrays). Returns the FP32 parameters."""
    torch = _torch()
    dev = torch.device("cuda", device)
    nin, n = x.shape
    nout = t.shape[0]
    X = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32), device=dev)
    Tt = torch.as_tensor(np.ascontiguousarray(t, dtype=np.float32), device=dev)
    W = torch.as_tensor(np.ascontiguousarray(w, dtype=np.float32), device=dev)
    p = torch.as_tensor(init_params(nin, nout, seed), device=dev)
    g = torch.zeros(NPARAM, dtype=torch.float32, device=dev)
    m1 = torch.zeros_like(g)
    m2 = torch.zeros_like(g)
    loss = torch.zeros(2, dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    step = 0
    nb = n // batch
    total = epochs * nb
    for ep in range(epochs):
        perm = torch.randperm(n, device=dev, generator=gen)
        loss.zero_()
        t0 = time.time()
        for b in range(nb):
            idx = perm[b * batch:(b + 1) * batch]
            xb = X[:, idx].contiguous()
            tb = Tt[:, idx].contiguous()
            wb = W[idx].contiguous()
            grad(p, xb, tb, wb, lnk_weight, g, loss)
            step += 1
            lr_t = lr * 0.5 * (1 + np.cos(np.pi * step / total))  # cosine decay
            check(lib().ocpf_mlp_adam(p.data_ptr(), g.data_ptr(), m1.data_ptr(), m2.data_ptr(), step,
                                      C.c_float(lr_t), None), "ocpf_mlp_adam")
        torch.cuda.synchronize(dev)
        l = loss.cpu().numpy() / (nb * batch)
        log(f"epoch {ep}: logistic {l[0]:.4f}  lnK mse {l[1]:.4f}  ({time.time() - t0:.1f} s)")
    return p.cpu().numpy()


def evaluate(init: Initializer, raw, t, w, device=0):
    """Accuracy figures of a trained network on held-out states."""
    torch = _torch()
    dev = torch.device("cuda", device)
    x = torch.as_tensor(init.normalise(raw), device=dev)
    p = torch.as_tensor(init.params, device=dev)
    y = forward(p, x, init.nc + 1).cpu().numpy()
    prob = 1 / (1 + np.exp(-y[0]))
    two = t[0] > 0.5
    conf = prob >= init.confidence
    lnk_err = np.abs(y[1:] - t[1:])[:, w > 0]
    return {"n": int(len(prob)), "accuracy": float(np.mean((prob >= 0.5) == two)),
            "confident_share": float(np.mean(conf)), "confident_two_phase_recall": float(np.mean(conf[two])),
            "confident_precision": float(np.mean(two[conf])) if conf.any() else 1.0,
            "lnk_mae": float(np.mean(lnk_err)) if lnk_err.size else 0.0,
            "lnk_p95": float(np.quantile(lnk_err, 0.95)) if lnk_err.size else 0.0}


def flash_dataset(fluid, n, seed, device=0, form="batched", steps=20):
    """n seeded states of the 1M-cell workload's distribution (70 % uniform,
    30 % near the envelope) flashed as fresh cells; returns raw features,
    targets and weights."""
    import torch
    from .flash import MixtureCompBatch
    from .workload import make_workload
    w = make_workload(fluid, n, seed, device)
    m = MixtureCompBatch(fluid, device)
    chunk = 1 << 20
    st = m.new_state(min(n, chunk))
    ts, ws = [], []
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        k = c1 - c0
        P = np.full(st.ncell, 1000.0); T = np.full(st.ncell, 100.0)
        N = np.tile(w["Ni"][c0:c0 + 1], (st.ncell, 1))
        P[:k], T[:k], N[:k] = w["P"][c0:c1], w["T"][c0:c1], w["Ni"][c0:c1]
        st.load(P, T, N)
        m.flash_fim(st, form=form, fresh=True)
        torch.cuda.synchronize()
        out = {"phaseNum": st.out["phaseNum"][:k].cpu().numpy(),
               "xij": st.out["xij"][:, :k].cpu().numpy().T.copy()}
        t, wt = targets_from_flash(out, fluid.nc)
        ts.append(t); ws.append(wt)
    m.close()
    return raw_features(w["P"], w["T"], w["Ni"]), np.hstack(ts), np.concatenate(ws)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1 << 23)
    ap.add_argument("--test", type=int, default=1 << 20)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--confidence", type=float, default=0.95)
    args = ap.parse_args()
    from .workload import bench_fluid
    fl = bench_fluid()
    t0 = time.time()
    raw, t, w = flash_dataset(fl, args.train, 7001)
    print(f"training set: {raw.shape[1]} states, two-phase {t[0].mean():.3f} ({time.time() - t0:.0f} s)")
    mean = raw.mean(axis=1)
    scale = raw.std(axis=1) + 1e-12
    init0 = Initializer(fl.nc, np.zeros(NPARAM, np.float32), mean, scale, args.confidence)
    params = train(init0.normalise(raw), t, w, epochs=args.epochs)
    init = Initializer(fl.nc, params, mean, scale, args.confidence,
                       meta={"train_states": raw.shape[1], "train_seed": 7001, "epochs": args.epochs})
    raw_h, t_h, w_h = flash_dataset(fl, args.test, 9001)
    ev = evaluate(init, raw_h, t_h, w_h)
    print("held-out:", ev)
    init.meta.update({f"heldout_{k}": v for k, v in ev.items()})
    init.save(args.out)
    print("saved", args.out)


if __name__ == "__main__":
    main()
