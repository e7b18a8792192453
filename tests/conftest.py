"""Shared test set-up: the ``gpu`` marker, import paths and the golden-fixture
loader."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ("spe5", "uniform_nc6", "warm_nc6", "uniform_nc3", "uniform_nc9", "uniform_nc12",
                "near_nc6", "restart_nc6", "config1_nc6")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    """Returns (fluid, inputs, reference outputs, fragile mask) of a fixture;
    the reference's per-field self-noise is in out['noise']."""
    from opencaeporo_b200.fluid import Controls, Fluid

    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    c = d["controls"]
    ctl = Controls(rr_maxit=int(c[0]), rr_tol=c[1], ssmsta_maxit=int(c[2]), ssmsta_tol=c[3],
                   ssmsta_eyt=c[4], nrsta_maxit=int(c[5]), nrsta_tol=c[6], ssmsp_maxit=int(c[7]),
                   ssmsp_tol=c[8], nrsp_maxit=int(c[9]), nrsp_tol=c[10], use_skip=bool(c[11]))
    nc = len(d["fluid_Tc"])
    fl = Fluid(nc=nc, Tc=d["fluid_Tc"], Pc=d["fluid_Pc"], Vc=d["fluid_Vc"], MW=d["fluid_MW"],
               Acf=d["fluid_Acf"], BIC=d["fluid_BIC"], OmegaA=d["fluid_OmegaA"],
               OmegaB=d["fluid_OmegaB"], Vshift=d["fluid_Vshift"], LBCcoef=d["fluid_LBCcoef"],
               pvtw=d["fluid_pvtw"], std_rho_w=float(d["fluid_std_rho_w"]), controls=ctl,
               name=str(d["fluid_name"]))
    inp = {"P": d["in_P"], "T": d["in_T"], "Ni": d["in_Ni"], "S": d["in_S"],
           "lastNP": d["in_lastNP"].astype(np.int32), "xij": d["in_xij"],
           "skip": {k: d[f"skipin_{k}"] for k in ("flag", "minEig", "P", "T", "z")}}
    out = {k[4:]: d[k] for k in d.files if k.startswith("out_")}
    out["skip"] = {k: d[f"skipout_{k}"] for k in ("flag", "minEig", "P", "T", "z")}
    out["noise"] = {k[6:]: d[k].astype(np.float64) for k in d.files if k.startswith("noise_")}
    return fl, inp, out, d["fragile"]


@pytest.fixture(scope="session")
def golden():
    return load_golden


def load_golden_impec(name="impec_nc6"):
    """(fluid, inputs, reference IMPEC outputs with their self-noise, fragile
    mask) of the FlashIMPEC fixture."""
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    fl, _, _, _ = _fluid_only(d)
    inp = {"P": d["in_P"], "T": d["in_T"], "Ni": d["in_Ni"], "lastNP": d["in_lastNP"].astype(np.int32),
           "xij": d["in_xij"], "skip": {k: d[f"skipin_{k}"] for k in ("flag", "minEig", "P", "T", "z")}}
    out = {k[4:]: d[k] for k in d.files if k.startswith("out_")}
    out["skip"] = {k: d[f"skipout_{k}"] for k in ("flag", "minEig", "P", "T", "z")}
    out["noise"] = {k[6:]: d[k].astype(np.float64) for k in d.files if k.startswith("noise_")}
    return fl, inp, out, d["fragile"]


def _fluid_only(d):
    from opencaeporo_b200.fluid import Controls, Fluid
    c = d["controls"]
    ctl = Controls(rr_maxit=int(c[0]), rr_tol=c[1], ssmsta_maxit=int(c[2]), ssmsta_tol=c[3],
                   ssmsta_eyt=c[4], nrsta_maxit=int(c[5]), nrsta_tol=c[6], ssmsp_maxit=int(c[7]),
                   ssmsp_tol=c[8], nrsp_maxit=int(c[9]), nrsp_tol=c[10], use_skip=bool(c[11]))
    nc = len(d["fluid_Tc"])
    fl = Fluid(nc=nc, Tc=d["fluid_Tc"], Pc=d["fluid_Pc"], Vc=d["fluid_Vc"], MW=d["fluid_MW"],
               Acf=d["fluid_Acf"], BIC=d["fluid_BIC"], OmegaA=d["fluid_OmegaA"],
               OmegaB=d["fluid_OmegaB"], Vshift=d["fluid_Vshift"], LBCcoef=d["fluid_LBCcoef"],
               pvtw=d["fluid_pvtw"], std_rho_w=float(d["fluid_std_rho_w"]), controls=ctl,
               name=str(d["fluid_name"]))
    return fl, None, None, None


def run_gpu_impec(fl, inp, form="plain"):
    """One FlashIMPEC of a fixture's inputs through ocpf_flash_impec on cuda:0."""
    import torch
    from opencaeporo_b200.flash import MixtureCompBatch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["Ni"])
    st.out["phaseNum"].copy_(torch.as_tensor(inp["lastNP"].astype(np.int32)))
    ncom = fl.nc + 1
    st.out["xij"].copy_(torch.as_tensor(np.ascontiguousarray(inp["xij"].reshape(n, 3 * ncom).T)))
    sk = inp["skip"]
    st.skip["flag"].copy_(torch.as_tensor(sk["flag"].astype(np.int32)))
    for k in ("minEig", "P", "T"):
        st.skip[k].copy_(torch.as_tensor(np.asarray(sk[k], dtype=np.float64)))
    st.skip["z"].copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(sk["z"]).T)))
    m.flash_impec(st, form=form)
    torch.cuda.synchronize()
    res = st.to_host()
    m.close()
    return res


def load_golden_init(name="init_nc6"):
    """(fluid, inputs, reference outputs of InitFlashFIM, of InitFlashIMPEC,
    fragile mask) of the initialisation fixture; each output dict carries
    its self-noise under ``noise``."""
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    fl, _, _, _ = _fluid_only(d)
    inp = {"P": d["in_P"], "T": d["in_T"], "z": d["in_z"], "S": d["in_S"], "Vpore": d["in_Vpore"]}
    out = {k[4:]: d[k] for k in d.files if k.startswith("out_")}
    out["skip"] = {k: d[f"skipout_{k}"] for k in ("flag", "minEig", "P", "T", "z")}
    out["noise"] = {k[6:]: d[k].astype(np.float64) for k in d.files if k.startswith("noise_")}
    outi = {k[5:]: d[k] for k in d.files if k.startswith("outi_")}
    outi["noise"] = {k[7:]: d[k].astype(np.float64) for k in d.files if k.startswith("noisei_")}
    # the reference's next FlashFIM from the initialised state
    nxt = {k[5:]: d[k] for k in d.files if k.startswith("out2_")}
    nxt["noise"] = {k[7:]: d[k].astype(np.float64) for k in d.files if k.startswith("noise2_")}
    nxt["fragile"] = d["fragile2"]
    out["next"] = nxt
    return fl, inp, out, outi, d["fragile"]


def run_gpu_init(fl, inp, impec=False, form="plain", init=None):
    """One InitFlashFIM (or InitFlashIMPEC) of a fixture's initial states
    through the C ABI on cuda:0; the host outputs carry ``Ni``."""
    import torch
    from opencaeporo_b200.flash import MixtureCompBatch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    m = MixtureCompBatch(fl)
    if init is not None:
        init.attach(m)
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["z"])
    m.init_flash(st, inp["Vpore"], S=inp["S"], impec=impec, form=form)
    torch.cuda.synchronize()
    res = st.to_host()
    res["Ni"] = st.Ni.cpu().numpy().T.copy()
    m.close()
    return res


def run_gpu(fl, inp, form="plain", init=None):
    """One flash of a fixture's inputs through the C ABI on cuda:0 (warm-start
    state and skip cache from the fixture); ``init``: a learned initialiser
    to attach (fast form). Returns host outputs."""
    import torch
    from opencaeporo_b200.flash import MixtureCompBatch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    m = MixtureCompBatch(fl)
    if init is not None:
        init.attach(m)
    n = len(inp["P"])
    st = m.new_state(n)
    st.load(inp["P"], inp["T"], inp["Ni"])
    o = st.out
    o["S"].copy_(torch.as_tensor(np.ascontiguousarray(inp["S"].T)))
    o["phaseNum"].copy_(torch.as_tensor(inp["lastNP"].astype(np.int32)))
    ncom = fl.nc + 1
    o["xij"].copy_(torch.as_tensor(np.ascontiguousarray(inp["xij"].reshape(n, 3 * ncom).T)))
    sk = inp["skip"]
    st.skip["flag"].copy_(torch.as_tensor(sk["flag"].astype(np.int32)))
    for k in ("minEig", "P", "T"):
        st.skip[k].copy_(torch.as_tensor(np.asarray(sk[k], dtype=np.float64)))
    st.skip["z"].copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(sk["z"]).T)))
    m.flash_fim(st, form=form)
    torch.cuda.synchronize()
    res = st.to_host()
    m.close()
    return res


FIMN_CALLS = ("fresh", "warm", "init")


def load_golden_fimn(name="fimn_nc6"):
    """(fluid, {call: (inputs, reference outputs with their self-noise under
    ``noise``, moved mask)}) of the FlashFIMn fixture, for the calls
    'fresh' (FlashFIMn of new bulks), 'warm' (FlashFIMn from a last step's
    state) and 'init' (InitFlashFIMn)."""
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    fl, _, _, _ = _fluid_only(d)
    sk_keys = ("flag", "minEig", "P", "T", "z")
    n1 = len(d["in1_P"])
    calls = {
        "fresh": ({"P": d["in1_P"], "T": d["in1_T"], "Ni": d["in1_Ni"], "S": np.zeros((n1, 3)),
                   "lastNP": np.zeros(n1, np.int32), "xij": np.zeros((n1, 3, fl.nc + 1)),
                   "skip": {k: np.zeros_like(d[f"skipin2_{k}"][:1].repeat(n1, axis=0)) for k in sk_keys}}, "1"),
        "warm": ({"P": d["in2_P"], "T": d["in2_T"], "Ni": d["in2_Ni"], "S": d["in2_S"],
                  "lastNP": d["in2_lastNP"].astype(np.int32), "xij": d["in2_xij"],
                  "skip": {k: d[f"skipin2_{k}"] for k in sk_keys}}, "2"),
        "init": ({"P": d["ini_P"], "T": d["ini_T"], "z": d["ini_z"], "S": d["ini_S"], "Vpore": d["ini_Vpore"]}, "i"),
    }
    out = {}
    for call, (inp, t) in calls.items():
        r = {k[len(t) + 4:]: d[k] for k in d.files if k.startswith(f"out{t}_")}
        r["skip"] = {k: d[f"skipout{t}_{k}"] for k in sk_keys}
        r["noise"] = {k[len(t) + 6:]: d[k].astype(np.float64) for k in d.files if k.startswith(f"noise{t}_")}
        out[call] = (inp, r, d[f"fragile{t}"])
    return fl, out


def run_gpu_fimn(fl, call, inp, form="plain"):
    """One FlashFIMn ('fresh', 'warm') or InitFlashFIMn ('init') of the
    fixture's inputs through the C ABI on cuda:0; host outputs with res,
    resPc (and Ni for 'init')."""
    import torch
    from opencaeporo_b200.flash import MixtureCompBatch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    m = MixtureCompBatch(fl)
    n = len(inp["P"])
    st = m.new_state(n)
    if call == "init":
        st.load(inp["P"], inp["T"], inp["z"])
        m.init_flash(st, inp["Vpore"], S=inp["S"], form=form, fimn=True)
    else:
        st.load(inp["P"], inp["T"], inp["Ni"])
        o = st.out
        o["S"].copy_(torch.as_tensor(np.ascontiguousarray(inp["S"].T)))
        o["phaseNum"].copy_(torch.as_tensor(inp["lastNP"].astype(np.int32)))
        ncom = fl.nc + 1
        o["xij"].copy_(torch.as_tensor(np.ascontiguousarray(inp["xij"].reshape(n, 3 * ncom).T)))
        sk = inp["skip"]
        st.skip["flag"].copy_(torch.as_tensor(sk["flag"].astype(np.int32)))
        for k in ("minEig", "P", "T"):
            st.skip[k].copy_(torch.as_tensor(np.asarray(sk[k], dtype=np.float64)))
        st.skip["z"].copy_(torch.as_tensor(np.ascontiguousarray(np.asarray(sk["z"]).T)))
        m.flash_fimn(st, form=form)
    torch.cuda.synchronize()
    res = st.to_host()
    if call == "init":
        res["Ni"] = st.Ni.cpu().numpy().T.copy()
    m.close()
    return res
