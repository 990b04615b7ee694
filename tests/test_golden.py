"""Golden vectors (tests/golden/*.npz, made by tests/golden/make_golden.py).

The CPU tests pin the oracle: it must reproduce every fixture.  The GPU tests
compare the library's forms with the fixtures, with the same criteria as the
oracle parity tests.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL_T = 1e-6
ATOL_Y = 1e-9


def _load(name):
    return np.load(os.path.join(GOLDEN, name))


def _padded45():
    from laminarsmoke_b200 import mech
    return mech.load("h2co+30")[0]


# ---- the oracle against its fixtures (CPU) ----

def test_oracle_rhs_golden(oracle_h2co):
    g = _load("h2co_rhs.npz")
    for k in range(g["y"].shape[0]):
        dy, qr = oracle_h2co.rhs(g["y"][k])
        np.testing.assert_allclose(dy, g["dy"][k], rtol=1e-13, atol=1e-300)
        assert abs(qr - g["qr"][k]) <= 1e-13 * abs(g["qr"][k])


@pytest.mark.parametrize("name", ["h2co_step.npz", "h2co_edge.npz", "h2co45_step.npz"])
def test_oracle_step_golden(oracle_h2co, name):
    from oracle.oracle import OracleMechanism
    g = _load(name)
    orc = oracle_h2co if name != "h2co45_step.npz" else OracleMechanism(_padded45())
    kw = {"tmin_chem": float(g["tmin_chem"])} if "tmin_chem" in g else {}
    dt = g["dt"] if g["dt"].ndim else float(g["dt"])
    Y, T, Q, st, cnt = orc.reaction_step(g["Y0"], g["T0"], dt, nthreads=1, **kw)
    np.testing.assert_array_equal(st, g["status"])
    np.testing.assert_array_equal(cnt, g["counters"])
    np.testing.assert_allclose(T, g["T"], rtol=1e-13)
    np.testing.assert_allclose(Y, g["Y"], rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(Q, g["Q"], rtol=1e-12, atol=1e-9)


def test_oracle_cv_step_golden(oracle_h2co):
    g = _load("h2co_cv_step.npz")
    Y, T, Q, st, cnt = oracle_h2co.reaction_step(g["Y0"], g["T0"], float(g["dt"]), nthreads=1, rho=g["rho"])
    np.testing.assert_array_equal(st, g["status"])
    np.testing.assert_array_equal(cnt, g["counters"])
    np.testing.assert_allclose(T, g["T"], rtol=1e-13)
    np.testing.assert_allclose(Y, g["Y"], rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(Q, g["Q"], rtol=1e-12, atol=1e-9)


def test_oracle_sources_golden(oracle_h2co):
    s = _load("h2co_step.npz")
    g = _load("h2co_sources.npz")
    RR, RT = oracle_h2co.compact_sources(s["Y0"], s["T0"], s["Y"], s["T"], 1e-5)
    np.testing.assert_allclose(RR, g["RR"], rtol=1e-13, atol=1e-300)
    np.testing.assert_allclose(RT, g["RT"], rtol=1e-13, atol=1e-300)
    for k in range(g["y"].shape[0]):
        si, se = oracle_h2co.steady_sources(g["y"][k], float(g["p"]))
        np.testing.assert_allclose(si, g["S_implicit"][k], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(se, g["S_explicit"][k], rtol=1e-12, atol=1e-300)


def test_oracle_global_ford_golden():
    from laminarsmoke_b200 import mech
    from oracle.oracle import OracleMechanism
    g = _load("ch4_1step.npz")
    Y, T, Q, st, cnt = OracleMechanism(mech.load("ch4_1step")[0]).reaction_step(
        g["Y0"], g["T0"], float(g["dt"]), nthreads=1)
    np.testing.assert_array_equal(st, g["status"])
    np.testing.assert_array_equal(cnt, g["counters"])
    np.testing.assert_allclose(T, g["T"], rtol=1e-13)
    np.testing.assert_allclose(Y, g["Y"], rtol=1e-12, atol=1e-18)


def test_oracle_rateforms_golden():
    import test_cabr
    import test_cheb
    import test_plog
    from oracle.oracle import OracleMechanism
    g = _load("rateforms_rhs.npz")
    for name, (dm, _) in (("plog", test_plog.plog_mechanism()), ("cheb", test_cheb.cheb_mechanism()),
                          ("cabr", test_cabr.cabr_mechanism(troe=True))):
        o = OracleMechanism(dm)
        ys = g[f"{name}_y"]
        for patm in (0.3, 2.0, 20.0):
            dy = np.array([o.rhs(ys[k], patm * 101325.0)[0] for k in range(ys.shape[0])])
            np.testing.assert_allclose(dy, g[f"{name}_dy_{patm}"], rtol=1e-13, atol=1e-300, err_msg=name)


def test_oracle_properties_golden(h2co):
    from oracle.properties import OracleProperties
    s = _load("h2co_step.npz")
    g = _load("h2co_properties.npz")
    f = OracleProperties(h2co[0]).evaluate(s["Y"], s["T"], g["p"], soret=True)
    for key, v in f.items():
        np.testing.assert_allclose(v, g[key], rtol=1e-13, atol=0., err_msg=key)


def test_oracle_drg_golden(oracle_h2co):
    g = _load("h2co_drg_step.npz")
    bands = tuple(tuple(b) for b in g["bands"])
    Y, T, Q, st, cnt, nsp, nrx = oracle_h2co.reaction_step_drg(g["Y0"], g["T0"], float(g["dt"]), list(g["key"]),
                                                               bands=bands, min_T=300.0)
    for got, key in ((st, "status"), (cnt, "counters"), (nsp, "n_species"), (nrx, "n_reactions")):
        np.testing.assert_array_equal(got, g[key], err_msg=key)
    np.testing.assert_allclose(T, g["T"], rtol=1e-13)
    np.testing.assert_allclose(Y, g["Y"], rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(Q, g["Q"], rtol=1e-12, atol=1e-9)


def test_oracle_sparse_sources_golden(oracle_h2co):
    g = _load("h2co_sparse_sources.npz")
    for k in range(g["y"].shape[0]):
        si, se = oracle_h2co.steady_sources_sparse(g["y"][k], float(g["p"]))
        np.testing.assert_allclose(si, g["S_implicit"][k], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(se, g["S_explicit"][k], rtol=1e-12, atol=1e-300)


def test_oracle_extended_rates_golden():
    import test_xfo
    import test_xplog
    from oracle.oracle import OracleMechanism
    g = _load("xrates_rhs.npz")
    for name, dm in (("xplog", test_xplog.xplog_mechanism()[0]), ("xfo", test_xfo.xfo_mechanism()[0])):
        o = OracleMechanism(dm)
        ys = g[f"{name}_y"]
        for patm in (0.3, 2.0, 20.0):
            dy = np.array([o.rhs(ys[k], patm * 101325.0)[0] for k in range(ys.shape[0])])
            np.testing.assert_allclose(dy, g[f"{name}_dy_{patm}"], rtol=1e-13, atol=1e-300, err_msg=name)


# ---- the library against the fixtures (GPU) ----

def _gpu_step(data, g, **kw):
    from laminarsmoke_b200 import lsg
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw)
    Ys = np.ascontiguousarray(g["Y0"].T)
    T = g["T0"].copy()
    dt = g["dt"] if g["dt"].ndim else float(g["dt"])
    Q, st, ns = ctx.step(Ys, T, dt)
    ctx.check()
    return Ys.T, T, Q, st, ns


@pytest.mark.gpu
def test_gpu_rhs_golden(h2co, cuda):
    import torch
    from laminarsmoke_b200 import lsg
    g = _load("h2co_rhs.npz")
    y = np.ascontiguousarray(g["y"].T)
    yd = torch.tensor(y, device=cuda)
    dyd = torch.zeros_like(yd)
    qr = torch.zeros(y.shape[1], dtype=torch.float64, device=cuda)
    ctx = lsg.ReactionStep(lsg.Mechanism(h2co[0]))
    ctx.rhs_device(yd, dyd, qr=qr)
    torch.cuda.synchronize()
    dy = dyd.cpu().numpy().T
    for k in range(y.shape[1]):
        np.testing.assert_allclose(dy[k], g["dy"][k], rtol=1e-11, atol=1e-12 * np.abs(g["dy"][k]).max())
    np.testing.assert_allclose(qr.cpu().numpy(), g["qr"], rtol=1e-11, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_gpu_step_golden(h2co, cuda, form):
    from laminarsmoke_b200 import lsg
    g = _load("h2co_step.npz")
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED)}[form]
    Y, T, Q, st, ns = _gpu_step(h2co[0], g, **kw)
    np.testing.assert_array_equal(st, g["status"])
    abs_Y = np.abs(Y - g["Y"]).max(axis=1)
    assert (np.abs(T - g["T"]) / g["T"]).max() <= RTOL_T
    assert np.mean(abs_Y <= ATOL_Y) >= 0.99 and abs_Y.max() <= 1e-7


@pytest.mark.gpu
def test_gpu_edge_golden(h2co, cuda):
    from laminarsmoke_b200 import lsg
    g = _load("h2co_edge.npz")
    Y, T, Q, st, ns = _gpu_step(h2co[0], g, tmin_chem=float(g["tmin_chem"]),
                                tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64)
    np.testing.assert_array_equal(st, g["status"])
    np.testing.assert_allclose(T, g["T"], rtol=RTOL_T)
    np.testing.assert_allclose(Y, g["Y"], atol=ATOL_Y)


@pytest.mark.gpu
def test_gpu_block_golden(cuda):
    g = _load("h2co45_step.npz")
    Y, T, Q, st, ns = _gpu_step(_padded45(), g)
    np.testing.assert_array_equal(st, g["status"])
    abs_Y = np.abs(Y - g["Y"]).max(axis=1)
    assert (np.abs(T - g["T"]) / g["T"]).max() <= RTOL_T
    assert np.mean(abs_Y <= ATOL_Y) >= 0.9 and abs_Y.max() <= 1e-7


@pytest.mark.gpu
def test_gpu_properties_golden(h2co, cuda):
    import torch
    from laminarsmoke_b200 import lsg
    s = _load("h2co_step.npz")
    g = _load("h2co_properties.npz")
    ctx = lsg.ReactionStep(lsg.Mechanism(h2co[0]))
    got = ctx.properties_device(torch.tensor(np.ascontiguousarray(s["Y"].T), device=cuda),
                                torch.tensor(s["T"], device=cuda), torch.tensor(g["p"], device=cuda), soret=True)
    torch.cuda.synchronize()
    for key, v in got.items():
        r = g[key].T if g[key].ndim == 2 else g[key]
        np.testing.assert_allclose(v.cpu().numpy(), r, rtol=1e-11, atol=1e-13 * float(np.max(np.abs(r))),
                                   err_msg=key)
