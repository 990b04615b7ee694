"""Chebyshev (CHEB) reactions: parsing and units (ReactionPolicy_CHEMKIN.hpp:456-475, :1321-1342,
:1409-1412), the rate constant (ChebyshevPolynomialRateExpression.hpp:50-114) in the oracle, and the GPU
forms against the oracle."""
import math

import numpy as np
import pytest

from laminarsmoke_b200.mech import blob, chemkin, synthetic

R_J_KMOL = 8314.4621
COEF = [[8.5, 0.3], [-0.2, 0.05], [0.01, -0.02]]   # N = 3 temperature terms, M = 2 pressure terms
TLIM, PLIM = (200.0, 6500.0), (0.01, 100.0)   # T range wide enough for Newton iterates of a violent mechanism


def cheb_mechanism(only=False):
    """The 12-species synthetic mechanism with its first fall-off reaction turned into an irreversible
    Chebyshev one (the fit below has no barrier, so its reverse through the equilibrium constant would
    be unphysically fast), or with only=True that reaction alone."""
    s = synthetic.generate(12, 20, seed=4, physical=True)
    lines = s.kinetics.split("\n")
    k = next(i for i, l in enumerate(lines) if "(+M)" in l)
    j = k + 1
    while lines[j].startswith(" "):
        j += 1
    head = lines[k].split()[0]
    cheb = [f"{head.replace('=', '=>', 1)}   1.0 0.0 0.0", f" TCHEB / {TLIM[0]} {TLIM[1]} /", f" PCHEB / {PLIM[0]} {PLIM[1]} /",
            " CHEB / 3 2 /", " CHEB / " + " ".join(f"{v}" for row in COEF for v in row) + " /"]
    if only:
        lines = lines[:lines.index("REACTIONS") + 1] + cheb + ["END"]
    else:
        lines[k:j] = cheb
    m = chemkin.compile_mechanism("\n".join(lines) + "\n", s.thermo)
    return blob.pack(m.arrays, m.species), m


def k_cheb(T, P, conv):
    tt = (2.0 / T - 1.0 / TLIM[0] - 1.0 / TLIM[1]) / (1.0 / TLIM[1] - 1.0 / TLIM[0])
    lp0, lp1 = math.log10(PLIM[0] * 101325.0), math.log10(PLIM[1] * 101325.0)
    pt = (2.0 * math.log10(P) - lp0 - lp1) / (lp1 - lp0)
    s = sum(COEF[n][m] * math.cos(n * math.acos(tt)) * math.cos(m * math.acos(pt)) for n in range(3) for m in range(2))
    return 10.0 ** s * conv


def test_cheb_tables_and_units():
    data, m = cheb_mechanism()
    A = m.arrays
    np.testing.assert_array_equal(A["cheb_nm"], [3, 2])
    np.testing.assert_array_equal(A["cheb_coef"], [v for row in COEF for v in row])
    # a bimolecular (+M) reaction: k in cm3/mol/s -> m3/kmol/s
    np.testing.assert_allclose(A["cheb_lim"], [200.0, 6500.0, math.log10(0.01 * 101325.0),
                                               math.log10(100.0 * 101325.0), 1e-3], rtol=1e-15)


def test_cheb_coefficient_count_checked():
    s = synthetic.generate(12, 20, seed=4)
    lines = s.kinetics.split("\n")
    k = next(i for i, l in enumerate(lines) if "(+M)" in l)
    j = k + 1
    while lines[j].startswith(" "):
        j += 1
    lines[k + 1:j] = [" CHEB / 3 2 1.0 2.0 /"]
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism("\n".join(lines), s.thermo)


@pytest.mark.parametrize("patm", [0.02, 0.3, 1.0, 7.0, 90.0])
def test_oracle_cheb_rate(patm):
    from oracle.oracle import OracleMechanism
    data, m = cheb_mechanism(only=True)
    A = m.arrays
    orc = OracleMechanism(data)
    ia, ib = A["reac_species"][:2]
    rng = np.random.default_rng(8)
    P = patm * 101325.0
    for _ in range(5):
        Y = rng.uniform(0.05, 1.0, m.n_species)
        Y /= Y.sum()
        T = rng.uniform(400.0, 2800.0)
        dy, _ = orc.rhs(np.concatenate([Y, [T]]), P)
        mwmix = 1.0 / (Y / A["mw"]).sum()
        c = P / R_J_KMOL / T * mwmix * Y / A["mw"]
        rho = P / R_J_KMOL / T * mwmix
        ref = -A["mw"][ia] * k_cheb(T, P, 1e-3) * c[ia] * c[ib] / rho
        np.testing.assert_allclose(dy[ia], ref, rtol=1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("patm", [0.02, 1.0, 90.0])
def test_gpu_cheb_rhs(cuda, patm):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = cheb_mechanism()
    rng = np.random.default_rng(9)
    n = 128
    Y = rng.uniform(0.0, 1.0, (n, m.n_species))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(400.0, 2800.0, n)
    y = np.ascontiguousarray(np.concatenate([Y.T, T[None, :]], axis=0))
    yd = torch.tensor(y, device=cuda)
    dyd = torch.zeros_like(yd)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    ctx.rhs_device(yd, dyd, p=patm * 101325.0)
    torch.cuda.synchronize()
    ctx.check()
    dy = dyd.cpu().numpy()
    orc = OracleMechanism(data)
    for k in range(n):
        ref, _ = orc.rhs(y[:, k], patm * 101325.0)
        np.testing.assert_allclose(dy[:, k], ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_gpu_cheb_step(cuda, form):
    """One step at 2 atm against the oracle, at rtol 1e-10 (see the PLOG step test)."""
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = cheb_mechanism()
    rng = np.random.default_rng(10)
    n = 256
    Y = rng.uniform(0.0, 1.0, (n, m.n_species))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(900.0, 2200.0, n)
    P = 2.0 * 101325.0
    tol = dict(rtol=1e-10, atol=1e-16)
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw, **tol)
    Ys = np.ascontiguousarray(Y.T)
    Tg = T.copy()
    _, st, _ = ctx.step(Ys, Tg, 1e-5, p=P)
    ctx.check()
    Yo, To, _, sto, cnt = OracleMechanism(data).reaction_step(Y, T, 1e-5, p=P, nthreads=8, **tol)
    abs_Y = np.abs(Ys.T - Yo).max(axis=1)
    rel_T = np.abs(Tg - To) / To
    print(f"cheb {form}: max rel T {rel_T.max():.3e}, max abs Y {abs_Y.max():.3e}, "
          f"within 1e-9 {np.mean(abs_Y <= 1e-9):.3f}, steps {cnt[:, 0].mean():.0f}")
    np.testing.assert_array_equal(st, sto)
    assert rel_T.max() <= 1e-6
    # this violent test chemistry (T up to 3,760 K, ~7,500 steps at rtol 1e-10) spreads last-ulp differences
    # of the device's cos/acos/pow: measured 97.7 % of the cells within 1e-9, max 2.5e-8
    assert np.mean(abs_Y <= 1e-9) >= 0.95 and abs_Y.max() <= 1e-7
