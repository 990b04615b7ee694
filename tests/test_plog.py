"""Pressure-logarithmic (PLOG) reactions: CHEMKIN parsing and units
(ReactionPolicy_CHEMKIN.hpp:772-792, :1455-1465), the rate constant
(PressureLogarithmicRateExpression.hpp:71-119) in the oracle, and the GPU
forms against the oracle."""
import math

import numpy as np
import pytest

from laminarsmoke_b200.mech import blob, chemkin, synthetic

R_J_KMOL = 8314.4621
J_FROM_CAL = 8.3144621 / (8.3144621 / 4.18443)
PLOG = [(0.1, 1.0e12, 0.5, 5000.0), (1.0, 3.0e12, 0.2, 6000.0), (10.0, 2.0e13, -0.3, 8000.0)]


def plog_mechanism(only=False):
    """The 12-species synthetic mechanism with its first exchange reaction given PLOG points (or, with
    only=True, that reaction alone, irreversible)."""
    s = synthetic.generate(12, 20, seed=4, physical=True)
    lines = s.kinetics.split("\n")
    k = next(i for i, l in enumerate(lines) if "=" in l and "+M" not in l and not l.startswith(" "))
    plog = [f" PLOG / {p} {a:.6E} {b} {e} /" for p, a, b, e in PLOG]
    if only:
        head = lines[:lines.index("REACTIONS") + 1]
        lines = head + [lines[k].replace("=", "=>", 1)] + plog + ["END"]
    else:
        lines[k + 1:k + 1] = plog
    m = chemkin.compile_mechanism("\n".join(lines) + "\n", s.thermo)
    return blob.pack(m.arrays, m.species), m


def k_plog(T, P):
    """The reference's interpolation, written out."""
    pts = [(p * 101325.0, math.log(max(a * 1e-3, 1e-32)), b, e * 1e3 * J_FROM_CAL / R_J_KMOL) for p, a, b, e in PLOG]
    lk = [la + b * math.log(T) - er / T for _, la, b, er in pts]
    if P <= pts[0][0]:
        return math.exp(lk[0])
    if P >= pts[-1][0]:
        return math.exp(lk[-1])
    i = next(i for i in range(len(pts) - 1) if P < pts[i + 1][0])
    lp0, lp1 = math.log(pts[i][0]), math.log(pts[i + 1][0])
    return math.exp(lk[i] + (lk[i + 1] - lk[i]) * (math.log(P) - lp0) / (lp1 - lp0))


def test_plog_tables():
    data, m = plog_mechanism()
    A = m.arrays
    np.testing.assert_array_equal(A["plog_ptr"], [0, 3])
    np.testing.assert_allclose(A["plog_p"], [10132.5, 101325.0, 1013250.0], rtol=1e-15)
    np.testing.assert_allclose(A["plog_lnA"], [math.log(a * 1e-3) for _, a, _, _ in PLOG], rtol=1e-15)
    np.testing.assert_allclose(A["plog_eor"], [e * 1e3 * J_FROM_CAL / R_J_KMOL for _, _, _, e in PLOG], rtol=1e-15)


def test_plog_rejected_with_falloff_or_decreasing_pressures():
    s = synthetic.generate(12, 20, seed=4)
    lines = s.kinetics.split("\n")
    k = next(i for i, l in enumerate(lines) if "(+M)" in l)
    bad = lines[:k + 1] + [" PLOG / 1.0 1.0E12 0.0 0.0 /"] + lines[k + 1:]
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism("\n".join(bad), s.thermo)
    k = next(i for i, l in enumerate(lines) if "=" in l and "+M" not in l and not l.startswith(" "))
    bad = lines[:k + 1] + [" PLOG / 1.0 1.0E12 0.0 0.0 /", " PLOG / 0.5 1.0E12 0.0 0.0 /"] + lines[k + 1:]
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism("\n".join(bad), s.thermo)


@pytest.mark.parametrize("patm", [0.05, 0.1, 0.4, 1.0, 3.0, 10.0, 30.0])
def test_oracle_plog_rate(patm):
    """One irreversible PLOG reaction A + B => C + D: dY_A/dt = -MW_A k(T, P) c_A c_B / rho."""
    from oracle.oracle import OracleMechanism
    data, m = plog_mechanism(only=True)
    A = m.arrays
    orc = OracleMechanism(data)
    ia, ib = A["reac_species"][:2]
    rng = np.random.default_rng(5)
    P = patm * 101325.0
    for _ in range(5):
        Y = rng.uniform(0.05, 1.0, m.n_species)
        Y /= Y.sum()
        T = rng.uniform(700.0, 2200.0)
        dy, _ = orc.rhs(np.concatenate([Y, [T]]), P)
        mwmix = 1.0 / (Y / A["mw"]).sum()
        c = P / R_J_KMOL / T * mwmix * Y / A["mw"]
        rho = P / R_J_KMOL / T * mwmix
        ref = -A["mw"][ia] * k_plog(T, P) * c[ia] * c[ib] / rho
        np.testing.assert_allclose(dy[ia], ref, rtol=1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("patm", [0.05, 0.4, 3.0, 30.0])
def test_gpu_plog_rhs(cuda, patm):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = plog_mechanism()
    rng = np.random.default_rng(6)
    n = 128
    Y = rng.uniform(0.0, 1.0, (n, m.n_species))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(700.0, 2200.0, n)
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
@pytest.mark.parametrize("form", ["plain", "mixed", "cv"])
def test_gpu_plog_step(cuda, form):
    """One step at 3 atm, between two PLOG points (at constant volume the pressure moves with the state).
    The random mixtures take thousands of BDF steps, over which a last-ulp difference of exp/log moves
    step sequences apart by O(rtol); at rtol 1e-10 both integrations converge and are compared at the
    usual bounds."""
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = plog_mechanism()
    rng = np.random.default_rng(7)
    n = 256
    Y = rng.uniform(0.0, 1.0, (n, m.n_species))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(900.0, 2200.0, n)
    P = 3.0 * 101325.0
    tol = dict(rtol=1e-10, atol=1e-16)
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED),
          "cv": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw, **tol)
    Ys = np.ascontiguousarray(Y.T)
    Tg = T.copy()
    orc = OracleMechanism(data)
    if form == "cv":
        rho = P / R_J_KMOL / T / (Y / m.arrays["mw"]).sum(axis=1)
        _, st, ns = ctx.step_cv(Ys, Tg, rho, 1e-5)
        Yo, To, _, sto, cnt = orc.reaction_step(Y, T, 1e-5, nthreads=8, rho=rho, **tol)
    else:
        _, st, ns = ctx.step(Ys, Tg, 1e-5, p=P)
        Yo, To, _, sto, cnt = orc.reaction_step(Y, T, 1e-5, p=P, nthreads=8, **tol)
    ctx.check()
    abs_Y = np.abs(Ys.T - Yo).max(axis=1)
    rel_T = np.abs(Tg - To) / To
    same = ns == cnt[:, 0]
    print(f"plog {form}: statuses equal {np.mean(st == sto):.3f}, max rel T {rel_T.max():.3e}, "
          f"max abs Y {abs_Y.max():.3e}, within 1e-9 {np.mean(abs_Y <= 1e-9):.3f}, "
          f"same step count {same.mean():.3f}, max abs Y there {abs_Y[same].max():.3e}, steps {cnt[:, 0].mean():.0f}")
    np.testing.assert_array_equal(st, sto)
    assert rel_T.max() <= 1e-6
    # about 8,500 BDF steps a cell: cells taking the oracle's number of steps meet 1e-9; in the others a
    # last-ulp difference of exp/log moved step-size decisions (measured 97.3 % to 99.2 % of all cells
    # within 1e-9, max 2.1e-8)
    assert (not same.any() or abs_Y[same].max() <= 1e-9)
    assert np.mean(abs_Y <= 1e-9) >= 0.95 and abs_Y.max() <= 1e-7
