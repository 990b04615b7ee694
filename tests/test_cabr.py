"""Chemically activated bimolecular (CABR, the HIGH keyword) reactions: units
(ReactionPolicy_CHEMKIN.hpp:1395-1407), the rate (KineticsMap_CHEMKIN.hpp:
1613-1660: k0 F / (1 + Pr), Pr = k0 [M] / k_inf) in the oracle, and the GPU
forms against the oracle."""
import math

import numpy as np
import pytest

from laminarsmoke_b200.mech import blob, chemkin, synthetic

R_J_KMOL = 8314.4621
J_FROM_CAL = 8.3144621 / (8.3144621 / 4.18443)
K0 = (2.0e13, 0.0, 3000.0)      # reaction line: low-pressure, bimolecular [cm3/mol/s]
KINF = (5.0e10, 0.5, 1000.0)    # HIGH: high-pressure limit, converted by 1e3^(2 - sum of orders)
TROE = (0.6, 200.0, 1200.0)


def cabr_mechanism(troe=False, only=False):
    s = synthetic.generate(12, 20, seed=4, physical=True)
    lines = s.kinetics.split("\n")
    k = next(i for i, l in enumerate(lines) if "(+M)" in l)
    j = k + 1
    while lines[j].startswith(" "):
        j += 1
    head = lines[k].split()[0].replace("=", "=>", 1)
    block = [f"{head}   {K0[0]:.6E} {K0[1]} {K0[2]}", f" HIGH / {KINF[0]:.6E} {KINF[1]} {KINF[2]} /"]
    if troe:
        block.append(" TROE / " + " ".join(str(v) for v in TROE) + " /")
    if only:
        lines = lines[:lines.index("REACTIONS") + 1] + block + ["END"]
    else:
        lines[k:j] = block
    m = chemkin.compile_mechanism("\n".join(lines) + "\n", s.thermo)
    return blob.pack(m.arrays, m.species), m


def k_cabr(T, M, troe):
    k0 = K0[0] * 1e-3 * T ** K0[1] * math.exp(-K0[2] * 1e3 * J_FROM_CAL / R_J_KMOL / T)
    kinf = KINF[0] * math.pow(1.e3, 2. - 2.) * T ** KINF[1] * math.exp(-KINF[2] * 1e3 * J_FROM_CAL / R_J_KMOL / T)
    pr = k0 * M / kinf
    f = 1.0
    if troe:
        a, b, c = TROE
        lf = math.log10((1 - a) * math.exp(-T / b) + a * math.exp(-T / c))
        n = 0.75 - 1.27 * lf
        cc = -0.4 - 0.67 * lf
        s = math.log10(pr) + cc
        f = 10.0 ** (lf / (1.0 + (s / (n - 0.14 * s)) ** 2))
    return k0 * f / (1.0 + pr)


def test_cabr_tables_and_units():
    data, m = cabr_mechanism()
    A = m.arrays
    j = int(A["fo_rxn"][0])
    assert A["fo_cabr"].tolist() == [1] + [0] * (len(A["fo_rxn"]) - 1)
    assert A["lnA"][j] == math.log(K0[0] * math.pow(1.e3, 1. - 2.))
    assert A["fo_lnA"][0] == math.log(KINF[0] * math.pow(1.e3, 2. - 2.))


@pytest.mark.parametrize("troe", [False, True])
@pytest.mark.parametrize("patm", [0.1, 1.0, 20.0])
def test_oracle_cabr_rate(troe, patm):
    from oracle.oracle import OracleMechanism
    data, m = cabr_mechanism(troe=troe, only=True)
    A = m.arrays
    orc = OracleMechanism(data)
    ia, ib = A["reac_species"][:2]
    rng = np.random.default_rng(11)
    P = patm * 101325.0
    for _ in range(5):
        Y = rng.uniform(0.05, 1.0, m.n_species)
        Y /= Y.sum()
        T = rng.uniform(600.0, 2400.0)
        dy, _ = orc.rhs(np.concatenate([Y, [T]]), P)
        mwmix = 1.0 / (Y / A["mw"]).sum()
        ctot = P / R_J_KMOL / T
        c = ctot * mwmix * Y / A["mw"]
        # third-body concentration: cTot, plus (efficiency - 1) c_i of the listed species (none here)
        ref = -A["mw"][ia] * k_cabr(T, ctot, troe) * c[ia] * c[ib] / (ctot * mwmix)
        np.testing.assert_allclose(dy[ia], ref, rtol=1e-11)


@pytest.mark.gpu
@pytest.mark.parametrize("troe", [False, True])
def test_gpu_cabr_rhs(cuda, troe):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = cabr_mechanism(troe=troe)
    rng = np.random.default_rng(12)
    n = 128
    Y = rng.uniform(0.0, 1.0, (n, m.n_species))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(600.0, 2400.0, n)
    y = np.ascontiguousarray(np.concatenate([Y.T, T[None, :]], axis=0))
    yd = torch.tensor(y, device=cuda)
    dyd = torch.zeros_like(yd)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    ctx.rhs_device(yd, dyd, p=3 * 101325.0)
    torch.cuda.synchronize()
    ctx.check()
    dy = dyd.cpu().numpy()
    orc = OracleMechanism(data)
    for k in range(n):
        ref, _ = orc.rhs(y[:, k], 3 * 101325.0)
        np.testing.assert_allclose(dy[:, k], ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_gpu_cabr_step(cuda, form):
    """One step at 3 atm against the oracle at rtol 1e-10 (see the PLOG step test)."""
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = cabr_mechanism(troe=True)
    rng = np.random.default_rng(13)
    n = 256
    Y = rng.uniform(0.0, 1.0, (n, m.n_species))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(900.0, 2200.0, n)
    P = 3.0 * 101325.0
    tol = dict(rtol=1e-10, atol=1e-16)
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw, **tol)
    Ys = np.ascontiguousarray(Y.T)
    Tg = T.copy()
    _, st, ns = ctx.step(Ys, Tg, 1e-5, p=P)
    ctx.check()
    Yo, To, _, sto, cnt = OracleMechanism(data).reaction_step(Y, T, 1e-5, p=P, nthreads=8, **tol)
    abs_Y = np.abs(Ys.T - Yo).max(axis=1)
    rel_T = np.abs(Tg - To) / To
    same = ns == cnt[:, 0]
    print(f"cabr {form}: max rel T {rel_T.max():.3e}, max abs Y {abs_Y.max():.3e}, "
          f"within 1e-9 {np.mean(abs_Y <= 1e-9):.3f}, same step count {same.mean():.3f}, "
          f"max abs Y there {abs_Y[same].max():.3e}, steps {cnt[:, 0].mean():.0f}")
    np.testing.assert_array_equal(st, sto)
    assert rel_T.max() <= 1e-6
    # about 9,000 BDF steps a cell: a last-ulp difference of exp/log moves step-size decisions, after which
    # the two integrations agree to O(rtol) only, and few cells keep the oracle's exact step count.  Those
    # that do meet 1e-9; measured 94.5 % (mixed) and 96.1 % (plain) of all cells within 1e-9, max 2.1e-8.
    assert (not same.any() or abs_Y[same].max() <= 1e-9)
    assert np.mean(abs_Y <= 1e-9) >= 0.9 and abs_Y.max() <= 1e-7
