"""Output fields beyond Y, T and Q (chemistry_DI.H): the compact Strang
scheme's source terms RR/RT (:236-281), the formation-rate fields (:293-326),
and the steady solvers' linearised sources (steady/linearModel.H:92-170).
CPU: the oracle against an independent numpy restatement and conservation
laws.  GPU: the library against the oracle on the same inputs.
"""
import math

import numpy as np
import pytest

from laminarsmoke_b200 import cells

R_J_KMOL = 8314.4621


def _numpy_sources(A, Y0, T0, Yf, Tf, dt, p=101325.0):
    mw = A["mw"]
    nc = mw.size
    mwmix = 1.0 / (Yf / mw).sum(axis=1)
    x = mwmix[:, None] * Yf / mw
    T = Tf[:, None]
    hi = T > A["t_mid"][None, :]
    ch = A["cp_ht"].reshape(nc, 5)
    cl = A["cp_lt"].reshape(nc, 5)
    poly = lambda c: c[None, :, 0] + T * c[None, :, 1] + T ** 2 * c[None, :, 2] + T ** 3 * c[None, :, 3] + T ** 4 * c[None, :, 4]
    cp = np.where(hi, poly(ch), poly(cl))
    cpmix = (cp * x).sum(axis=1) * R_J_KMOL / mwmix
    rho = p * mwmix / R_J_KMOL / Tf
    RR = rho[:, None] * (Yf - Y0) / dt
    RT = rho * cpmix * (Tf - T0) / dt
    return RR, RT


def _states(h2co, n, seed):
    _, species, A = h2co
    return cells.h2co_mixing(species, A["mw"], n, seed=seed)


def test_oracle_compact_sources(h2co, oracle_h2co):
    _, species, A = h2co
    Y0, T0 = _states(h2co, 256, 51)
    Yf, Tf, _, st, _ = oracle_h2co.reaction_step(Y0, T0, 1e-5, nthreads=8)
    RR, RT = oracle_h2co.compact_sources(Y0, T0, Yf, Tf, 1e-5)
    RRn, RTn = _numpy_sources(A, Y0, T0, Yf, Tf, 1e-5)
    np.testing.assert_allclose(RR, RRn, rtol=1e-9, atol=1e-12 * np.abs(RRn).max())
    np.testing.assert_allclose(RT, RTn, rtol=1e-9, atol=1e-12 * np.abs(RTn).max())
    # mass: sum_i RR_i = rho (sum Yf - sum Y0) / dt = 0 for normalised fields
    assert np.abs(RR.sum(axis=1)).max() <= 1e-10 * np.abs(RR).max()
    # a zero step gives zero sources; with the energy equation off RT is left alone
    RR0, RT0 = oracle_h2co.compact_sources(Y0, T0, Yf, Tf, np.where(np.arange(256) % 2 == 0, 0.0, 1e-5))
    assert np.all(RR0[::2] == 0) and np.all(RT0[::2] == 0)
    np.testing.assert_array_equal(RR0[1::2], RR[1::2])
    _, RTe = oracle_h2co.compact_sources(Y0, T0, Yf, Tf, 1e-5, energy=False)
    assert np.all(RTe == 0)


def test_oracle_formation_rates(h2co, oracle_h2co):
    _, species, A = h2co
    Y, T = _states(h2co, 64, 52)
    for k in range(64):
        y = np.concatenate([Y[k], [T[k]]])
        out = oracle_h2co.formation_rates(y)
        dy, _ = oracle_h2co.rhs(y)
        rho = 101325.0 / R_J_KMOL / T[k] / (Y[k] / A["mw"]).sum()
        np.testing.assert_allclose(out, rho * dy[:-1], rtol=1e-12, atol=1e-14 * np.abs(out).max())
        assert abs(out.sum()) <= 1e-12 * np.abs(out).sum()


@pytest.mark.gpu
def test_gpu_compact_sources(h2co, oracle_h2co, cuda):
    import torch
    from laminarsmoke_b200 import lsg
    Y0, T0 = _states(h2co, 4096, 53)
    ctx = lsg.ReactionStep(lsg.Mechanism(h2co[0]))
    Y0d = torch.tensor(np.ascontiguousarray(Y0.T), device=cuda)
    T0d = torch.tensor(T0, device=cuda)
    Yfd, Tfd = Y0d.clone(), T0d.clone()
    ctx.step_device(Yfd, Tfd, 1e-5)
    dt = np.where(np.arange(4096) % 7 == 0, 0.0, 1e-5)
    dtd = torch.tensor(dt, device=cuda)
    RRd = torch.empty_like(Y0d)
    RTd = torch.empty_like(T0d)
    ctx.compact_sources_device(Y0d, T0d, Yfd, Tfd, dtd, RRd, RTd)
    torch.cuda.synchronize()
    ctx.check()
    Yf, Tf = Yfd.cpu().numpy().T, Tfd.cpu().numpy()
    RR, RT = oracle_h2co.compact_sources(Y0, T0, Yf, Tf, dt)
    np.testing.assert_allclose(RRd.cpu().numpy().T, RR, rtol=1e-13, atol=0)
    np.testing.assert_allclose(RTd.cpu().numpy(), RT, rtol=1e-13, atol=0)
    assert np.all(RRd.cpu().numpy()[:, ::7] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("mech_name", ["h2co", "h2co+30"])
def test_gpu_formation_rates(h2co, cuda, mech_name):
    import torch
    from laminarsmoke_b200 import lsg, mech
    from laminarsmoke_b200.mech import blob
    from oracle.oracle import OracleMechanism
    data, species = mech.load(mech_name)
    A, _ = blob.unpack(data)
    Y, T = cells.h2co_mixing(species[:14], A["mw"][:14], 512, seed=54)
    k = len(species) - 14
    if k:
        Y = np.concatenate([Y * 0.9, np.full((512, k), 0.1 / k)], axis=1)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    out = torch.zeros(len(species), 640, dtype=torch.float64, device=cuda)
    ctx.formation_rates_device(Yd, Td, out)
    torch.cuda.synchronize()
    ctx.check()
    g = out.cpu().numpy()[:, :512].T
    orc = OracleMechanism(data)
    rtol = 1e-11 if k == 0 else 1e-9
    for c in range(512):
        ref = orc.formation_rates(np.concatenate([Y[c], [T[c]]]))
        np.testing.assert_allclose(g[c], ref, rtol=rtol, atol=1e-12 * np.abs(ref).max())


def _steady_ref(orc, y, p=101325.0):
    """linearModel::reactionSourceTerms + ::reactionJacobian (steady/linearModel.H:92-170) written out with
    the oracle's formation rates and heat release."""
    nc = y.size - 1

    def sources(yy):
        yc = yy.copy()
        yc[:nc] = np.maximum(yc[:nc], 0.0)
        s = np.empty(nc + 1)
        s[:nc] = orc.formation_rates(yc, p)
        s[nc] = orc.rhs(yc, p)[1]
        return s
    s0 = sources(y)
    zero_der = math.sqrt(float(np.float32(1.175494351e-38)))
    eta2 = math.sqrt(2.220446049250313e-16)
    si = np.empty(nc + 1)
    se = np.empty(nc + 1)
    for k in range(nc + 1):
        ew = 1.0 / (1e-12 + 1e-7 * abs(y[k]))
        hj = eta2 * abs(max(y[k], 1.0 / ew))
        hj = max(hj, 1.0 / ew)
        hj = max(hj, zero_der)
        d = min(hj, 1.e-3 + 1e-3 * abs(y[k]))
        yp = y.copy()
        yp[k] += d
        j = (sources(yp)[k] - s0[k]) * (1.0 / d)
        si[k] = j
        se[k] = s0[k] - j * y[k]
    return si, se


def test_oracle_steady_sources(h2co, oracle_h2co):
    Y, T = _states(h2co, 16, 55)
    Y[0, 3] = -1e-12   # a slightly negative mass fraction: clipped in the source, perturbed unclipped
    for c in range(16):
        y = np.concatenate([Y[c], [T[c]]])
        si, se = oracle_h2co.steady_sources(y)
        ri, re = _steady_ref(oracle_h2co, y)
        np.testing.assert_allclose(si, ri, rtol=1e-13, atol=1e-300)
        np.testing.assert_allclose(se, re, rtol=1e-13, atol=1e-12 * np.abs(re).max())


@pytest.mark.gpu
def test_gpu_steady_sources(h2co, oracle_h2co, cuda):
    """Device against oracle.  A one-sided difference carries the rounding of S_k amplified by 1/dy_k, so
    each J_k is compared within 1e-6 |J_k| plus 64 eps |S_k| / dy_k."""
    import torch
    from laminarsmoke_b200 import lsg
    Y, T = _states(h2co, 512, 56)
    p = np.random.default_rng(57).uniform(0.8e5, 1.2e5, 512)
    ctx = lsg.ReactionStep(lsg.Mechanism(h2co[0]))
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    n = Y.shape[1] + 1
    Si = torch.zeros(n, 600, dtype=torch.float64, device=cuda)
    Se = torch.zeros(n, 600, dtype=torch.float64, device=cuda)
    ctx.steady_sources_device(Yd, Td, Si, Se, p=torch.tensor(p, device=cuda))
    torch.cuda.synchronize()
    ctx.check()
    si, se = Si.cpu().numpy()[:, :512].T, Se.cpu().numpy()[:, :512].T
    worst = 0.0
    for c in range(512):
        y = np.concatenate([Y[c], [T[c]]])
        ri, re = oracle_h2co.steady_sources(y, p[c])
        s0 = re + ri * y
        ew = 1.0 / (1e-12 + 1e-7 * np.abs(y))
        hj = np.maximum(np.maximum(math.sqrt(2.220446049250313e-16) * np.abs(np.maximum(y, 1.0 / ew)), 1.0 / ew),
                        math.sqrt(float(np.float32(1.175494351e-38))))
        d = np.minimum(hj, 1e-3 + 1e-3 * np.abs(y))
        tol = 1e-6 * np.abs(ri) + 64 * 2.220446049250313e-16 * np.abs(s0) / d
        err = np.abs(si[c] - ri)
        worst = max(worst, float((err / np.maximum(tol, 1e-300)).max()))
        assert np.all(err <= tol), (c, err / tol)
        np.testing.assert_allclose(se[c] + si[c] * y, s0, rtol=1e-10, atol=1e-12 * np.abs(s0).max())
    print(f"worst J error / tolerance {worst:.3f}")
