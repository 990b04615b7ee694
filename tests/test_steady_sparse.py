"""The steady solvers' default linearisation (sparseJacobian true; steady/linearModel.H:172-232 with
maps/JacobianSparsityPatternMap.hpp:427-560): the oracle, and the CUDA form (lsg_steady_sources_sparse_device)
against it.

Checks: the analytic species diagonal against the formula written out for a one-reaction mechanism; the T
entry equal to the dense path's; the speciesEquations / energyEquation switches; and, as a sanity bound,
agreement with the dense forward-difference diagonal for the fast species, whose own concentration term
dominates (the analytic form leaves out the density's dependence on omega).
"""
import math

import numpy as np
import pytest


def test_species_diagonal_one_reaction():
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    from oracle.oracle import OracleMechanism
    data, sp = mech.load("ch4_1step")
    A, _ = blob.unpack(data)
    o = OracleMechanism(data)
    rng = np.random.default_rng(2)
    P = 2e5
    MW = A["mw"]
    nu = np.zeros(len(sp))
    for s, v in zip(A["reac_species"], A["reac_nu"]):
        nu[s] -= v
    for s, v in zip(A["prod_species"], A["prod_nu"]):
        nu[s] += v
    for _ in range(20):
        Y = rng.uniform(0, 1, len(sp))
        Y[rng.integers(len(sp))] = 0.0                      # floored at 1e-13
        Y /= Y.sum()
        T = rng.uniform(800, 2400)
        si, se = o.steady_sources_sparse(np.concatenate([Y, [T]]), P)
        om = np.maximum(Y, 1e-13)
        rho = P / 8314.4621 / T / np.sum(om / MW)
        c = om * rho / MW
        k = math.exp(A["lnA"][0] + A["beta"][0] * math.log(T) - A["e_over_r"][0] / T)
        rf = k * np.prod([c[s] ** v for s, v in zip(A["ford_species"], A["ford_val"])])
        J = np.zeros(len(sp))
        for s, v in zip(A["ford_species"], A["ford_val"]):
            J[s] += nu[s] * v * rf / om[s]
        np.testing.assert_allclose(si[:-1], J * MW, rtol=1e-13, atol=0.)


@pytest.fixture(scope="module")
def states(h2co):
    from laminarsmoke_b200 import cells
    from oracle.oracle import OracleMechanism
    data, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 48, seed=7)
    return OracleMechanism(data), Y, T


def test_temperature_entry_and_switches(states):
    o, Y, T = states
    for k in range(0, 48, 6):
        y = np.concatenate([Y[k], [T[k]]])
        d_imp, d_exp = o.steady_sources(y, 1.5e5)
        s_imp, s_exp = o.steady_sources_sparse(y, 1.5e5)
        assert s_imp[-1] == d_imp[-1] and s_exp[-1] == d_exp[-1]
        n_imp, n_exp = o.steady_sources_sparse(y, 1.5e5, species=False)
        assert np.all(n_imp[:-1] == 0.) and n_imp[-1] == s_imp[-1]
        S = d_exp + d_imp * y                                   # the source terms themselves
        np.testing.assert_allclose(n_exp[:-1], S[:-1], rtol=1e-12, atol=1e-12 * np.abs(S[:-1]).max())
        e_imp, _ = o.steady_sources_sparse(y, 1.5e5, energy=False)
        assert e_imp[-1] == 0. and np.array_equal(e_imp[:-1], s_imp[:-1])


def test_fast_species_agree_with_the_dense_diagonal(states):
    o, Y, T = states
    rel = []
    for k in range(48):
        y = np.concatenate([Y[k], [T[k]]])
        d, _ = o.steady_sources(y, 1.5e5)
        s, _ = o.steady_sources_sparse(y, 1.5e5)
        fast = np.abs(d[:-1]) > 1e5
        rel += list(np.abs(s[:-1][fast] / d[:-1][fast] - 1.))
    rel = np.array(rel)
    assert rel.size > 100
    assert np.median(rel) < 1e-3 and rel.max() < 0.1


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2co", "ch4", "ch4_1step"])
@pytest.mark.parametrize("species,energy", [(1, 1), (1, 0), (0, 1)])
def test_gpu_steady_sources_sparse(cuda, name, species, energy):
    """Device against oracle on states with some zero and negative mass fractions (floored at 1e-13), per-cell
    pressure: the species diagonal is analytic (1e-9 relative, the fall-off part a 1e-4 difference of the
    correction in both); the temperature entry a one-sided difference (1e-6 relative plus the rounding of S
    amplified by 1/dT); S_explicit + S_implicit y reproduces S."""
    import torch
    from laminarsmoke_b200 import lsg, mech
    from laminarsmoke_b200.mech import blob
    from oracle.oracle import OracleMechanism
    data, sp = mech.load(name)
    A, _ = blob.unpack(data)
    rng = np.random.default_rng(61)
    n = 256
    Y = 10.0 ** rng.uniform(-12, 0, (n, len(sp)))
    Y[rng.random((n, len(sp))) < 0.05] = 0.0
    Y[rng.random((n, len(sp))) < 0.02] = -1e-12
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(800.0, 2400.0, n)
    p = rng.uniform(0.8e5, 3e5, n)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    Si = torch.zeros(len(sp) + 1, n, dtype=torch.float64, device=cuda)
    Se = torch.zeros_like(Si)
    ctx.steady_sources_sparse_device(torch.tensor(np.ascontiguousarray(Y.T), device=cuda),
                                     torch.tensor(T, device=cuda), Si, Se, p=torch.tensor(p, device=cuda),
                                     species=species, energy=energy)
    torch.cuda.synchronize()
    ctx.check()
    si, se = Si.cpu().numpy().T, Se.cpu().numpy().T
    o = OracleMechanism(data)
    for c in range(n):
        y = np.concatenate([Y[c], [T[c]]])
        ri, re = o.steady_sources_sparse(y, p[c], species=bool(species), energy=bool(energy))
        s0 = re + ri * y
        np.testing.assert_allclose(si[c, :-1], ri[:-1], rtol=1e-9, atol=1e-12 * np.abs(ri[:-1]).max() + 1e-300)
        dT = min(max(math.sqrt(2.220446049250313e-16) * y[-1], 1e-12 + 1e-7 * y[-1]), 1e-3 + 1e-3 * y[-1])
        tolT = 1e-6 * abs(ri[-1]) + 64 * 2.220446049250313e-16 * abs(s0[-1]) / dT
        assert abs(si[c, -1] - ri[-1]) <= tolT, (c, si[c, -1], ri[-1])
        np.testing.assert_allclose(se[c] + si[c] * y, s0, rtol=1e-10, atol=1e-12 * np.abs(s0).max())
