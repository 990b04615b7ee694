"""The analytic Jacobian (lsg_jacobian_device, lsg_options.jacobian = LSG_JACOBIAN_ANALYTIC).

The reference builds the Newton matrix's Jacobian by forward differences only (KernelDense.hpp:111-193;
its UserDefinedJacobian is unimplemented, :96-109).  The library's species columns are exact derivatives
of the rate expressions.  They are checked column by column against central differences of the oracle's
right-hand side (truncation O(h^2)) on several mechanisms and rate forms, and the reaction step of the
round scheme that uses them is checked against the oracle."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu


def _synthetic_sri_rev():
    from laminarsmoke_b200.mech import blob, chemkin, synthetic
    s = synthetic.generate(16, 40, seed=12, physical=True, frac_sri=0.15, frac_rev=0.3)
    m = chemkin.compile_mechanism(s.kinetics, s.thermo)
    return blob.pack(m.arrays, m.species), m.species


def _mech(name):
    from laminarsmoke_b200 import mech
    if name == "sri_rev":
        return _synthetic_sri_rev()
    return mech.load(name)


def _states(data, species, n, seed):
    from laminarsmoke_b200.mech import blob
    A, _ = blob.unpack(data)
    fuel = {"H2": 0.5, "CO": 0.5} if "CO" in species and "CH4" not in species else {"CH4": 1.0}
    if "CH4" not in species and "CO" not in species:
        fuel = {"H2": 1.0}
    rng = np.random.default_rng(seed)
    yf, ya = cells.fuel_air_mass(species, A["mw"], fuel, {"O2": 0.21, "N2": 0.79})
    Z = rng.uniform(0.0, 0.5, n)
    Y = Z[:, None] * yf[None, :] + (1.0 - Z)[:, None] * ya[None, :]
    others = [i for i, s in enumerate(species) if s not in tuple(fuel) + ("O2", "N2")]
    Y[:, others] = 10.0 ** rng.uniform(-8.0, -2.0, (n, len(others)))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(900.0, 2400.0, n)
    return Y, T


def _central(orc, y, j, p):
    # The temperature row sums species enthalpy terms that cancel to a small net rate, so its rounding is
    # eps times the sum of their magnitudes, far above eps |f|.  A species step of 1e-5 |y_j| alone makes
    # that rounding ~1e-6 of the column for a radical at 1e-8 (1e-11 steps).  The right-hand side is a low-order
    # rational function of the mass fractions (products of concentrations of order <= 2, the mixture
    # molecular weight), so a step floored at 1e-9 and kept within half of y_j adds no measurable truncation
    # (checked against steps 4x and 16x larger: within 0.6 of the bound below on H2/CO).
    if j < len(y) - 1:
        h = 1e-5 * max(abs(y[j]), 1e-4)
        if y[j] > 0:
            h = min(h, 0.5 * y[j])
    else:
        h = 1e-5 * y[j]
    yp, ym = y.copy(), y.copy()
    yp[j] += h
    ym[j] -= h
    return (orc.rhs(yp, p)[0] - orc.rhs(ym, p)[0]) / (2 * h), h


@pytest.mark.parametrize("name", ["h2co", "ch4", "ch4_1step", "sri_rev"])
def test_analytic_jacobian_against_central_differences(cuda, name):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, species = _mech(name)
    n = len(species) + 1
    Y, T = _states(data, species, 24, 3)
    y = np.ascontiguousarray(np.concatenate([Y.T, T[None, :]], axis=0))
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    J = torch.zeros((24, n, n), dtype=torch.float64, device=cuda)
    ctx.jacobian_device(torch.tensor(y, device=cuda), J)
    torch.cuda.synchronize()
    ctx.check()
    Jg = J.cpu().numpy()
    orc = OracleMechanism(data)
    worst = 0.0
    for k in range(24):
        yk = y[:, k].copy()
        f0 = orc.rhs(yk)[0]
        for j in range(n):
            ref, h = _central(orc, yk, j, 101325.0)
            # a central difference carries the rounding of f amplified by 1/h, and its own truncation; the
            # bound allows 1e-6 of the column plus 256 eps |f| / h per entry.  The device's temperature
            # column is itself a forward difference with hT = sqrt(eps) T: its rounding, 64 eps |f| / hT, is
            # added there (f is a sum with cancellation: measured up to 14 eps |f| / hT)
            eps = 2.220446049250313e-16
            tol = 1e-6 * np.abs(ref).max() + 256 * eps * np.abs(f0) / h
            if j == n - 1:
                tol = tol + 64 * eps * np.abs(f0) / (np.sqrt(eps) * max(abs(yk[j]), 1.0))
            err = np.abs(Jg[k, :, j] - ref)
            worst = max(worst, float((err / np.maximum(tol, 1e-300)).max()))
            assert np.all(err <= tol), (name, k, j, float((err / np.maximum(tol, 1e-300)).max()))
    print(f"{name}: worst column error / bound against central differences {worst:.3f}")


@pytest.mark.parametrize("rtol,atol,frac", [(1e-7, 1e-12, 0.97), (1e-10, 1e-16, 0.99)])
def test_round_scheme_with_analytic_jacobian(cuda, h2co, rtol, atol, frac):
    """The round scheme with the analytic Jacobian against the oracle (which differentiates numerically,
    as the reference does): identical statuses, T within 1e-6, Y within 1e-9 in most cells and 1e-7 in
    all; one RHS call per Jacobian (its temperature column) instead of n."""
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, species, A = h2co
    n = 2048
    Y, T = cells.h2co_mixing(species, A["mw"], n, seed=4)
    ctx = lsg.ReactionStep(lsg.Mechanism(data), tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED,
                           jacobian=lsg.LSG_JACOBIAN_ANALYTIC, rtol=rtol, atol=atol)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    st = torch.zeros(n, dtype=torch.int32, device=cuda)
    cnt = torch.zeros((n, lsg.NCOUNTERS), dtype=torch.int64, device=cuda)
    ctx.step_device(Yd, Td, 1e-5, status=st, counters=cnt)
    torch.cuda.synchronize()
    ctx.check()
    Yo, To, _, sto, co = OracleMechanism(data).reaction_step(Y, T, 1e-5, rtol=rtol, atol=atol, nthreads=8)
    c = cnt.cpu().numpy()
    np.testing.assert_array_equal(st.cpu().numpy(), sto)
    assert (c[:, 7] == c[:, 2]).all()          # one RHS call per Jacobian
    dT = np.abs(Td.cpu().numpy() - To) / To
    dY = np.abs(Yd.cpu().numpy().T - Yo).max(axis=1)
    print(f"analytic J rtol {rtol:g}: max rel T {dT.max():.2e}, max abs Y {dY.max():.2e}, within 1e-9 "
          f"{np.mean(dY <= 1e-9):.4f}; steps/cell {c[:, 0].mean():.1f} (oracle {co[:, 0].mean():.1f}), "
          f"RHS/cell {c[:, 1].mean() + c[:, 7].mean():.1f} (oracle {co[:, 1].mean() + co[:, 7].mean():.1f})")
    assert dT.max() <= 1e-6
    assert np.mean(dY <= 1e-9) >= frac and dY.max() <= 1e-7
