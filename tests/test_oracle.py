"""The CPU oracle (test infrastructure) against physical invariants of the reference method.

The reference ships no tests or golden vectors for this path, so the oracle is
checked against invariants the reference's equations satisfy exactly."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells


def _mix(h2co, n=64, seed=11):
    _, species, A = h2co
    return cells.h2co_mixing(species, A["mw"], n, seed=seed)


def test_rhs_conserves_mass(h2co, oracle_h2co):
    Y, T = _mix(h2co, 32)
    for k in range(Y.shape[0]):
        y = np.concatenate([Y[k], [T[k]]])
        dy, qr = oracle_h2co.rhs(y)
        scale = np.abs(dy[:-1]).sum()
        assert abs(dy[:-1].sum()) <= 1e-13 * scale + 1e-300


def test_rhs_conserves_elements(h2co, oracle_h2co):
    _, species, A = h2co
    comp = {"H2": (2, 0, 0), "O2": (0, 2, 0), "H2O": (2, 1, 0), "H2O2": (2, 2, 0), "O": (0, 1, 0), "H": (1, 0, 0),
            "OH": (1, 1, 0), "HO2": (1, 2, 0), "CO": (0, 1, 1), "CO2": (0, 2, 1), "HCO": (1, 1, 1),
            "HE": (0, 0, 0), "AR": (0, 0, 0), "N2": (0, 0, 0)}
    E = np.array([comp[s] for s in species], float)
    Y, T = _mix(h2co, 16)
    for k in range(Y.shape[0]):
        dy, _ = oracle_h2co.rhs(np.concatenate([Y[k], [T[k]]]))
        moles = dy[:-1] / A["mw"]
        flux = np.abs(moles)[:, None] * E
        assert np.all(np.abs(moles @ E) <= 1e-12 * flux.sum(0) + 1e-300)


def test_energy_equation_is_enthalpy_conserving(h2co, oracle_h2co):
    """dT/dt = -sum(h_i dY_i)/cp  <=>  d(h_mix)/dt = 0 for the constant-pressure reactor."""
    _, species, A = h2co
    Y, T = _mix(h2co, 16)
    for k in range(Y.shape[0]):
        y = np.concatenate([Y[k], [T[k]]])
        dy, qr = oracle_h2co.rhs(y)
        eps = 1e-3
        yp = y + eps * dy / max(1.0, np.abs(dy[-1]) / 10.0)
        # finite-difference check of dh/dt ~ 0 is dominated by truncation; check the sign of QR instead
        assert np.isfinite(qr)
        assert np.sign(dy[-1]) == np.sign(qr) or qr == 0.0


def test_step_statuses_and_normalisation(h2co, oracle_h2co):
    Y, T = _mix(h2co, 128)
    Y2, T2, Q, st, cnt = oracle_h2co.reaction_step(Y, T, 1e-5, nthreads=4)
    assert np.all(st == 2)
    np.testing.assert_allclose(Y2.sum(1), 1.0, rtol=0, atol=4e-16)
    assert np.all(Y2 >= 0.0)
    assert np.all(cnt[:, 0] > 0)


def test_enthalpy_conserved_over_a_step(h2co, oracle_h2co):
    """Mixture enthalpy at constant p is invariant; integrator error bounded by the tolerances."""
    _, species, A = h2co
    Y, T = _mix(h2co, 64)
    Y2, T2, Q, st, cnt = oracle_h2co.reaction_step(Y, T, 1e-4, nthreads=4)

    def hmix(Yc, Tc):
        raw = A["nasa_raw"].reshape(-1, 18)
        out = 0.0
        for i in range(len(species)):
            a = raw[i, 0:7] if Tc > A["t_mid"][i] else raw[i, 7:14]
            h_rt = a[0] + a[1] / 2 * Tc + a[2] / 3 * Tc ** 2 + a[3] / 4 * Tc ** 3 + a[4] / 5 * Tc ** 4 + a[5] / Tc
            out += Yc[i] / A["mw"][i] * h_rt * 8314.4621 * Tc
        return out
    for k in range(0, 64, 4):
        h0, h1 = hmix(Y[k] / Y[k].sum(), T[k]), hmix(Y2[k], T2[k])
        assert abs(h1 - h0) <= 1e-4 * (abs(h0) + 1e5)


def test_skip_below_tmin_only_normalises(h2co, oracle_h2co):
    Y, T = _mix(h2co, 8)
    Y = Y * 1.01
    Y2, T2, Q, st, cnt = oracle_h2co.reaction_step(Y, T, 1e-5, tmin_chem=5000.0, nthreads=1)
    assert np.all(st == 0)
    np.testing.assert_allclose(Y2, Y / Y.sum(1, keepdims=True), rtol=1e-15)
    np.testing.assert_array_equal(T2, T)


def test_max_steps_returns_last_accepted_state(h2co, oracle_h2co):
    Y, T = _mix(h2co, 4)
    Y2, T2, Q, st, cnt = oracle_h2co.reaction_step(Y, T, 1e-5, max_steps=3, nthreads=1)
    assert np.all(st == -1)
    assert np.all(cnt[:, 0] == 3)
    assert np.all(np.isfinite(Y2)) and np.all(np.isfinite(T2))


def test_illegal_initial_temperature(h2co, oracle_h2co):
    Y, T = _mix(h2co, 3)
    T = np.array([150.0, 7000.0, 1500.0])
    Y2, T2, Q, st, cnt = oracle_h2co.reaction_step(Y, T, 1e-5, nthreads=1)
    assert list(st) == [-9, -9, 2]


def test_sequential_solver_state_matches_independent_without_failures(h2co, oracle_h2co):
    Y, T = _mix(h2co, 32, seed=5)
    a = oracle_h2co.reaction_step(Y, T, 1e-5, nthreads=1)
    b = oracle_h2co.reaction_step(Y, T, 1e-5, nthreads=1, sequential_state=True)
    if a[4][:, 6].sum() == 0:   # no convergence failure -> no carried state change
        np.testing.assert_array_equal(a[0], b[0])


def test_saturated_order_state_changes_results(h2co, oracle_h2co):
    """A solver object that has seen many convergence failures behaves differently (max order 4, alfa2 = 0)."""
    Y, T = _mix(h2co, 32, seed=6)
    a = oracle_h2co.reaction_step(Y, T, 1e-4, nthreads=2)
    b = oracle_h2co.reaction_step(Y, T, 1e-4, nthreads=2, alfa2_4=0.0, alfa2_5=0.0, maximum_order=4)
    assert not np.array_equal(a[4][:, 0], b[4][:, 0])


def _umix(A, species, Yc, Tc):
    """Mixture internal energy per unit mass, u = sum_i Y_i (h_i - R T) / MW_i."""
    raw = A["nasa_raw"].reshape(-1, 18)
    out = 0.0
    for i in range(len(species)):
        a = raw[i, 0:7] if Tc > A["t_mid"][i] else raw[i, 7:14]
        h_rt = a[0] + a[1] / 2 * Tc + a[2] / 3 * Tc ** 2 + a[3] / 4 * Tc ** 3 + a[4] / 5 * Tc ** 4 + a[5] / Tc
        out += Yc[i] / A["mw"][i] * (h_rt - 1.0) * 8314.4621 * Tc
    return out


def test_constant_volume_step_conserves_internal_energy(h2co, oracle_h2co):
    """Constant-volume reactor (BatchReactorHomogeneousConstantVolume.H:148-199): the mixture internal
    energy of the closed cell is invariant, the enthalpy is not, and T rises more than at constant p."""
    _, species, A = h2co
    Y, T = _mix(h2co, 64)
    Yn = Y / Y.sum(axis=1, keepdims=True)
    rho = 101325.0 * (1.0 / (Yn / A["mw"]).sum(axis=1)) / 8314.4621 / T
    Yv, Tv, Q, st, cnt = oracle_h2co.reaction_step(Y, T, 1e-4, nthreads=4, rho=rho)
    Yp, Tp, _, _, _ = oracle_h2co.reaction_step(Y, T, 1e-4, nthreads=4)
    assert np.all(st == 2)
    np.testing.assert_allclose(Yv.sum(axis=1), 1.0, rtol=1e-12)
    hot = 0
    for k in range(0, 64, 2):
        u0, u1 = _umix(A, species, Yn[k], T[k]), _umix(A, species, Yv[k], Tv[k])
        assert abs(u1 - u0) <= 1e-4 * (abs(u0) + 1e5)
        if Tp[k] - T[k] > 50.0:
            hot += 1
            assert Tv[k] - T[k] > Tp[k] - T[k]
    assert hot > 0

