"""DRG-reduced integration in the oracle (solvers/laminarSMOKE/unsteady/DRG.hpp, chemistry_DRG.H).

These tests pin the oracle's restatement (tests/test_gpu_drg.py checks the CUDA form against it): the analysis' limits
(epsilon 0 and 1, monotonicity, inert species), the reduced system with every species kept
reproducing the full step, the solver options that reach only cell 0, the epsilon carried over
between cells, and the temperature cut.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def setup(h2co):
    from laminarsmoke_b200 import cells
    from oracle.oracle import OracleMechanism
    data, species, A = h2co
    o = OracleMechanism(data)
    Y, T = cells.h2co_mixing(species, A["mw"], 48, seed=21)
    key = [species.index(s) for s in ("H2", "O2", "CO")]
    return o, species, A, Y, T, key


def _conc(A, y, T, p=101325.0):
    MW = A["mw"]
    x = (1. / np.sum(y / MW)) * y / MW
    return p / 8314.4621 / T * x


def test_analysis_limits(setup):
    o, species, A, Y, T, key = setup
    inert = {species.index(s) for s in ("HE", "AR", "N2")}
    for k in (0, 17, 40):
        c = _conc(A, Y[k], T[k])
        imp0, drop0 = o.drg_analysis(T[k], 101325., c, 0.0, key)
        assert set(imp0) == set(range(len(species))) - inert and drop0 == []
        imp1, drop1 = o.drg_analysis(T[k], 101325., c, 1.0, key)
        assert imp1 == sorted(key) and len(drop1) == o.n_reactions
        prev = set(imp0)
        for eps in (1e-4, 1e-3, 1e-2, 1e-1):
            imp, drop = o.drg_analysis(T[k], 101325., c, eps, key)
            assert set(key) <= set(imp) <= prev
            prev = set(imp)


def test_all_species_kept_reproduces_the_full_step(setup):
    o, species, A, Y, T, key = setup
    everyone = list(range(len(species)))
    Yn = Y / Y.sum(axis=1, keepdims=True)
    Yd, Td, Qd, std, _, nsp, nrx = o.reaction_step_drg(Yn, T, 1e-5, everyone, bands=((1e6, 0.0),), min_T=0.0,
                                                        first_cell_options_only=False)
    Yf, Tf, Qf, stf, _ = o.reaction_step(Yn, T, 1e-5, nthreads=1)
    assert np.all(nsp == len(species)) and np.all(nrx == o.n_reactions)
    np.testing.assert_array_equal(std, stf)
    np.testing.assert_allclose(Td, Tf, rtol=1e-12)
    np.testing.assert_allclose(Yd, Yf, rtol=1e-10, atol=1e-16)


def test_solver_options_reach_cell_zero_only(setup):
    o, species, A, Y, T, key = setup
    kw = dict(bands=((1e6, 1e-2),), min_T=300.0)
    Yr, Tr, Qr, _, cr, nsp_r, _ = o.reaction_step_drg(Y, T, 1e-5, key, first_cell_options_only=True, **kw)
    Ya, Ta, Qa, _, ca, nsp_a, _ = o.reaction_step_drg(Y, T, 1e-5, key, first_cell_options_only=False, **kw)
    np.testing.assert_array_equal(nsp_r, nsp_a)             # the analysis does not depend on the solver
    assert Tr[0] == Ta[0] and np.array_equal(Yr[0], Ya[0]) and np.array_equal(cr[0], ca[0])
    assert not np.array_equal(cr[1:], ca[1:])                # default tolerances elsewhere


def test_epsilon_carries_over_between_cells(setup):
    o, species, A, Y, T, key = setup
    hot = int(np.argmax(T))
    cold = int(np.argmin(T))
    assert T[cold] < 1000. < T[hot]
    bands = ((1000., 0.0),)       # below 1000 K epsilon 0; above it no band applies
    one = o.reaction_step_drg(Y[[hot]], T[[hot]], 1e-5, key, bands=bands, epsilon0=1.0, min_T=0.0)
    two = o.reaction_step_drg(Y[[cold, hot]], T[[cold, hot]], 1e-5, key, bands=bands, epsilon0=1.0, min_T=0.0)
    assert one[5][0] == len(key)                            # epsilon0 = 1: the key species only
    assert two[5][1] > len(key)                             # after the cold cell epsilon is 0


def test_cells_at_or_below_min_temperature_are_left_alone(setup):
    o, species, A, Y, T, key = setup
    cut = float(np.median(T))
    Yd, Td, _, st, cnt, nsp, nrx = o.reaction_step_drg(Y, T, 1e-5, key, min_T=cut)
    cold = T <= cut
    np.testing.assert_array_equal(Yd[cold], Y[cold])
    np.testing.assert_array_equal(Td[cold], T[cold])
    assert np.all(nsp[cold] == 0) and np.all(nrx[cold] == 0) and np.all(cnt[cold] == 0)
    assert np.all(nsp[~cold] >= len(key))
