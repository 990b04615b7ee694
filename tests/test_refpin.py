"""The oracle's integrator pinned to the reference's own code.

oracle/refpin compiles the reference's dense BDF integrator class templates --
MultiValueSolver< MethodGear< KernelDense<...> > > from
solvers/openSMOKEpp4laminarSMOKE/math/native-ode-solvers/{MultiValueSolver,MethodGear,
KernelDense,OdeSolverUtilities}.{h,hpp} -- unchanged, from the reference checkout,
against small stand-ins for Eigen and two OpenSMOKE helpers, and drives it with the
oracle's right-hand side and the per-cell calls of chemistry_DI.H:92-169.  On the same
cells the oracle's restated integrator (oracle.cpp, class Gear) must give the same
results bit for bit: Y, T, Q, statuses and all eight per-cell counters.  This pins
the integrator (finite-difference Jacobian, G = I - h r0 J and its LU, Newton
correction, step/order control, Gear constants) and the driver's pre- and
post-processing to the reference's code; the oracle's RHS (thermodynamics and
kinetics maps) remains a restatement.

The library exists only where the reference sources were present at build time
(oracle/_ref, built by __graft_entry__.build()); without it these tests skip.
"""
import os

import numpy as np
import pytest

from laminarsmoke_b200 import cells

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

pytestmark = pytest.mark.skipif(
    not __import__("oracle.oracle", fromlist=["refpin_available"]).refpin_available(),
    reason="oracle/_ref/liblsmoke_refpin.so not built (reference sources absent at build time)")


def _both(data, Y, T, dt, **kw):
    from oracle.oracle import OracleMechanism, ReferenceIntegrator
    o = OracleMechanism(data).reaction_step(Y, T, dt, nthreads=8, **kw)
    r = ReferenceIntegrator(data).reaction_step(Y, T, dt, nthreads=8, **kw)
    return o, r


def _assert_identical(o, r, label):
    Yo, To, Qo, sto, co = o
    Yr, Tr, Qr, str_, cr = r
    np.testing.assert_array_equal(sto, str_, err_msg=label)
    ok = sto >= 0   # a failed cell: the reference hands back its stale solution, the oracle its last state
    np.testing.assert_array_equal(co[ok], cr[ok], err_msg=label)
    np.testing.assert_array_equal(Yo[ok], Yr[ok], err_msg=label)
    np.testing.assert_array_equal(To[ok], Tr[ok], err_msg=label)
    np.testing.assert_array_equal(Qo[ok], Qr[ok], err_msg=label)


def test_refpin_h2co_mixing(h2co):
    data, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 1024, seed=3)
    _assert_identical(*_both(data, Y, T, 1e-5), "h2co mixing")


def test_refpin_h2co_uneven_subset(h2co):
    """Cold frozen, igniting and near-equilibrium cells of the benchmark workload."""
    data, species, A = h2co
    Y, T = cells.h2co_uneven(species, A["mw"], 1 << 20,
                             cells.pool_from_file(os.path.join(GOLDEN, "h2co_hot_pool.npz")), seed=2)
    pick = np.sort(np.random.default_rng(5).choice(Y.shape[0], 2048, replace=False))
    _assert_identical(*_both(data, Y[pick], T[pick], 1e-5), "h2co uneven")


@pytest.mark.parametrize("name", ["h2co_step.npz", "h2co_edge.npz"])
def test_refpin_reproduces_golden_fixtures(h2co, name):
    """The reference's integrator reproduces the committed golden vectors exactly."""
    from oracle.oracle import ReferenceIntegrator
    g = np.load(os.path.join(GOLDEN, name))
    kw = {"tmin_chem": float(g["tmin_chem"])} if "tmin_chem" in g else {}
    dt = g["dt"] if g["dt"].ndim else float(g["dt"])
    Y, T, Q, st, cnt = ReferenceIntegrator(h2co[0]).reaction_step(g["Y0"], g["T0"], dt, nthreads=1, **kw)
    np.testing.assert_array_equal(st, g["status"])
    np.testing.assert_array_equal(cnt, g["counters"])
    np.testing.assert_array_equal(T, g["T"])
    np.testing.assert_array_equal(Y, g["Y"])
    np.testing.assert_array_equal(Q, g["Q"])


def test_refpin_tight_tolerances(h2co):
    data, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 256, seed=7)
    _assert_identical(*_both(data, Y, T, 1e-5, rtol=1e-10, atol=1e-16), "h2co rtol 1e-10")


def test_refpin_edge_options(h2co):
    """Skipped cells, energy off, a step limit that ends cells with status -1, per-cell dt."""
    data, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 256, seed=8)
    dt = np.random.default_rng(2).uniform(1e-6, 3e-5, 256)
    _assert_identical(*_both(data, Y, T, dt, tmin_chem=1500.0), "tmin_chem")
    _assert_identical(*_both(data, Y, T, 1e-5, energy=False), "energy off")
    _assert_identical(*_both(data, Y, T, 1e-5, max_steps=20), "max_steps")


@pytest.mark.parametrize("name", ["ch4", "h2"])
def test_refpin_other_mechanisms(name):
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load(name)
    A, _ = blob.unpack(data)
    fuel = {"ch4": {"CH4": 1.0}, "h2": {"H2": 1.0}}[name]
    yf, ya = cells.fuel_air_mass(species, A["mw"], fuel, {"O2": 0.21, "N2": 0.79})
    rng = np.random.default_rng(4)
    Z = rng.uniform(0.0, 0.3, 256)
    Y = Z[:, None] * yf[None, :] + (1.0 - Z)[:, None] * ya[None, :]
    others = [i for i, s in enumerate(species) if s not in tuple(fuel) + ("O2", "N2")]
    Y[:, others] = 10.0 ** rng.uniform(-10.0, -4.0, (256, len(others)))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(1000.0, 2200.0, 256)
    _assert_identical(*_both(data, Y, T, 1e-5), name)


def test_refpin_sri_rev_mechanism():
    from laminarsmoke_b200.mech import blob, chemkin, synthetic
    s = synthetic.generate(16, 40, seed=12, physical=True, frac_sri=0.15, frac_rev=0.3)
    m = chemkin.compile_mechanism(s.kinetics, s.thermo)
    data = blob.pack(m.arrays, m.species)
    Y, T = cells.synthetic_mixing(m.species, m.arrays["mw"], 128, seed=3, t_range=(900.0, 2200.0))
    _assert_identical(*_both(data, Y, T, 1e-5), "SRI/REV")
