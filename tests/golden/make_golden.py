"""Regenerate the golden vectors of the reaction-step path from the oracle.

    python tests/golden/make_golden.py

The oracle (oracle/oracle.cpp, the FP64 restatement of the reference step) is
the only source: the reference itself cannot be compiled here, so these
fixtures pin the oracle against later changes and give the GPU tests fixed
expected outputs.  Inputs are seeded (numpy PCG64, seeds below):

* h2co_rhs.npz      -- 64 H2/CO mixing states y = [Y(14), T]: dy/dt and QR;
* h2co_step.npz     -- 256 H2/CO mixing cells, one step dt = 1e-5, rtol 1e-7,
                       atol 1e-12: Y, T, Q, ODE status, counters;
* h2co_edge.npz     -- 4 cells: T at tmin_chem (skipped), a cold frozen
                       mixture, a hot equilibrium-near state, a 1 us step;
* h2co45_step.npz   -- 32 cells of the H2/CO chemistry padded with 30 inert
                       species (45 components, the block-per-cell form);
* h2co_cv_step.npz  -- 64 cells of the constant-volume reactor at their own
                       densities;
* h2co_sources.npz  -- compact-scheme sources of the h2co_step cells and the
                       steady solvers' linearised sources of 32 states;
* ch4_1step.npz     -- 64 cells of the global one-step CH4 mechanism (FORD);
* rateforms_rhs.npz -- RHS of the PLOG, Chebyshev and CABR test mechanisms
                       (tests/test_plog.py, test_cheb.py, test_cabr.py) at
                       32 states and three pressures each;
* h2co_properties.npz -- the property update (oracle/properties.py) of the
                       h2co_step result at 1 and 3 atm, with Soret terms;
* h2co_drg_step.npz -- a DRG-reduced step of 48 cells (key species H2, O2,
                       CO; epsilon 1e-3 below 1000 K, 1e-2 above);
* h2co_sparse_sources.npz -- the steady solvers' analytic-diagonal sources of
                       32 states at 1.5 bar;
* xrates_rhs.npz    -- RHS of the PLOGMX/PLOGSP and LOWMX/LOWSP test
                       mechanisms (tests/test_xplog.py, test_xfo.py) at 32
                       states and three pressures each.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from laminarsmoke_b200 import cells, mech  # noqa: E402
from laminarsmoke_b200.mech import blob  # noqa: E402
from oracle.oracle import OracleMechanism  # noqa: E402


def padded_states(k, n, seed):
    data, species = mech.load(f"h2co+{k}")
    A, _ = blob.unpack(data)
    Y, T = cells.h2co_mixing(species[:14], A["mw"][:14], n, seed=seed)
    return data, np.concatenate([Y * 0.9, np.full((n, k), 0.1 / k)], axis=1), T


def edge_states(species, mw):
    Y, T = cells.h2co_mixing(species, mw, 4, seed=41)
    T = np.array([250.0, 400.0, 2300.0, 1500.0])
    dt = np.array([1e-5, 1e-5, 1e-5, 1e-6])
    return Y, T, dt


def main():
    data, species = mech.load("h2co")
    A, _ = blob.unpack(data)
    orc = OracleMechanism(data)

    Y, T = cells.h2co_mixing(species, A["mw"], 64, seed=31)
    y = np.concatenate([Y, T[:, None]], axis=1)
    dy = np.zeros_like(y)
    qr = np.zeros(64)
    for k in range(64):
        dy[k], qr[k] = orc.rhs(y[k])
    np.savez_compressed(os.path.join(HERE, "h2co_rhs.npz"), y=y, dy=dy, qr=qr)

    Y, T = cells.h2co_mixing(species, A["mw"], 256, seed=32)
    Yo, To, Qo, sto, cnt = orc.reaction_step(Y, T, 1e-5, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "h2co_step.npz"), Y0=Y, T0=T, dt=1e-5, Y=Yo, T=To, Q=Qo,
                        status=sto, counters=cnt)

    Y, T, dt = edge_states(species, A["mw"])
    Yo, To, Qo, sto, cnt = orc.reaction_step(Y, T, dt, tmin_chem=300.0, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "h2co_edge.npz"), Y0=Y, T0=T, dt=dt, tmin_chem=300.0, Y=Yo, T=To,
                        Q=Qo, status=sto, counters=cnt)

    data45, Y, T = padded_states(30, 32, seed=33)
    Yo, To, Qo, sto, cnt = OracleMechanism(data45).reaction_step(Y, T, 1e-5, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "h2co45_step.npz"), Y0=Y, T0=T, dt=1e-5, Y=Yo, T=To, Q=Qo,
                        status=sto, counters=cnt)

    Y, T = cells.h2co_mixing(species, A["mw"], 64, seed=34)
    Y = Y / Y.sum(axis=1, keepdims=True)
    rho = np.random.default_rng(35).uniform(0.5, 2.0, 64) * 101325.0 / ((Y / A["mw"]).sum(axis=1) * 8314.4621 * T)
    Yo, To, Qo, sto, cnt = orc.reaction_step(Y, T, 1e-5, nthreads=1, rho=rho)
    np.savez_compressed(os.path.join(HERE, "h2co_cv_step.npz"), Y0=Y, T0=T, rho=rho, dt=1e-5, Y=Yo, T=To, Q=Qo,
                        status=sto, counters=cnt)

    g = np.load(os.path.join(HERE, "h2co_step.npz"))
    RR, RT = orc.compact_sources(g["Y0"], g["T0"], g["Y"], g["T"], 1e-5)
    Y, T = cells.h2co_mixing(species, A["mw"], 32, seed=36)
    ys = np.concatenate([Y, T[:, None]], axis=1)
    si = np.zeros_like(ys)
    se = np.zeros_like(ys)
    for k in range(32):
        si[k], se[k] = orc.steady_sources(ys[k], 1.5e5)
    np.savez_compressed(os.path.join(HERE, "h2co_sources.npz"), RR=RR, RT=RT, y=ys, p=1.5e5, S_implicit=si,
                        S_explicit=se)

    d1, sp1 = mech.load("ch4_1step")
    A1, _ = blob.unpack(d1)
    rng = np.random.default_rng(37)
    Y = rng.uniform(0.0, 1.0, (64, len(sp1)))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(900.0, 2200.0, 64)
    Yo, To, Qo, sto, cnt = OracleMechanism(d1).reaction_step(Y, T, 1e-5, nthreads=1)
    np.savez_compressed(os.path.join(HERE, "ch4_1step.npz"), Y0=Y, T0=T, dt=1e-5, Y=Yo, T=To, Q=Qo,
                        status=sto, counters=cnt)

    sys.path.insert(0, os.path.dirname(HERE))
    import test_cabr
    import test_cheb
    import test_plog
    out = {}
    for name, (dm, mm) in (("plog", test_plog.plog_mechanism()), ("cheb", test_cheb.cheb_mechanism()),
                           ("cabr", test_cabr.cabr_mechanism(troe=True))):
        o = OracleMechanism(dm)
        rng = np.random.default_rng(38)
        Y = rng.uniform(0.0, 1.0, (32, mm.n_species))
        Y /= Y.sum(axis=1, keepdims=True)
        T = rng.uniform(700.0, 2400.0, 32)
        ys = np.concatenate([Y, T[:, None]], axis=1)
        for patm in (0.3, 2.0, 20.0):
            out[f"{name}_y"] = ys
            out[f"{name}_dy_{patm}"] = np.array([o.rhs(ys[k], patm * 101325.0)[0] for k in range(32)])
    np.savez_compressed(os.path.join(HERE, "rateforms_rhs.npz"), **out)

    from oracle.properties import OracleProperties
    g = np.load(os.path.join(HERE, "h2co_step.npz"))
    p = np.where(np.arange(g["T"].size) % 2 == 0, 101325.0, 3.0 * 101325.0)
    f = OracleProperties(data).evaluate(g["Y"], g["T"], p, soret=True)
    np.savez_compressed(os.path.join(HERE, "h2co_properties.npz"), p=p, **f)

    Y, T = cells.h2co_mixing(species, A["mw"], 48, seed=40)
    key = [species.index(n) for n in ("H2", "O2", "CO")]
    bands = ((1000., 1e-3), (1e6, 1e-2))
    Yd, Td, Qd, std, cnt, nsp, nrx = orc.reaction_step_drg(Y, T, 1e-5, key, bands=bands, min_T=300.0)
    np.savez_compressed(os.path.join(HERE, "h2co_drg_step.npz"), Y0=Y, T0=T, dt=1e-5, key=np.array(key),
                        bands=np.array(bands), Y=Yd, T=Td, Q=Qd, status=std, counters=cnt, n_species=nsp,
                        n_reactions=nrx)

    Y, T = cells.h2co_mixing(species, A["mw"], 32, seed=41)
    ys = np.concatenate([Y, T[:, None]], axis=1)
    si = np.zeros_like(ys)
    se = np.zeros_like(ys)
    for k in range(32):
        si[k], se[k] = orc.steady_sources_sparse(ys[k], 1.5e5)
    np.savez_compressed(os.path.join(HERE, "h2co_sparse_sources.npz"), y=ys, p=1.5e5, S_implicit=si,
                        S_explicit=se)

    import test_xfo
    import test_xplog
    out = {}
    for name, dm in (("xplog", test_xplog.xplog_mechanism()[0]), ("xfo", test_xfo.xfo_mechanism()[0])):
        o = OracleMechanism(dm)
        rng = np.random.default_rng(42)
        Y = rng.uniform(0.0, 1.0, (32, o.n_species))
        Y /= Y.sum(axis=1, keepdims=True)
        T = rng.uniform(700.0, 2400.0, 32)
        ys = np.concatenate([Y, T[:, None]], axis=1)
        out[f"{name}_y"] = ys
        for patm in (0.3, 2.0, 20.0):
            out[f"{name}_dy_{patm}"] = np.array([o.rhs(ys[k], patm * 101325.0)[0] for k in range(32)])
    np.savez_compressed(os.path.join(HERE, "xrates_rhs.npz"), **out)


if __name__ == "__main__":
    main()
