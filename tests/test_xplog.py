"""Extended PLOG reactions (PLOGMX / PLOGSP): CHEMKIN parsing and units (ReactionPolicy_CHEMKIN.hpp:793-880,
:1467-1471), the bath-weighted rate constant (ExtendedPressureLogarithmicRateExpression.hpp:162-202) in the
oracle; the device library accepts such mechanisms (its kernels evaluate them, tests/test_gpu_extended.py)."""
import ctypes as C
import math

import numpy as np
import pytest

from laminarsmoke_b200.mech import blob, chemkin, synthetic

R_J_KMOL = 8314.4621
J_FROM_CAL = 8.3144621 / (8.3144621 / 4.18443)
MIX = [(0.1, 1.0e12, 0.5, 5000.0), (1.0, 3.0e12, 0.2, 6000.0), (10.0, 2.0e13, -0.3, 8000.0)]
BATH = [(0.5, 4.0e12, 0.1, 4000.0), (5.0, 9.0e12, 0.0, 4500.0)]


def xplog_mechanism(bath_first=False):
    """The 12-species synthetic mechanism reduced to its first exchange reaction, irreversible, with a
    mixture table and a table for the bath species that is not a reactant of it."""
    s = synthetic.generate(12, 20, seed=4, physical=True)
    lines = s.kinetics.split("\n")
    k = next(i for i, l in enumerate(lines) if "=" in l and "+M" not in l and not l.startswith(" "))
    head = lines[:lines.index("REACTIONS") + 1]
    m0 = chemkin.compile_mechanism(s.kinetics, s.thermo)
    reac = set(int(v) for v in m0.arrays["reac_species"][m0.arrays["reac_ptr"][0]:m0.arrays["reac_ptr"][1]])
    bath = next(n for i, n in enumerate(m0.species) if i not in reac)
    mix = [f" PLOGMX / {p} {a:.6E} {b} {e} /" for p, a, b, e in MIX]
    sp = [f" PLOGSP / {bath} {p} {a:.6E} {b} {e} /" for p, a, b, e in BATH]
    body = (sp + mix) if bath_first else (mix + sp)
    lines = head + [lines[k].replace("=", "=>", 1)] + body + ["END"]
    m = chemkin.compile_mechanism("\n".join(lines) + "\n", s.thermo)
    return blob.pack(m.arrays, m.species), m, m.species.index(bath)


def _k(points, T, P):
    pts = [(p * 101325.0, math.log(max(a * 1e-3, 1e-32)), b, e * 1e3 * J_FROM_CAL / R_J_KMOL) for p, a, b, e in points]
    lk = [la + b * math.log(T) - er / T for _, la, b, er in pts]
    if P <= pts[0][0]:
        return math.exp(lk[0])
    if P >= pts[-1][0]:
        return math.exp(lk[-1])
    i = next(i for i in range(len(pts) - 1) if P < pts[i + 1][0])
    lp0, lp1 = math.log(pts[i][0]), math.log(pts[i + 1][0])
    return math.exp(lk[i] + (lk[i + 1] - lk[i]) * (math.log(P) - lp0) / (lp1 - lp0))


def test_xplog_tables():
    _, m, ib = xplog_mechanism()
    A = m.arrays
    np.testing.assert_array_equal(A["xplog_rxn"], [0])
    np.testing.assert_array_equal(A["xplog_bath_ptr"], [0, 2])
    np.testing.assert_array_equal(A["xplog_bath_sp"], [-1, ib])
    np.testing.assert_array_equal(A["xplog_ptr"], [0, 3, 5])
    np.testing.assert_allclose(A["xplog_p"], [p * 101325.0 for p, *_ in MIX + BATH], rtol=1e-15)
    np.testing.assert_allclose(A["xplog_lnA"], [math.log(a * 1e-3) for _, a, _, _ in MIX + BATH], rtol=1e-15)
    np.testing.assert_allclose(A["xplog_eor"], [e * 1e3 * J_FROM_CAL / R_J_KMOL for *_, e in MIX + BATH],
                               rtol=1e-15)
    _, m2, _ = xplog_mechanism(bath_first=True)   # baths in order of first appearance
    np.testing.assert_array_equal(m2.arrays["xplog_bath_sp"], [ib, -1])


@pytest.mark.parametrize("bad", ["no_mixture", "decreasing", "negative_A", "with_plog", "unknown_bath"])
def test_xplog_rejections(bad):
    s = synthetic.generate(12, 20, seed=4)
    lines = s.kinetics.split("\n")
    k = next(i for i, l in enumerate(lines) if "=" in l and "+M" not in l and not l.startswith(" "))
    sp0 = s.kinetics.split("SPECIES")[1].split()[0]
    extra = {
        "no_mixture": [f" PLOGSP / {sp0} 1.0 1.0E12 0.0 0.0 /"],
        "decreasing": [" PLOGMX / 1.0 1.0E12 0.0 0.0 /", " PLOGMX / 0.5 1.0E12 0.0 0.0 /"],
        "negative_A": [" PLOGMX / 1.0 -1.0E12 0.0 0.0 /"],
        "with_plog": [" PLOG / 1.0 1.0E12 0.0 0.0 /", " PLOGMX / 1.0 1.0E12 0.0 0.0 /"],
        "unknown_bath": [" PLOGMX / 1.0 1.0E12 0.0 0.0 /", " PLOGSP / NOTASPECIES 1.0 1.0E12 0.0 0.0 /"],
    }[bad]
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism("\n".join(lines[:k + 1] + extra + lines[k + 1:]), s.thermo)


@pytest.mark.parametrize("patm", [0.05, 0.3, 1.0, 3.0, 30.0])
def test_oracle_xplog_rate(patm):
    """A + B => C + D with k = (c_bath k_bath + (cTot - c_bath) k_mix) / cTot."""
    from oracle.oracle import OracleMechanism
    data, m, ib = xplog_mechanism()
    A = m.arrays
    orc = OracleMechanism(data)
    ia, ib2 = A["reac_species"][:2]
    rng = np.random.default_rng(8)
    P = patm * 101325.0
    for _ in range(5):
        Y = rng.uniform(0.05, 1.0, m.n_species)
        Y /= Y.sum()
        T = rng.uniform(700.0, 2200.0)
        dy, _ = orc.rhs(np.concatenate([Y, [T]]), P)
        mwmix = 1.0 / (Y / A["mw"]).sum()
        c = P / R_J_KMOL / T * mwmix * Y / A["mw"]
        ctot = c.sum()
        k = (c[ib] * _k(BATH, T, P) + (ctot - c[ib]) * _k(MIX, T, P)) / ctot
        rho = P / R_J_KMOL / T * mwmix
        np.testing.assert_allclose(dy[ia], -A["mw"][ia] * k * c[ia] * c[ib2] / rho, rtol=1e-11)


def test_device_library_accepts_xplog_mechanisms_without_gpu():
    from laminarsmoke_b200 import lsg
    data, _, _ = xplog_mechanism()
    buf = (C.c_ubyte * len(data)).from_buffer_copy(data)
    h = C.c_void_p()
    assert lsg.lib().lsg_mech_load_blob(C.cast(buf, C.c_void_p), len(data), 0, C.byref(h)) not in (-2, -5)   # parsed and accepted (no GPU here: the upload fails, LSG_ERR_CUDA)
