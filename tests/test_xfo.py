"""Extended fall-off reactions (LOWMX/LOWSP with TROEMX/TROESP/SRIMX/SRISP): CHEMKIN parsing and units
(ReactionPolicy_CHEMKIN.hpp:639-730, 984-1070, 1126-1215, 1415-1453), the bath-weighted rate constant
(ExtendedFallOff.hpp:170-240) in the oracle, and the device library accepting such mechanisms (its kernels
evaluate them; tests/test_gpu_extended.py compares them with the oracle)."""
import ctypes as C
import math

import numpy as np
import pytest

from laminarsmoke_b200.mech import blob, chemkin, synthetic

R_J_KMOL = 8314.4621
J_FROM_CAL = 8.3144621 / (8.3144621 / 4.18443)
KINF = (2.818001e11, 0.7725, 28043.862)                  # the reaction line: k_inf
LOW_MIX = (1.292317e16, 0.1325, 10402.975)
TROE_MIX = (0.3254, 265.58, 3908.30, 8121.96)
LOW_N2 = (6.0e15, 0.0, 9000.0)
SRI_N2 = (0.5, 200.0, 800.0, 1.2, 0.1)
EFF = {"H2O": 5.71, "CO2": 6.60}


def xfo_lines(reversible=False):
    arrow = "=" if reversible else "=>"
    return [f"H+S011(+M){arrow}OH(+M)   {KINF[0]:.6E} {KINF[1]} {KINF[2]}",
            f" LOWMX/ {LOW_MIX[0]:.6E} {LOW_MIX[1]} {LOW_MIX[2]} /",
            " TROEMX/ " + " ".join(str(v) for v in TROE_MIX) + " /",
            f" LOWSP/ N2 {LOW_N2[0]:.6E} {LOW_N2[1]} {LOW_N2[2]} /",
            " SRISP/ N2 " + " ".join(str(v) for v in SRI_N2) + " /",
            " " + "".join(f"{k}/{v}/" for k, v in EFF.items())]


def xfo_mechanism(body=None):
    s = synthetic.generate(12, 20, seed=4, physical=True)
    lines = s.kinetics.split("\n")
    head = lines[:lines.index("REACTIONS") + 1]
    m = chemkin.compile_mechanism("\n".join(head + (body or xfo_lines()) + ["END"]) + "\n", s.thermo)
    return blob.pack(m.arrays, m.species), m


def _k(T, c, sp):
    e_conv = 1e3 * J_FROM_CAL
    kinf = KINF[0] * 1e-3 * T ** KINF[1] * math.exp(-KINF[2] * (e_conv / R_J_KMOL) / T)
    ctot = c.sum()
    M = ctot + sum((v - 1.0) * c[sp.index(k)] for k, v in EFF.items())

    def kb(low, form, par):
        k0 = low[0] * 1e-6 * T ** low[1] * math.exp(-low[2] * (e_conv / R_J_KMOL) / T)
        Pr = k0 / kinf * M
        F = 1.0
        if form == "troe":
            a, t3, t1, t2 = par
            Fc = (1 - a) * math.exp(-T / t3) + a * math.exp(-T / t1) + math.exp(-t2 / T)
            lf = math.log10(Fc)
            cc, n = -0.4 - 0.67 * lf, 0.75 - 1.27 * lf
            e = math.log10(Pr) + cc
            F = 10 ** (lf / (1 + (e / (n - 0.14 * e)) ** 2))
        elif form == "sri":
            a, b, cpar, d, ee = par
            X = 1 / (1 + math.log10(Pr) ** 2)
            F = (a * math.exp(-b / T) + math.exp(-T / cpar)) ** X * d * T ** ee
        return kinf * Pr / (1 + Pr) * F

    cn2 = c[sp.index("N2")]
    return (cn2 * kb(LOW_N2, "sri", SRI_N2) + (ctot - cn2) * kb(LOW_MIX, "troe", TROE_MIX)) / ctot


def test_xfo_tables():
    _, m = xfo_mechanism()
    A = m.arrays
    sp = m.species
    np.testing.assert_array_equal(A["xfo_rxn"], [0])
    np.testing.assert_array_equal(A["xfo_bath_sp"], [-1, sp.index("N2")])
    np.testing.assert_array_equal(A["xfo_type"], [1, 2])
    np.testing.assert_array_equal(A["xfo_par_ptr"], [0, 4, 9])
    np.testing.assert_allclose(A["xfo_par"], list(TROE_MIX) + list(SRI_N2), rtol=1e-15)
    e_conv = 1e3 * J_FROM_CAL
    np.testing.assert_allclose(A["xfo_kinf"], [KINF[0] * 1e-3, KINF[1], KINF[2] * (e_conv / R_J_KMOL)], rtol=1e-15)
    np.testing.assert_allclose(A["xfo_low"], [LOW_MIX[0] * 1e-6, LOW_MIX[1], LOW_MIX[2] * (e_conv / R_J_KMOL),
                                              LOW_N2[0] * 1e-6, LOW_N2[1], LOW_N2[2] * (e_conv / R_J_KMOL)],
                               rtol=1e-15)
    np.testing.assert_array_equal(A["xfo_tb_sp"], [sp.index(k) for k in EFF])
    np.testing.assert_allclose(A["xfo_tb_eff_m1"], [v - 1.0 for v in EFF.values()], rtol=1e-15)
    assert len(A["fo_rxn"]) == 0 and len(A["tb_rxn"]) == 0     # not a plain fall-off or third-body reaction


@pytest.mark.parametrize("bad", ["no_mixture", "two_low", "with_troe", "bath_efficiency", "not_pressure_dependent",
                                 "explicit_rev"])
def test_xfo_rejections(bad):
    body = xfo_lines(reversible=bad == "explicit_rev")
    if bad == "no_mixture":
        body = [body[0]] + body[3:]
    elif bad == "two_low":
        body = body + [" LOWSP/ N2 1.0E15 0.0 0.0 /"]
    elif bad == "with_troe":
        body = body + [" TROE/ 0.5 100. 1000. /"]
    elif bad == "bath_efficiency":
        body = body[:-1] + [" N2/2.0/"]
    elif bad == "not_pressure_dependent":
        body = ["H+S011=>OH   1.0E12 0.0 0.0"] + body[1:-1]
    elif bad == "explicit_rev":
        body = body + [" REV/ 1.0E10 0.0 0.0 /"]
    with pytest.raises(chemkin.ChemkinError):
        xfo_mechanism(body)


@pytest.mark.parametrize("patm", [0.01, 0.3, 1.0, 10.0, 100.0])
def test_oracle_xfo_rate(patm):
    """H + S011 (+M) => OH: dY_H/dt = -MW_H k c_H c_S011 / rho with the bath-weighted k."""
    from oracle.oracle import OracleMechanism
    data, m = xfo_mechanism()
    A = m.arrays
    sp = m.species
    orc = OracleMechanism(data)
    ih, i2 = sp.index("H"), sp.index("S011")
    rng = np.random.default_rng(9)
    P = patm * 101325.0
    for _ in range(5):
        Y = rng.uniform(0.05, 1.0, m.n_species)
        Y /= Y.sum()
        T = rng.uniform(700.0, 2200.0)
        dy, _ = orc.rhs(np.concatenate([Y, [T]]), P)
        mwmix = 1.0 / (Y / A["mw"]).sum()
        c = P / R_J_KMOL / T * mwmix * Y / A["mw"]
        rho = P / R_J_KMOL / T * mwmix
        np.testing.assert_allclose(dy[ih], -A["mw"][ih] * _k(T, c, sp) * c[ih] * c[i2] / rho, rtol=1e-11)


def test_device_library_accepts_xfo_mechanisms_without_gpu():
    from laminarsmoke_b200 import lsg
    data, _ = xfo_mechanism()
    buf = (C.c_ubyte * len(data)).from_buffer_copy(data)
    h = C.c_void_p()
    assert lsg.lib().lsg_mech_load_blob(C.cast(buf, C.c_void_p), len(data), 0, C.byref(h)) not in (-2, -5)   # parsed and accepted (no GPU here: the upload fails, LSG_ERR_CUDA)
