"""CHEMKIN compiler: hand-computed known answers for the reference's preprocessing rules."""
import math
import os

import numpy as np
import pytest

from laminarsmoke_b200.mech import blob, chemkin, synthetic

# The reference checkout (its run/kinetic-mechanisms CHEMKIN files) is named by LSMOKE_REFERENCE_ROOT;
# the tests that recompile its files are skipped when the variable is unset.
REF_ROOT = os.environ.get("LSMOKE_REFERENCE_ROOT", "")
KM = os.path.join(REF_ROOT, "run", "kinetic-mechanisms") if REF_ROOT else ""
REF = os.path.join(KM, "POLIMI_H2CO_1412") + os.sep if KM else ""
have_ref = bool(REF) and os.path.exists(REF)

R_J_KMOL = 8314.4621
J_FROM_CAL = 8.3144621 / (8.3144621 / 4.18443)


def test_h2co_dimensions(h2co):
    data, species, A = h2co
    assert species == ["H2", "O2", "H2O", "H2O2", "O", "H", "OH", "HO2", "CO", "CO2", "HCO", "HE", "AR", "N2"]
    assert list(A["dims"]) == [14, 33]
    assert len(A["rev_thermo"]) == 29 and len(A["rev_explicit"]) == 0
    assert len(A["tb_rxn"]) == 5 and list(A["fo_rxn"]) == [2, 12, 16]
    assert list(A["fo_type"]) == [1, 1, 0]   # Troe, Troe, Lindemann


def test_molecular_weights_float_rounded_elements(h2co):
    _, species, A = h2co
    H, O, C, N = 1.008000016212463, 15.998999595642090, 12.010999679565430, 14.0069999694824
    mw = dict(zip(species, A["mw"]))
    assert mw["H2"] == 0.0 + H * 2.0
    assert mw["O2"] == 0.0 + O * 2.0
    assert mw["N2"] == 0.0 + N * 2.0
    assert mw["AR"] == 39.948001861572270
    assert mw["CO2"] == (0.0 + C * 1.0) + O * 2.0


def test_unit_conversion_bimolecular(h2co):
    _, _, A = h2co
    # H+O2=OH+O  .9600E+15 -.200 16625.0 (cal/mol, cm3/mol/s)
    a = 0.96e15 * (math.pow(1.e3, 1. - 2.) / math.pow(1., 1. - 2.))
    assert A["lnA"][0] == math.log(a)
    assert A["beta"][0] == -0.2
    assert A["e_over_r"][0] == (16625.0 * (1.e3 * J_FROM_CAL)) / R_J_KMOL
    # J_FROM_CAL is computed as R_J_mol / R_cal_mol (it rounds to 4.18443 in double)


def test_low_swap_and_falloff_units(h2co):
    _, _, A = h2co
    # H+O2(+M)=HO2(+M) main line .5580E+13 .400 .0 ; LOW/ .8400E+18 -.800 .0/
    k0 = 0.84e18 * (math.pow(1.e3, -2.) / math.pow(1., -2.))
    kinf = 0.558e13 * (math.pow(1.e3, 1. - 2.) / math.pow(1., 1. - 2.))
    assert A["lnA"][2] == math.log(k0)     # "direct" constant is k0
    assert A["beta"][2] == -0.8
    assert A["fo_lnA"][0] == math.log(kinf)
    assert A["fo_beta"][0] == 0.4
    assert (A["fo_a"][0], A["fo_b"][0], A["fo_c"][0], A["fo_d"][0]) == (0.5, 1.0e-30, 1.0e30, 0.0)
    # TROE with 4 parameters
    assert (A["fo_a"][1], A["fo_b"][1], A["fo_c"][1], A["fo_d"][1]) == (0.7346, 94.0, 1756.0, 5182.0)


def test_third_body_units_and_efficiencies(h2co):
    _, species, A = h2co
    # H2+M=H+H+M .1115E+15 .000 96081.0 ; sum of reactant orders = 1 + 1 (M)
    j = 7
    assert A["lnA"][j] == math.log(0.1115e15 * math.pow(1.e3, 1. - 2.))
    k = list(A["tb_rxn"]).index(j)
    sl = slice(A["tb_ptr"][k], A["tb_ptr"][k + 1])
    eff = dict(zip([species[s] for s in A["tb_species"][sl]], A["tb_eff_m1"][sl]))
    assert eff == {"H2": 2.5 - 1., "H2O": 12.0 - 1., "AR": 0.5 - 1., "CO": 1.9 - 1., "CO2": 3.8 - 1.}
    # products H+H merged into one entry with nu = 2
    ps = slice(A["prod_ptr"][j], A["prod_ptr"][j + 1])
    assert [species[s] for s in A["prod_species"][ps]] == ["H"]
    assert list(A["prod_nu"][ps]) == [2.0]
    assert A["delta_nu"][j] == 1.0


def test_irreversible_and_duplicates(h2co):
    _, _, A = h2co
    # 4 irreversible reactions ('=>'); the DUPLICATE pair stays two reactions
    assert int((A["is_reversible"] == 0).sum()) == 4
    assert A["lnA"][18] != A["lnA"][19]


def test_formation_list_order_matches_buckets(h2co):
    _, species, A = h2co
    # species H: reactant entries first (bucket order, reactions ascending), then products
    i = species.index("H")
    sl = slice(A["fr_ptr"][i], A["fr_ptr"][i + 1])
    coef = A["fr_coef"][sl]
    neg = np.where(coef < 0)[0]
    pos = np.where(coef > 0)[0]
    assert neg.max() < pos.min()
    assert 2.0 in coef  # H produced with nu = 2 by H2+M=H+H+M


def test_nasa_tables(h2co):
    _, species, A = h2co
    k = species.index("H2O")
    raw = A["nasa_raw"].reshape(-1, 18)[k]
    assert A["dh_ht"][6 * k + 2] == (1. / 3.) * raw[2]
    assert A["ds_lt"][6 * k + 3] == (1. / 3.) * raw[10]
    assert A["t_mid"][k] == raw[16]


def test_blob_roundtrip(h2co):
    data, species, A = h2co
    A2, sp2 = blob.unpack(blob.pack(A, species))
    assert sp2 == species
    for k in A:
        np.testing.assert_array_equal(A[k], A2[k])


@pytest.mark.skipif(not have_ref, reason="reference CHEMKIN files not present")
def test_packaged_blob_matches_fresh_compile(h2co):
    m = chemkin.compile_files(REF + "POLIMI_H2CO_1412.CKI", REF + "POLIMI_TOT_NOX_1412.CKT",
                              trc_path=REF + "POLIMI_TOT_NOX_1412.TRC")
    assert blob.pack(m.arrays, m.species) == h2co[0]


def test_tmid_correction_is_off_by_default():
    s = synthetic.generate(20, 30, seed=7)
    a = chemkin.compile_mechanism(s.kinetics, s.thermo)
    b = chemkin.compile_mechanism(s.kinetics, s.thermo, tmid_correct=True)
    assert not np.array_equal(a.arrays["cp_lt"], b.arrays["cp_lt"])


def test_parser_rejects_unknown_species():
    kin = "ELEMENTS\nH\nEND\nSPECIES\nH H2\nEND\nREACTIONS\nH+X=H2 1.0 0.0 0.0\nEND\n"
    s = synthetic.generate(12, 10, seed=1)
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism(kin, s.thermo)


@pytest.mark.parametrize("ns,nr", [(120, 800)])
def test_synthetic_mechanism_is_element_balanced(ns, nr):
    s = synthetic.generate(ns, nr, seed=1201)
    m = chemkin.compile_mechanism(s.kinetics, s.thermo)
    assert m.n_species == ns and m.n_reactions == nr
    comp = np.array([s.compositions[n] for n in m.species], dtype=float)
    A = m.arrays
    for j in range(nr):
        lhs = sum(A["reac_nu"][q] * comp[A["reac_species"][q]] for q in range(A["reac_ptr"][j], A["reac_ptr"][j + 1]))
        rhs = sum(A["prod_nu"][q] * comp[A["prod_species"][q]] for q in range(A["prod_ptr"][j], A["prod_ptr"][j + 1]))
        np.testing.assert_array_equal(lhs, rhs)
    assert len(A["tb_rxn"]) == round(0.15 * nr) and len(A["fo_rxn"]) == round(0.10 * nr)


def test_compile_command_line(tmp_path):
    """python -m laminarsmoke_b200.mech compile writes the same blob as the library call."""
    import subprocess
    import sys
    from laminarsmoke_b200.mech import blob, chemkin, synthetic
    sm = synthetic.generate(12, 30, seed=7)
    kin, thermo = sm.kinetics, sm.thermo
    (tmp_path / "k.cki").write_text(kin)
    (tmp_path / "t.ckt").write_text(thermo)
    out = tmp_path / "m.lsmech"
    r = subprocess.run([sys.executable, "-m", "laminarsmoke_b200.mech", "compile", str(tmp_path / "k.cki"),
                        str(tmp_path / "t.ckt"), "-o", str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    m = chemkin.compile_mechanism(kin, thermo)
    assert out.read_bytes() == blob.pack(m.arrays, m.species)
    r = subprocess.run([sys.executable, "-m", "laminarsmoke_b200.mech", "info", str(out)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and f"{m.n_species} species" in r.stdout


def _ford_case(extra=""):
    s = synthetic.generate(12, 10, seed=1)
    a, b, c = list(s.compositions)[:3]
    kin = (f"ELEMENTS\nC H O N\nEND\nSPECIES\n{a} {b} {c}\nEND\nREACTIONS\n"
           f"{a}+{b}=>{c} 1.0E13 0.5 1000.\nFORD /{a} 0.7/\nFORD /{c} 0.2/\n{extra}END\n")
    return kin, s.thermo


def test_ford_orders_and_units():
    """FORD (ReactionPolicy_CHEMKIN.hpp:511-545): the reactant coefficients are the starting orders, a FORD
    species replaces its order or is appended, the list is sorted by species, and the units of A follow
    the sum of the orders (0.7 + 1 + 0.2 = 1.9): A [m, kmol, s] = 1e13 * 1e3^(1 - 1.9)."""
    kin, thermo = _ford_case()
    m = chemkin.compile_mechanism(kin, thermo)
    A = m.arrays
    np.testing.assert_array_equal(A["reac_nu"], [1.0, 1.0])
    np.testing.assert_array_equal(A["ford_ptr"], [0, 3])
    np.testing.assert_array_equal(A["ford_species"], [0, 1, 2])
    np.testing.assert_array_equal(A["ford_val"], [0.7, 1.0, 0.2])
    assert A["lnA"][0] == math.log(1.0e13 * math.pow(1.e3, 1. - 1.9))


def test_ford_absent_keeps_the_blob_unchanged(h2co):
    assert "ford_val" not in h2co[2]


def test_rord_is_rejected_like_the_reference():
    kin, thermo = _ford_case("RORD /X 1.0/\n")
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism(kin, thermo)


def test_global_ch4_one_step():
    """The reference's GLOBAL_CH4_1step: CH4 + 2 O2 => CO2 + 2 H2O with FORD /CH4 1/ /O2 1/, so the rate
    law is second order and A = 1e15 cm3/mol/s = 1e12 m3/kmol/s."""
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    A, species = blob.unpack(mech.load("ch4_1step")[0])
    assert species == ["CH4", "O2", "CO2", "H2O", "N2"]
    np.testing.assert_array_equal(A["reac_nu"], [1.0, 2.0])
    np.testing.assert_array_equal(A["ford_val"], [1.0, 1.0])
    assert A["lnA"][0] == math.log(1.0e15 * math.pow(1.e3, 1. - 2.0))
    assert A["e_over_r"][0] == 20000.0 * 1.e3 * J_FROM_CAL / R_J_KMOL


def test_oracle_rhs_global_ch4_rate_law():
    """Oracle RHS of the one-step CH4 mechanism against the rate law written out by hand:
    r = k [CH4] [O2], dY_i/dt = MW_i nu_i r / rho."""
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    from oracle.oracle import OracleMechanism
    data, species = mech.load("ch4_1step")
    A, _ = blob.unpack(data)
    mw = A["mw"]
    orc = OracleMechanism(data)
    rng = np.random.default_rng(3)
    for _ in range(20):
        Y = rng.uniform(0.01, 1.0, 5)
        Y /= Y.sum()
        T = rng.uniform(800.0, 2200.0)
        dy, _ = orc.rhs(np.concatenate([Y, [T]]))
        ctot = 101325.0 / R_J_KMOL / T
        mwmix = 1.0 / (Y / mw).sum()
        c = ctot * mwmix * Y / mw
        k = math.exp(A["lnA"][0] - A["e_over_r"][0] / T)
        r = k * c[0] * c[1]
        rho = ctot * mwmix
        nu = np.array([-1.0, -2.0, 1.0, 2.0, 0.0])
        np.testing.assert_allclose(dy[:5], mw * nu * r / rho, rtol=1e-12, atol=1e-300)


@pytest.mark.skipif(not (KM and os.path.exists(os.path.join(KM, "GLOBAL_CH4_1step"))),
                    reason="LSMOKE_REFERENCE_ROOT unset or its CHEMKIN files not present")
@pytest.mark.parametrize("name,key", [("GLOBAL_CH4_1step", "ch4_1step"), ("GLOBAL_H2_1step", "h2_1step")])
def test_packaged_global_blobs_match_fresh_compile(name, key):
    from laminarsmoke_b200 import mech
    d = os.path.join(KM, name) + os.sep
    m = chemkin.compile_files(d + name + ".CKI", d + name + ".CKT", trc_path=d + name + ".TRC")
    assert blob.pack(m.arrays, m.species) == mech.load(key)[0]


@pytest.mark.parametrize("bad", [
    "H2+O2=OH+OH 1.0E13 X 0.0",              # not a number where beta stands
    "2.x H2+O2=H2O2 1.0E13 0.0 0.0",          # bad stoichiometric coefficient
    "H2+M=H+H+M 1.0E13 0.0 0.0\n H2O/1..0/",  # bad efficiency
    "H2+O2=OH+OH 1.0E13 0.0 0.0\n LOW / 1.0 2.0 /",   # LOW with two numbers, no (+M)
    "H2+O2=OH+OH 1.0E13 0.0 0.0\nEND = ",     # '=' on the END line
])
def test_malformed_reactions_raise_chemkin_errors(bad):
    """Malformed input raises ChemkinError naming the line, never another exception (a fuzz of the
    packaged mechanism's text found these)."""
    s = synthetic.generate(12, 10, seed=1)
    names = " ".join(n for n in ("H2", "O2", "OH", "H", "H2O2", "H2O") if n in s.compositions)
    kin = f"ELEMENTS\nC H O N\nEND\nSPECIES\n{names}\nEND\nREACTIONS\n{bad}\nEND\n"
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism(kin, s.thermo)


def test_malformed_thermo_raises_chemkin_error():
    """A NASA record with a broken number raises ChemkinError naming the record (thermo fuzzing found
    plain ValueErrors here)."""
    s = synthetic.generate(12, 10, seed=1)
    lines = s.thermo.split("\n")
    k = next(i for i, l in enumerate(lines) if l.rstrip().endswith("2"))
    lines[k] = lines[k][:10] + "1.2.3e+00" + lines[k][19:]
    with pytest.raises(chemkin.ChemkinError):
        chemkin.compile_mechanism(s.kinetics, "\n".join(lines))


def test_compile_command_line_with_transport(tmp_path):
    """--transport writes the same blob as compile_mechanism(..., transport_text=...)."""
    import subprocess
    import sys
    from laminarsmoke_b200.mech import synthetic
    s = synthetic.generate(12, 30, seed=7)
    tr = synthetic.transport_text(s)
    for nm, text in (("k.cki", s.kinetics), ("t.ckt", s.thermo), ("tr.trc", tr)):
        (tmp_path / nm).write_text(text)
    out = tmp_path / "m.lsmech"
    r = subprocess.run([sys.executable, "-m", "laminarsmoke_b200.mech", "compile", str(tmp_path / "k.cki"),
                        str(tmp_path / "t.ckt"), "--transport", str(tmp_path / "tr.trc"), "-o", str(out)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    m = chemkin.compile_mechanism(s.kinetics, s.thermo, transport_text=tr)
    assert out.read_bytes() == blob.pack(m.arrays, m.species)
    r = subprocess.run([sys.executable, "-m", "laminarsmoke_b200.mech", "info", str(out)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "transport fits: yes" in r.stdout
