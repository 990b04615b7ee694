"""CHEMKIN mechanism compiler: kinetics (.CKI) + thermodynamics (.CKT) -> packed tables.

This is the offline preprocessing step of the reaction-step path.  The reference
runs ``openSMOKEppCHEMKINPreProcessor`` once per mechanism; it writes
``kinetics.xml`` which the solvers load at start-up.  This module performs the
same transformations and produces the numbers the reference's maps hold after
reading that XML, so that the GPU kernels and the CPU oracle see identical
coefficients:

* CHEMKIN text clean-up: comments after ``!`` dropped, tabs become blanks
  (``kernel/thermo/InputFileCHEMKIN.hpp:89-104``).
* NASA-7 records, fixed-width fields and element columns 25-44 + 74-78
  (``kernel/thermo/ThermoPolicy_CHEMKIN.hpp:85-369``); the first record of a
  species name wins (``kernel/thermo/ThermoReaderPolicy_CHEMKIN.hpp:186``).
* Molecular weight = sum over the record's elements, in record order, of
  the float-rounded atomic weights (``kernel/thermo/AtomicElementMap.hpp:41-145``,
  ``kernel/thermo/AtomicComposition.hpp:77-84``).
* NASA coefficients are NOT corrected at T_mid: the preprocessor's
  ``ThermodynamicConsistency()`` calls are commented out
  (``openSMOKEppCHEMKINPreProcessor/CHEMKIN_PreProcessor.C:313-328``); the
  correction routine is kept here behind ``tmid_correction=True`` for study only.
* Reaction grammar: ``(+M)``, ``(+SPECIES)``, trailing ``+M``, ``<=>/=>/=``,
  species merged and sorted by index (``kernel/kinetics/KineticsUtilityFunctions.hpp:71-305,661-700``,
  ``kernel/kinetics/ReactionPolicy_CHEMKIN.hpp:122-1357``).
* LOW swap: for fall-off reactions the main-line Arrhenius becomes k_inf and the
  LOW parameters become the "direct" constant k0 (``ReactionPolicy_CHEMKIN.hpp:599-640``).
* Units to m, kmol, s, J with cal->J = R_J_mol / R_cal_mol
  (``ReactionPolicy_CHEMKIN.hpp:1359-1501``, ``math/PhysicalConstants.h:19-25``,
  ``math/Conversions.h:112``).
* XML values: lnA = log|A| (log(1e-100) for A = 0), E_over_R = E / 8314.4621,
  efficiencies stored minus one (``preprocessing/PreProcessorKineticsPolicy_CHEMKIN.hpp:2134-2260``,
  ``maps/KineticsMap_CHEMKIN.hpp:643-664,734-789``).  The XML text is written
  with 17-19 significant digits, so the text round trip is exact and is skipped.
* Stoichiometric lists bucketed by coefficient 1, 2, 3, 1/2, other, species-major
  with reactions ascending (``PreProcessorKineticsPolicy_CHEMKIN.hpp:858-1106``).
* NASA-derived tables Cp, DH, DS as ``maps/ThermodynamicsMap_CHEMKIN.hpp:263-343``.

All floating-point expressions below are evaluated in IEEE double precision
in the same order as the reference's C++ (Python floats are doubles and are
never contracted into FMAs; ``math.log``/``math.pow`` call the C library).
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# --- physical constants (math/PhysicalConstants.h:19-25) ---------------------
R_J_MOL = 8.3144621
R_CAL_MOL = 8.3144621 / 4.18443
R_J_KMOL = 8314.4621
NAV_MOL = 6.0221417930e23
J_FROM_EV = 1.6021765314e-19
J_FROM_CAL = R_J_MOL / R_CAL_MOL  # math/Conversions.h:112

# --- atomic weights (kernel/thermo/AtomicElementMap.hpp:41-145), the subset the
# mechanisms of this project use plus the common light elements.  Values are the
# reference's own float-rounded numbers.
ATOMIC_WEIGHTS = {
    "E": 0.0,
    "H": 1.008000016212463,
    "HE": 4.002999782562256,
    "LI": 6.93900,
    "BE": 9.01220,
    "B": 10.81100,
    "C": 12.010999679565430,
    "N": 14.0069999694824,
    "O": 15.998999595642090,
    "F": 18.99840,
    "NE": 20.18300,
    "NA": 22.98980,
    "MG": 24.31200,
    "AL": 26.98150,
    "SI": 28.08600,
    "P": 30.97380,
    "S": 32.06,
    "CL": 35.45300,
    "AR": 39.948001861572270,
    "K": 39.10200,
    "CA": 40.08000,
    "D": 2.01410,
}

TAG_SIMPLE, TAG_THIRDBODY, TAG_LINDEMANN, TAG_TROE, TAG_SRI = 0, 1, 2, 3, 4
FALLOFF_TAGS = (TAG_LINDEMANN, TAG_TROE, TAG_SRI)


class ChemkinError(ValueError):
    """Raised when a CHEMKIN file cannot be interpreted."""


def _good_lines(text: str) -> List[str]:
    """InputFileCHEMKIN: strip ``!`` comments, tabs -> blanks, drop blank lines."""
    out = []
    for raw in text.splitlines():
        line = raw.rstrip("\r")
        k = line.find("!")
        if k >= 0:
            line = line[:k]
        line = line.replace("\t", " ")
        if line.strip(" ") == "":
            continue
        out.append(line)
    return out


# --------------------------------------------------------------------------
# Thermodynamics
# --------------------------------------------------------------------------
@dataclass
class ThermoRecord:
    name: str
    elements: List[Tuple[str, float]]
    params: List[float]  # 1-based like the reference: [0]=unused,[1]=Tlow,[2]=Tmid,[3]=Thigh,[4..10]=HT,[11..17]=LT

    @property
    def mw(self) -> float:
        mw = 0.0
        for name, coeff in self.elements:
            if name not in ATOMIC_WEIGHTS:
                raise ChemkinError(f"unknown element {name} in species {self.name}")
            mw += ATOMIC_WEIGHTS[name] * coeff
        return mw


def _fixed_fields(line: str, widths: Sequence[int]) -> List[str]:
    out, pos = [], 0
    for w in widths:
        out.append(line[pos:pos + w])
        pos += w
    return out


def _parse_thermo_record(block: List[str], tdefault: Tuple[float, float, float]) -> ThermoRecord:
    line0 = block[0]
    if len(line0) < 80 or line0[79] != "1":
        raise ChemkinError("Expected 1 at column 80")
    words = _fixed_fields(line0, (16, 2, 6, 20, 1, 10, 10, 8, 5, 1, 1, 20))
    name = words[0].upper().strip().split(" ")[0].strip() if words[0].strip() else ""
    first = 1
    additional = ""
    if len(words[11]) > 0 and words[11][0] == "&":
        additional = block[1]
        first += 1
    atomic = words[3] + words[8]
    elements: List[Tuple[str, float]] = []
    toks = _fixed_fields(atomic, (2, 3) * 9)
    for k in range(0, len(toks), 2):
        nm, num = toks[k].strip(), toks[k + 1].strip()
        if nm != "" and not nm[0].isdigit():
            try:
                elements.append((nm.upper(), float(num)))
            except ValueError as exc:
                raise ChemkinError(f"bad atomic coefficient for {name}") from exc
    if additional:
        t = additional.split()
        for k in range(0, len(t) - 1, 2):
            elements.append((t[k].upper(), float(t[k + 1])))
    tl, tm, th = tdefault
    if words[5].strip():
        tl = float(words[5].strip())
    if words[6].strip():
        th = float(words[6].strip())
    if words[7].strip():
        tm = float(words[7].strip())
    if tl > tm or tm > th:
        raise ChemkinError(f"wrong temperature sequence for {name}")
    if len(block) < first + 3:
        raise ChemkinError(f"incomplete NASA record for {name}")
    l2, l3, l4 = block[first], block[first + 1], block[first + 2]
    for ln, tag in ((l2, "2"), (l3, "3"), (l4, "4")):
        if len(ln) < 80 or ln[79] != tag:
            raise ChemkinError(f"Expected {tag} at column 80 ({name})")
    nums = _fixed_fields(l2, (15,) * 5) + _fixed_fields(l3, (15,) * 5) + _fixed_fields(l4, (15,) * 4)
    coeffs = []
    for s in nums:
        s = s.replace("e 0", "E+0", 1).replace("E 0", "E+0", 1).strip()
        coeffs.append(float(s))
    params = [0.0, tl, tm, th] + coeffs
    return ThermoRecord(name=name, elements=elements, params=params)


def read_thermo(text: str) -> Dict[str, ThermoRecord]:
    """ThermoReaderPolicy_CHEMKIN::ReadFromASCIIFile: first record of a name wins."""
    lines = _good_lines(text)
    head = lines[0].split()
    if not head or head[0] not in ("THERMO", "thermo") or len(head) > 2:
        raise ChemkinError("Expected THERMO || THERMO ALL")
    t = lines[1].split()
    if len(t) != 3:
        raise ChemkinError("Wrong number of temperature ranges")
    try:
        tdef = (float(t[0]), float(t[1]), float(t[2]))
    except ValueError:
        raise ChemkinError("the THERMO line must give three default temperatures") from None
    starts = []
    end = None
    for j in range(2, len(lines)):
        word = lines[j][:15].strip()
        try:
            float(word)
            continue
        except ValueError:
            pass
        tok = word.split()
        if tok and tok[0] in ("END", "end") and len(tok) == 1:
            end = j
            break
        if tok and tok[0] in ("TEMP", "temp"):
            continue
        if len(lines[j]) >= 80 and lines[j][79] == "1":
            starts.append(j)
    starts.append(end if end is not None else len(lines))
    recs: Dict[str, ThermoRecord] = {}
    for a, b in zip(starts[:-1], starts[1:]):
        try:
            rec = _parse_thermo_record(lines[a:b], tdef)
        except ChemkinError:
            raise
        except ValueError as exc:
            raise ChemkinError(f"bad thermodynamic record: {lines[a].strip()[:40]}: {exc}") from None
        recs.setdefault(rec.name, rec)
    return recs


def tmid_correction(rec: ThermoRecord) -> None:
    """ThermoPolicy_CHEMKIN::CheckThermodynamicConsistency (ThermoPolicy_CHEMKIN.hpp:609-670).

    Not part of the reference's preprocessing path (its calls are commented out);
    available for experiments only.
    """
    p = rec.params
    R = R_J_MOL / (rec.mw * 1.e-3)
    T = p[2]
    lt = math.log(T)
    cp_plus = (p[4] + T * (p[5] + T * (p[6] + T * (p[7] + T * p[8])))) * R
    cp_minus = (p[11] + T * (p[12] + T * (p[13] + T * (p[14] + T * p[15])))) * R
    h_plus = ((p[4] + T * (p[5] / 2. + T * (p[6] / 3. + T * (p[7] / 4. + T * p[8] / 5.)))) + p[9] / T) * T * R
    h_minus = ((p[11] + T * (p[12] / 2. + T * (p[13] / 3. + T * (p[14] / 4. + T * p[15] / 5.)))) + p[16] / T) * T * R
    s_plus = ((p[4] * lt + T * (p[5] + T * (p[6] / 2. + T * (p[7] / 3. + T * p[8] / 4.)))) + p[10]) * R
    s_minus = ((p[11] * lt + T * (p[12] + T * (p[13] / 2. + T * (p[14] / 3. + T * p[15] / 4.)))) + p[17]) * R
    e_cp = abs(cp_plus - cp_minus) / (0.50 * (cp_plus + cp_minus))
    e_h = abs(h_plus - h_minus) / (0.50 * (h_plus + h_minus))
    e_s = abs(s_plus - s_minus) / (0.50 * (s_plus + s_minus))
    if e_cp > 1.e-3 or e_h > 1.e-3 or e_s > 1.e-3:
        return
    p[11] = cp_plus / R - (cp_minus / R - p[11])
    h_minus = ((p[11] + T * (p[12] / 2. + T * (p[13] / 3. + T * (p[14] / 4. + T * p[15] / 5.)))) + p[16] / T) * T * R
    p[16] = h_plus / R - (h_minus / R - p[16])
    s_minus = ((p[11] * lt + T * (p[12] + T * (p[13] / 2. + T * (p[14] / 3. + T * p[15] / 4.)))) + p[17]) * R
    p[17] = s_plus / R - (s_minus / R - p[17])


# --------------------------------------------------------------------------
# Kinetics
# --------------------------------------------------------------------------
@dataclass
class Reaction:
    reactants: List[Tuple[int, float]] = field(default_factory=list)  # sorted by species, merged
    products: List[Tuple[int, float]] = field(default_factory=list)
    reversible: bool = False
    explicit_rev: bool = False
    tag: int = TAG_SIMPLE
    A: float = 0.0
    beta: float = 0.0
    E: float = 0.0
    A_inf: float = 0.0
    beta_inf: float = 0.0
    E_inf: float = 0.0
    A_rev: float = 0.0
    beta_rev: float = 0.0
    E_rev: float = 0.0
    troe: List[float] = field(default_factory=list)
    sri: List[float] = field(default_factory=list)
    tb_species: List[int] = field(default_factory=list)
    tb_eff: List[float] = field(default_factory=list)
    pd_species: int = -1
    duplicate: bool = False
    ford: bool = False   # FORD given: forward_orders replace the reactant coefficients in the rate law
    plog: List[Tuple[float, float, float, float]] = field(default_factory=list)   # PLOG (p [atm], A, beta, E)
    plog_table: List[Tuple[float, float, float, float, float]] = field(default_factory=list)  # (p [Pa], ln p, ln A, beta, E/R) SI
    # PLOGMX / PLOGSP: (bath species index, -1 for the mixture; p [atm], A, beta, E) per line, and per bath in
    # order of first appearance its SI table [(p [Pa], ln p, ln A, beta, E/R)]
    xplog: List[Tuple[int, float, float, float, float]] = field(default_factory=list)
    xplog_table: List[Tuple[int, List[Tuple[float, float, float, float, float]]]] = field(default_factory=list)
    # LOWMX/LOWSP, TROEMX/TROESP, SRIMX/SRISP: (kind "low" | "troe" | "sri", bath index (-1 mixture), values)
    # per line, and per bath in order of first appearance (bath, A0, beta0, E0/R, type 0/1/2, parameters) SI
    xfo: List[Tuple[str, int, List[float]]] = field(default_factory=list)
    xfo_table: List[Tuple[int, float, float, float, int, List[float]]] = field(default_factory=list)
    xfo_kinf: Tuple[float, float, float] = (0., 0., 0.)   # (A_inf, beta_inf, E_inf/R) SI
    cheb: List[float] = field(default_factory=list)   # CHEB numbers as given: N, M, a_11 .. a_NM
    cheb_T: List[float] = field(default_factory=list)  # TCHEB (Tmin, Tmax) [K]
    cheb_P: List[float] = field(default_factory=list)  # PCHEB (Pmin, Pmax) [atm]
    cheb_conv: float = 1.0
    cabr: bool = False   # HIGH given: chemically activated bimolecular reaction (k0 on the line, k_inf in HIGH)
    forward_orders: List[Tuple[int, float]] = field(default_factory=list)
    text: str = ""


def _split_species_side(side: str) -> List[Tuple[str, float]]:
    """SeparateSpeciesAndStoichiometricCoefficients (KineticsUtilityFunctions.hpp:159-229)."""
    line = side.replace("(+M)", "+$PDR$").replace("(+m)", "+$PDR$")
    m = re.search(r"[(][+].*[)]", line, flags=re.IGNORECASE)
    if m:
        orig = m.group(0)
        name = orig.replace("(+", "+$PDS$")[:-1]
        line = line.replace(orig, name)
    line += "\n"
    line = line.replace("++", "$PLUS$+").replace("+\n", "$PLUS$")
    line = line.replace("+M\n", "+$TBR$").replace("+m\n", "+$TBR$")
    line = line.replace("\n", "")
    out = []
    for tok in [t for t in line.split("+") if t != ""]:
        tok = tok.replace("$PLUS$", "+")
        if not (tok[0].isdigit() or tok[0] == "."):
            out.append((tok, 1.0))
        else:
            j = 0
            while j < len(tok) and (tok[j].isdigit() or tok[j] == "."):
                j += 1
            if j == len(tok):
                raise ChemkinError(f"bad species token {tok}")
            try:
                out.append((tok[j:], float(tok[:j])))
            except ValueError:
                raise ChemkinError(f"bad stoichiometric coefficient in species token {tok}") from None
    return out


def _reorder_clean(pairs: List[Tuple[int, float]]) -> List[Tuple[int, float]]:
    """ReorderPairsOfVectors + CleanPairsOfVectors (KineticsUtilityFunctions.hpp:71-117)."""
    s = sorted(pairs, key=lambda p: p[0])
    idx = [p[0] for p in s]
    nu = [p[1] for p in s]
    for i in range(len(idx) - 1, 0, -1):
        if idx[i] == idx[i - 1]:
            nu[i - 1] += nu[i]
            idx[i] = -1
    return [(i, v) for i, v in zip(idx, nu) if i != -1]


def _species_value(line: str, what: str) -> Tuple[str, float]:
    """`KEY /SPECIES value/` (ReadReactionKeyWordPlusCoefficients with two tokens)."""
    a, b = line.find("/"), line.rfind("/")
    toks = line[a + 1:b].split() if 0 <= a < b else []
    if len(toks) != 2:
        raise ChemkinError(f"{what}: expected /SPECIES value/ in: {line.strip()}")
    try:
        return toks[0], float(toks[1])
    except ValueError:
        raise ChemkinError(f"{what}: bad value in: {line.strip()}") from None


def _slash_numbers(line: str, counts: Sequence[int], what: str) -> List[float]:
    parts = [p for p in line.strip().split("/") if p != ""]
    if len(parts) != 2:
        raise ChemkinError(f"{what}: syntax error")
    nums = parts[1].split()
    if len(nums) not in counts:
        raise ChemkinError(f"{what}: wrong number of arguments")
    try:
        return [float(x) for x in nums]
    except ValueError:
        raise ChemkinError(f"{what}: the coefficients are not numbers in: {line.strip()}") from None


def _parse_reaction(lines: List[str], species_index: Dict[str, int],
                    a_units: str, e_units: str) -> Reaction:
    if not lines:
        raise ChemkinError("a reaction line is missing its data (a '=' on the END line?)")
    first = lines[0]
    toks = first.split()
    if len(toks) < 4:
        raise ChemkinError(f"wrong number of arguments: {first}")
    r = Reaction(text=first.strip())
    try:
        r.A, r.beta, r.E = float(toks[-3]), float(toks[-2]), float(toks[-1])
    except ValueError:
        raise ChemkinError(f"the reaction line must end with A, beta and E: {first.strip()}") from None
    recon = "".join(toks[:-3])
    k = recon.find("<=>")
    if k >= 0:
        r.reversible, lhs, rhs = True, recon[:k], recon[k + 3:]
    else:
        k = recon.find("=>")
        if k >= 0:
            r.reversible, lhs, rhs = False, recon[:k], recon[k + 2:]
        else:
            k = recon.find("=")
            if k < 0:
                raise ChemkinError(f"missing = in {first}")
            r.reversible, lhs, rhs = True, recon[:k], recon[k + 1:]
    left = _split_species_side(lhs)
    right = _split_species_side(rhs)

    pdr = "none"
    third_body = False
    for side in (left, right):
        tags = [i for i, (s, _) in enumerate(side) if s == "$PDR$"]
        if len(tags) > 1:
            raise ChemkinError("pressure dependent tag used more than once")
        if tags:
            pdr = "all"
            side.pop(tags[0])
    for side in (left, right):
        tags = [i for i, (s, _) in enumerate(side) if s.startswith("$PDS$")]
        if len(tags) > 1:
            raise ChemkinError("pressure dependent tag used more than once")
        if tags:
            if pdr == "all":
                raise ChemkinError("two pressure-dependence tags")
            pdr = "partial"
            nm = side[tags[0]][0].replace("$PDS$", "")
            if nm not in species_index:
                raise ChemkinError(f"unknown species {nm}")
            if r.pd_species != -1 and r.pd_species != species_index[nm]:
                raise ChemkinError("inconsistent (+SPECIES) third body")
            r.pd_species = species_index[nm]
            side.pop(tags[0])
    for side in (left, right):
        tags = [i for i, (s, _) in enumerate(side) if s == "$TBR$"]
        if len(tags) > 1:
            raise ChemkinError("third body tag used more than once")
        if tags:
            if pdr != "none":
                raise ChemkinError("third body reaction not specified correctly")
            side.pop(tags[0])
            third_body = True

    def to_idx(side):
        out = []
        for s, v in side:
            if s not in species_index:
                raise ChemkinError(f"species not available: {s}")
            out.append((species_index[s], v))
        return _reorder_clean(out)

    r.reactants = to_idx(left)
    r.products = to_idx(right)

    i_low = i_troe = i_sri = i_lind = i_high = False
    for line in lines[1:]:
        k = line.find("/")
        keyword = line[:k].strip() if k >= 0 else line.split()[0]
        if keyword in species_index:
            parts = [p for p in line.strip().split("/")]
            if line.strip()[-1] != "/":
                raise ChemkinError("third body efficiencies: syntax error")
            parts = [p for p in parts if p != ""]
            if len(parts) % 2 != 0:
                raise ChemkinError("third body efficiencies: syntax error")
            for q in range(0, len(parts), 2):
                nm = parts[q].strip()
                if nm not in species_index:
                    raise ChemkinError(f"third body efficiencies: unknown species {nm}")
                r.tb_species.append(species_index[nm])
                try:
                    r.tb_eff.append(float(parts[q + 1].strip()))
                except ValueError:
                    raise ChemkinError(f"third body efficiencies: bad value in: {line.strip()}") from None
            if r.pd_species != -1:
                raise ChemkinError("third body reactions require (+M)")
            continue
        kw = keyword.upper()
        if kw == "LOW":
            if pdr == "none":
                raise ChemkinError("LOW only for pressure-dependent reactions")
            if r.xfo:
                raise ChemkinError("LOW cannot be combined with LOWMX/LOWSP")
            c = _slash_numbers(line, (3,), "LOW")
            i_low = True
            if not i_troe and not i_sri:
                i_lind = True
            r.A_inf, r.beta_inf, r.E_inf = r.A, r.beta, r.E
            r.A, r.beta, r.E = c
            if r.A_inf < 0.:
                raise ChemkinError("negative frequency factor in LOW reaction")
        elif kw == "HIGH":
            # ReactionPolicy_CHEMKIN.hpp:553-575: the high-pressure limit of a chemically activated
            # bimolecular (CABR) reaction; the reaction line keeps the low-pressure k0
            if pdr == "none":
                raise ChemkinError("HIGH only for pressure-dependent reactions")
            if i_low or r.cheb or r.plog:
                raise ChemkinError("HIGH cannot be combined with LOW/CHEB/PLOG")
            c = _slash_numbers(line, (3,), "HIGH")
            i_high = True
            if not i_troe and not i_sri:
                i_lind = True
            r.A_inf, r.beta_inf, r.E_inf = c
            r.cabr = True
        elif kw == "TROE":
            if pdr == "none":
                raise ChemkinError("TROE only for pressure-dependent reactions")
            if r.xfo:
                raise ChemkinError("TROE cannot be combined with the extended fall-off options")
            r.troe = _slash_numbers(line, (3, 4), "TROE")
            i_troe, i_lind = True, False
        elif kw == "SRI":
            if pdr == "none":
                raise ChemkinError("SRI only for pressure-dependent reactions")
            if r.xfo:
                raise ChemkinError("SRI cannot be combined with the extended fall-off options")
            r.sri = _slash_numbers(line, (3, 5), "SRI")
            i_sri, i_lind = True, False
        elif kw == "REV":
            c = _slash_numbers(line, (3,), "REV")
            if not r.reversible:
                raise ChemkinError("REV used on an irreversible reaction")
            r.A_rev, r.beta_rev, r.E_rev = c
            r.explicit_rev = True
        elif kw == "FORD":
            # ReactionPolicy_CHEMKIN.hpp:511-545: the order of one species in the forward rate law; the
            # reactant coefficients are the starting orders, a species not among the reactants is appended
            nm, val = _species_value(line, "FORD")
            if nm not in species_index:
                raise ChemkinError(f"FORD: species not available: {nm}")
            if not r.ford:
                r.forward_orders = list(r.reactants)
                r.ford = True
            si = species_index[nm]
            for q, (sq, _) in enumerate(r.forward_orders):
                if sq == si:
                    r.forward_orders[q] = (si, val)
                    break
            else:
                r.forward_orders.append((si, val))
        elif kw == "PLOG":
            # ReactionPolicy_CHEMKIN.hpp:772-792: one (p [atm], A, beta, E) point per line
            if third_body or pdr != "none" or i_low or i_troe or i_sri or r.xplog:
                raise ChemkinError("PLOG cannot be combined with third bodies or LOW/TROE/SRI")
            r.plog.append(tuple(_slash_numbers(line, (4,), "PLOG")))
        elif kw in ("LOWMX", "LOWSP", "TROEMX", "TROESP", "SRIMX", "SRISP"):
            # ReactionPolicy_CHEMKIN.hpp:639-730, 984-1070, 1126-1215: the extended fall-off form, per bath
            # (the mixture: ...MX; one species: ...SP) its low-pressure limit and optionally Troe or SRI
            if pdr == "none":
                raise ChemkinError(f"{kw} can be used only for pressure-dependent reactions")
            if i_low or i_high or i_troe or i_sri or r.cheb or r.cheb_T or r.cheb_P or r.plog or r.xplog:
                raise ChemkinError(f"{kw} cannot be combined with LOW/HIGH/TROE/SRI/CHEB/PLOG/PLOGMX")
            kind = {"LOW": "low", "TRO": "troe", "SRI": "sri"}[kw[:3]]
            counts = {"low": (3,), "troe": (3, 4), "sri": (3, 5)}[kind]
            if kw.endswith("MX"):
                r.xfo.append((kind, -1, _slash_numbers(line, counts, kw)))
            else:
                a, b = line.find("/"), line.rfind("/")
                tok = line[a + 1:b].split() if 0 <= a < b else []
                if len(tok) - 1 not in counts:
                    raise ChemkinError(f"{kw}: wrong number of arguments in: {line.strip()}")
                if tok[0] not in species_index:
                    raise ChemkinError(f"{kw}: bath species not available: {tok[0]}")
                try:
                    vals = [float(t) for t in tok[1:]]
                except ValueError:
                    raise ChemkinError(f"{kw}: the coefficients are not numbers in: {line.strip()}") from None
                r.xfo.append((kind, species_index[tok[0]], vals))
        elif kw in ("PLOGMX", "PLOGSP"):
            # ReactionPolicy_CHEMKIN.hpp:793-880: a PLOG table for the mixture (PLOGMX) or for one bath species
            # (PLOGSP), one point (p [atm], A, beta, E) per line
            if third_body:
                raise ChemkinError(f"{kw} cannot be used for third-body reactions")
            if i_low or i_high or i_troe or i_sri or r.cheb or r.cheb_T or r.cheb_P or r.plog or r.xfo:
                raise ChemkinError(f"{kw} cannot be combined with LOW/HIGH/TROE/SRI/CHEB/PLOG/LOWMX")
            if kw == "PLOGMX":
                r.xplog.append((-1,) + tuple(_slash_numbers(line, (4,), kw)))
            else:
                a, b = line.find("/"), line.rfind("/")
                tok = line[a + 1:b].split() if 0 <= a < b else []
                if len(tok) != 5:
                    raise ChemkinError(f"{kw}: expected /SPECIES p A beta E/ in: {line.strip()}")
                if tok[0] not in species_index:
                    raise ChemkinError(f"{kw}: bath species not available: {tok[0]}")
                try:
                    vals = tuple(float(t) for t in tok[1:])
                except ValueError:
                    raise ChemkinError(f"{kw}: the coefficients are not numbers in: {line.strip()}") from None
                r.xplog.append((species_index[tok[0]],) + vals)
        elif kw == "CHEB":
            # ReactionPolicy_CHEMKIN.hpp:456-475: every number between the slashes, over as many lines as needed
            if pdr != "all":
                raise ChemkinError("CHEB needs a (+M) pressure-dependent reaction")
            if i_low or i_troe or i_sri or r.plog:
                raise ChemkinError("CHEB cannot be combined with LOW/TROE/SRI/PLOG")
            a, b = line.find("/"), line.rfind("/")
            try:
                r.cheb += [float(t) for t in line[a + 1:b].split()]
            except ValueError:
                raise ChemkinError(f"CHEB: the coefficients are not numbers in: {line.strip()}") from None
        elif kw in ("TCHEB", "PCHEB"):
            if pdr != "all":
                raise ChemkinError(f"{kw} needs a (+M) pressure-dependent reaction")
            lim = _slash_numbers(line, (2,), kw)
            if (r.cheb_T if kw == "TCHEB" else r.cheb_P):
                raise ChemkinError(f"{kw} is used more than once")
            (r.cheb_T if kw == "TCHEB" else r.cheb_P).extend(lim)
        elif kw == "RORD":
            raise ChemkinError("option RORD is not available (ReactionPolicy_CHEMKIN.hpp:908-913 rejects it)")
        elif kw in ("DUP", "DUPLICATE"):
            r.duplicate = True
        elif kw == "UNITS":
            raise ChemkinError("per-reaction UNITS is not supported by this compiler")
        else:
            raise ChemkinError(f"option {keyword} is not supported by this compiler")

    if r.ford:   # ReorderPairsOfVectors + CleanPairsOfVectors of the orders (ReactionPolicy_CHEMKIN.hpp:1266-1271)
        r.forward_orders = _reorder_clean(r.forward_orders)
    if pdr == "all" and not i_low and not i_high and not r.cheb and not r.xfo:
        raise ChemkinError("no pressure dependence option defined")
    if pdr == "partial" and not i_low and not i_high:
        raise ChemkinError("no pressure dependence option defined")
    if r.cheb:
        # REACTION_CHEBYSHEV (ReactionPolicy_CHEMKIN.hpp:1299, :1321-1342): its k replaces the Arrhenius one;
        # no third-body or fall-off factor; default limits 300-2500 K and 0.001-100 atm
        if i_low:
            raise ChemkinError("CHEB cannot be combined with LOW")
        n_, m_ = int(r.cheb[0]), int(r.cheb[1])
        if n_ * m_ != len(r.cheb) - 2:
            raise ChemkinError(f"CHEB: expected {n_ * m_} coefficients, given {len(r.cheb) - 2}")
        r.cheb_T = r.cheb_T or [300., 2500.]
        r.cheb_P = r.cheb_P or [0.001, 100.]
        r.tag = TAG_SIMPLE
    elif r.xfo:
        # REACTION_EXTENDEDFALLOFF (ReactionPolicy_CHEMKIN.hpp:1300-1301): the kinetics tables keep it as a
        # simple reaction; the extended fall-off tables carry k
        if r.explicit_rev:
            raise ChemkinError("explicitly reversible extended fall-off reactions are not allowed")
        r.tag = TAG_SIMPLE
    elif not third_body and pdr == "none":
        r.tag = TAG_SIMPLE
    elif third_body:
        r.tag = TAG_THIRDBODY
    elif i_lind and (i_low or i_high):
        r.tag = TAG_LINDEMANN
    elif i_troe and (i_low or i_high):
        r.tag = TAG_TROE
    elif i_sri and (i_low or i_high):
        r.tag = TAG_SRI
    else:
        raise ChemkinError("unsupported pressure-dependent form")
    if r.A < 0. and r.tag != TAG_SIMPLE:
        raise ChemkinError("negative frequency factors only for simple reactions")
    if r.plog and r.tag != TAG_SIMPLE:
        raise ChemkinError("PLOG cannot be used for third-body or fall-off reactions")
    if r.xplog and r.tag != TAG_SIMPLE:
        raise ChemkinError("PLOGMX/PLOGSP cannot be used for third-body or fall-off reactions")
    _convert_units(r, a_units, e_units)
    return r


def _convert_units(r: Reaction, a_units: str, e_units: str) -> None:
    """ConversionFactors + ReactionOrders + ConvertUnits (ReactionPolicy_CHEMKIN.hpp:1359-1501)."""
    e_conv = {
        "CAL": 1.e3 * J_FROM_CAL,
        "KCAL": 1.e6 * J_FROM_CAL,
        "JOUL": 1.e3,
        "KJOU": 1.e6,
        "EVOL": 1.e3 * NAV_MOL * J_FROM_EV,
        "KELV": 1.e3 * R_J_MOL,
    }[e_units]
    a_conv = 1. if a_units == "MOLE" else NAV_MOL
    a_line, e_line = r.A, r.E   # the reaction line's values before conversion
    sum_lr = 0.   # ReactionOrders: the sums of the rate-law orders (lambda), FORD included
    for _, v in (r.forward_orders if r.ford else r.reactants):
        sum_lr += v
    sum_lp = 0.
    for _, v in r.products:
        sum_lp += v
    if r.tag == TAG_THIRDBODY:
        sum_lr += 1.
        if r.reversible:
            sum_lp += 1.
    if r.tag in FALLOFF_TAGS and r.cabr:   # ConvertUnits, CABR branch (ReactionPolicy_CHEMKIN.hpp:1395-1407)
        r.E *= e_conv
        r.E_inf *= e_conv
        r.A *= math.pow(1.e3, 1. - sum_lr) / math.pow(a_conv, 1. - sum_lr)
        r.A_inf *= math.pow(1.e3, 2. - sum_lr) / math.pow(a_conv, 2. - sum_lr)
        if r.explicit_rev:
            raise ChemkinError("explicitly reversible CABR reactions are not allowed")
    elif r.tag in FALLOFF_TAGS:
        r.E *= e_conv
        r.E_inf *= e_conv
        r.A *= math.pow(1.e3, -sum_lr) / math.pow(a_conv, -sum_lr)
        r.A_inf *= math.pow(1.e3, 1. - sum_lr) / math.pow(a_conv, 1. - sum_lr)
        if r.explicit_rev:
            raise ChemkinError("explicitly reversible falloff reactions are not allowed")
    else:
        r.E *= e_conv
        r.A *= math.pow(1.e3, 1. - sum_lr) / math.pow(a_conv, 1. - sum_lr)
        if r.cheb:   # ConvertUnits for REACTION_CHEBYSHEV (ReactionPolicy_CHEMKIN.hpp:1409-1412)
            r.cheb_conv = math.pow(1.e3, 1. - sum_lr) / math.pow(a_conv, 1. - sum_lr)
        if r.plog:
            # PressureLogarithmicRateExpression::Setup (PressureLogarithmicRateExpression.hpp:71-101), with the
            # conversion factors ConvertUnits appends (ReactionPolicy_CHEMKIN.hpp:1460-1465)
            conv_a = math.pow(1.e3, 1. - sum_lr) / math.pow(a_conv, 1. - sum_lr)
            last = -math.inf
            for pa, a_, b_, e_ in r.plog:
                if a_ < 0.:
                    raise ChemkinError("PLOG needs non-negative frequency factors")
                pp = pa * 101325.
                if pp <= last:
                    raise ChemkinError("PLOG pressures must be increasing")
                last = pp
                r.plog_table.append((pp, math.log(pp), math.log(max(a_ * conv_a, 1.e-32)), b_, e_ * e_conv / R_J_KMOL))
        if r.xfo:
            # ExtendedFallOff::Setup (ExtendedFallOff.hpp:71-169) with the conversion factors of ConvertUnits
            # (ReactionPolicy_CHEMKIN.hpp:1415-1453): k_inf from the reaction line, a low-pressure limit per
            # bath, the mixture's required; a bath takes one low-pressure line and at most one Troe or SRI line
            conv_a0 = math.pow(1.e3, -sum_lr) / math.pow(a_conv, -sum_lr)
            order: List[int] = []
            for _, sp, _ in r.xfo:
                if sp not in order:
                    order.append(sp)
            for sp in order:
                kinds = [kd for kd, sq, _ in r.xfo if sq == sp]
                if kinds.count("low") != 1 or len(kinds) > 2:
                    raise ChemkinError("extended fall-off: each bath needs one LOW line and at most one TROE or SRI")
            if -1 not in order:
                raise ChemkinError("extended fall-off needs the low-pressure parameters of the mixture (LOWMX)")
            for sp in order:
                if sp != -1 and sp in r.tb_species and r.tb_eff[r.tb_species.index(sp)] != 1.:
                    raise ChemkinError("extended fall-off: the third-body efficiency of a bath species must be 1")
                low = next(v for kd, sq, v in r.xfo if sq == sp and kd == "low")
                extra = [(kd, v) for kd, sq, v in r.xfo if sq == sp and kd != "low"]
                kind, par = (extra[0] if extra else ("low", []))
                r.xfo_table.append((sp, low[0] * conv_a0, low[1], low[2] * (e_conv / R_J_KMOL),
                                    {"low": 0, "troe": 1, "sri": 2}[kind], list(par)))
            conv_ainf = math.pow(1.e3, 1. - sum_lr) / math.pow(a_conv, 1. - sum_lr)
            r.xfo_kinf = (a_line * conv_ainf, r.beta, e_line * (e_conv / R_J_KMOL))
        if r.xplog:
            # ExtendedPressureLogarithmicRateExpression::Setup (:84-160) with the conversion factors of
            # ConvertUnits (ReactionPolicy_CHEMKIN.hpp:1467-1471): baths in order of first appearance, each
            # table with increasing pressures and non-negative A; a mixture table (PLOGMX) is required
            conv_a = math.pow(1.e3, 1. - sum_lr) / math.pow(a_conv, 1. - sum_lr)
            order: List[int] = []
            for sp, *_ in r.xplog:
                if sp not in order:
                    order.append(sp)
            if -1 not in order:
                raise ChemkinError("PLOGSP needs the kinetic parameters of the mixture (PLOGMX)")
            for sp in order:
                pts, last = [], -math.inf
                for sq, pa, a_, b_, e_ in r.xplog:
                    if sq != sp:
                        continue
                    if a_ < 0.:
                        raise ChemkinError("PLOGMX/PLOGSP need non-negative frequency factors")
                    pp = pa * 101325.
                    if pp <= last:
                        raise ChemkinError("PLOGMX/PLOGSP pressures must be increasing")
                    last = pp
                    pts.append((pp, math.log(pp), math.log(max(a_ * conv_a, 1.e-32)), b_, e_ * e_conv / R_J_KMOL))
                r.xplog_table.append((sp, pts))
        if r.explicit_rev:
            r.E_rev *= e_conv
            r.A_rev *= math.pow(1.e3, 1. - sum_lp) / math.pow(a_conv, 1. - sum_lp)


_A_UNIT_TAGS = {"MOLEC": "MOLEC", "MOLECULES": "MOLEC", "MOLE": "MOLE", "MOLES": "MOLE"}
_E_UNIT_TAGS = {
    "CAL": "CAL", "CAL/MOLE": "CAL", "EVOL": "EVOL", "EVOLTS": "EVOL",
    "JOUL": "JOUL", "JOULES/MOLE": "JOUL", "KCAL": "KCAL", "KCAL/MOLE": "KCAL",
    "KJOU": "KJOU", "KJOULES/MOLE": "KJOU", "KELV": "KELV", "KELVINS": "KELV",
}


def read_kinetics(text: str) -> Tuple[List[str], List[Reaction]]:
    """PreProcessorKineticsPolicy_CHEMKIN::ReadFromASCIIFile + KineticsFromASCIIFile (:66-560)."""
    lines = _good_lines(text)
    ir = None
    for j, ln in enumerate(lines):
        if "REACTIONS" in ln or "reactions" in ln:
            ir = j
            break
    if ir is None:
        raise ChemkinError("No REACTIONS keyword found")
    spec_lines = []
    end_lines = []
    for j in range(ir):
        ln = lines[j].replace("SPECIES", "SPEC").replace("species", "SPEC").replace("end", "END")
        if "SPEC" in ln:
            spec_lines.append(j)
        if "END" in ln:
            end_lines.append(j)
    if not spec_lines:
        raise ChemkinError("No SPECIES section found")
    last = spec_lines[0]
    for e in end_lines:
        if e < ir:
            last = e
    last = max(last, spec_lines[-1])
    txt = " ".join(lines[spec_lines[0]:last + 1]).strip()
    for a in ("SPECIES", "species", "SPEC", "spec", "END", "end"):
        txt = txt.replace(a, " ")
    species = txt.split()
    if len(set(species)) != len(species):
        raise ChemkinError("a species is declared more than once")
    species_index = {s: i for i, s in enumerate(species)}

    a_units, e_units = "MOLE", "CAL"
    head = lines[ir].split()
    if len(head) > 3:
        raise ChemkinError("wrong number of arguments on the REACTIONS line")
    for tag in head[1:]:
        t = tag.upper()
        if t in _E_UNIT_TAGS:
            e_units = _E_UNIT_TAGS[t]
        elif t in _A_UNIT_TAGS:
            a_units = _A_UNIT_TAGS[t]
        else:
            raise ChemkinError(f"wrong units on the REACTIONS line: {tag}")

    iend = None
    for j in range(ir, len(lines)):
        if "END" in lines[j] or "end" in lines[j]:
            iend = j + 1
            break
    if iend is None:
        raise ChemkinError("Missing END keyword after the reactions")
    starts = [j for j in range(iend) if "=" in lines[j]]
    starts.append(iend - 1)
    reactions = []
    for a, b in zip(starts[:-1], starts[1:]):
        reactions.append(_parse_reaction(lines[a:b], species_index, a_units, e_units))
    return species, reactions


# --------------------------------------------------------------------------
# Packed mechanism
# --------------------------------------------------------------------------
@dataclass
class Mechanism:
    """Compiled mechanism tables (0-based indices), the contents of the packed blob."""
    species: List[str]
    reactions: List[Reaction]
    thermo: List[ThermoRecord]
    arrays: Dict[str, np.ndarray] = field(default_factory=dict)

    @property
    def n_species(self) -> int:
        return len(self.species)

    @property
    def n_reactions(self) -> int:
        return len(self.reactions)

    def index(self, name: str) -> int:
        return self.species.index(name)


def _bucket(nu: float) -> int:
    if nu == 1.:
        return 0
    if nu == 2.:
        return 1
    if nu == 3.:
        return 2
    if nu == 0.5:
        return 3
    return 4


def build_tables(species: List[str], reactions: List[Reaction], thermo: List[ThermoRecord]) -> Dict[str, np.ndarray]:
    nc, nr = len(species), len(reactions)
    f64 = np.float64
    A: Dict[str, np.ndarray] = {}
    A["dims"] = np.array([nc, nr], dtype=np.int32)

    # --- thermodynamics: SetCoefficients (ThermodynamicsMap_CHEMKIN.hpp:263-343)
    one_third = 1. / 3.
    mw = np.zeros(nc, f64)
    cp_ht = np.zeros((nc, 5), f64); cp_lt = np.zeros((nc, 5), f64)
    dh_ht = np.zeros((nc, 6), f64); dh_lt = np.zeros((nc, 6), f64)
    ds_ht = np.zeros((nc, 6), f64); ds_lt = np.zeros((nc, 6), f64)
    tm = np.zeros(nc, f64); tl = np.zeros(nc, f64); th = np.zeros(nc, f64)
    raw = np.zeros((nc, 18), f64)
    for k, rec in enumerate(thermo):
        p = rec.params
        c = list(p[4:11]) + list(p[11:18]) + [p[1], p[3], p[2], rec.mw]
        raw[k] = c
        cp_ht[k] = c[0:5]
        cp_lt[k] = c[7:12]
        dh_ht[k] = [c[0], 0.50 * c[1], one_third * c[2], 0.25 * c[3], 0.20 * c[4], c[5]]
        dh_lt[k] = [c[7], 0.50 * c[8], one_third * c[9], 0.25 * c[10], 0.20 * c[11], c[12]]
        ds_ht[k] = [c[0], c[1], 0.50 * c[2], one_third * c[3], 0.25 * c[4], c[6]]
        ds_lt[k] = [c[7], c[8], 0.50 * c[9], one_third * c[10], 0.25 * c[11], c[13]]
        tl[k], th[k], tm[k] = c[14], c[15], c[16]
        mw[k] = c[17]
    A.update(mw=mw, nasa_raw=raw.ravel(), cp_ht=cp_ht.ravel(), cp_lt=cp_lt.ravel(),
             dh_ht=dh_ht.ravel(), dh_lt=dh_lt.ravel(), ds_ht=ds_ht.ravel(), ds_lt=ds_lt.ravel(),
             t_mid=tm, t_low=tl, t_high=th)

    # --- kinetic parameters (PreProcessorKineticsPolicy_CHEMKIN.hpp:2134-2176)
    lnA = np.zeros(nr, f64); beta = np.zeros(nr, f64); eor = np.zeros(nr, f64)
    sign = np.ones(nr, np.int32)
    for j, r in enumerate(reactions):
        lnA[j] = math.log(1.e-100) if r.A == 0. else math.log(abs(r.A))
        if r.A < 0.:
            sign[j] = -1
        beta[j] = r.beta
        eor[j] = r.E / R_J_KMOL
    A.update(lnA=lnA, beta=beta, e_over_r=eor, a_sign=sign)

    rev = [j for j, r in enumerate(reactions) if r.reversible]
    rev_th = [j for j, r in enumerate(reactions) if r.reversible and not r.explicit_rev]
    rev_ex = [j for j, r in enumerate(reactions) if r.reversible and r.explicit_rev]
    is_rev = np.zeros(nr, np.int32); is_rev[rev] = 1
    A["is_reversible"] = is_rev
    A["rev_thermo"] = np.array(rev_th, np.int32)
    A["rev_explicit"] = np.array(rev_ex, np.int32)
    A["lnA_rev"] = np.array([math.log(1.e-100) if reactions[j].A_rev == 0. else math.log(reactions[j].A_rev)
                             for j in rev_ex], f64)
    A["beta_rev"] = np.array([reactions[j].beta_rev for j in rev_ex], f64)
    A["e_over_r_rev"] = np.array([reactions[j].E_rev / R_J_KMOL for j in rev_ex], f64)

    # change of moles (PreProcessorKineticsPolicy_CHEMKIN.hpp:1153, ReactionPolicy_CHEMKIN.hpp:1495-1500)
    dnu = np.zeros(nr, f64)
    for j, r in enumerate(reactions):
        sr = 0.
        for _, v in r.reactants:
            sr += v
        sp = 0.
        for _, v in r.products:
            sp += v
        dnu[j] = sp - sr
    A["delta_nu"] = dnu

    # --- third body reactions
    tb = [j for j, r in enumerate(reactions) if r.tag == TAG_THIRDBODY]
    ptr, sp, eff = [0], [], []
    for j in tb:
        r = reactions[j]
        sp += r.tb_species
        eff += [e - 1. for e in r.tb_eff]
        ptr.append(len(sp))
    A["tb_rxn"] = np.array(tb, np.int32)
    A["tb_ptr"] = np.array(ptr, np.int32)
    A["tb_species"] = np.array(sp, np.int32)
    A["tb_eff_m1"] = np.array(eff, f64)

    # --- fall-off reactions (KineticsMap_CHEMKIN.hpp:669-789)
    fo = [j for j, r in enumerate(reactions) if r.tag in FALLOFF_TAGS]
    ftype, flnA, fbeta, feor = [], [], [], []
    fa, fb, fc, fd, fe, fsingle = [], [], [], [], [], []
    fptr, fsp, feff = [0], [], []
    for j in fo:
        r = reactions[j]
        ftype.append({TAG_LINDEMANN: 0, TAG_TROE: 1, TAG_SRI: 2}[r.tag])
        flnA.append(math.log(r.A_inf))
        fbeta.append(r.beta_inf)
        feor.append(r.E_inf / R_J_KMOL)
        a = b = c = d = e = 0.
        if r.tag == TAG_TROE:
            a, b, c = r.troe[0], r.troe[1], r.troe[2]
            if len(r.troe) == 4:
                d = r.troe[3]
        elif r.tag == TAG_SRI:
            a, b, c = r.sri[0], r.sri[1], r.sri[2]
            if len(r.sri) == 5:
                d, e = r.sri[3], r.sri[4]
            else:
                d, e = 1., 0.
        fa.append(a); fb.append(b); fc.append(c); fd.append(d); fe.append(e)
        fsingle.append(r.pd_species)
        if r.pd_species == -1:
            fsp += r.tb_species
            feff += [x - 1. for x in r.tb_eff]
        fptr.append(len(fsp))
    A["fo_rxn"] = np.array(fo, np.int32)
    A["fo_type"] = np.array(ftype, np.int32)
    A["fo_lnA"] = np.array(flnA, f64)
    A["fo_beta"] = np.array(fbeta, f64)
    A["fo_e_over_r"] = np.array(feor, f64)
    A["fo_a"] = np.array(fa, f64); A["fo_b"] = np.array(fb, f64); A["fo_c"] = np.array(fc, f64)
    A["fo_d"] = np.array(fd, f64); A["fo_e"] = np.array(fe, f64)
    A["fo_single"] = np.array(fsingle, np.int32)
    A["fo_ptr"] = np.array(fptr, np.int32)
    A["fo_species"] = np.array(fsp, np.int32)
    A["fo_eff_m1"] = np.array(feff, f64)
    if any(reactions[j].cabr for j in fo):   # chemically activated bimolecular slots, only when present
        A["fo_cabr"] = np.array([1 if reactions[j].cabr else 0 for j in fo], np.int32)

    # --- stoichiometry per reaction (species ascending; merged)
    rptr, rsp, rnu = [0], [], []
    pptr, psp, pnu = [0], [], []
    for r in reactions:
        for s, v in r.reactants:
            rsp.append(s); rnu.append(v)
        rptr.append(len(rsp))
        for s, v in r.products:
            psp.append(s); pnu.append(v)
        pptr.append(len(psp))
    A["reac_ptr"] = np.array(rptr, np.int32); A["reac_species"] = np.array(rsp, np.int32)
    A["reac_nu"] = np.array(rnu, f64)
    A["prod_ptr"] = np.array(pptr, np.int32); A["prod_species"] = np.array(psp, np.int32)
    A["prod_nu"] = np.array(pnu, f64)
    if any(r.plog for r in reactions):
        # pressure-logarithmic reactions (KineticsMap_CHEMKIN.hpp:1341-1348): their k replaces the Arrhenius one
        prx, pptr2, pv = [], [0], {k: [] for k in ("p", "lnp", "lnA", "beta", "eor")}
        for j, r in enumerate(reactions):
            if r.plog:
                prx.append(j)
                for pp, lp, la, b_, er in r.plog_table:
                    pv["p"].append(pp); pv["lnp"].append(lp); pv["lnA"].append(la); pv["beta"].append(b_)
                    pv["eor"].append(er)
                pptr2.append(len(pv["p"]))
        A["plog_rxn"] = np.array(prx, np.int32); A["plog_ptr"] = np.array(pptr2, np.int32)
        for k, v in pv.items():
            A["plog_" + k] = np.array(v, f64)
    if any(r.xfo for r in reactions):
        # extended fall-off reactions (KineticsMap_CHEMKIN.hpp:1672-1681; ExtendedFallOff::KineticConstant,
        # ExtendedFallOff.hpp:170-240): k_inf (A, beta, E/R), efficiencies - 1, per bath the low-pressure limit,
        # the form (0 Lindemann, 1 Troe, 2 SRI) and its parameters
        xr, kinf, tbp, tbs, tbe, bp, bs, low, bty, pp, par = [], [], [0], [], [], [0], [], [], [], [0], []
        for j, r in enumerate(reactions):
            if not r.xfo:
                continue
            xr.append(j)
            kinf += list(r.xfo_kinf)
            tbs += r.tb_species
            tbe += [e - 1. for e in r.tb_eff]
            tbp.append(len(tbs))
            for sp, a0, b0, e0, ty, pr in r.xfo_table:
                bs.append(sp); low += [a0, b0, e0]; bty.append(ty); par += pr; pp.append(len(par))
            bp.append(len(bs))
        A["xfo_rxn"] = np.array(xr, np.int32); A["xfo_kinf"] = np.array(kinf, f64)
        A["xfo_tb_ptr"] = np.array(tbp, np.int32); A["xfo_tb_sp"] = np.array(tbs, np.int32)
        A["xfo_tb_eff_m1"] = np.array(tbe, f64)
        A["xfo_bath_ptr"] = np.array(bp, np.int32); A["xfo_bath_sp"] = np.array(bs, np.int32)
        A["xfo_low"] = np.array(low, f64); A["xfo_type"] = np.array(bty, np.int32)
        A["xfo_par_ptr"] = np.array(pp, np.int32); A["xfo_par"] = np.array(par, f64)
    if any(r.xplog for r in reactions):
        # extended PLOG reactions (KineticsMap_CHEMKIN.hpp:1662-1670; ExtendedPressureLogarithmicRateExpression::
        # KineticConstant, :162-202): per reaction its baths (species index, -1 the mixture), per bath its points
        xrx, bptr, bsp, qptr = [], [0], [], [0]
        xv = {k: [] for k in ("p", "lnp", "lnA", "beta", "eor")}
        for j, r in enumerate(reactions):
            if not r.xplog:
                continue
            xrx.append(j)
            for sp, pts in r.xplog_table:
                bsp.append(sp)
                for pp, lp, la, b_, er in pts:
                    xv["p"].append(pp); xv["lnp"].append(lp); xv["lnA"].append(la); xv["beta"].append(b_)
                    xv["eor"].append(er)
                qptr.append(len(xv["p"]))
            bptr.append(len(bsp))
        A["xplog_rxn"] = np.array(xrx, np.int32); A["xplog_bath_ptr"] = np.array(bptr, np.int32)
        A["xplog_bath_sp"] = np.array(bsp, np.int32); A["xplog_ptr"] = np.array(qptr, np.int32)
        for k, v in xv.items():
            A["xplog_" + k] = np.array(v, f64)
    if any(r.cheb for r in reactions):
        # Chebyshev reactions (ChebyshevPolynomialRateExpression::Setup, :50-75): per reaction N, M, the
        # N x M coefficients by rows and (Tmin, Tmax, log10 Pmin, log10 Pmax, conversion) with P in Pa
        crx, cnm, cptr, cco, clim = [], [], [0], [], []
        for j, r in enumerate(reactions):
            if r.cheb:
                crx.append(j)
                cnm += [int(r.cheb[0]), int(r.cheb[1])]
                cco += list(r.cheb[2:])
                cptr.append(len(cco))
                clim += [r.cheb_T[0], r.cheb_T[1], math.log10(r.cheb_P[0] * 101325.),
                         math.log10(r.cheb_P[1] * 101325.), r.cheb_conv]
        A["cheb_rxn"] = np.array(crx, np.int32); A["cheb_nm"] = np.array(cnm, np.int32)
        A["cheb_ptr"] = np.array(cptr, np.int32); A["cheb_coef"] = np.array(cco, f64)
        A["cheb_lim"] = np.array(clim, f64)
    if any(r.ford for r in reactions):
        # forward rate-law orders (StoichiometricMap lambda lists), only when some reaction has FORD;
        # without them the reactant coefficients are the orders
        optr, osp, oval = [0], [], []
        for r in reactions:
            for sp, v in (r.forward_orders if r.ford else r.reactants):
                osp.append(sp); oval.append(v)
            optr.append(len(osp))
        A["ford_ptr"] = np.array(optr, np.int32); A["ford_species"] = np.array(osp, np.int32)
        A["ford_val"] = np.array(oval, f64)

    # --- formation-rate lists in the reference's accumulation order
    # (StoichiometricMap.hpp:656-729): per species, reactant buckets 1,2,3,1/2,other
    # then product buckets 1,2,3,1/2,other; reactions ascending inside a bucket.
    fr_ptr, fr_rxn, fr_coef = [0], [], []
    for i in range(nc):
        for side, sgn in (("r", -1.), ("p", 1.)):
            for bk in range(5):
                for j, r in enumerate(reactions):
                    lst = r.reactants if side == "r" else r.products
                    for s, v in lst:
                        if s == i and _bucket(v) == bk:
                            fr_rxn.append(j)
                            fr_coef.append(sgn * v)
        fr_ptr.append(len(fr_rxn))
    A["fr_ptr"] = np.array(fr_ptr, np.int32)
    A["fr_rxn"] = np.array(fr_rxn, np.int32)
    A["fr_coef"] = np.array(fr_coef, f64)
    return A


def compile_mechanism(kinetics_text: str, thermo_text: str, tmid_correct: bool = False,
                      transport_text: str = None) -> Mechanism:
    """Compile CHEMKIN kinetics + thermodynamics (+ transport) text into a :class:`Mechanism`.

    With a transport file the tables also carry the fitted species transport
    properties (``tr_*``, mech/transport.py) that the property update uses."""
    species, reactions = read_kinetics(kinetics_text)
    db = read_thermo(thermo_text)
    thermo = []
    for s in species:
        key = s.upper()
        if key not in db:
            raise ChemkinError(f"no thermodynamic data for species {s}")
        rec = db[key]
        rec = ThermoRecord(name=rec.name, elements=list(rec.elements), params=list(rec.params))
        if tmid_correct:
            tmid_correction(rec)
        thermo.append(rec)
    mech = Mechanism(species=species, reactions=reactions, thermo=thermo)
    mech.arrays = build_tables(species, reactions, thermo)
    if transport_text is not None:
        from .transport import transport_tables
        mech.arrays.update(transport_tables(species, mech.arrays, transport_text))
    return mech


def compile_files(cki_path: str, ckt_path: str, tmid_correct: bool = False, trc_path: str = None) -> Mechanism:
    with open(cki_path, "r", encoding="latin-1") as f:
        kin = f.read()
    with open(ckt_path, "r", encoding="latin-1") as f:
        th = f.read()
    tr = None
    if trc_path is not None:
        with open(trc_path, "r", encoding="latin-1") as f:
            tr = f.read()
    return compile_mechanism(kin, th, tmid_correct=tmid_correct, transport_text=tr)
