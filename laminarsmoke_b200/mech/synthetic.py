"""Seeded synthetic C/H/O/N mechanisms written as CHEMKIN text.

The large-mechanism workloads of this project (120 species / 800 reactions and
500 species / 3 000 reactions) have no public mechanism behind them; they are
generated here from a seed and then go through the same CHEMKIN compiler as a
real mechanism, so the parser, the LOW swap and the unit conversions are
exercised on them too.

Construction:

* species are C_c H_h O_o N_n atom vectors (several isomers per composition,
  each with its own thermodynamics); a fixed set of named species (N2, O2, H2,
  H2O, CO, CO2, CH4, H, O, OH, HO2) is always present so fuel/air mixtures and
  the Burke-Schumann flame fields can be defined;
* reactions are element-balanced: bimolecular exchanges A+B=C+D found through
  an index of pair compositions, and recombinations A+B(+M)=C(+M) /
  A+B+M=C+M found through an index of single-species compositions;
* A is log-uniform in [1e6, 1e14] (CHEMKIN mol-cm-s units), beta ~ U[-2, 2],
  Ea ~ U[0, 60] kcal/mol; 15 % third-body reactions, 10 % Troe fall-off;
  optionally (frac_sri, frac_rev; both 0 by default, which leaves the draws of
  the packaged mechanisms unchanged) SRI fall-off reactions with 3 or 5
  parameters and exchange reactions with explicit reverse constants (REV);
* NASA-7 polynomials are least-squares fits of a smooth random cp(T) on
  [300, T_mid] and [T_mid, 3500] K; a6/a7 come from a bounded formation
  enthalpy (|Hf| <= 50 kcal/mol) and standard entropy, made continuous at T_mid,
  which keeps |dG/RT| of every reaction well below the exp() overflow range.

With ``physical=True`` the same draws are shaped by two physical bounds:
every activation energy is raised by the reaction's endothermicity at 298 K
(so no reverse rate constant exceeds its forward one by more than exp(dS/R)),
and forward rate constants at 2000 K are capped at 1e14 cm3/mol/s (1e17
cm6/mol2/s for third-body and 1e20 for fall-off low-pressure limits).  The
unbounded mechanisms give time scales near 1e-13 s and many cells that no
integrator finishes; the bounded ones integrate like real chemistry.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass
from typing import Dict, List, Tuple

import numpy as np

R_CAL = 1.98720425864083  # cal/mol/K, only used to shape synthetic enthalpies

NAMED = {
    "N2": (0, 0, 0, 2), "O2": (0, 0, 2, 0), "H2": (0, 2, 0, 0), "H2O": (0, 2, 1, 0),
    "CO": (1, 0, 1, 0), "CO2": (1, 0, 2, 0), "CH4": (1, 4, 0, 0), "H": (0, 1, 0, 0),
    "O": (0, 0, 1, 0), "OH": (0, 1, 1, 0), "HO2": (0, 1, 2, 0),
}


@dataclass
class SyntheticMechanism:
    kinetics: str
    thermo: str
    species: List[str]
    compositions: Dict[str, Tuple[int, int, int, int]]


def _fmt15(x: float) -> str:
    s = f"{x: .8E}"
    return s.rjust(15)[:15]


def _nasa_lines(name: str, comp, tmid: float, ht: np.ndarray, lt: np.ndarray) -> List[str]:
    els = ""
    for sym, cnt in zip(("C", "H", "O", "N"), comp):
        if cnt:
            els += f"{sym:<2s}{cnt:>3d}"
    els = els.ljust(20)[:20]
    l1 = f"{name:<16s}{'':2s}{'SYN':<6s}{els}G{300.0:10.2f}{3500.0:10.2f}{tmid:8.2f}{'':5s}{'':1s}1"
    assert len(l1) == 80, (len(l1), l1)
    c = list(ht) + list(lt)
    l2 = "".join(_fmt15(v) for v in c[0:5]) + "    2"
    l3 = "".join(_fmt15(v) for v in c[5:10]) + "    3"
    l4 = "".join(_fmt15(v) for v in c[10:14]) + " " * 19 + "4"
    return [l1, l2, l3, l4]


def _fit_nasa(rng: np.random.Generator, natoms: int, tmid: float):
    """Random smooth cp/R(T) -> (HT, LT) NASA-7 arrays (a1..a7)."""
    cp0 = 2.5 + 0.5 * natoms * rng.uniform(0.6, 1.0)
    cpinf = cp0 + 1.5 * natoms * rng.uniform(0.5, 1.0) + 0.5
    tc = rng.uniform(600.0, 1600.0)
    w = rng.uniform(300.0, 900.0)

    def cp(t):
        return cp0 + (cpinf - cp0) * (0.5 + 0.5 * np.tanh((t - tc) / w))

    def fit(lo, hi):
        t = np.linspace(lo, hi, 60)
        ts = t / 1000.0
        M = np.stack([ts ** k for k in range(5)], axis=1)
        a, *_ = np.linalg.lstsq(M, cp(t), rcond=None)
        return np.array([a[k] / 1000.0 ** k for k in range(5)])

    lt = fit(300.0, tmid)
    ht = fit(tmid, 3500.0)
    hf = rng.uniform(-50000.0, 50000.0) / R_CAL  # Hf/R [K]
    s0 = rng.uniform(18.0, 40.0) + 1.5 * natoms  # S0/R

    def hpoly(a, t):
        return a[0] * t + a[1] / 2 * t ** 2 + a[2] / 3 * t ** 3 + a[3] / 4 * t ** 4 + a[4] / 5 * t ** 5

    def spoly(a, t):
        return a[0] * math.log(t) + a[1] * t + a[2] / 2 * t ** 2 + a[3] / 3 * t ** 3 + a[4] / 4 * t ** 4

    a6_lt = hf - hpoly(lt, 298.15)
    a7_lt = s0 - spoly(lt, 298.15)
    a6_ht = (hpoly(lt, tmid) + a6_lt) - hpoly(ht, tmid)
    a7_ht = (spoly(lt, tmid) + a7_lt) - spoly(ht, tmid)
    return np.concatenate([ht, [a6_ht, a7_ht]]), np.concatenate([lt, [a6_lt, a7_lt]]), hf


def generate(n_species: int, n_reactions: int, seed: int,
             frac_thirdbody: float = 0.15, frac_troe: float = 0.10, physical: bool = False,
             frac_sri: float = 0.0, frac_rev: float = 0.0) -> SyntheticMechanism:
    rng = np.random.default_rng(seed)
    cmax = 2 if n_species <= 200 else 4
    hmax = 6 if n_species <= 200 else 10
    omax = 2 if n_species <= 200 else 3
    pool = [c for c in itertools.product(range(cmax + 1), range(hmax + 1), range(omax + 1), (0,))
            if sum(c) > 0]
    names: List[str] = []
    comps: Dict[str, Tuple[int, int, int, int]] = {}
    for nm, c in NAMED.items():
        names.append(nm)
        comps[nm] = c
    k = 0
    while len(names) < n_species:
        c = pool[int(rng.integers(len(pool)))] if k >= len(pool) else pool[k]
        k += 1
        nm = f"S{len(names):03d}"
        names.append(nm)
        comps[nm] = tuple(int(x) for x in c)

    # thermodynamics
    th_lines = ["THERMO ALL", "   300.000  1000.000  3500.000"]
    hf_r: Dict[str, float] = {}   # formation enthalpy / R [K]
    for nm in names:
        comp = comps[nm]
        tmid = float(rng.choice([800.0, 1000.0, 1200.0, 1400.0]))
        ht, lt, hf_r[nm] = _fit_nasa(rng, sum(comp), tmid)
        th_lines += _nasa_lines(nm, comp, tmid, ht, lt)
    th_lines.append("END")

    # composition indices
    idx = {nm: i for i, nm in enumerate(names)}
    by_comp: Dict[Tuple[int, ...], List[int]] = {}
    for nm in names:
        by_comp.setdefault(comps[nm], []).append(idx[nm])
    pair_index: Dict[Tuple[int, ...], List[Tuple[int, int]]] = {}
    ns = len(names)
    for i in range(ns):
        ci = comps[names[i]]
        for j in range(i, ns):
            cj = comps[names[j]]
            s = tuple(a + b for a, b in zip(ci, cj))
            pair_index.setdefault(s, []).append((i, j))
    recomb_targets = [(pair, c) for c, lst in by_comp.items() for pair in pair_index.get(c, [])]

    n_tb = int(round(frac_thirdbody * n_reactions))
    n_troe = int(round(frac_troe * n_reactions))
    n_sri = int(round(frac_sri * n_reactions))
    kinds = (["tb"] * n_tb + ["troe"] * n_troe + ["sri"] * n_sri
             + ["ex"] * (n_reactions - n_tb - n_troe - n_sri))
    rng.shuffle(kinds)
    seen = set()
    lines = ["ELEMENTS", "C H O N", "END", "SPECIES"]
    for q in range(0, ns, 8):
        lines.append(" ".join(names[q:q + 8]))
    lines += ["END", "REACTIONS"]
    bath_eff = [n for n in ("H2O", "CO2", "H2", "CO") if n in idx]

    def arrh(reac=(), prod=(), kcap=1.e14):
        A = 10.0 ** rng.uniform(6.0, 14.0)
        b = rng.uniform(-2.0, 2.0)
        Ea = rng.uniform(0.0, 60000.0)
        if physical:
            dh = R_CAL * (sum(hf_r[names[q]] for q in prod) - sum(hf_r[names[q]] for q in reac))   # cal/mol
            Ea += max(0.0, dh)
            A = min(A, kcap / 2000.0 ** b)
        return A, b, Ea

    for kind in kinds:
        for _attempt in range(10000):
            if kind == "ex":
                i, j = (int(x) for x in rng.integers(ns, size=2))
                s = tuple(a + b for a, b in zip(comps[names[i]], comps[names[j]]))
                cands = [p for p in pair_index.get(s, []) if set(p).isdisjoint({i, j})]
                if not cands:
                    continue
                c, d = cands[int(rng.integers(len(cands)))]
                key = ("ex",) + tuple(sorted([tuple(sorted((i, j))), tuple(sorted((c, d)))]))
                if key in seen:
                    continue
                seen.add(key)
                A, b, Ea = arrh((i, j), (c, d))
                lines.append(f"{'+'.join(_side(names, i, j))}={'+'.join(_side(names, c, d))}"
                             f"   {A:.6E} {b:.4f} {Ea:.3f}")
                if frac_rev > 0.0 and rng.uniform() < frac_rev:
                    # explicit reverse rate constants: k_r = k_f(T) / K_eq(298 K)-like ratio, kept in the
                    # collision limit; the reverse barrier is the forward one less the reaction enthalpy
                    dh = R_CAL * (hf_r[names[c]] + hf_r[names[d]] - hf_r[names[i]] - hf_r[names[j]])
                    Ar = min(A * 10.0 ** rng.uniform(-1.0, 1.0), 1.e14 / 2000.0 ** b)
                    lines.append(f" REV/ {Ar:.6E} {b:.4f} {max(0.0, Ea - dh):.3f} /")
                break
            else:
                (i, j), target = recomb_targets[int(rng.integers(len(recomb_targets)))]
                cands = by_comp[target]
                t = cands[int(rng.integers(len(cands)))]
                if t in (i, j):
                    continue
                key = (kind, tuple(sorted((i, j))), t)
                if key in seen:
                    continue
                seen.add(key)
                A, b, Ea = arrh((i, j), (t,), 1.e17 if kind == "tb" else 1.e14)
                left = "+".join(_side(names, i, j))
                effs = "".join(f"{n}/{rng.uniform(1.5, 8.0):.2f}/" for n in bath_eff
                               if idx[n] not in (i, j, t))
                if kind == "tb":
                    lines.append(f"{left}+M={names[t]}+M   {A:.6E} {b:.4f} {Ea:.3f}")
                elif kind == "sri":
                    lines.append(f"{left}(+M)={names[t]}(+M)   {A:.6E} {b:.4f} {Ea:.3f}")
                    A0 = min(A * 10.0 ** rng.uniform(3.0, 7.0), 1.e20 / 2000.0 ** (b - 1.0))
                    lines.append(f" LOW/ {A0:.6E} {b - 1.0:.4f} {Ea * 0.5:.3f} /")
                    sri = [rng.uniform(0.3, 1.5), rng.uniform(100.0, 800.0), rng.uniform(800.0, 3000.0)]
                    if rng.uniform() < 0.5:
                        sri += [rng.uniform(0.8, 1.2), rng.uniform(-0.3, 0.3)]
                    lines.append(" SRI/ " + " ".join(f"{v:.4f}" for v in sri) + " /")
                else:
                    lines.append(f"{left}(+M)={names[t]}(+M)   {A:.6E} {b:.4f} {Ea:.3f}")
                    A0 = A * 10.0 ** rng.uniform(3.0, 7.0)
                    b0 = b - rng.uniform(0.0, 2.0)
                    E0 = Ea * rng.uniform(0.0, 1.0)
                    if physical:
                        A0 = min(A0, 1.e20 / 2000.0 ** b0)
                    lines.append(f" LOW/ {A0:.6E} {b0:.4f} {E0:.3f} /")
                    lines.append(f" TROE/ {rng.uniform(0.1, 0.9):.4f} {rng.uniform(50, 500):.2f} "
                                 f"{rng.uniform(500, 5000):.2f} {rng.uniform(2000, 9000):.2f} /")
                if effs:
                    lines.append(" " + effs)
                break
        else:
            raise RuntimeError("could not place a reaction; enlarge the species pool")
    lines.append("END")
    return SyntheticMechanism(kinetics="\n".join(lines) + "\n", thermo="\n".join(th_lines) + "\n",
                              species=names, compositions=comps)


def _side(names, i, j):
    return [names[i], names[j]]


def transport_text(s: SyntheticMechanism) -> str:
    """A CHEMKIN transport file for a synthetic mechanism: per species the molecule shape from its atom
    count (1 atom, 2 linear, more non-linear) and Lennard-Jones parameters from smooth correlations with
    its size (sigma 2.3 + 0.45 n^0.6 A, epsilon/k 60 + 3.5 MW K), no dipole, polarizability 1.5 A^3 for
    the molecules, Zrot 4 (linear) or 1.5.  Stand-in data that exercises the transport fits and the
    property update at the synthetic mechanisms' sizes; not a physical property set."""
    lines = []
    for nm in s.species:
        c, h, o, n = s.compositions[nm]
        natoms = c + h + o + n
        shape = 0 if natoms == 1 else (1 if natoms == 2 else 2)
        mw = 12.011 * c + 1.008 * h + 15.999 * o + 14.007 * n
        sigma = 2.3 + 0.45 * natoms ** 0.6
        eps = 60.0 + 3.5 * mw
        alpha = 0.0 if natoms == 1 else 1.5
        zrot = 0.0 if natoms == 1 else (4.0 if shape == 1 else 1.5)
        lines.append(f"{nm:<16} {shape} {eps:9.3f} {sigma:7.3f} 0.000 {alpha:6.3f} {zrot:7.3f}")
    return "\n".join(lines) + "\nEND\n"
