"""Transport data of a CHEMKIN mechanism: Lennard-Jones records -> fitted species properties.

The mixture property update after each reaction step (solvers/laminarSMOKE/
properties.H:40-190) evaluates species viscosities, conductivities, binary
diffusivities and thermal-diffusion ratios from polynomial fits in T that the
reference's preprocessor computes once from the CHEMKIN transport file
(solvers/openSMOKEpp4laminarSMOKE/preprocessing/
PreProcessorSpeciesPolicy_CHEMKIN_WithTransport.hpp).  This module restates
that preprocessing:

* ``read_transport`` -- the transport file: per species the molecule shape
  (0 atom, 1 linear, 2 non-linear), epsilon/k [K], sigma [A], dipole moment
  [Debye], polarizability [A^3] and the rotational relaxation number at 298 K;
* ``SpeciesTransport`` -- Chapman-Enskog kinetic theory at one temperature
  (:217-534): viscosity (5.1), thermal conductivity by the Warnatz
  translational/rotational/vibrational split (5.17-5.34), binary diffusion
  coefficients (5.31) with the Stockmayer corrections of the pair potential
  for polar/non-polar pairs (5.9-5.14), and thermal-diffusion ratios
  (5.54-5.57) for the species up to 20 kg/kmol;
* ``fit`` -- least squares on 10 temperatures from 300 to 3600 K (:536-689):
  cubics in ln T for ln(eta), ln(lambda) and ln(D_jk at 1 bar), cubics in T
  for the thermal-diffusion ratios.

The reduced collision integrals come from the tabulated Stockmayer values
(``data/collision_integrals.npz``), interpolated as the reference does
(CollisionIntegralMatrices.hpp:187-455): three-point quadratics in T* and
then in delta*, with the tabulated high-T* polynomials beyond T* = 75.

The fits enter the packed mechanism as

* ``tr_eta``, ``tr_lambda`` -- [nc, 4] coefficients of ln(eta) [kg/m/s] and
  ln(lambda) [W/m/K] in powers of ln T;
* ``tr_gamma`` -- [nc (nc - 1) / 2, 4] coefficients of ln(D_jk P) [m^2/s bar]
  in powers of ln T, pairs j < k in row order;
* ``tr_teta`` -- [n_teta, nc, 4] coefficients of the thermal-diffusion ratio
  theta_ij in powers of T, for the light species ``tr_iteta`` [n_teta].
"""
from __future__ import annotations

import functools
import math
import os
from dataclasses import dataclass
from typing import Dict, List, Sequence

import numpy as np

R_J_MOL = 8.3144621            # PhysicalConstants.h:20
R_J_KMOL = 8314.4621           # PhysicalConstants.h:24
K_BOLTZMANN = 1.3806504e-23    # PhysicalConstants.h:17 [J/K]
MAX_MW_THERMAL_DIFFUSION = 20.  # PhysicalConstants.h:44 [kg/kmol]
_BOLTZMANN_ERG = K_BOLTZMANN * 1.e7
_MU_MIN = 1.e-38
_ZROTA = 0.5 * math.pi ** 1.5
_ZROTB = 2.0 + 0.25 * math.pi ** 2
_ZROTC = math.pi ** 1.5
_TWO_OVER_PI = 2. / math.pi
_FIVE_OVER_3R = 5. / (3. * R_J_MOL)
FIT_TMIN, FIT_TMAX, FIT_POINTS = 300., 3600., 10


class TransportError(ValueError):
    pass


@dataclass
class TransportRecord:
    name: str
    shape: int          # 0 atom, 1 linear, 2 non-linear
    eps_over_kb: float  # [K]
    sigma: float        # [A]
    mu: float           # dipole moment [Debye]
    alpha: float        # polarizability [A^3]
    zrot298: float      # rotational relaxation collision number at 298 K


def read_transport(text: str) -> Dict[str, TransportRecord]:
    """CHEMKIN transport file: one species per line, name then six numbers;
    '!' starts a comment.  As TransportReaderPolicy_CHEMKIN::ReadFromASCIIFile
    (kernel/transport/TransportReaderPolicy_CHEMKIN.hpp:52-79) reads it, the
    first line containing END or end ends the file and the first record of a
    species is the one kept.  Keys are upper-case names."""
    db: Dict[str, TransportRecord] = {}
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].strip()
        if "END" in line or "end" in line:
            break
        if not line:
            continue
        tok = line.split()
        if len(tok) < 7:
            raise TransportError(f"transport record needs 7 fields: {raw!r}")
        try:
            shape = int(float(tok[1]))
            vals = [float(v) for v in tok[2:7]]
        except ValueError as e:
            raise TransportError(f"bad transport record {raw!r}") from e
        if shape not in (0, 1, 2):
            raise TransportError(f"bad molecule shape {shape} for {tok[0]}")
        db.setdefault(tok[0].upper(), TransportRecord(tok[0], shape, *vals))
    return db


@functools.lru_cache(maxsize=1)
def _tables():
    from . import DATA
    with np.load(os.path.join(DATA, "collision_integrals.npz")) as z:
        return {k: np.array(z[k]) for k in z.files}


def _count_below(v: np.ndarray, x: float) -> int:
    """1-based index of the last tabulated value below x (the bisection of
    OpenSMOKEVector::LocateInSortedVector on an increasing vector)."""
    return int(np.count_nonzero(v < x))


def _quad3(x1, x2, x3, f1, f2, f3, x):
    a2 = (f2 - f1) / (x2 - x1)
    a3 = (f3 - f1 - a2 * (x3 - x1)) / ((x3 - x1) * (x3 - x2))
    return f1 + (x - x1) * (a2 + a3 * (x - x2))


def _omega(table: np.ndarray, high, tstar: float, dstar: float) -> float:
    ts, ds = _tables()["t_star"], _tables()["delta_star"]
    if tstar > ts[35]:
        return high[0] + tstar * (high[1] + tstar * (high[2] - tstar * high[3]))
    it = 1 if tstar < ts[1] else _count_below(ts, tstar)
    x1, x2, x3 = ts[it - 1], ts[it], ts[it + 1]

    def along_t(col):
        return _quad3(x1, x2, x3, table[it - 1, col], table[it, col], table[it + 1, col], tstar)

    if abs(dstar) <= 1.e-5:
        return along_t(0)
    if dstar < ds[1]:
        idx = 1
    elif dstar > ds[6]:
        idx = 6
    else:
        idx = _count_below(ds, dstar)
    y = [along_t(idx - 1), along_t(idx), along_t(idx + 1)]
    return _quad3(ds[idx - 1], ds[idx], ds[idx + 1], y[0], y[1], y[2], dstar)


def omega11(tstar: float, dstar: float) -> float:
    """Omega(1,1)*: CollisionIntegral11 (CollisionIntegralMatrices.hpp:187-312)."""
    tstar = max(tstar, 0.09)
    return _omega(_tables()["omega11"], (.623, -.136e-2, .346e-5, .343e-8), tstar, dstar)


def omega22(tstar: float, dstar: float) -> float:
    """Omega(2,2)*: Omega22k (CollisionIntegralMatrices.hpp:314-455); a T*
    below 0.09 is replaced by 1, as there."""
    if tstar < 0.09:
        tstar = 1.0
    return _omega(_tables()["omega22"], (.703, -.146e-2, .357e-5, .343e-8), tstar, dstar)


class SpeciesTransport:
    """Kinetic-theory species properties of one mechanism (the preprocessor's state)."""

    def __init__(self, species: Sequence[str], mw: np.ndarray, cp_ht: np.ndarray, cp_lt: np.ndarray,
                 t_mid: np.ndarray, records: Dict[str, TransportRecord]):
        nc = len(species)
        self.nc = nc
        self.mw = np.asarray(mw, float)
        self.cp_ht = np.asarray(cp_ht, float).reshape(nc, 5)
        self.cp_lt = np.asarray(cp_lt, float).reshape(nc, 5)
        self.t_mid = np.asarray(t_mid, float)
        recs = []
        for s in species:
            r = records.get(s.upper())
            if r is None:
                raise TransportError(f"no transport data for species {s}")
            recs.append(r)
        self.shape = np.array([r.shape for r in recs])
        self.eps_kb = np.array([r.eps_over_kb for r in recs])
        self.sigma = np.array([r.sigma for r in recs])
        self.alpha = np.array([r.alpha for r in recs])
        self.zrot298 = np.array([r.zrot298 for r in recs])
        mu = np.array([r.mu for r in recs]) * 1.e-6              # Debye -> sqrt(A^3 erg)
        mu[mu < _MU_MIN] = 0.
        self.mu = mu
        self.eps = _BOLTZMANN_ERG * self.eps_kb                    # [erg]
        self.mu_star = mu / np.sqrt(self.eps * self.sigma ** 3)
        self.light = [i for i in range(nc) if self.mw[i] <= MAX_MW_THERMAL_DIFFUSION]
        # collision-pair parameters (InitializeMassDiffusivity, :261-273)
        self.delta_jk = np.zeros((nc, nc))
        self.coeff_djk = np.zeros((nc, nc))
        for j in range(nc):
            for k in range(nc):
                e, s = self.pair_potential(j, k)
                mujk = math.sqrt(mu[j] * mu[k]) / math.sqrt(e * _BOLTZMANN_ERG * s ** 3)
                self.delta_jk[j, k] = 0.5 * mujk ** 2
                mjk = 2. * self.mw[j] * self.mw[k] / (self.mw[j] + self.mw[k])
                self.coeff_djk[j, k] = 2.6693e-7 / (math.sqrt(mjk) * s ** 2)
        # conductivity constants (InitializeThermalConductivity, :275-302)
        aux = np.sqrt(self.eps_kb / 298.)
        self.f298 = 1. + aux * (_ZROTA + aux * (_ZROTB + aux * _ZROTC))
        self.cv_trans = 1.5 * R_J_MOL
        self.cv_rot = np.where(self.shape == 0, 0., np.where(self.shape == 1, R_J_MOL, self.cv_trans))
        self.coeff_dkk = 2.6693e-7 / (np.sqrt(self.mw) * self.sigma ** 2)
        self.coeff_eta = 26.693e-7 * np.sqrt(self.mw) / self.sigma ** 2

    def pair_potential(self, j: int, k: int):
        """epsilon_jk/k [K] and sigma_jk [A] with the polar/non-polar
        correction (LennardJonesPotentialAndCollisionDiameter, :217-253)."""
        e = math.sqrt(self.eps_kb[j] * self.eps_kb[k])
        s = 0.5 * (self.sigma[j] + self.sigma[k])
        for n, p in ((j, k), (k, j)):
            if self.mu[n] == 0. and self.mu[p] != 0.:
                a_star = self.alpha[n] / self.sigma[n] ** 3
                xsi = 1. + 0.25 * a_star * self.mu_star[p] ** 2 * math.sqrt(self.eps[p] / self.eps[n])
                e *= xsi * xsi
                s *= xsi ** (-1. / 6.)
                break
        return e, s

    def cp_mass(self, T: float) -> np.ndarray:
        """Species cp [J/kg/K] from the NASA polynomials (ThermoPolicy_CHEMKIN::cp,
        kernel/thermo/ThermoPolicy_CHEMKIN.hpp:371-379)."""
        out = np.empty(self.nc)
        for i in range(self.nc):
            a = self.cp_ht[i] if T > self.t_mid[i] else self.cp_lt[i]
            r = R_J_MOL / (self.mw[i] * 1.e-3)
            out[i] = (a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4])))) * r
        return out

    def viscosity(self, T: float) -> np.ndarray:
        """[kg/m/s] (SingleSpeciesViscosity, :525-534; the species delta* stays 0)."""
        kb_over_eps = 1. / self.eps_kb
        om = np.array([omega22(T * kb_over_eps[k], 0.) for k in range(self.nc)])   # TkStar = T kb/eps
        return self.coeff_eta * math.sqrt(T) / om

    def conductivity(self, T: float) -> np.ndarray:
        """[W/m/K] (SpeciesThermalConductivities, :323-336, 419-500)."""
        eta = self.viscosity(T)
        aux = np.sqrt(self.eps_kb * (1. / T))     # ComputeFT: sqrt(eps/k uT)
        fT = 1. + aux * (_ZROTA + aux * (_ZROTB + aux * _ZROTC))
        zrot = self.zrot298 * self.f298 / fT
        cv = self.cp_mass(T) - R_J_KMOL * (1. / self.mw)     # SpeciesCv (WithoutTransport.hpp:95-99)
        cv_vib = cv * self.mw * 1.e-3 - self.cv_trans - self.cv_rot
        rho = 100. / (R_J_MOL * T) * self.mw
        kb_over_eps = 1. / self.eps_kb
        om11 = np.array([omega11(T * kb_over_eps[k], 0.) for k in range(self.nc)])
        dkk = self.coeff_dkk * T ** 1.5 / om11
        lam = np.empty(self.nc)
        for k in range(self.nc):
            f_vib = rho[k] * dkk[k] / eta[k]
            A = 2.5 - f_vib
            B = zrot[k] + _TWO_OVER_PI * (_FIVE_OVER_3R * self.cv_rot[k] + f_vib)
            f_trans = 2.50 * (1. - _TWO_OVER_PI * self.cv_rot[k] / self.cv_trans * A / B)
            umw = 1. / self.mw[k]
            if self.shape[k] == 0:
                lam[k] = eta[k] * umw * (f_trans * self.cv_trans)
            else:
                f_rot = f_vib * (1. + _TWO_OVER_PI * A / B)
                lam[k] = eta[k] * umw * (f_trans * self.cv_trans + f_rot * self.cv_rot[k] + f_vib * cv_vib[k])
        return lam * 1000.

    def binary_diffusivity(self, T: float, p_bar: float = 1.) -> np.ndarray:
        """D_jk [m^2/s] (BinaryDiffusionCoefficients, :390-417).  The reduced
        temperature uses the uncorrected pair potential, as there."""
        D = np.zeros((self.nc, self.nc))
        tp = T ** 1.5 / p_bar
        for j in range(self.nc):
            for k in range(j + 1, self.nc):
                ts = T / math.sqrt(self.eps_kb[j] * self.eps_kb[k])
                D[j, k] = D[k, j] = self.coeff_djk[j, k] * tp / omega11(ts, self.delta_jk[j, k])
        for k in range(self.nc):
            D[k, k] = self.coeff_dkk[k] * tp / omega11(T * (1. / self.eps_kb[k]), 0.)
        return D

    def thermal_diffusion_ratios(self, T: float) -> np.ndarray:
        """theta_ij for the light species i (SpeciesThermalDiffusionRatios, :349-388)."""
        tab = _tables()
        out = np.zeros((len(self.light), self.nc))
        for a, k in enumerate(self.light):
            for j in range(self.nc):
                e, _ = self.pair_potential(k, j)
                t = math.log(T / e)
                pw = [t ** n for n in range(7)]
                A = float(np.dot(tab["fit_astar"], pw))
                B = float(np.dot(tab["fit_bstar"], pw))
                C = float(np.dot(tab["fit_cstar"], pw))
                out[a, j] = (7.5 * (2. * A + 5.) * (6. * C - 5.) / (A * (16. * A - 12. * B + 55.)) *
                             (self.mw[k] - self.mw[j]) / (self.mw[k] + self.mw[j]))
        return out


def _solve_full_pivot(M: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """Gaussian elimination with complete pivoting (the 4 x 4 normal
    equations are solved with a full-pivoting LU in the reference)."""
    A = np.array(M, float)
    B = np.array(rhs, float)
    n = A.shape[0]
    perm = list(range(n))
    for c in range(n):
        sub = np.abs(A[c:, c:])
        r, q = np.unravel_index(int(np.argmax(sub)), sub.shape)
        r += c
        q += c
        A[[c, r]] = A[[r, c]]
        B[[c, r]] = B[[r, c]]
        A[:, [c, q]] = A[:, [q, c]]
        perm[c], perm[q] = perm[q], perm[c]
        for i in range(c + 1, n):
            f = A[i, c] / A[c, c]
            A[i, c:] -= f * A[c, c:]
            B[i] -= f * B[c]
    X = np.zeros_like(B)
    for i in range(n - 1, -1, -1):
        X[i] = (B[i] - A[i, i + 1:] @ X[i + 1:]) / A[i, i]
    out = np.zeros_like(X)
    for c in range(n):
        out[perm[c]] = X[c]
    return out


def fit_temperatures() -> List[float]:
    """The 10 fitting temperatures, accumulated as in Fitting (:538-560)."""
    dT = (FIT_TMAX - FIT_TMIN) / float(FIT_POINTS - 1)
    out, T = [], FIT_TMIN
    for _ in range(FIT_POINTS):
        out.append(T)
        T += dT
    return out


def _lsq(X: np.ndarray, Y: np.ndarray) -> np.ndarray:
    return _solve_full_pivot(X.T @ X, X.T @ Y)


def fit(st: SpeciesTransport) -> Dict[str, np.ndarray]:
    """Fitted coefficient arrays of the packed mechanism (Fitting, :536-689)."""
    Ts = fit_temperatures()
    nc = st.nc
    Xl = np.array([[1., math.log(T), math.log(T) ** 2, math.log(T) ** 3] for T in Ts])
    eta = np.array([np.log(st.viscosity(T)) for T in Ts])
    lam = np.array([np.log(st.conductivity(T)) for T in Ts])
    D = [st.binary_diffusivity(T, 1.) for T in Ts]
    pairs = [(j, k) for j in range(nc) for k in range(j + 1, nc)]
    gam = np.array([[math.log(Dt[j, k]) for (j, k) in pairs] for Dt in D]).reshape(len(Ts), len(pairs))
    out = {
        "tr_eta": _lsq(Xl, eta).T.copy(),
        "tr_lambda": _lsq(Xl, lam).T.copy(),
        "tr_gamma": (_lsq(Xl, gam).T.copy() if pairs else np.zeros((0, 4))),
    }
    nT = len(st.light)
    if nT:
        Xt = np.array([[1., T, T * T, T * T * T] for T in Ts])
        th = np.array([st.thermal_diffusion_ratios(T).ravel() for T in Ts])
        out["tr_teta"] = _lsq(Xt, th).T.reshape(nT, nc, 4).copy()
    else:
        out["tr_teta"] = np.zeros((0, nc, 4))
    out["tr_iteta"] = np.array(st.light, np.int32)
    return {k: (v if v.dtype == np.int32 else np.ascontiguousarray(v, np.float64).ravel()) for k, v in out.items()}


def transport_tables(species: Sequence[str], arrays: Dict[str, np.ndarray], text: str) -> Dict[str, np.ndarray]:
    """The ``tr_*`` arrays for a compiled mechanism's tables and a transport file's text."""
    st = SpeciesTransport(species, arrays["mw"], arrays["cp_ht"], arrays["cp_lt"], arrays["t_mid"],
                          read_transport(text))
    return fit(st)
