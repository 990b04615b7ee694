"""Seeded synthetic cell states for the reaction-step workloads.

Every generator returns cell-major mass fractions ``Y[ncells, NC]`` (rows sum
to one) and temperatures ``T[ncells]``; the seed is part of the workload name.

* ``h2co_mixing``   -- T ~ U[900, 2200] K, mixture fraction Z ~ U[0, 1] between
  fuel (0.5 H2 / 0.5 CO by mole) and air (0.21 O2 / 0.79 N2 by mole), mixed in
  mass; radicals H, O, OH, HO2, H2O2, HCO log-uniform in [1e-10, 1e-3], then
  renormalised (4 096 cells in the CPU-runnable case).
* ``h2co_uneven``   -- 30 % cold frozen mixing states T ~ U[300, 600] K, 20 %
  near-ignition T ~ U[950, 1150] K with radicals at 1e-8, 50 % hot
  near-equilibrium states: a pool of 4 096 hot mixtures (T ~ U[1800, 2300] K)
  integrated for 10 ms by a caller-supplied integrator (``pool_from_file`` reads
  the pool the CPU oracle integrated once), then sampled with a relative
  perturbation of at most 1e-3.
* ``synthetic_mixing`` -- for the synthetic mechanisms: CH4/air mixing states
  with every other species log-uniform in [1e-10, 1e-3], T ~ U[lo, hi].
* ``coflow_fields`` -- 2D axisymmetric 200 x 400 mesh: Gaussian temperature ridge
  300-2100 K along the stoichiometric surface and Z from a Burke-Schumann
  profile; the fuel is CH4 or a mix of H2 and CO.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

RADICALS_H2CO = ("H", "O", "OH", "HO2", "H2O2", "HCO")


def _mass_from_mole(x: np.ndarray, mw: np.ndarray) -> np.ndarray:
    y = x * mw
    return y / y.sum(axis=-1, keepdims=True)


def fuel_air_mass(species: Sequence[str], mw: np.ndarray, fuel: dict, air: dict):
    nc = len(species)
    xf = np.zeros(nc)
    xa = np.zeros(nc)
    for k, v in fuel.items():
        xf[species.index(k)] = v
    for k, v in air.items():
        xa[species.index(k)] = v
    return _mass_from_mole(xf, mw), _mass_from_mole(xa, mw)


def h2co_mixing(species: List[str], mw: np.ndarray, ncells: int, seed: int = 1,
                t_range: Tuple[float, float] = (900.0, 2200.0)):
    rng = np.random.default_rng(seed)
    yf, ya = fuel_air_mass(species, mw, {"H2": 0.5, "CO": 0.5}, {"O2": 0.21, "N2": 0.79})
    Z = rng.uniform(0.0, 1.0, ncells)
    Y = Z[:, None] * yf[None, :] + (1.0 - Z)[:, None] * ya[None, :]
    for r in RADICALS_H2CO:
        Y[:, species.index(r)] = 10.0 ** rng.uniform(-10.0, -3.0, ncells)
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(*t_range, ncells)
    return Y, T


Integrator = Callable[[np.ndarray, np.ndarray, float], Tuple[np.ndarray, np.ndarray]]


def pool_digest(Y: np.ndarray, T: np.ndarray) -> str:
    """SHA-256 of a pool's initial states (float64, C order)."""
    import hashlib
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(Y, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(T, dtype=np.float64).tobytes())
    return h.hexdigest()


def pool_from_file(path: str) -> Integrator:
    """An integrate_pool callable for h2co_uneven that returns the integrated pool stored in `path`
    (written once by the CPU oracle), after checking that the pool's initial states are the ones the
    file was made from."""
    d = np.load(path)
    want = bytes(d["sha256_initial"]).decode()

    def integrate(Yp, Tp, dt):
        if pool_digest(Yp, Tp) != want or float(d["dt"]) != dt:
            raise ValueError(f"{path} was made from other initial pool states")
        return d["Y"].copy(), d["T"].copy()
    return integrate


def h2co_uneven(species: List[str], mw: np.ndarray, ncells: int, integrate_pool: Integrator,
                seed: int = 2, pool_size: int = 4096, pool_seed: int = 2):
    """Config with per-cell BDF step counts spread over two orders of magnitude."""
    rng = np.random.default_rng(seed)
    n_cold = int(round(0.3 * ncells))
    n_ign = int(round(0.2 * ncells))
    n_hot = ncells - n_cold - n_ign
    yf, ya = fuel_air_mass(species, mw, {"H2": 0.5, "CO": 0.5}, {"O2": 0.21, "N2": 0.79})
    rad = [species.index(r) for r in RADICALS_H2CO]

    def mix(n):
        Z = rng.uniform(0.0, 1.0, n)
        return Z[:, None] * yf[None, :] + (1.0 - Z)[:, None] * ya[None, :]

    # cold frozen mixing states
    Yc = mix(n_cold)
    Yc[:, rad] = 10.0 ** rng.uniform(-10.0, -6.0, (n_cold, len(rad)))
    Tc = rng.uniform(300.0, 600.0, n_cold)
    # near-ignition states, radicals at 1e-8
    Yi = mix(n_ign)
    Yi[:, rad] = 1e-8
    Ti = rng.uniform(950.0, 1150.0, n_ign)
    # hot near-equilibrium states from an integrated pool; the pool has its own random stream (pool_seed),
    # so it is the same whatever the number of cells and the seed of the rest
    prng = np.random.default_rng([pool_seed, 1])
    Zp = prng.uniform(0.0, 1.0, pool_size)
    Yp = Zp[:, None] * yf[None, :] + (1.0 - Zp)[:, None] * ya[None, :]
    Yp[:, rad] = 10.0 ** prng.uniform(-6.0, -3.0, (pool_size, len(rad)))
    Yp /= Yp.sum(axis=1, keepdims=True)
    Tp = prng.uniform(1800.0, 2300.0, pool_size)
    Yp, Tp = integrate_pool(Yp, Tp, 1.0e-2)
    pick = rng.integers(0, pool_size, n_hot)
    Yh = Yp[pick] * (1.0 + rng.uniform(-1e-3, 1e-3, (n_hot, len(species))))
    Th = Tp[pick] * (1.0 + rng.uniform(-1e-3, 1e-3, n_hot))
    Y = np.concatenate([Yc, Yi, Yh])
    T = np.concatenate([Tc, Ti, Th])
    Y = np.maximum(Y, 0.0)
    Y /= Y.sum(axis=1, keepdims=True)
    perm = rng.permutation(ncells)
    return Y[perm], T[perm]


def synthetic_mixing(species: List[str], mw: np.ndarray, ncells: int, seed: int,
                     t_range: Tuple[float, float]):
    rng = np.random.default_rng(seed)
    yf, ya = fuel_air_mass(species, mw, {"CH4": 1.0}, {"O2": 0.21, "N2": 0.79})
    Z = rng.uniform(0.0, 0.3, ncells)
    Y = Z[:, None] * yf[None, :] + (1.0 - Z)[:, None] * ya[None, :]
    others = [i for i, s in enumerate(species) if s not in ("CH4", "O2", "N2")]
    Y[:, others] = 10.0 ** rng.uniform(-10.0, -3.0, (ncells, len(others)))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(*t_range, ncells)
    return Y, T


def stoichiometric_z(species: Sequence[str], mw: np.ndarray, fuel: dict) -> float:
    """Stoichiometric mixture fraction of `fuel` (mole fractions of H2, CO, CH4)
    against air (0.21 O2 / 0.79 N2 by mole)."""
    o2_per_mol = {"H2": 0.5, "CO": 0.5, "CH4": 2.0}
    o2 = sum(v * o2_per_mol[k] for k, v in fuel.items())
    m_fuel = sum(v * mw[species.index(k)] for k, v in fuel.items())
    m_air = o2 / 0.21 * (0.21 * mw[species.index("O2")] + 0.79 * mw[species.index("N2")])
    return m_fuel / (m_fuel + m_air)


def coflow_fields(species: List[str], mw: np.ndarray, nr: int = 200, nz: int = 400, seed: int = 5,
                  fuel: Optional[dict] = None):
    """Burke-Schumann coflow: fuel jet radius a, coflow radius b; T ridge at Z_st.
    `fuel` defaults to CH4; any mole-fraction mix of H2, CO and CH4 works (the
    ridge follows its stoichiometric mixture fraction)."""
    rng = np.random.default_rng(seed)
    fuel = fuel or {"CH4": 1.0}
    yf, ya = fuel_air_mass(species, mw, fuel, {"O2": 0.21, "N2": 0.79})
    r = (np.arange(nr) + 0.5) / nr          # radius / coflow radius
    z = (np.arange(nz) + 0.5) / nz * 20.0   # axial distance / jet radius
    a = 0.25
    R, Zax = np.meshgrid(r, z, indexing="ij")
    # leading-order Burke-Schumann mixture fraction: diffusion-broadened top hat
    w = 0.02 + 0.05 * np.sqrt(Zax)
    Zmix = 0.5 * (1.0 - np.tanh((R - a) / w))
    z_st = stoichiometric_z(species, mw, fuel)
    T = 300.0 + 1800.0 * np.exp(-((Zmix - z_st) / 0.05) ** 2) * (1.0 - np.exp(-Zax / 0.5))
    Zf = Zmix.ravel()
    Y = Zf[:, None] * yf[None, :] + (1.0 - Zf)[:, None] * ya[None, :]
    others = [i for i, s in enumerate(species) if s not in tuple(fuel) + ("O2", "N2")]
    Y[:, others] = 10.0 ** rng.uniform(-10.0, -4.0, (Zf.size, len(others)))
    Y /= Y.sum(axis=1, keepdims=True)
    return Y, T.ravel()
