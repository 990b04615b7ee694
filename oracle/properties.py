"""CPU restatement of the per-cell property update -- test infrastructure only.

Only tests/ and __graft_entry__.smoke() use this module, as the checker; the
product path never imports it.

It follows the reference's property loop over the cells
(solvers/laminarSMOKE/properties.H:40-190) and the maps it calls:

* mole fractions and mixture molecular weight:
  ThermodynamicsMap_CHEMKIN::MoleFractions_From_MassFractions (maps/
  ThermodynamicsMap_CHEMKIN.hpp:429-434);
* cTot = p / (R T), psi = cTot MWmix / p, h = sum x_i h_i / MWmix
  (properties.H:93-96; hMolar_Mixture_From_MoleFractions :514-520);
* cp, cv = (cp_molar - R) / MWmix and species cp_i / MW_i
  (properties.H:103-122; cpMolar_Mixture_From_MoleFractions :506-512,
  cpMolar_Species :560-564), only when the energy equation is solved or the
  Lewis-number diffusivities need them;
* mu by Wilke's rule with the fitted species viscosities
  (TransportPropertiesMap_CHEMKIN.hpp:729-766, 959-1001), lambda by the
  Mathur-Saxena combination (:690-727, 947-957);
* the simplified transport option mu = mu0 (T/T0)^beta0, lambda = mu cp / Pr0
  (properties.H:124-133);
* mixture-averaged diffusion coefficients from the binary fits at the cell's
  pressure, with mole fractions shifted by 1e-14 (gamma :798-859,
  gammaMix :1032-1059), or lambda / (rho cp Le_i) with Lewis numbers
  (properties.H:140-162);
* thermal diffusion: theta_i = sum_j theta_ij x_i x_j for the light species
  (teta :768-796, tetaMix :1103-1117) and Dsoret = Dmix_i theta_i MW_i / MWmix
  (properties.H:177-189).
"""
from __future__ import annotations

import numpy as np

from laminarsmoke_b200.mech import blob

R_J_KMOL = 8314.4621
THRESHOLD = 1.e-14
MU0, T0, BETA0, PR0 = 1.8405e-5, 300., 0.6759, 0.7


class OracleProperties:
    def __init__(self, data: bytes):
        A, species = blob.unpack(data)
        if "tr_eta" not in A:
            raise ValueError("the mechanism has no transport data")
        nc = int(A["dims"][0])
        self.nc = nc
        self.species = species
        self.mw = np.asarray(A["mw"], float)
        self.cp_ht = np.asarray(A["cp_ht"], float).reshape(nc, 5)
        self.cp_lt = np.asarray(A["cp_lt"], float).reshape(nc, 5)
        self.dh_ht = np.asarray(A["dh_ht"], float).reshape(nc, 6)
        self.dh_lt = np.asarray(A["dh_lt"], float).reshape(nc, 6)
        self.t_mid = np.asarray(A["t_mid"], float)
        self.eta = np.asarray(A["tr_eta"], float).reshape(nc, 4)
        self.lam = np.asarray(A["tr_lambda"], float).reshape(nc, 4)
        self.gam = np.asarray(A["tr_gamma"], float).reshape(-1, 4)
        self.iteta = np.asarray(A["tr_iteta"], int)
        self.teta = np.asarray(A["tr_teta"], float).reshape(len(self.iteta), nc, 4)

    def evaluate(self, Y, T, p, energy=True, lewis=None, simplified=False, soret=False):
        """Y [ncells, nc], T and p [ncells].  Returns a dict of fields;
        lewis (nc Lewis numbers) selects the Lewis-number diffusivities."""
        Y = np.asarray(Y, float)
        T = np.asarray(T, float)
        p = np.asarray(p, float) * np.ones_like(T)
        nc = self.nc
        n = T.size
        u = np.zeros(n)
        for i in range(nc):
            u = u + Y[:, i] / self.mw[i]
        MW = 1. / u
        X = MW[:, None] * Y / self.mw[None, :]
        out = {"X": X, "MWmix": MW}
        cTot = p / R_J_KMOL / T
        psi = cTot * MW / p
        out["cTot"], out["psi"] = cTot, psi
        hi = T[:, None] > self.t_mid[None, :]
        T2, T3, T4 = T * T, T * T * T, T * T * T * T
        dh = np.where(hi[:, :, None], self.dh_ht[None], self.dh_lt[None])
        h_rt = (dh[:, :, 0] + T[:, None] * dh[:, :, 1] + T2[:, None] * dh[:, :, 2] + T3[:, None] * dh[:, :, 3]
                + T4[:, None] * dh[:, :, 4] + (1. / T)[:, None] * dh[:, :, 5])
        h = np.zeros(n)
        for i in range(nc):
            h = h + h_rt[:, i] * X[:, i]
        out["h"] = h * (R_J_KMOL * T) / MW
        lnT = np.log(T)
        pw = np.stack([np.ones(n), lnT, lnT * lnT, lnT * lnT * lnT], axis=1)
        eta = np.exp(pw @ self.eta.T)
        # Wilke (etaMix)
        sumK = X.copy()
        sq = np.sqrt(eta)
        usq = 1. / sq
        for k in range(nc):
            for j in range(k + 1, nc):
                phi_sup = 1. / np.sqrt(8. * (1. + self.mw[k] / self.mw[j]))
                phi_inf = 1. / np.sqrt(8. * (1. + self.mw[j] / self.mw[k]))
                r14 = np.sqrt(np.sqrt(self.mw[j] / self.mw[k]))
                d = sq[:, k] * usq[:, j] * r14
                sumK[:, k] += X[:, j] * phi_sup * (1. + d) * (1. + d)
                sumK[:, j] += X[:, k] * phi_inf * (1. + 1. / d) * (1. + 1. / d)
        mu = np.zeros(n)
        for k in range(nc):
            mu = mu + X[:, k] * eta[:, k] / sumK[:, k]
        out["mu"] = mu
        lewis_mode = lewis is not None
        if energy or lewis_mode:
            lam_s = np.exp(pw @ self.lam.T)
            s1 = np.zeros(n)
            s2 = np.zeros(n)
            for k in range(nc):
                s1 = s1 + X[:, k] * lam_s[:, k]
                s2 = s2 + X[:, k] / lam_s[:, k]
            out["lambda"] = 0.5 * (s1 + 1. / s2)
            cpc = np.where(hi[:, :, None], self.cp_ht[None], self.cp_lt[None])
            cp_r = cpc[:, :, 0] + T[:, None] * cpc[:, :, 1] + T2[:, None] * cpc[:, :, 2] + \
                T3[:, None] * cpc[:, :, 3] + T4[:, None] * cpc[:, :, 4]
            cpm = np.zeros(n)
            for k in range(nc):
                cpm = cpm + cp_r[:, k] * X[:, k]
            cpm = cpm * R_J_KMOL
            out["cv"] = (cpm - R_J_KMOL) / MW
            out["cp"] = cpm / MW
            out["cp_species"] = cp_r * R_J_KMOL / self.mw[None, :]
        if simplified:
            out["mu"] = MU0 * (T / T0) ** BETA0
            if "cp" in out:   # lambda and cp are fields only with the energy equation or Lewis numbers
                out["lambda"] = out["mu"] * out["cp"] / PR0
        if lewis_mode:
            coef = out["lambda"] / (p * psi) / out["cp"]
            out["Dmix"] = coef[:, None] / np.asarray(lewis, float)[None, :]
        else:
            p_bar = p / 1.e5
            xc = (X + THRESHOLD) / (1. + THRESHOLD * nc)
            MWc = np.zeros(n)
            for i in range(nc):
                MWc = MWc + xc[:, i] * self.mw[i]
            acc = np.zeros((n, nc))
            q = 0
            for k in range(nc):
                for j in range(k + 1, nc):
                    g = p_bar / np.exp(pw @ self.gam[q])
                    acc[:, j] += xc[:, k] * g
                    acc[:, k] += xc[:, j] * g
                    q += 1
            out["Dmix"] = (MWc[:, None] - xc * self.mw[None, :]) / (MWc[:, None] * acc)
        if soret:
            tp = np.stack([np.ones(n), T, T2, T3], axis=1)
            ds = np.zeros((n, len(self.iteta)))
            for a, i in enumerate(self.iteta):
                th = np.zeros(n)
                for j in range(nc):
                    th = th + (tp @ self.teta[a, j]) * X[:, i] * X[:, j]
                ds[:, a] = out["Dmix"][:, i] * th * self.mw[i] / MW
            out["Dsoret"] = ds
        return out
