"""Property update after the step (properties.H:40-190): transport fits, the oracle, the CUDA kernel.

CPU tests pin the transport preprocessing (kinetic theory against measured
gas properties, fit quality, table interpolation) and the oracle's mixture
rules (limits they must reach); GPU tests compare the kernel with the oracle
on the same cells through the C ABI.
"""
import math

import numpy as np
import pytest

# records of the standard CHEMKIN transport database (shape, eps/k, sigma, dipole, polarizability, Zrot)
TRC = """
N2   1   97.530   3.621   0.000   1.760   4.000
O2   1  107.400   3.458   0.000   1.600   3.800
H2   1   38.000   2.920   0.000   0.790 280.000
H2O  2  572.400   2.605   1.844   0.000   4.000   ! polar
AR   0  136.500   3.330   0.000   0.000   0.000
"""
RTOL_GPU = 1e-11


def _n2_o2_h2_h2o_ar():
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob, transport as tr
    A, species = blob.unpack(mech.load("h2co")[0])
    idx = [species.index(s) for s in ("N2", "O2", "H2", "H2O", "AR")]
    nc = len(species)
    cp_ht = np.asarray(A["cp_ht"]).reshape(nc, 5)[idx]
    cp_lt = np.asarray(A["cp_lt"]).reshape(nc, 5)[idx]
    st = tr.SpeciesTransport(["N2", "O2", "H2", "H2O", "AR"], np.asarray(A["mw"])[idx], cp_ht, cp_lt,
                             np.asarray(A["t_mid"])[idx], tr.read_transport(TRC))
    return st


def test_collision_integrals_at_table_nodes():
    from laminarsmoke_b200.mech import transport as tr
    tab = tr._tables()
    for i in (2, 9, 20, 30):
        for j in (0, 3, 6):
            d = tab["delta_star"][j] if j else 0.
            assert abs(tr.omega22(tab["t_star"][i], d) - tab["omega22"][i, j]) < 1e-12
            assert abs(tr.omega11(tab["t_star"][i], d) - tab["omega11"][i, j]) < 1e-12
    assert abs(tr.omega22(1.0, 0.) - 1.593) < 1e-12   # Lennard-Jones Omega(2,2)* at T* = 1


def test_kinetic_theory_against_measured_gas_properties():
    st = _n2_o2_h2_h2o_ar()
    eta = st.viscosity(300.)
    lam = st.conductivity(300.)
    D = st.binary_diffusivity(300., 1.01325)
    # measured at 300 K, 1 atm: mu [Pa s], lambda [W/m/K], D [m2/s]
    assert eta[0] == pytest.approx(1.78e-5, rel=0.03)     # N2
    assert eta[1] == pytest.approx(2.07e-5, rel=0.03)     # O2
    assert eta[2] == pytest.approx(8.9e-6, rel=0.03)      # H2
    assert eta[4] == pytest.approx(2.27e-5, rel=0.03)     # Ar
    assert lam[0] == pytest.approx(0.0259, rel=0.05)
    assert lam[2] == pytest.approx(0.182, rel=0.05)
    assert lam[4] == pytest.approx(0.0177, rel=0.05)
    assert D[1, 0] == pytest.approx(2.0e-5, rel=0.08)     # O2-N2
    assert D[2, 0] == pytest.approx(7.8e-5, rel=0.08)     # H2-N2
    assert np.allclose(D, D.T)


def test_polar_pair_correction_is_symmetric():
    st = _n2_o2_h2_h2o_ar()
    for j in range(5):
        for k in range(5):
            assert st.pair_potential(j, k) == pytest.approx(st.pair_potential(k, j), rel=1e-15)
    e_plain = math.sqrt(st.eps_kb[0] * st.eps_kb[3])
    assert st.pair_potential(0, 3)[0] > e_plain          # N2-H2O: the polar correction raises epsilon
    assert st.pair_potential(0, 1)[0] == pytest.approx(math.sqrt(st.eps_kb[0] * st.eps_kb[1]))


def test_fits_reproduce_kinetic_theory():
    from laminarsmoke_b200.mech import transport as tr
    st = _n2_o2_h2_h2o_ar()
    f = tr.fit(st)
    eta_c = f["tr_eta"].reshape(5, 4)
    lam_c = f["tr_lambda"].reshape(5, 4)
    gam_c = f["tr_gamma"].reshape(-1, 4)
    pairs = [(j, k) for j in range(5) for k in range(j + 1, 5)]
    for T in tr.fit_temperatures():
        pw = np.array([1., math.log(T), math.log(T) ** 2, math.log(T) ** 3])
        np.testing.assert_allclose(np.exp(eta_c @ pw), st.viscosity(T), rtol=0.01)
        np.testing.assert_allclose(np.exp(lam_c @ pw), st.conductivity(T), rtol=0.02)
        D = st.binary_diffusivity(T)
        np.testing.assert_allclose(np.exp(gam_c @ pw), [D[j, k] for j, k in pairs], rtol=0.01)
    assert list(f["tr_iteta"]) == [2, 3]                  # H2 and H2O are the species up to 20 kg/kmol


def test_thermal_diffusion_ratio_signs():
    st = _n2_o2_h2_h2o_ar()
    th = st.thermal_diffusion_ratios(1000.)
    assert th.shape == (2, 5)
    assert th[0, 2] == 0.                                 # H2 with itself
    assert th[0, 0] < 0. and th[0, 4] < 0.                # the light species goes to the hot side


def test_compiled_mechanisms_carry_transport():
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    for name in ("h2co", "h2", "ch4", "ch4_1step", "h2_1step"):
        A, species = blob.unpack(mech.load(name)[0])
        nc = len(species)
        assert A["tr_eta"].size == 4 * nc and A["tr_gamma"].size == 2 * nc * (nc - 1)
        light = [i for i in range(nc) if A["mw"][i] <= 20.]
        assert list(A["tr_iteta"]) == light
    A, _ = blob.unpack(mech.load("h2co+8")[0])
    assert not [k for k in A if k.startswith("tr_")]


def _cells(data, species, n, seed):
    from laminarsmoke_b200 import cells
    from laminarsmoke_b200.mech import blob
    A, _ = blob.unpack(data)
    rng = np.random.default_rng(seed)
    try:
        Y, T = cells.h2co_mixing(species, A["mw"], n, seed=seed)
    except ValueError:   # a mechanism without the H2/CO species: uniform random states
        Y = None
    if Y is None:
        Y = rng.uniform(0., 1., (n, len(species)))
        Y /= Y.sum(axis=1, keepdims=True)
        T = rng.uniform(300., 2500., n)
    p = rng.uniform(0.5, 5.0, n) * 101325.
    return Y, T, p


def test_oracle_limits(h2co):
    from oracle.properties import OracleProperties
    data, species = h2co[0], h2co[1]
    o = OracleProperties(data)
    nc = o.nc
    Y, T, p = _cells(data, species, 64, 3)
    f = o.evaluate(Y, T, p, soret=True)
    np.testing.assert_allclose(f["X"].sum(axis=1), 1., rtol=1e-14)
    np.testing.assert_allclose(f["cTot"] * 8314.4621 * T, p, rtol=1e-14)
    np.testing.assert_allclose(f["psi"] * p, p * f["MWmix"] / (8314.4621 * T), rtol=1e-14)
    # cp = dh/dT at fixed composition
    fp = o.evaluate(Y, T + 1e-3, p)
    fm = o.evaluate(Y, T - 1e-3, p)
    np.testing.assert_allclose((fp["h"] - fm["h"]) / 2e-3, f["cp"], rtol=1e-6)
    assert np.all(f["cp"] > f["cv"]) and np.all(f["Dmix"] > 0.)
    # a pure gas: Wilke and Mathur-Saxena give the species values
    n2 = species.index("N2")
    Yp = np.zeros((1, nc))
    Yp[0, n2] = 1.
    g = o.evaluate(Yp, np.array([1200.]), np.array([101325.]))
    lt = math.log(1200.)
    pw = np.array([1., lt, lt * lt, lt ** 3])
    assert g["mu"][0] == pytest.approx(math.exp(o.eta[n2] @ pw), rel=1e-14)
    assert g["lambda"][0] == pytest.approx(math.exp(o.lam[n2] @ pw), rel=1e-14)
    # a trace of H2 in N2 diffuses with the binary coefficient, scaled by the pressure
    h2 = species.index("H2")
    Yt = np.zeros((1, nc))
    Yt[0, n2] = 1. - 1e-9
    Yt[0, h2] = 1e-9
    j, k = sorted((h2, n2))
    q = [(a, b) for a in range(nc) for b in range(a + 1, nc)].index((j, k))
    for patm in (1., 4.):
        d = o.evaluate(Yt, np.array([1200.]), np.array([patm * 101325.]))["Dmix"][0, h2]
        assert d == pytest.approx(math.exp(o.gam[q] @ pw) / (patm * 101325. / 1e5), rel=1e-6)
    # Lewis numbers: D = lambda / (rho cp Le)
    le = np.linspace(0.3, 1.5, nc)
    fl = o.evaluate(Y, T, p, lewis=le)
    rho = p * fl["psi"]
    np.testing.assert_allclose(fl["Dmix"], (fl["lambda"] / (rho * fl["cp"]))[:, None] / le[None, :], rtol=1e-14)
    fs = o.evaluate(Y, T, p, simplified=True)
    np.testing.assert_allclose(fs["mu"], 1.8405e-5 * (T / 300.) ** 0.6759, rtol=1e-14)
    np.testing.assert_allclose(fs["lambda"], fs["mu"] * fs["cp"] / 0.7, rtol=1e-14)


# ---- the CUDA kernel against the oracle ----

def _compare(got: dict, ref: dict, rtol=RTOL_GPU):
    for key, v in got.items():
        r = ref[key]
        g = v.cpu().numpy() if hasattr(v, "cpu") else v
        r = r.T if r.ndim == 2 else r
        np.testing.assert_allclose(g, r, rtol=rtol, atol=0., err_msg=key)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2co", "ch4", "h2_1step"])
def test_gpu_properties_match_oracle(cuda, name):
    import torch
    from laminarsmoke_b200 import lsg, mech
    from oracle.properties import OracleProperties
    data, species = mech.load(name)
    Y, T, p = _cells(data, species, 3000, 11)
    ref = OracleProperties(data).evaluate(Y, T, p, soret=True)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    got = ctx.properties_device(Yd, torch.tensor(T, device=cuda), torch.tensor(p, device=cuda), soret=True)
    torch.cuda.synchronize()
    assert set(got) == set(lsg.PROPERTY_FIELDS)
    _compare(got, ref)


@pytest.mark.gpu
def test_gpu_properties_options_and_host_entry(h2co, cuda):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.properties import OracleProperties
    data, species = h2co[0], h2co[1]
    nc = len(species)
    Y, T, p = _cells(data, species, 777, 12)
    o = OracleProperties(data)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    le = np.linspace(0.3, 1.5, nc)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    got = ctx.properties_device(Yd, Td, p_scalar=2.5e5, lewis=torch.tensor(le, device=cuda), soret=True)
    torch.cuda.synchronize()
    _compare(got, o.evaluate(Y, T, np.full_like(T, 2.5e5), lewis=le, soret=True))
    got = ctx.properties_device(Yd, Td, p_scalar=2.5e5, energy=False, simplified=True)
    torch.cuda.synchronize()
    assert "lambda" not in got and "cp" not in got
    _compare(got, o.evaluate(Y, T, np.full_like(T, 2.5e5), energy=False, simplified=True))
    host = ctx.properties(np.ascontiguousarray(Y.T), T, p=p, soret=True)
    _compare(host, o.evaluate(Y, T, p, soret=True))


@pytest.mark.gpu
def test_gpu_properties_without_transport_data(cuda):
    import torch
    from laminarsmoke_b200 import lsg, mech
    data, species = mech.load("h2co+8")
    m = lsg.Mechanism(data)
    assert m.transport_info() == (False, [])
    ctx = lsg.ReactionStep(m)
    Y = torch.full((len(species), 4), 1. / len(species), dtype=torch.float64, device=cuda)
    with pytest.raises(lsg.LsgError):
        ctx.properties_device(Y, torch.full((4,), 1000., dtype=torch.float64, device=cuda))


def test_transport_file_errors():
    from laminarsmoke_b200.mech import transport as tr
    with pytest.raises(tr.TransportError):
        tr.read_transport("N2 1 97.53 3.621 0.0 1.76\n")               # six fields
    with pytest.raises(tr.TransportError):
        tr.read_transport("N2 3 97.53 3.621 0.0 1.76 4.0\n")           # shape 3
    with pytest.raises(tr.TransportError):
        tr.read_transport("N2 1 97.53 abc 0.0 1.76 4.0\n")
    db = tr.read_transport("! comment\n\nn2 1 97.53 3.621 0.0 1.76 4.0 ! trailing\nN2 1 1 1 1 1 1\n"
                           "END\nO2 1 1 1 1 1 1\n")
    assert list(db) == ["N2"] and db["N2"].sigma == 3.621   # case-insensitive; first record kept; END stops
    st_args = _n2_o2_h2_h2o_ar()
    with pytest.raises(tr.TransportError):
        tr.SpeciesTransport(["N2", "XX"], st_args.mw[:2], st_args.cp_ht[:2], st_args.cp_lt[:2], st_args.t_mid[:2],
                            tr.read_transport(TRC))


def test_compile_with_transport_rejects_missing_species(tmp_path):
    import subprocess
    import sys
    from laminarsmoke_b200.mech import synthetic
    s = synthetic.generate(12, 10, seed=3)
    (tmp_path / "k.cki").write_text(s.kinetics)
    (tmp_path / "t.ckt").write_text(s.thermo)
    (tmp_path / "tr.trc").write_text(TRC)                                # lacks most of the species
    r = subprocess.run([sys.executable, "-m", "laminarsmoke_b200.mech", "compile", str(tmp_path / "k.cki"),
                        str(tmp_path / "t.ckt"), "--transport", str(tmp_path / "tr.trc"), "-o",
                        str(tmp_path / "m.lsmech")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "no transport data" in r.stderr


def test_synthetic_transport_120_species():
    """The 120-species synthetic mechanism with synthetic transport records: fits, oracle fields, and the
    library's host-side checks (on a machine without a GPU the load gets as far as the CUDA call)."""
    import ctypes as C
    from laminarsmoke_b200 import lsg, mech
    from oracle.properties import OracleProperties
    data, sp = mech.load("syn120t")
    o = OracleProperties(data)
    rng = np.random.default_rng(1)
    Y = rng.uniform(0, 1, (16, len(sp)))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(400, 2500, 16)
    f = o.evaluate(Y, T, np.full(16, 1e5), soret=True)
    assert all(np.isfinite(v).all() for v in f.values())
    assert np.all(f["mu"] > 0) and np.all(f["Dmix"] > 0) and f["Dsoret"].shape == (16, len(o.iteta))
    buf = (C.c_ubyte * len(data)).from_buffer_copy(data)
    h = C.c_void_p()
    rc = lsg.lib().lsg_mech_load_blob(C.cast(buf, C.c_void_p), len(data), 0, C.byref(h))
    assert rc in (0, -3)                                  # LSG_OK with a GPU, LSG_ERR_CUDA without one
    if rc == 0:
        lsg.lib().lsg_mech_destroy(h)
