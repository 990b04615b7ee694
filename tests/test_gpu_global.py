"""The reference's global one-step mechanisms (GLOBAL_CH4_1step, GLOBAL_H2_1step):
reactions whose forward rate law has orders given by FORD instead of the
stoichiometric coefficients.  RHS and reaction step of the plain and mixed
forms against the oracle."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu

RTOL_T = 1e-6
ATOL_Y = 1e-9
FUELS = {"ch4_1step": {"CH4": 1.0}, "h2_1step": {"H2": 1.0}}


def _states(name, n, seed):
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load(name)
    A, _ = blob.unpack(data)
    rng = np.random.default_rng(seed)
    yf, ya = cells.fuel_air_mass(species, A["mw"], FUELS[name], {"O2": 0.21, "N2": 0.79})
    Z = rng.uniform(0.0, 0.15, n)
    Y = Z[:, None] * yf[None, :] + (1.0 - Z)[:, None] * ya[None, :]
    burnt = [i for i, s in enumerate(species) if s in ("CO2", "H2O")]
    Y[:, burnt] = rng.uniform(0.0, 0.1, (n, len(burnt)))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(900.0, 2200.0, n)
    return data, Y, T


@pytest.mark.parametrize("name", ["ch4_1step", "h2_1step"])
def test_global_rhs(cuda, name):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, Y, T = _states(name, 256, 61)
    y = np.ascontiguousarray(np.concatenate([Y.T, T[None, :]], axis=0))
    yd = torch.tensor(y, device=cuda)
    dyd = torch.zeros_like(yd)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    ctx.rhs_device(yd, dyd)
    torch.cuda.synchronize()
    ctx.check()
    dy = dyd.cpu().numpy()
    orc = OracleMechanism(data)
    for k in range(256):
        ref, _ = orc.rhs(y[:, k])
        np.testing.assert_allclose(dy[:, k], ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("name", ["ch4_1step", "h2_1step"])
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_global_step(cuda, name, form):
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, Y, T = _states(name, 2048, 62)
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw)
    Ys = np.ascontiguousarray(Y.T)
    Tg = T.copy()
    _, st, _ = ctx.step(Ys, Tg, 1e-5)
    ctx.check()
    Yo, To, _, sto, _ = OracleMechanism(data).reaction_step(Y, T, 1e-5, nthreads=8)
    np.testing.assert_array_equal(st, sto)
    abs_Y = np.abs(Ys.T - Yo).max(axis=1)
    print(f"{name} {form}: max rel T err {(np.abs(Tg - To) / To).max():.3e}, max abs Y err {abs_Y.max():.3e}")
    assert (np.abs(Tg - To) / To).max() <= RTOL_T
    assert np.mean(abs_Y <= ATOL_Y) >= 0.99 and abs_Y.max() <= 1e-7
