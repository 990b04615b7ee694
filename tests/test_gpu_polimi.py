"""The reference's detailed mechanisms besides H2/CO: POLIMI_H2_1412 (10
components) and POLIMI_CH4_SKELETAL_1412 (25 components, which takes the
32-lane solver groups of the round scheme).  Reaction step of the plain and
mixed forms against the oracle on seeded fuel/air mixing states."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu

RTOL_T = 1e-6
ATOL_Y = 1e-9
FUELS = {"h2": {"H2": 1.0}, "ch4": {"CH4": 1.0}}


def _states(name, n, seed):
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load(name)
    A, _ = blob.unpack(data)
    rng = np.random.default_rng(seed)
    yf, ya = cells.fuel_air_mass(species, A["mw"], FUELS[name], {"O2": 0.21, "N2": 0.79})
    Z = rng.uniform(0.0, 0.3, n)
    Y = Z[:, None] * yf[None, :] + (1.0 - Z)[:, None] * ya[None, :]
    minor = [i for i, s in enumerate(species) if s not in tuple(FUELS[name]) + ("O2", "N2")]
    Y[:, minor] = 10.0 ** rng.uniform(-10.0, -4.0, (n, len(minor)))
    Y /= Y.sum(axis=1, keepdims=True)
    T = rng.uniform(900.0, 2200.0, n)
    return data, Y, T


@pytest.mark.parametrize("name", ["h2", "ch4"])
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_polimi_step(cuda, name, form):
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, Y, T = _states(name, 1024, 71)
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw)
    Ys = np.ascontiguousarray(Y.T)
    Tg = T.copy()
    _, st, _ = ctx.step(Ys, Tg, 1e-5)
    ctx.check()
    Yo, To, _, sto, _ = OracleMechanism(data).reaction_step(Y, T, 1e-5, nthreads=8)
    np.testing.assert_array_equal(st, sto)
    rel_T = np.abs(Tg - To) / To
    abs_Y = np.abs(Ys.T - Yo).max(axis=1)
    print(f"{name} {form}: max rel T err {rel_T.max():.3e}, max abs Y err {abs_Y.max():.3e}, "
          f"cells within Y bound {np.mean(abs_Y <= ATOL_Y):.4f}")
    assert rel_T.max() <= RTOL_T
    assert np.mean(abs_Y <= ATOL_Y) >= 0.99 and abs_Y.max() <= 1e-7
