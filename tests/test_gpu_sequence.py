"""Device-resident sequences of reaction steps on the coflow mesh.

A CFD run calls the chemistry once per time step with the state kept in
device memory and the start time advancing by dt.  These tests take a seeded
subset of the 200 x 400 Burke-Schumann coflow mesh (H2/CO fuel; half the cells
from the flame ridge, half from the rest), run several successive steps on one
set of device arrays, and compare with the oracle taking the same steps on the
host.  The 121-component case (the H2/CO chemistry padded with inert species)
runs the block-per-cell form.
"""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu

RTOL_T = 1e-6
ATOL_Y = 1e-9
FUEL = {"H2": 0.5, "CO": 0.5}
DT = 1e-5


def _coflow_subset(species, mw, ncells, seed=7):
    Y, T = cells.coflow_fields(species, mw, fuel=FUEL)
    rng = np.random.default_rng(seed)
    hot = np.flatnonzero(T > 900.0)
    cold = np.flatnonzero(T <= 900.0)
    idx = np.concatenate([rng.choice(hot, ncells // 2, replace=False),
                          rng.choice(cold, ncells - ncells // 2, replace=False)])
    return np.ascontiguousarray(Y[idx]), T[idx].copy()


def _sequence(data, Y, T, nsteps, **kw):
    """(GPU Y, T, failures), (oracle Y, T, failures) after `nsteps` steps."""
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device="cuda")
    Td = torch.tensor(T, device="cuda")
    fails = ctx.step_sequence_device(Yd, Td, DT, nsteps)
    ctx.check()
    orc = OracleMechanism(data)
    Yo, To = Y, T
    bad = np.zeros(T.size, dtype=bool)
    for k in range(nsteps):
        Yo, To, _, sto, _ = orc.reaction_step(Yo, To, DT, t0=k * DT, nthreads=8)
        bad |= sto < 0
    return (Yd.cpu().numpy().T, Td.cpu().numpy(), fails), (Yo, To, int(bad.sum()))


def _compare(g, o, frac_y):
    (Yg, Tg, fg), (Yo, To, fo) = g, o
    rel_T = np.abs(Tg - To) / To
    abs_Y = np.abs(Yg - Yo).max(axis=1)
    print(f"max rel T err {rel_T.max():.3e}, max abs Y err {abs_Y.max():.3e}, "
          f"cells within Y bound {np.mean(abs_Y <= ATOL_Y):.4f}, failures gpu {fg} oracle {fo}")
    assert fg == fo == 0
    assert rel_T.max() <= RTOL_T
    assert np.mean(abs_Y <= ATOL_Y) >= frac_y
    assert abs_Y.max() <= 1e-7


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_coflow_sequence_h2co(h2co, cuda, form):
    from laminarsmoke_b200 import lsg
    data, species, A = h2co
    Y, T = _coflow_subset(species, A["mw"], 2048)
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED)}[form]
    g, o = _sequence(data, Y, T, 5, **kw)
    _compare(g, o, 0.99)


def test_coflow_sequence_block_121(cuda):
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load("h2co+106")
    A, _ = blob.unpack(data)
    Y, T = _coflow_subset(species, A["mw"], 128)
    g, o = _sequence(data, Y, T, 3)
    _compare(g, o, 0.9)


@pytest.mark.parametrize("name,tile,precision", [("h2co", 1, 0), ("h2co", 3, 1), ("h2co+30", 4, 0),
                                                 ("h2co+30", 4, 1), ("h2co", 2, 1), ("h2co", 5, 1)],
                         ids=["plain", "persistent", "block-fp64", "block-tc", "rounds", "group"])
def test_sequence_graph_equals_step_by_step(cuda, name, tile, precision):
    """lsg_reaction_step_sequence_device captures the steps into a CUDA graph (the round scheme, whose
    rounds wait on the host, runs them one by one): its result must be the one of the same steps
    made one call at a time, bit for bit, on the first call and on the replay."""
    import torch
    from laminarsmoke_b200 import lsg, mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load(name)
    A, _ = blob.unpack(data)
    Y, T = _coflow_subset(species[:14], A["mw"][:14], 256)
    if len(species) > 14:
        Yp = np.zeros((len(T), len(species)))
        Yp[:, :14] = 0.5 * Y
        Yp[:, 14:] = 0.5 / (len(species) - 14)
        Y = Yp
    m = lsg.Mechanism(data)
    nsteps = 4
    ref = lsg.ReactionStep(m, tile=tile, precision=precision)
    Yr = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Tr = torch.tensor(T, device=cuda)
    for k in range(nsteps):
        ref.step_device(Yr, Tr, DT, t0=k * DT)
    torch.cuda.synchronize()
    ref.check()
    ctx = lsg.ReactionStep(m, tile=tile, precision=precision)
    Yg = torch.empty_like(Yr)
    Tg = torch.empty_like(Tr)
    for call in range(2):
        Yg.copy_(torch.tensor(np.ascontiguousarray(Y.T), device=cuda))
        Tg.copy_(torch.tensor(T, device=cuda))
        used = ctx.step_sequence_graph(Yg, Tg, DT, nsteps)
        torch.cuda.synchronize()
        ctx.check()
        assert used == (tile != 2)
        assert torch.equal(Yg, Yr) and torch.equal(Tg, Tr), f"call {call}"
