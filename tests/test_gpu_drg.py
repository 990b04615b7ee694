"""The DRG-reduced reaction step on the GPU (lsg_reaction_step_drg_device) against the oracle.

The oracle restates solvers/laminarSMOKE/unsteady/chemistry_DRG.H with DRG.hpp (tests/test_drg.py pins it):
per cell above min_T, the analysis at the cell's state, the reduced system integrated by a fresh solver,
the solver options reaching cell 0 only (the reference's behaviour) or every cell, the epsilon of the
previous analysed cell kept for a cell above every temperature band.  The GPU form is the plain warp
kernel (FP64, the reference's operation order) on the reduced system up to 31 species, one block per
cell above.  Criteria: identical statuses,
important-species and kept-reaction counts; T within 1e-6 relative and Y within 1e-9 absolute in every
cell integrated with the configured tolerances; the cells integrated with the solver's defaults
(relative 1e-5) within 1e-6 / 1e-7, most within 1e-9.
"""
import os

import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _run(ctx, Y, T, key, cuda, **kw):
    import torch
    n = T.size
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    Q = torch.zeros(n, dtype=torch.float64, device=cuda)
    st = torch.full((n,), 99, dtype=torch.int32, device=cuda)
    nsp = torch.full((n,), -1, dtype=torch.int32, device=cuda)
    nrx = torch.full((n,), -1, dtype=torch.int32, device=cuda)
    cnt = torch.zeros((n, 8), dtype=torch.int64, device=cuda)
    ctx.step_drg_device(Yd, Td, 1e-5, key, Q=Q, status=st, n_species=nsp, n_reactions=nrx, counters=cnt, **kw)
    torch.cuda.synchronize()
    ctx.check()
    return (Yd.cpu().numpy().T, Td.cpu().numpy(), Q.cpu().numpy(), st.cpu().numpy(), cnt.cpu().numpy(),
            nsp.cpu().numpy(), nrx.cpu().numpy())


def _compare(got, ref, strict_mask):
    Yg, Tg, Qg, sg, cg, ng, rg = got
    Yo, To, Qo, so, co, no, ro = ref
    np.testing.assert_array_equal(sg, so)
    np.testing.assert_array_equal(ng, no)
    np.testing.assert_array_equal(rg, ro)
    dT = np.abs(Tg - To) / To
    dY = np.abs(Yg - Yo).max(axis=1)
    assert dT.max() <= 1e-6, dT.max()
    assert dY[strict_mask].max() <= 1e-9, dY[strict_mask].max()
    loose = ~strict_mask
    if loose.any():
        assert dY[loose].max() <= 1e-7 and np.mean(dY[loose] <= 1e-9) >= 0.9, (dY[loose].max(),
                                                                               np.mean(dY[loose] <= 1e-9))
    same = (cg == co).all(axis=1)
    print(f"DRG: max rel T {dT.max():.2e}, max abs Y {dY.max():.2e}, same counters {same.mean():.3f}, "
          f"species kept {ng.min()}-{ng.max()} of {Yg.shape[1]}")


@pytest.mark.parametrize("first_only", [True, False], ids=["cell0-options", "all-options"])
def test_drg_step_against_oracle(cuda, h2co, oracle_h2co, first_only):
    from laminarsmoke_b200 import lsg
    data, species, A = h2co
    n = 384
    Y, T = cells.h2co_mixing(species, A["mw"], n, seed=23)
    T[::7] = 280.0          # skipped cells (at or below min_T)
    T[3::11] = 2300.0       # above every band: the previous analysed cell's epsilon
    key = [species.index(s) for s in ("H2", "O2", "CO")]
    bands = ((1200.0, 1e-3), (1800.0, 3e-2))
    kw = dict(bands=bands, epsilon0=1e-2, min_T=300.0, first_cell_options_only=first_only)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    got = _run(ctx, Y, T, key, cuda, **kw)
    ref = oracle_h2co.reaction_step_drg(Y, T, 1e-5, key, **kw)
    strict = np.ones(n, dtype=bool)
    if first_only:
        strict[1:] = False
    _compare(got, ref, strict)
    assert (got[5][T <= 300.0] == 0).all() and (got[3][T <= 300.0] == 0).all()
    np.testing.assert_array_equal(got[0][T <= 300.0], Y[T <= 300.0])


def test_drg_step_all_species_kept_equals_full_step(cuda, h2co):
    """epsilon 0 keeps every reacting species and reaction: the reduced system is the full one, so with the
    options on every cell the step equals the plain form's (the inert species, never reached, keep their
    values, which the full system also does)."""
    import torch
    from laminarsmoke_b200 import lsg
    data, species, A = h2co
    n = 128
    Y, T = cells.h2co_mixing(species, A["mw"], n, seed=24)
    Y /= Y.sum(axis=1, keepdims=True)
    ctx = lsg.ReactionStep(lsg.Mechanism(data), tile=lsg.LSG_TILE_WARP)
    everyone = list(range(len(species)))
    got = _run(ctx, Y, T, everyone, cuda, bands=((1e6, 0.0),), epsilon0=0.0, min_T=0.0,
               first_cell_options_only=False)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    st = torch.zeros(n, dtype=torch.int32, device=cuda)
    ctx.step_device(Yd, Td, 1e-5, status=st)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got[3], st.cpu().numpy())
    np.testing.assert_allclose(got[1], Td.cpu().numpy(), rtol=1e-12)
    np.testing.assert_allclose(got[0], Yd.cpu().numpy().T, rtol=1e-10, atol=1e-16)


def test_drg_golden(cuda, h2co):
    """The oracle-made 48-cell DRG fixture (tests/golden/h2co_drg_step.npz)."""
    from laminarsmoke_b200 import lsg
    data, species, A = h2co
    g = np.load(os.path.join(HERE, "golden", "h2co_drg_step.npz"))
    bands = tuple(tuple(b) for b in g["bands"])
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    got = _run(ctx, g["Y0"], g["T0"], list(g["key"]), cuda, bands=bands, min_T=300.0)
    ref = (g["Y"], g["T"], g["Q"], g["status"], g["counters"], g["n_species"], g["n_reactions"])
    strict = np.zeros(g["T"].size, dtype=bool)
    strict[0] = True
    _compare(got, ref, strict)


def test_drg_rejects_bad_arguments(cuda, h2co):
    import torch
    from laminarsmoke_b200 import lsg
    data, species, A = h2co
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    Y = torch.full((len(species), 4), 1.0 / len(species), dtype=torch.float64, device=cuda)
    T = torch.full((4,), 1500.0, dtype=torch.float64, device=cuda)
    for key in ([], [len(species)], [-1]):
        with pytest.raises(lsg.LsgError):
            ctx.step_drg_device(Y, T, 1e-5, key)
    with pytest.raises(lsg.LsgError):
        ctx.step_drg_device(Y, T, 1e-5, [0], bands=tuple((1e3 + k, 1e-2) for k in range(17)))


@pytest.mark.parametrize("pad,first_only", [(106, False), (150, False), (106, True)],
                         ids=["n121-bt128", "n165-bt256", "n121-cell0-options"])
def test_drg_block_form_against_oracle(cuda, pad, first_only):
    """Above 31 species the DRG step runs one block per cell (drg_block_kernel): H2/CO chemistry padded with
    inert species, which the search never reaches, against the oracle on the same mechanism.  The block form
    sums over threads in tree order, so a few cells may take another step sequence: statuses and counts
    identical, T within 1e-6, Y within 1e-9 in 90 % of the cells and 1e-7 in all."""
    from laminarsmoke_b200 import lsg, mech
    from laminarsmoke_b200.mech import blob
    from oracle.oracle import OracleMechanism
    data, species = mech.load(f"h2co+{pad}")
    A, _ = blob.unpack(data)
    n = 96
    Y, T = cells.h2co_mixing(species[:14], A["mw"][:14], n, seed=25)
    Yp = np.zeros((n, len(species)))
    Yp[:, :14] = 0.5 * Y
    Yp[:, 14:] = 0.5 / (len(species) - 14)
    T[::9] = 280.0
    key = [species.index(s) for s in ("H2", "O2", "CO")]
    kw = dict(bands=((1200.0, 1e-3), (1e6, 1e-2)), epsilon0=1e-2, min_T=300.0, first_cell_options_only=first_only)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    Yg, Tg, Qg, sg, cg, ng, rg = _run(ctx, Yp, T, key, cuda, **kw)
    Yo, To, Qo, so, co, no, ro = OracleMechanism(data).reaction_step_drg(Yp, T, 1e-5, key, **kw)
    np.testing.assert_array_equal(sg, so)
    np.testing.assert_array_equal(ng, no)
    np.testing.assert_array_equal(rg, ro)
    assert ng.max() <= 14
    dT = np.abs(Tg - To) / To
    dY = np.abs(Yg - Yo).max(axis=1)
    print(f"DRG block form, {len(species)} species: max rel T {dT.max():.2e}, max abs Y {dY.max():.2e}, "
          f"within 1e-9 {np.mean(dY <= 1e-9):.3f}")
    assert dT.max() <= 1e-6
    assert np.mean(dY <= 1e-9) >= 0.9 and dY.max() <= 1e-7


def test_drg_host_entry_equals_device_entry(cuda, h2co):
    """lsg_reaction_step_drg (host fields, staged through the context) gives the device entry's results bit for
    bit, and leaves Q of the skipped cells as the caller had it."""
    from laminarsmoke_b200 import lsg
    data, species, A = h2co
    n = 200
    Y, T = cells.h2co_mixing(species, A["mw"], n, seed=26)
    T[::10] = 280.0
    key = [species.index(s) for s in ("H2", "O2", "CO")]
    kw = dict(bands=((1200.0, 1e-3), (1e6, 1e-2)), epsilon0=1e-2, min_T=300.0, first_cell_options_only=True)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    Yd, Td, Qd, sd, _, nd, rd = _run(ctx, Y, T, key, cuda, **kw)
    Yh = np.ascontiguousarray(Y.T).copy()
    Th = T.copy()
    Qh, sh, nh, rh = ctx.step_drg(Yh, Th, 1e-5, key, **kw)
    np.testing.assert_array_equal(sh, sd)
    np.testing.assert_array_equal(nh, nd)
    np.testing.assert_array_equal(rh, rd)
    np.testing.assert_array_equal(Th, Td)
    np.testing.assert_array_equal(Yh.T, Yd)
    np.testing.assert_array_equal(Qh, Qd)
    assert (Qh[T <= 300.0] == 0.0).all()
