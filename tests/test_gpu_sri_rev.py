"""SRI fall-off (KineticsMap_CHEMKIN.hpp:1538-1544) and explicit reverse rate constants (REV,
:1243-1255) on the GPU.  Neither occurs in the reference's H2/CO mechanism, so a 16-species
synthetic mechanism supplies them: 15 % SRI fall-off reactions (3- and 5-parameter forms), 10 %
Troe, 15 % third-body, 30 % of the exchange reactions with REV.  RHS of every form against the
oracle at 1e-11 through lsg_rhs_device (the warp and block bodies; the round-scheme and persistent
bodies are reached through the step), and the reaction step of every form at rtol 1e-10."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sri_rev():
    from laminarsmoke_b200.mech import blob, chemkin, synthetic
    s = synthetic.generate(16, 40, seed=12, physical=True, frac_sri=0.15, frac_rev=0.3)
    m = chemkin.compile_mechanism(s.kinetics, s.thermo)
    A = m.arrays
    assert 2 in set(A["fo_type"].tolist()) and len(A["rev_explicit"]) > 0
    return blob.pack(A, m.species), m


def test_mechanism_has_both_forms(sri_rev):
    _, m = sri_rev
    A = m.arrays
    assert int((A["fo_type"] == 2).sum()) >= 4
    assert len(A["rev_explicit"]) >= 5


@pytest.mark.parametrize("tile", [1, 4], ids=["warp", "block"])
def test_sri_rev_rhs(cuda, sri_rev, tile):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = sri_rev
    Y, T = cells.synthetic_mixing(m.species, m.arrays["mw"], 256, seed=5, t_range=(700.0, 2400.0))
    y = np.ascontiguousarray(np.concatenate([Y.T, T[None, :]], axis=0))
    yd = torch.tensor(y, device=cuda)
    dyd = torch.zeros_like(yd)
    ctx = lsg.ReactionStep(lsg.Mechanism(data), tile=tile)
    ctx.rhs_device(yd, dyd)
    torch.cuda.synchronize()
    ctx.check()
    dy = dyd.cpu().numpy()
    orc = OracleMechanism(data)
    for k in range(256):
        ref, _ = orc.rhs(y[:, k])
        np.testing.assert_allclose(dy[:, k], ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("form", ["plain", "rounds", "persistent", "block", "group"])
def test_sri_rev_step(cuda, sri_rev, form):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = sri_rev
    n = 256
    Y, T = cells.synthetic_mixing(m.species, m.arrays["mw"], n, seed=3, t_range=(900.0, 2200.0))
    kw = {"plain": dict(tile=1, precision=0), "rounds": dict(tile=2, precision=1),
          "persistent": dict(tile=3, precision=1), "block": dict(tile=4, precision=0),
          "group": dict(tile=5, precision=1)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), rtol=1e-10, atol=1e-16, **kw)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    st = torch.zeros(n, dtype=torch.int32, device=cuda)
    ctx.step_device(Yd, Td, 1e-5, status=st)
    torch.cuda.synchronize()
    ctx.check()
    Yo, To, _, sto, _ = OracleMechanism(data).reaction_step(Y, T, 1e-5, rtol=1e-10, atol=1e-16, nthreads=8)
    np.testing.assert_array_equal(st.cpu().numpy(), sto)
    dT = np.abs(Td.cpu().numpy() - To) / To
    dY = np.abs(Yd.cpu().numpy().T - Yo).max(axis=1)
    print(f"SRI/REV {form}: max rel T {dT.max():.2e}, max abs Y {dY.max():.2e}, "
          f"within 1e-9 {np.mean(dY <= 1e-9):.4f}")
    assert dT.max() <= 1e-6
    assert np.mean(dY <= 1e-9) >= 0.97 and dY.max() <= 1e-7
