"""Extended PLOG (PLOGMX / PLOGSP; KineticsMap_CHEMKIN.hpp:1662-1670) and extended fall-off (LOWMX / LOWSP
with TROEMX / SRISP; :1672-1681) on the GPU: the 12-species synthetic mechanism with its first exchange
reaction given a mixture and a bath-species PLOG table, and with a reversible extended fall-off reaction
added.  RHS of the warp and block bodies against the oracle at several pressures (1e-11), and the reaction
step of every form at rtol 1e-10."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells
from laminarsmoke_b200.mech import blob, chemkin, synthetic

pytestmark = pytest.mark.gpu


def _mechanism(kind):
    from tests.test_xfo import xfo_lines
    from tests.test_xplog import BATH, MIX
    s = synthetic.generate(12, 20, seed=4, physical=True)
    lines = s.kinetics.split("\n")
    if kind == "xplog":
        m0 = chemkin.compile_mechanism(s.kinetics, s.thermo)
        k = next(i for i, l in enumerate(lines) if "=" in l and "+M" not in l and not l.startswith(" "))
        reac = set(int(v) for v in m0.arrays["reac_species"][m0.arrays["reac_ptr"][0]:m0.arrays["reac_ptr"][1]])
        bath = next(n for i, n in enumerate(m0.species) if i not in reac)
        extra = [f" PLOGMX / {p} {a:.6E} {b} {e} /" for p, a, b, e in MIX]
        extra += [f" PLOGSP / {bath} {p} {a:.6E} {b} {e} /" for p, a, b, e in BATH]
        lines[k + 1:k + 1] = extra
    else:
        end = len(lines) - 1 - lines[::-1].index("END")
        lines[end:end] = xfo_lines(reversible=True)
    m = chemkin.compile_mechanism("\n".join(lines) + "\n", s.thermo)
    key = "xplog_rxn" if kind == "xplog" else "xfo_rxn"
    assert key in m.arrays
    return blob.pack(m.arrays, m.species), m


@pytest.mark.parametrize("kind", ["xplog", "xfo"])
@pytest.mark.parametrize("tile", [1, 4], ids=["warp", "block"])
@pytest.mark.parametrize("patm", [0.3, 2.0, 20.0])
def test_extended_rhs(cuda, kind, tile, patm):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = _mechanism(kind)
    Y, T = cells.synthetic_mixing(m.species, m.arrays["mw"], 128, seed=5, t_range=(700.0, 2400.0))
    y = np.ascontiguousarray(np.concatenate([Y.T, T[None, :]], axis=0))
    yd = torch.tensor(y, device=cuda)
    dyd = torch.zeros_like(yd)
    ctx = lsg.ReactionStep(lsg.Mechanism(data), tile=tile)
    P = patm * 101325.0
    ctx.rhs_device(yd, dyd, p=P)
    torch.cuda.synchronize()
    ctx.check()
    dy = dyd.cpu().numpy()
    orc = OracleMechanism(data)
    for k in range(128):
        ref, _ = orc.rhs(y[:, k], P)
        np.testing.assert_allclose(dy[:, k], ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("kind", ["xplog", "xfo"])
@pytest.mark.parametrize("form", ["plain", "rounds", "persistent", "block", "group"])
def test_extended_step(cuda, kind, form):
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, m = _mechanism(kind)
    n = 256
    P = 3.0 * 101325.0
    Y, T = cells.synthetic_mixing(m.species, m.arrays["mw"], n, seed=3, t_range=(900.0, 2200.0))
    kw = {"plain": dict(tile=1, precision=0), "rounds": dict(tile=2, precision=1, jacobian=1),
          "persistent": dict(tile=3, precision=1), "block": dict(tile=4, precision=0),
          "group": dict(tile=5, precision=1)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), rtol=1e-10, atol=1e-16, **kw)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    st = torch.zeros(n, dtype=torch.int32, device=cuda)
    ctx.step_device(Yd, Td, 1e-5, p=P, status=st)
    torch.cuda.synchronize()
    ctx.check()
    Yo, To, _, sto, _ = OracleMechanism(data).reaction_step(Y, T, 1e-5, p=P, rtol=1e-10, atol=1e-16, nthreads=8)
    np.testing.assert_array_equal(st.cpu().numpy(), sto)
    dT = np.abs(Td.cpu().numpy() - To) / To
    dY = np.abs(Yd.cpu().numpy().T - Yo).max(axis=1)
    print(f"{kind} {form}: max rel T {dT.max():.2e}, max abs Y {dY.max():.2e}, within 1e-9 {np.mean(dY <= 1e-9):.4f}")
    assert dT.max() <= 1e-6
    assert np.mean(dY <= 1e-9) >= 0.95 and dY.max() <= 1e-7
