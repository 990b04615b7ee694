"""Constant-volume reactor (chemistry_DI.H with constPressureBatchReactor
false; BatchReactorHomogeneousConstantVolume.H:148-199): every form against
the oracle, each cell at its own density."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu

RTOL_T = 1e-6
ATOL_Y = 1e-9


def _cv_states(name, n, seed):
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load(name)
    A, _ = blob.unpack(data)
    Y, T = cells.h2co_mixing(species[:14], A["mw"][:14], n, seed=seed)
    k = len(species) - 14
    if k:
        Y = np.concatenate([Y * 0.9, np.full((n, k), 0.1 / k)], axis=1)
    Y /= Y.sum(axis=1, keepdims=True)
    rng = np.random.default_rng(seed + 1)
    rho = rng.uniform(0.5, 2.0, n) * 101325.0 / ((Y / A["mw"]).sum(axis=1) * 8314.4621 * T)
    return data, Y, T, rho


@pytest.mark.parametrize("name,form,n,frac", [
    ("h2co", "plain", 1024, 0.97), ("h2co", "mixed", 1024, 0.97), ("h2co", "persistent", 1024, 0.97),
    ("h2co", "group", 1024, 0.97), ("h2co+30", "block", 128, 0.85)])
def test_cv_step(cuda, name, form, n, frac):
    """Statuses equal the oracle's; T within 1e-6 everywhere; Y within 1e-9 in every cell whose solver took
    the oracle's path (all eight counters equal) and within 1e-7 in the others (an ulp of exp/log flips a
    step-size or order decision there); at least `frac` of the cells on the oracle's path."""
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    data, Y, T, rho = _cv_states(name, n, 81)
    kw = {"plain": dict(tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64),
          "mixed": dict(tile=lsg.LSG_TILE_LANE, precision=lsg.LSG_PRECISION_MIXED),
          "persistent": dict(tile=lsg.LSG_TILE_PERSISTENT, precision=lsg.LSG_PRECISION_MIXED),
          "group": dict(tile=lsg.LSG_TILE_GROUP, precision=lsg.LSG_PRECISION_MIXED),
          "block": dict(precision=lsg.LSG_PRECISION_FP64)}[form]
    ctx = lsg.ReactionStep(lsg.Mechanism(data), **kw)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    st = torch.zeros(n, dtype=torch.int32, device=cuda)
    cnt = torch.zeros((n, lsg.NCOUNTERS), dtype=torch.int64, device=cuda)
    ctx.step_cv_device(Yd, Td, torch.tensor(rho, device=cuda), 1e-5, status=st, counters=cnt)
    torch.cuda.synchronize()
    ctx.check()
    Yo, To, _, sto, co = OracleMechanism(data).reaction_step(Y, T, 1e-5, nthreads=8, rho=rho)
    np.testing.assert_array_equal(st.cpu().numpy(), sto)
    rel_T = np.abs(Td.cpu().numpy() - To) / To
    abs_Y = np.abs(Yd.cpu().numpy().T - Yo).max(axis=1)
    same = (cnt.cpu().numpy() == co).all(axis=1)
    print(f"{name} {form}: max rel T err {rel_T.max():.3e}, max abs Y err {abs_Y.max():.3e}, "
          f"cells within Y bound {np.mean(abs_Y <= ATOL_Y):.4f}, on the oracle's path {same.mean():.4f}, "
          f"max abs Y there {abs_Y[same].max():.3e}")
    assert rel_T.max() <= RTOL_T
    assert same.mean() >= frac and abs_Y[same].max() <= ATOL_Y and abs_Y.max() <= 1e-7


def test_cv_device_call_and_constant_pressure_unchanged(h2co, cuda):
    """The device-array call gives the host call's result, and the constant-pressure calls of the same
    context are unaffected by an earlier constant-volume call."""
    import torch
    from laminarsmoke_b200 import lsg
    data, Y, T, rho = _cv_states("h2co", 512, 82)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    Ys = np.ascontiguousarray(Y.T)
    Tg = T.copy()
    ctx.step_cv(Ys, Tg, rho, 1e-5)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    ctx.step_cv_device(Yd, Td, torch.tensor(rho, device=cuda), 1e-5)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(Yd.cpu().numpy(), Ys)
    np.testing.assert_array_equal(Td.cpu().numpy(), Tg)
    Yp = np.ascontiguousarray(Y.T)
    Tp = T.copy()
    ctx.step(Yp, Tp, 1e-5)
    ctx2 = lsg.ReactionStep(lsg.Mechanism(data))
    Yq = np.ascontiguousarray(Y.T)
    Tq = T.copy()
    ctx2.step(Yq, Tq, 1e-5)
    np.testing.assert_array_equal(Yp, Yq)
    np.testing.assert_array_equal(Tp, Tq)
