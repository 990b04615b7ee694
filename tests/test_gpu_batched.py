"""Lane-per-cell batched reaction step (FP64 LU and mixed FP32 LU) against the CPU oracle."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu

RTOL_T = 1e-6
ATOL_Y = 1e-9


@pytest.fixture(scope="module")
def gpu_h2co(h2co, cuda):
    from laminarsmoke_b200 import lsg
    return lsg.Mechanism(h2co[0])


def _run(gpu_h2co, oracle_h2co, Y, T, dt, precision, **kw):
    from laminarsmoke_b200 import lsg
    ctx = lsg.ReactionStep(gpu_h2co, tile=lsg.LSG_TILE_LANE, precision=precision,
                           **{k: v for k, v in kw.items() if k in ("max_steps", "tmin_chem", "rtol", "atol")})
    Ys = np.ascontiguousarray(Y.T)
    Tg = T.copy()
    Q, st, ns = ctx.step(Ys, Tg, dt)
    ctx.check()
    Yo, To, Qo, sto, cnt = oracle_h2co.reaction_step(Y, T, dt, nthreads=8, **kw)
    return (Ys.T, Tg, Q, st, ns), (Yo, To, Qo, sto, cnt)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64-lu", "fp32-lu"])
def test_batched_parity_mixing_states(h2co, oracle_h2co, gpu_h2co, precision):
    _, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 4096, seed=1)
    (Yg, Tg, Qg, stg, nsg), (Yo, To, Qo, sto, cnt) = _run(gpu_h2co, oracle_h2co, Y, T, 1e-5, precision)
    np.testing.assert_array_equal(stg, sto)
    rel_T = np.abs(Tg - To) / To
    abs_Y = np.abs(Yg - Yo).max(axis=1)
    same = nsg == cnt[:, 0]
    print(f"precision={precision}: max rel T err {rel_T.max():.3e}, max abs Y err {abs_Y.max():.3e}, "
          f"p99 abs Y err {np.quantile(abs_Y, 0.99):.3e}, identical step counts {same.mean():.4f}, "
          f"cells within Y bound {np.mean(abs_Y <= ATOL_Y):.4f}")
    assert rel_T.max() <= RTOL_T
    assert np.mean(abs_Y <= ATOL_Y) >= 0.99
    assert abs_Y.max() <= 1e-7


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64-lu", "fp32-lu"])
def test_batched_tight_tolerances(h2co, oracle_h2co, gpu_h2co, precision):
    _, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 1024, seed=21)
    (Yg, Tg, Qg, stg, nsg), (Yo, To, Qo, sto, cnt) = _run(gpu_h2co, oracle_h2co, Y, T, 1e-5, precision,
                                                          rtol=1e-10, atol=1e-16)
    rel_T = np.abs(Tg - To) / To
    abs_Y = np.abs(Yg - Yo).max(axis=1)
    print(f"tight precision={precision}: max rel T err {rel_T.max():.3e}, max abs Y err {abs_Y.max():.3e}")
    assert rel_T.max() <= RTOL_T
    assert abs_Y.max() <= ATOL_Y


def test_batched_edge_cases(h2co, oracle_h2co, gpu_h2co):
    _, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 8, seed=4)
    Y[0, 3] = -1e-6
    Y[1] *= 1.01
    T[2] = 7000.0
    T[3] = 250.0
    (Yg, Tg, Qg, stg, nsg), (Yo, To, Qo, sto, cnt) = _run(gpu_h2co, oracle_h2co, Y, T, 1e-5, 1, tmin_chem=260.0)
    np.testing.assert_array_equal(stg, sto)
    assert stg[2] == -9 and stg[3] == 0
    np.testing.assert_allclose(Tg, To, rtol=RTOL_T)
    np.testing.assert_allclose(Yg, Yo, atol=1e-8)
    (Yg, Tg, Qg, stg, nsg), (Yo, To, Qo, sto, cnt) = _run(gpu_h2co, oracle_h2co, Y, T, 1e-5, 1, max_steps=5)
    np.testing.assert_array_equal(stg, sto)
    np.testing.assert_allclose(Tg, To, rtol=1e-9)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_autotuner_picks_a_measured_form(h2co, oracle_h2co, gpu_h2co, precision):
    """With tile AUTO and autotune on, the first step times the candidate forms on
    its own cells, keeps the fastest, and the step it then runs matches the oracle."""
    import torch
    from laminarsmoke_b200 import lsg
    _, species, A = h2co
    Y, T = cells.h2co_mixing(species, A["mw"], 4096, seed=31)
    ctx = lsg.ReactionStep(gpu_h2co, precision=precision, tile=lsg.LSG_TILE_AUTO, autotune=1)
    assert ctx.tuning() is None
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device="cuda")
    Td = torch.tensor(T, device="cuda")
    st = torch.zeros(4096, dtype=torch.int32, device="cuda")
    ctx.step_device(Yd, Td, 1e-5, status=st)
    torch.cuda.synchronize()
    ctx.check()
    tile, width, rates = ctx.tuning()
    print(f"autotune precision={precision}: tile {tile} width {width} rates {rates}")
    tried = {k: v for k, v in rates.items() if v > 0}
    assert len(tried) >= 3 if precision == 0 else len(tried) >= 2
    best = max(tried, key=tried.get)
    assert (tile, width) == {"rounds16": (lsg.LSG_TILE_LANE, 16), "rounds32": (lsg.LSG_TILE_LANE, 32),
                             "plain_warp": (lsg.LSG_TILE_WARP, 0),
                             "persistent": (lsg.LSG_TILE_PERSISTENT, 0), "group_4": (lsg.LSG_TILE_GROUP, 4),
                             "group_2": (lsg.LSG_TILE_GROUP, 2)}[best]
    Yo, To, Qo, sto, cnt = oracle_h2co.reaction_step(Y, T, 1e-5, nthreads=8)
    np.testing.assert_array_equal(st.cpu().numpy(), sto)
    assert np.max(np.abs(Td.cpu().numpy() - To) / To) <= RTOL_T
    abs_Y = np.abs(Yd.cpu().numpy().T - Yo).max(axis=1)
    assert np.mean(abs_Y <= ATOL_Y) >= 0.99 and abs_Y.max() <= 1e-7
