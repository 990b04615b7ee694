"""The mixed-precision form of large mechanisms on the tensor cores.

lsg_build_and_invert_g_device runs the factorisation that the mixed-precision block form uses in place
of KernelDense::BuildAndFactorizeMatrixG (KernelDense.hpp:195-220): G^-1 of G = I - hr0 J by blocked
Gauss-Jordan elimination with partial pivoting, the rank-32 updates as split-TF32 tcgen05 products.
It is checked against the FP64 inverse, on random matrices and on the oracle's finite-difference
Jacobians of a 121-component state at BDF step sizes; then the reaction step of the mixed block form
(which solves with that inverse inside the FP64 Newton iteration) against the oracle."""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu


def _tc_inverse(ctx, Js, hs, cuda):
    """Js: list of n x n FP64 Jacobians; returns the FP32 inverses of I - h J as n x n arrays."""
    import torch
    n = Js[0].shape[0]
    J = torch.tensor(np.stack([j.T for j in Js]).copy(), device=cuda)      # column-major per matrix
    h = torch.tensor(np.asarray(hs, dtype=np.float64), device=cuda)
    inv = torch.zeros((len(Js), n, n), dtype=torch.float32, device=cuda)
    ctx.build_and_invert_g_device(J, h, inv)
    torch.cuda.synchronize()
    ctx.check()
    return [x.T.astype(np.float64) for x in inv.cpu().numpy()]


@pytest.mark.parametrize("n", [32, 45, 64, 100, 121, 128, 129, 200, 256, 301, 501, 512])
def test_tc_inverse_random(cuda, h2co, n):
    """Up to 128 one 128-row tile in TMEM; above, the in-place multi-tile inverse in global memory.  G is
    kept well conditioned (|h J| <= 0.5 in norm) so that the bound is the FP32 rounding of the
    elimination, which grows with n."""
    from laminarsmoke_b200 import lsg
    ctx = lsg.ReactionStep(lsg.Mechanism(h2co[0]))
    rng = np.random.default_rng(n)
    nm = 40 if n <= 128 else 12
    Js = [rng.normal(size=(n, n)) for _ in range(nm)]
    hs = rng.uniform(0.2, 1.0, nm) * 0.5 / (2.0 * np.sqrt(n))
    tol = 1e-5 if n <= 128 else 4e-5
    worst = 0.0
    for X, J, h in zip(_tc_inverse(ctx, Js, hs, cuda), Js, hs):
        G = np.eye(n) - h * J
        Xe = np.linalg.inv(G)
        worst = max(worst, float(np.abs(X @ G - np.eye(n)).max()))
        assert np.abs(X - Xe).max() <= tol * np.abs(Xe).max()
        assert np.abs(X @ G - np.eye(n)).max() <= tol
    print(f"n={n}: worst |X G - I| {worst:.2e}")


@pytest.mark.parametrize("pad", [106, 286], ids=["n121", "n301"])
def test_tc_inverse_chemistry_jacobians(cuda, pad):
    """Finite-difference Jacobians of H2/CO states padded to 121 or 301 components (condition numbers 1e4
    to 1e8): entrywise error of the FP32 inverse against the FP64 one, relative to its largest entry."""
    from laminarsmoke_b200 import lsg, mech
    from laminarsmoke_b200.mech import blob
    from oracle.oracle import OracleMechanism
    data, species = mech.load(f"h2co+{pad}")
    A, _ = blob.unpack(data)
    om = OracleMechanism(data)
    Y, T = cells.h2co_mixing(species[:14], A["mw"][:14], 8, seed=1)
    Js, hs = [], []
    for k in range(8):
        y = np.zeros(len(species) + 1)
        y[:14] = 0.5 * Y[k]
        y[14:-1] = 0.5 / (len(species) - 14)
        y[-1] = T[k]
        for h in (1e-8, 1e-7, 1e-6):
            Js.append(om.fd_jacobian(y, h))
            hs.append(0.5 * h)
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    worst = worst_res = 0.0
    for X, J, h in zip(_tc_inverse(ctx, Js, hs, cuda), Js, hs):
        G = np.eye(J.shape[0]) - h * J
        Xe = np.linalg.inv(G)
        err = np.abs(X - Xe).max() / np.abs(Xe).max()
        res = np.abs(X @ G - np.eye(J.shape[0])).max()
        worst, worst_res = max(worst, err), max(worst_res, res)
    print(f"n={J.shape[0]}: worst entrywise relative error of the split-TF32 inverse {worst:.2e}, "
          f"worst |X G - I| {worst_res:.2e}")
    assert worst <= 1e-4
    # the simplified Newton iteration with X in place of G^-1 contracts while |I - X G| < 1
    assert worst_res <= 0.5


def _padded_states(n, seed):
    from laminarsmoke_b200 import mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load("h2co+106")
    A, _ = blob.unpack(data)
    Y, T = cells.h2co_mixing(species[:14], A["mw"][:14], n, seed=seed)
    Yp = np.zeros((n, len(species)))
    Yp[:, :14] = 0.5 * Y
    Yp[:, 14:] = 0.5 / (len(species) - 14)
    return data, Yp, T


@pytest.mark.parametrize("rtol,atol,frac", [(1e-7, 1e-12, 0.7), (1e-10, 1e-16, 0.9)])
def test_tc_block_step_against_oracle(cuda, rtol, atol, frac):
    """The mixed-precision block form (121 components: H2/CO chemistry with 106 inert species) against
    the oracle: identical statuses, relative T error <= 1e-6 in every cell, absolute Y error <= 1e-9 in
    most cells and <= 1e-7 in all (the FP32 inverse changes the Newton iterates, so the step sequences
    of some cells differ from the oracle's by O(rtol))."""
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    n = 64
    data, Y, T = _padded_states(n, 5)
    ctx = lsg.ReactionStep(lsg.Mechanism(data), precision=lsg.LSG_PRECISION_MIXED, rtol=rtol, atol=atol)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    st = torch.zeros(n, dtype=torch.int32, device=cuda)
    cnt = torch.zeros((n, lsg.NCOUNTERS), dtype=torch.int64, device=cuda)
    ctx.step_device(Yd, Td, 1e-5, status=st, counters=cnt)
    torch.cuda.synchronize()
    ctx.check()
    Yo, To, _, sto, co = OracleMechanism(data).reaction_step(Y, T, 1e-5, rtol=rtol, atol=atol, nthreads=8)
    np.testing.assert_array_equal(st.cpu().numpy(), sto)
    dT = np.abs(Td.cpu().numpy() - To) / To
    dY = np.abs(Yd.cpu().numpy().T - Yo).max(axis=1)
    c = cnt.cpu().numpy()
    print(f"TC block rtol {rtol:g}: max rel T {dT.max():.2e}, max abs Y {dY.max():.2e}, within 1e-9 "
          f"{np.mean(dY <= 1e-9):.3f}; factorisations/cell {c[:, 3].mean():.1f} (oracle {co[:, 3].mean():.1f}), "
          f"solves/cell {c[:, 4].mean():.1f} (oracle {co[:, 4].mean():.1f})")
    assert c[:, 3].sum() > 0
    assert dT.max() <= 1e-6
    assert np.mean(dY <= 1e-9) >= frac and dY.max() <= 1e-7


def test_large_autotuner_times_both_factorisations(cuda):
    """With autotune on, the mixed-precision block form's first call times the FP64 LU factors against the
    tensor-core inverse on one wave of the FP64 form's blocks and keeps the faster; the step it then takes
    matches the oracle with the criteria above."""
    import torch
    from laminarsmoke_b200 import lsg
    from oracle.oracle import OracleMechanism
    n = 512
    data, Y, T = _padded_states(n, 7)
    ctx = lsg.ReactionStep(lsg.Mechanism(data), precision=lsg.LSG_PRECISION_MIXED, autotune=1)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    Td = torch.tensor(T, device=cuda)
    st = torch.zeros(n, dtype=torch.int32, device=cuda)
    ctx.step_device(Yd, Td, 1e-5, status=st)
    torch.cuda.synchronize()
    ctx.check()
    tile, width, rates = ctx.tuning()
    print(f"large autotuner: {rates}, chosen {'tensor-core inverse' if width else 'FP64 LU factors'}")
    assert tile == lsg.LSG_TILE_BLOCK
    assert rates["block_fp64_lu"] > 0 and rates["block_tc_inverse"] > 0
    assert width == int(rates["block_tc_inverse"] > rates["block_fp64_lu"])
    pick = np.arange(0, n, 8)
    Yo, To, _, sto, _ = OracleMechanism(data).reaction_step(Y[pick], T[pick], 1e-5, nthreads=8)
    np.testing.assert_array_equal(st.cpu().numpy()[pick], sto)
    dT = np.abs(Td.cpu().numpy()[pick] - To) / To
    dY = np.abs(Yd.cpu().numpy().T[pick] - Yo).max(axis=1)
    assert dT.max() <= 1e-6
    assert np.mean(dY <= 1e-9) >= 0.7 and dY.max() <= 1e-7
