"""The reaction step that allocates no device memory (lsg_reaction_step_device_noalloc).

Callers such as a CFD solver that hands all free device memory to its own pool
allocator, or one that keeps cudaMalloc/cudaFree (which synchronise the device)
out of its time loop, use this entry point.  It runs the persistent lane kernel
with its work space in a fixed 16 MiB device array, so it must give the same
cells the same answers as the context-based call of that kernel, call after
call (the array keeps the previous call's contents), agree with the CPU oracle,
and it must refuse a mechanism whose work space does not fit.

This file is collected last on purpose: it runs after every other test.
"""
import numpy as np
import pytest

from laminarsmoke_b200 import cells

pytestmark = pytest.mark.gpu

RTOL_T = 1e-6
ATOL_Y = 1e-9


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64-lu", "fp32-lu"])
def test_noalloc_matches_context_call_twice(h2co, oracle_h2co, cuda, precision):
    import torch
    from laminarsmoke_b200 import lsg
    _, species, A = h2co
    mech = lsg.Mechanism(h2co[0])
    # more cells than the fixed array has slots, so slots are reused through the queue
    n = 12000
    Y, T = cells.h2co_mixing(species, A["mw"], n, seed=3)
    Y0 = torch.tensor(np.ascontiguousarray(Y.T), device=cuda)
    T0 = torch.tensor(T, device=cuda)

    ctx = lsg.ReactionStep(mech, tile=lsg.LSG_TILE_PERSISTENT, precision=precision)
    Yr, Tr = Y0.clone(), T0.clone()
    str_ = torch.zeros(n, dtype=torch.int32, device=cuda)
    nsr = torch.zeros(n, dtype=torch.int32, device=cuda)
    Qr = torch.zeros(n, dtype=torch.float64, device=cuda)
    ctx.step_device(Yr, Tr, 1e-5, Q=Qr, status=str_, nsteps=nsr)
    ctx.check()
    ctx.close()

    opt = lsg.default_options(precision=precision)
    for call in range(2):
        Yn, Tn = Y0.clone(), T0.clone()
        stn = torch.full((n,), 99, dtype=torch.int32, device=cuda)
        nsn = torch.zeros(n, dtype=torch.int32, device=cuda)
        Qn = torch.zeros(n, dtype=torch.float64, device=cuda)
        lsg.step_device_noalloc(mech, Yn, Tn, 1e-5, options=opt, Q=Qn, status=stn, nsteps=nsn)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(stn.cpu().numpy(), str_.cpu().numpy(), err_msg=f"call {call}")
        np.testing.assert_array_equal(nsn.cpu().numpy(), nsr.cpu().numpy(), err_msg=f"call {call}")
        np.testing.assert_allclose(Tn.cpu().numpy(), Tr.cpu().numpy(), rtol=RTOL_T, err_msg=f"call {call}")
        np.testing.assert_allclose(Yn.cpu().numpy(), Yr.cpu().numpy(), rtol=0, atol=ATOL_Y, err_msg=f"call {call}")
        np.testing.assert_allclose(Qn.cpu().numpy(), Qr.cpu().numpy(), rtol=1e-9, atol=1e-6, err_msg=f"call {call}")
    # and against the oracle on 512 of the cells, with the criteria of the other step tests: identical
    # statuses, T within 1e-6 relative, Y within 1e-9 absolute in 99 % of the cells and 1e-7 in all
    pick = np.arange(0, n, n // 512)[:512]
    Yo, To, _, sto, _ = oracle_h2co.reaction_step(Y[pick], T[pick], 1e-5, nthreads=8)
    Yg, Tg = Yn.cpu().numpy().T[pick], Tn.cpu().numpy()[pick]
    np.testing.assert_array_equal(stn.cpu().numpy()[pick], sto)
    assert float(np.max(np.abs(Tg - To) / To)) <= RTOL_T
    dY = np.abs(Yg - Yo).max(axis=1)
    assert (dY <= ATOL_Y).mean() >= 0.99 and dY.max() <= 1e-7, (float((dY <= ATOL_Y).mean()), float(dY.max()))
    mech.close()


def test_noalloc_rejects_mechanism_beyond_scratch(cuda):
    import torch
    from laminarsmoke_b200 import lsg, mech as mechs
    data, species = mechs.load("syn120")
    mech = lsg.Mechanism(data)
    n = 64
    Y = torch.full((len(species), n), 1.0 / len(species), dtype=torch.float64, device=cuda)
    T = torch.full((n,), 1500.0, dtype=torch.float64, device=cuda)
    with pytest.raises(lsg.LsgError) as info:
        lsg.step_device_noalloc(mech, Y, T, 1e-5)
    assert info.value.code == lsg.LSG_ERR_SCRATCH
    assert "scratch" in str(info.value)
    mech.close()


_FRESH = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from laminarsmoke_b200 import cells, lsg, mech as mechs
from laminarsmoke_b200.mech import blob
data, species = mechs.load("h2co")
A, _ = blob.unpack(data)
dev = torch.device("cuda:0")
m = lsg.Mechanism(data)                       # loads the kernels and commits the fixed array
n = 4096
Y, T = cells.h2co_mixing(species, A["mw"], n, seed=9)
Yd = torch.tensor(np.ascontiguousarray(Y.T), device=dev)
Td = torch.tensor(T, device=dev)
st = torch.full((n,), 99, dtype=torch.int32, device=dev)
torch.cuda.synchronize()
# a pool allocator takes (nearly) all free device memory
hog = None
margin = 32 << 20
free, _ = torch.cuda.mem_get_info()
while hog is None and free > margin:
    try:
        hog = torch.empty(free - margin, dtype=torch.uint8, device=dev)
    except torch.OutOfMemoryError:
        margin *= 2
left, _ = torch.cuda.mem_get_info()
lsg.step_device_noalloc(m, Yd, Td, 1e-5, status=st)
s = st.cpu().numpy()
assert ((s == 2) | (s == 0)).all(), np.unique(s)
print(f"OK free before the call: {left >> 20} MiB")
"""


def test_noalloc_first_call_after_pool_takes_memory(cuda):
    """In a fresh process: load the mechanism, let a stand-in pool allocator take all but a few MiB of
    the free device memory, then make the first no-allocation call.  It must succeed: everything it
    needs was committed when the mechanism was loaded."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
