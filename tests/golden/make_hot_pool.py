"""Writes h2co_hot_pool.npz: the near-equilibrium pool of the uneven-stiffness H2/CO workload
(laminarsmoke_b200.cells.h2co_uneven, seed 2, any cell count).

The workload's hot cells are samples of 4,096 hot mixtures (T ~ U[1800, 2300] K) integrated
for 10 ms.  That integration is done once, here, by the CPU oracle, and stored, so that every
consumer of the workload (the GPU arm and the CPU reference arm of bench.py, the GPU tests)
integrates identical cells.  The file keeps the integrated states and a SHA-256 of the initial
states they came from; cells.pool_from_file checks it.

    python tests/golden/make_hot_pool.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main():
    from laminarsmoke_b200 import cells, mech
    from laminarsmoke_b200.mech import blob
    from oracle.oracle import OracleMechanism
    data, species = mech.load("h2co")
    arrays, _ = blob.unpack(data)
    om = OracleMechanism(data)
    out = {}

    def integrate(Yp, Tp, dt):
        Y2, T2, _, st, _ = om.reaction_step(Yp, Tp, dt, nthreads=os.cpu_count() or 1)
        assert (st == 2).all()
        out["Y"], out["T"], out["dt"] = Y2, T2, np.float64(dt)
        out["sha256_initial"] = np.bytes_(cells.pool_digest(Yp, Tp))
        return Y2, T2

    cells.h2co_uneven(species, arrays["mw"], 4096, integrate, seed=2)   # the pool does not depend on the cell count
    path = os.path.join(HERE, "h2co_hot_pool.npz")
    np.savez_compressed(path, **out)
    print(path, out["Y"].shape)


if __name__ == "__main__":
    main()
