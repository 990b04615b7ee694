"""Run one reaction step of a named synthetic workload on the GPU (a fixed case
for profiling and quick checks).

  python -m laminarsmoke_b200.run_case --workload h2co_mixing --cells 65536 --form mixed

Workloads (seeded, see laminarsmoke_b200.cells): h2co_mixing (T ~ U[900, 2200] K
mixtures of H2/CO fuel and air with radicals), h2co_uneven (cold / igniting /
near-equilibrium thirds; the pool is prepared with the plain step), coflow (the
200 x 400 Burke-Schumann coflow mesh with H2/CO fuel, 80,000 cells, advanced by
--steps successive device-resident steps; --cells below 80,000 takes an evenly
strided subset).  Forms: plain (warp-per-cell FP64), mixed (round scheme, FP32
factors), batched64 (round scheme, FP64 factors), persistent (persistent lane
kernel, FP32 factors), group / group64 (fused lane-group kernel, FP32 / FP64
factors), auto (the library's choice: the autotuner for up to 31 species, the
block-per-cell form above).  --mech h2co+K pads the H2/CO chemistry
with K inert species (h2co+106: 121 species).

  python -m laminarsmoke_b200.run_case --workload coflow --mech h2co+106 --steps 50 --form auto

tc_inverse inverts --cells seeded well-conditioned matrices G = I - h J of order --n (32 to 512) with the
mixed-precision form's tensor-core inverse (lsg_build_and_invert_g_device), --steps times:

  python -m laminarsmoke_b200.run_case --workload tc_inverse --n 121 --cells 4096
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=("h2co_mixing", "h2co_uneven", "coflow", "tc_inverse"),
                    default="h2co_mixing")
    ap.add_argument("--n", type=int, default=121, help="matrix order of the tc_inverse workload")
    ap.add_argument("--cells", type=int, default=65536)
    ap.add_argument("--form", choices=("plain", "mixed", "batched64", "persistent", "group", "group64", "auto"),
                    default="mixed")
    ap.add_argument("--mech", default="h2co", help="h2co or h2co+K (K inert species)")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--dt", type=float, default=1e-5)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args(argv)
    import torch
    from laminarsmoke_b200 import cells, lsg, mech
    from laminarsmoke_b200.mech import blob
    data, species = mech.load(args.mech)
    arrays, _ = blob.unpack(data)
    m = lsg.Mechanism(data)
    forms = {"plain": (lsg.LSG_TILE_WARP, lsg.LSG_PRECISION_FP64),
             "mixed": (lsg.LSG_TILE_LANE, lsg.LSG_PRECISION_MIXED),
             "batched64": (lsg.LSG_TILE_LANE, lsg.LSG_PRECISION_FP64),
             "persistent": (lsg.LSG_TILE_PERSISTENT, lsg.LSG_PRECISION_MIXED),
             "group": (lsg.LSG_TILE_GROUP, lsg.LSG_PRECISION_MIXED),
             "group64": (lsg.LSG_TILE_GROUP, lsg.LSG_PRECISION_FP64),
             "auto": (lsg.LSG_TILE_AUTO, lsg.LSG_PRECISION_MIXED)}
    tile, prec = forms[args.form]
    ctx = lsg.ReactionStep(m, tile=tile, precision=prec)
    if args.workload == "tc_inverse":
        return tc_inverse(ctx, args)
    if args.workload == "h2co_mixing":
        Y, T = cells.h2co_mixing(species, arrays["mw"], args.cells, seed=args.seed)
    elif args.workload == "coflow":
        Y, T = cells.coflow_fields(species, arrays["mw"], seed=args.seed, fuel={"H2": 0.5, "CO": 0.5})
        if args.cells < T.size:
            idx = np.linspace(0, T.size - 1, args.cells).astype(np.int64)
            Y, T = Y[idx], T[idx]
        args.cells = T.size
    else:
        plain = lsg.ReactionStep(m, tile=lsg.LSG_TILE_WARP, precision=lsg.LSG_PRECISION_FP64)

        def pool(Yp, Tp, dt):
            Yd = torch.tensor(np.ascontiguousarray(Yp.T), device="cuda")
            Td = torch.tensor(Tp, device="cuda")
            plain.step_device(Yd, Td, dt)
            torch.cuda.synchronize()
            return np.ascontiguousarray(Yd.cpu().numpy().T), Td.cpu().numpy()
        Y, T = cells.h2co_uneven(species, arrays["mw"], args.cells, pool, seed=args.seed)
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device="cuda")
    Td = torch.tensor(T, device="cuda")
    status = torch.zeros(args.cells, dtype=torch.int32, device="cuda")
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record()
    fails = ctx.step_sequence_device(Yd, Td, args.dt, args.steps, status=status)
    t1.record()
    torch.cuda.synchronize()
    ctx.check()
    ms = t0.elapsed_time(t1)
    st = status.cpu().numpy()
    print(f"{args.form} {args.workload} {args.mech} {args.cells} cells x {args.steps} steps: {ms:.1f} ms, "
          f"{args.cells * args.steps / (ms * 1e-3):.4e} cells*steps/s, cells failing in any step {fails}, "
          f"last statuses {dict(zip(*np.unique(st, return_counts=True)))}")
    return 0


def tc_inverse(ctx, args) -> int:
    import torch
    n, nm = args.n, args.cells
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    J = torch.randn((nm, n, n), dtype=torch.float64, device="cuda", generator=g)
    h = (0.2 + 0.8 * torch.rand(nm, dtype=torch.float64, device="cuda", generator=g)) * 0.5 / (2.0 * n ** 0.5)
    inv = torch.empty((nm, n, n), dtype=torch.float32, device="cuda")
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.build_and_invert_g_device(J, h, inv)   # first call: work matrices, kernel attributes
    torch.cuda.synchronize()
    t0.record()
    for _ in range(args.steps):
        ctx.build_and_invert_g_device(J, h, inv)
    t1.record()
    torch.cuda.synchronize()
    ctx.check()
    ms = t0.elapsed_time(t1) / args.steps
    G = torch.eye(n, dtype=torch.float64, device="cuda") - h[:4, None, None] * J[:4].transpose(1, 2)
    X = inv[:4].transpose(1, 2).double()
    res = (X @ G - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max().item()
    flops = 2.0 * n ** 3 * nm   # Gauss-Jordan inverse: 2 n^3
    print(f"tc_inverse n={n} x {nm}: {ms:.3f} ms per call, {nm / (ms * 1e-3):.4e} inverses/s, "
          f"{flops / (ms * 1e-3) / 1e12:.2f} TFLOP/s (2 n^3 per inverse), max |X G - I| {res:.2e}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
