"""Time the property update (lsg_properties_device, lsg_properties) on one GPU.

    python -m laminarsmoke_b200.run_properties --mech h2co --cells 1048576

Cells are H2/CO mixing states (uniform random states for other mechanisms)
at pressures from 0.5 to 5 atm; every field is requested, with Soret terms
and mixture-averaged diffusivities.  The device time is taken with CUDA
events on the launching stream over ``--reps`` launches after warm-up; the
inputs and outputs of a launch (hundreds of MB at a million cells) exceed
the 126 MB L2.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mech", default="h2co")
    ap.add_argument("--cells", type=int, default=1 << 20)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args(argv)

    import torch
    from . import cells, lsg, mech
    from .mech import blob

    data, species = mech.load(a.mech)
    A, _ = blob.unpack(data)
    nc = len(species)
    rng = np.random.default_rng(5)
    try:
        Y, T = cells.h2co_mixing(species, A["mw"], a.cells, seed=5)
    except ValueError:
        Y = rng.uniform(0., 1., (a.cells, nc))
        Y /= Y.sum(axis=1, keepdims=True)
        T = rng.uniform(300., 2500., a.cells)
    p = rng.uniform(0.5, 5.0, a.cells) * 101325.
    ctx = lsg.ReactionStep(lsg.Mechanism(data))
    nt = len(ctx.mech.transport_info()[1])
    dev = torch.device("cuda:0")
    Yd = torch.tensor(np.ascontiguousarray(Y.T), device=dev)
    Td = torch.tensor(T, device=dev)
    pd = torch.tensor(p, device=dev)
    stream = torch.cuda.current_stream()
    for _ in range(a.warmup):
        ctx.properties_device(Yd, Td, pd, soret=True)
    torch.cuda.synchronize()
    launches0 = ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.reps):
        ctx.properties_device(Yd, Td, pd, soret=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    # algorithmic bytes per cell: Y, T, p in; X, 8 scalars, species cp, Dmix, Dsoret out
    bytes_cell = 8 * (nc + 2) + 8 * (3 * nc + 8 + nt)
    # host entry: copies in, kernel, copies out
    Yh = np.ascontiguousarray(Y.T)
    ctx.properties(Yh, T, p=p, soret=True)
    t0 = time.perf_counter()
    reps_h = 3
    for _ in range(reps_h):
        ctx.properties(Yh, T, p=p, soret=True)
    host_s = (time.perf_counter() - t0) / reps_h
    print(json.dumps({
        "workload": f"property update, {a.mech} ({nc} species, {nt} with Soret terms), {a.cells} cells",
        "cells_per_s": a.cells / (ms * 1e-3), "ms_per_launch": ms,
        "algorithmic_bytes_per_cell": bytes_cell, "achieved_GBps": bytes_cell * a.cells / (ms * 1e-3) / 1e9,
        "kernel_launches": ctx.launches() - launches0,
        "host_entry_cells_per_s": a.cells / host_s, "host_entry_ms": host_s * 1e3,
    }))


if __name__ == "__main__":
    main()
