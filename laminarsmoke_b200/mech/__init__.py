"""Mechanism preprocessing: CHEMKIN compiler, packed blob format, seeded synthetic mechanisms.

``load(name)`` returns ``(blob_bytes, species_names)`` for the mechanisms the
workloads of this project use:

* ``"h2co"``    -- POLIMI_H2CO_1412 (14 species, 33 reactions), compiled from the
                   reference's CHEMKIN files into ``data/POLIMI_H2CO_1412.lsmech``
                   by ``mech/build_data.py``;
* ``"syn120"``  -- seeded synthetic C1-C2 mechanism, 120 species / 800 reactions;
* ``"syn500"``  -- seeded synthetic mechanism, 500 species / 3 000 reactions.
"""
from __future__ import annotations

import functools
import os
from typing import List, Tuple

from . import blob as _blob

DATA = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "data")

SYNTHETIC = {
    "syn120": (120, 800, 1201),
    "syn500": (500, 3000, 5003),
}


@functools.lru_cache(maxsize=8)
def load(name: str) -> Tuple[bytes, List[str]]:
    if name == "h2co":
        path = os.path.join(DATA, "POLIMI_H2CO_1412.lsmech")
        with open(path, "rb") as f:
            data = f.read()
        _, species = _blob.unpack(data)
        return data, species
    if name in SYNTHETIC:
        from . import chemkin, synthetic
        ns, nr, seed = SYNTHETIC[name]
        s = synthetic.generate(ns, nr, seed)
        m = chemkin.compile_mechanism(s.kinetics, s.thermo)
        return _blob.pack(m.arrays, m.species), m.species
    raise KeyError(f"unknown mechanism {name!r}")
