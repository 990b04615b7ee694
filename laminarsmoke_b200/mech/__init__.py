"""Mechanism preprocessing: CHEMKIN compiler, packed blob format, seeded synthetic mechanisms.

``load(name)`` returns ``(blob_bytes, species_names)`` for the mechanisms the
workloads of this project use:

* ``"h2co"``    -- POLIMI_H2CO_1412 (14 species, 33 reactions), compiled from the
                   reference's CHEMKIN files into ``data/POLIMI_H2CO_1412.lsmech``
                   by ``mech/build_data.py``;
* ``"h2"``, ``"ch4"`` -- POLIMI_H2_1412 (9 species, 20 reactions) and
                   POLIMI_CH4_SKELETAL_1412 (24 species, 155 reactions), from the
                   reference's files likewise;
* ``"ch4_1step"``, ``"h2_1step"`` -- the reference's global one-step CH4 and H2
                   mechanisms (forward reaction orders given by FORD), in
                   ``data/GLOBAL_*_1step.lsmech``;
* ``"syn120"``  -- seeded synthetic C1-C2 mechanism, 120 species / 800 reactions;
* ``"syn500"``  -- seeded synthetic mechanism, 500 species / 3 000 reactions;
* ``"syn120p"``, ``"syn500p"`` -- the same mechanisms with physically bounded
                   activation energies and rate constants (integrable);
* ``"syn120t"``  -- ``syn120p`` compiled with synthetic transport records
                   (``synthetic.transport_text``), for the property update at
                   120 species;
* ``"h2co+K"``  -- POLIMI_H2CO_1412 with K chemically inert copies of N2 added
                   (``pad_inert``): the H2/CO chemistry in a mechanism of 14 + K
                   species, which exercises the large-mechanism path with
                   realistic stiffness.
"""
from __future__ import annotations

import functools
import os
from typing import List, Tuple

from . import blob as _blob

DATA = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "data")

SYNTHETIC = {
    "syn120": (120, 800, 1201, False),
    "syn500": (500, 3000, 5003, False),
    # the same draws under physical bounds on barriers and rate constants (mech/synthetic.py)
    "syn120p": (120, 800, 1201, True),
    "syn500p": (500, 3000, 5003, True),
}


def pad_inert(data: bytes, k: int, template: str = "N2") -> Tuple[bytes, List[str]]:
    """The mechanism in `data` with `k` extra species that take part in no
    reaction and have the thermodynamics and molecular weight of `template`
    (collision efficiency 1 wherever third bodies appear)."""
    import numpy as np
    A, species = _blob.unpack(data)
    A = {key: np.array(v) for key, v in A.items()}
    t = species.index(template)
    nc = int(A["dims"][0])
    per = {"mw": 1, "t_mid": 1, "t_low": 1, "t_high": 1, "cp_ht": 5, "cp_lt": 5, "dh_ht": 6, "dh_lt": 6,
           "ds_ht": 6, "ds_lt": 6, "nasa_raw": A["nasa_raw"].size // nc}
    for key, w in per.items():
        row = A[key][t * w:(t + 1) * w]
        A[key] = np.concatenate([A[key]] + [row] * k)
    for key in [key for key in A if key.startswith("tr_")]:
        del A[key]    # the padded mechanism carries no transport data
    A["fr_ptr"] = np.concatenate([A["fr_ptr"], np.full(k, A["fr_ptr"][-1], A["fr_ptr"].dtype)])
    A["dims"] = np.array([nc + k, A["dims"][1]], A["dims"].dtype)
    names = list(species) + [f"INERT{i + 1}" for i in range(k)]
    return _blob.pack(A, names), names


@functools.lru_cache(maxsize=8)
def load(name: str) -> Tuple[bytes, List[str]]:
    if name.startswith("h2co+"):
        return pad_inert(load("h2co")[0], int(name[5:]))
    files = {"h2co": "POLIMI_H2CO_1412", "h2": "POLIMI_H2_1412", "ch4": "POLIMI_CH4_SKELETAL_1412",
             "ch4_1step": "GLOBAL_CH4_1step", "h2_1step": "GLOBAL_H2_1step"}
    if name in files:
        path = os.path.join(DATA, files[name] + ".lsmech")
        with open(path, "rb") as f:
            data = f.read()
        _, species = _blob.unpack(data)
        return data, species
    if name == "syn120t":
        from . import chemkin, synthetic
        s = synthetic.generate(120, 800, 1201, physical=True)
        m = chemkin.compile_mechanism(s.kinetics, s.thermo, transport_text=synthetic.transport_text(s))
        return _blob.pack(m.arrays, m.species), m.species
    if name in SYNTHETIC:
        from . import chemkin, synthetic
        ns, nr, seed, physical = SYNTHETIC[name]
        s = synthetic.generate(ns, nr, seed, physical=physical)
        m = chemkin.compile_mechanism(s.kinetics, s.thermo)
        return _blob.pack(m.arrays, m.species), m.species
    raise KeyError(f"unknown mechanism {name!r}")
