"""Extract the reduced collision-integral tables into ``data/collision_integrals.npz``.

The tables are the published Stockmayer-potential collision integrals of
Monchick & Mason (J. Chem. Phys. 35:1676, 1961) that CHEMKIN's TRANFIT and
OpenSMOKE++'s preprocessor interpolate: Omega(1,1)* and Omega(2,2)* on 37
reduced temperatures T* x 8 reduced dipole moments delta*, and the 7-term
fits in ln T* of the ratios A*, B*, C* used for thermal diffusion.  The
numbers must be the same as the reference preprocessor's for the transport
fits to agree, so they are read from its table file
(solvers/openSMOKEpp4laminarSMOKE/preprocessing/CollisionIntegralMatrices.hpp:76-180)
rather than typed in::

    python -m laminarsmoke_b200.mech.make_collision_tables /path/to/laminarSMOKE

The output file is committed; nothing at run time needs the reference.
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

from . import DATA

_NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"


def _block(text: str, name: str) -> np.ndarray:
    m = re.search(r"CollisionIntegralMatrices::" + name + r"\s*=\s*\(Eigen::\w+\(([\d,\s]+)\)\s*<<(.*?)\)\.finished\(\)",
                  text, re.S)
    if not m:
        raise ValueError(f"table {name} not found")
    shape = tuple(int(v) for v in m.group(1).split(","))
    vals = np.array([float(v) for v in re.findall(_NUM, m.group(2))])
    if vals.size != int(np.prod(shape)):
        raise ValueError(f"table {name}: {vals.size} values for shape {shape}")
    return vals.reshape(shape)


def _scalar(text: str, name: str) -> float:
    m = re.search(r"CollisionIntegralMatrices::" + name + r"\s*=\s*(" + _NUM + r")\s*;", text)
    if not m:
        raise ValueError(f"constant {name} not found")
    return float(m.group(1))


def extract(path: str) -> dict:
    with open(path, "r", encoding="latin-1") as f:
        text = f.read()
    out = {
        "delta_star": _block(text, "deltaStar"),
        "t_star": _block(text, "TStar"),
        "omega11": _block(text, "O37_8"),     # Omega(1,1)*: diffusion
        "omega22": _block(text, "P37_8"),     # Omega(2,2)*: viscosity and conductivity
    }
    for r in "ABC":
        out[f"fit_{r.lower()}star"] = np.array([_scalar(text, f"FIT{r}STAR_{i}") for i in range(1, 8)])
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    root = argv[0] if argv else os.environ.get("LSMOKE_REFERENCE_ROOT", "")
    if not root:
        raise SystemExit("usage: give the reference checkout as the first argument or in LSMOKE_REFERENCE_ROOT")
    src = os.path.join(root, "solvers/openSMOKEpp4laminarSMOKE/preprocessing/CollisionIntegralMatrices.hpp")
    tabs = extract(src)
    out = os.path.join(DATA, "collision_integrals.npz")
    np.savez(out, **tabs)
    print(out, {k: v.shape for k, v in tabs.items()})


if __name__ == "__main__":
    main()
