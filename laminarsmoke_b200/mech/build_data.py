"""Compile the reference's CHEMKIN mechanisms into packed blobs under ``data/``.

Run in a checkout that has the reference next to it::

    python -m laminarsmoke_b200.mech.build_data /path/to/laminarSMOKE

The output files are committed, so nothing at run time needs the reference.
"""
from __future__ import annotations

import os
import sys

from . import DATA, blob, chemkin

MECHS = {
    "POLIMI_H2CO_1412": ("run/kinetic-mechanisms/POLIMI_H2CO_1412/POLIMI_H2CO_1412.CKI",
                         "run/kinetic-mechanisms/POLIMI_H2CO_1412/POLIMI_TOT_NOX_1412.CKT"),
    "POLIMI_H2_1412": ("run/kinetic-mechanisms/POLIMI_H2_1412/POLIMI_H2_1412.CKI",
                       "run/kinetic-mechanisms/POLIMI_H2_1412/POLIMI_TOT_NOX_1412.CKT"),
    "POLIMI_CH4_SKELETAL_1412": ("run/kinetic-mechanisms/POLIMI_CH4_SKELETAL_1412/POLIMI_CH4_SKELETAL_1412.CKI",
                                 "run/kinetic-mechanisms/POLIMI_CH4_SKELETAL_1412/POLIMI_TOT_NOX_1412.CKT"),
    # global one-step mechanisms with forward reaction orders (FORD)
    "GLOBAL_CH4_1step": ("run/kinetic-mechanisms/GLOBAL_CH4_1step/GLOBAL_CH4_1step.CKI",
                         "run/kinetic-mechanisms/GLOBAL_CH4_1step/GLOBAL_CH4_1step.CKT"),
    "GLOBAL_H2_1step": ("run/kinetic-mechanisms/GLOBAL_H2_1step/GLOBAL_H2_1step.CKI",
                        "run/kinetic-mechanisms/GLOBAL_H2_1step/GLOBAL_H2_1step.CKT"),
}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    root = argv[0] if argv else "/root/reference"
    os.makedirs(DATA, exist_ok=True)
    for name, (cki, ckt) in MECHS.items():
        m = chemkin.compile_files(os.path.join(root, cki), os.path.join(root, ckt))
        out = os.path.join(DATA, name + ".lsmech")
        with open(out, "wb") as f:
            f.write(blob.pack(m.arrays, m.species))
        print(f"{out}: {m.n_species} species, {m.n_reactions} reactions")


if __name__ == "__main__":
    main()
