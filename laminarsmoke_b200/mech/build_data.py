"""Compile the reference's CHEMKIN mechanisms into packed blobs under ``data/``.

Run in a checkout that has the reference next to it::

    python -m laminarsmoke_b200.mech.build_data /path/to/laminarSMOKE

The output files are committed, so nothing at run time needs the reference.
"""
from __future__ import annotations

import os
import sys

from . import DATA, blob, chemkin

_K = "run/kinetic-mechanisms/"
# kinetics, thermodynamics, transport
MECHS = {
    "POLIMI_H2CO_1412": (_K + "POLIMI_H2CO_1412/POLIMI_H2CO_1412.CKI", _K + "POLIMI_H2CO_1412/POLIMI_TOT_NOX_1412.CKT",
                         _K + "POLIMI_H2CO_1412/POLIMI_TOT_NOX_1412.TRC"),
    "POLIMI_H2_1412": (_K + "POLIMI_H2_1412/POLIMI_H2_1412.CKI", _K + "POLIMI_H2_1412/POLIMI_TOT_NOX_1412.CKT",
                       _K + "POLIMI_H2_1412/POLIMI_TOT_NOX_1412.TRC"),
    "POLIMI_CH4_SKELETAL_1412": (_K + "POLIMI_CH4_SKELETAL_1412/POLIMI_CH4_SKELETAL_1412.CKI",
                                 _K + "POLIMI_CH4_SKELETAL_1412/POLIMI_TOT_NOX_1412.CKT",
                                 _K + "POLIMI_CH4_SKELETAL_1412/POLIMI_TOT_NOX_1412.TRC"),
    # global one-step mechanisms with forward reaction orders (FORD)
    "GLOBAL_CH4_1step": (_K + "GLOBAL_CH4_1step/GLOBAL_CH4_1step.CKI", _K + "GLOBAL_CH4_1step/GLOBAL_CH4_1step.CKT",
                         _K + "GLOBAL_CH4_1step/GLOBAL_CH4_1step.TRC"),
    "GLOBAL_H2_1step": (_K + "GLOBAL_H2_1step/GLOBAL_H2_1step.CKI", _K + "GLOBAL_H2_1step/GLOBAL_H2_1step.CKT",
                        _K + "GLOBAL_H2_1step/GLOBAL_H2_1step.TRC"),
}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    root = argv[0] if argv else os.environ.get("LSMOKE_REFERENCE_ROOT", "")
    if not root:
        raise SystemExit("usage: give the reference checkout as the first argument or in LSMOKE_REFERENCE_ROOT")
    os.makedirs(DATA, exist_ok=True)
    for name, (cki, ckt, trc) in MECHS.items():
        m = chemkin.compile_files(os.path.join(root, cki), os.path.join(root, ckt), trc_path=os.path.join(root, trc))
        out = os.path.join(DATA, name + ".lsmech")
        with open(out, "wb") as f:
            f.write(blob.pack(m.arrays, m.species))
        print(f"{out}: {m.n_species} species, {m.n_reactions} reactions")


if __name__ == "__main__":
    main()
