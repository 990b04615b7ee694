"""Mechanism compiler command line.

    python -m laminarsmoke_b200.mech compile KIN.CKI THERMO.CKT -o mech.lsmech [--tmid-correction]
                                            [--transport TRANSPORT.TRC]
    python -m laminarsmoke_b200.mech info mech.lsmech

`compile` turns CHEMKIN kinetics and thermodynamics files into the packed
blob that lsg_mech_load_file / lsg_mech_load_blob read (it takes the place of
the reference's pre-processor output, kinetics.xml).  With a CHEMKIN
transport file the blob also carries the fitted species transport properties
that the property update (lsg_properties_device) evaluates.
"""
from __future__ import annotations

import argparse
import sys

from . import blob, chemkin


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m laminarsmoke_b200.mech")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("compile", help="CHEMKIN kinetics + thermo -> blob")
    c.add_argument("kinetics")
    c.add_argument("thermo")
    c.add_argument("-o", "--output", required=True)
    c.add_argument("--tmid-correction", action="store_true",
                   help="make cp, h, s continuous at T_mid (the pre-processor's optional correction)")
    c.add_argument("--transport", default=None, help="CHEMKIN transport file (Lennard-Jones records)")
    i = sub.add_parser("info", help="print the sizes of a blob")
    i.add_argument("blob")
    args = ap.parse_args(argv)
    if args.cmd == "compile":
        try:
            m = chemkin.compile_files(args.kinetics, args.thermo, tmid_correct=args.tmid_correction,
                                      trc_path=args.transport)
        except (chemkin.ChemkinError, ValueError) as e:
            print(f"error: {e}", file=sys.stderr)
            return 1
        with open(args.output, "wb") as f:
            f.write(blob.pack(m.arrays, m.species))
        print(f"{args.output}: {m.n_species} species, {m.n_reactions} reactions")
        return 0
    with open(args.blob, "rb") as f:
        arrays, species = blob.unpack(f.read())
    dims = arrays["dims"]
    print(f"{args.blob}: {int(dims[0])} species, {int(dims[1])} reactions")
    extras = [f"{len(arrays[k])} {what}" for k, what in (
        ("plog_rxn", "PLOG"), ("cheb_rxn", "CHEB"), ("xplog_rxn", "PLOGMX/PLOGSP"),
        ("xfo_rxn", "LOWMX/LOWSP")) if k in arrays]
    if extras:
        print("  reactions with " + ", ".join(extras))
    if "tr_eta" in arrays:
        print(f"  transport fits: yes ({len(arrays['tr_iteta'])} species with thermal-diffusion ratios)")
    else:
        print("  transport fits: no")
    return 0


if __name__ == "__main__":
    sys.exit(main())
