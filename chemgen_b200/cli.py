"""generate_chemistry.py: the reference's generator CLI with the CUDA target.

Mirrors ``generate_chemistry.py`` of the reference (flags at
``generate_chemistry.py:7-54``; getrates mode at ``:72-87``) for the one path
this package implements:

    python generate_chemistry.py --mode getrates --mech chem.inp --therm therm.dat \\
        --language cuda --output getrates_mech.cu [--build]

``--language cuda`` writes the mechanism-specialised sm_100a kernels
(``<output>``), the packed mechanism blob (``<output stem>.blob``) that
``chemgen_create`` / ``chemgen_init_constants`` load, and with ``--build``
the compiled module ``<output stem>.so`` that registers the kernels with
libchemgen_b200.so when loaded.  ``--mode blob`` writes only the blob.
The reference's Python and Fortran targets are not part of this package.
"""
from __future__ import annotations

import argparse
import os
import sys

from .mechanism import load_mechanism
from .pack import pack


def parse_arguments(argv=None):
    ap = argparse.ArgumentParser(description="Generate B200 getrates kernels from a Chemkin/Cantera mechanism")
    ap.add_argument("--mode", choices=["getrates", "blob"], required=True)
    ap.add_argument("--mech", help="Chemkin mechanism (chem.inp) or Cantera YAML")
    ap.add_argument("--therm", help="Chemkin thermo data (therm.dat)")
    ap.add_argument("--yaml_file", help="Cantera YAML mechanism (used instead of --mech)")
    ap.add_argument("--output", required=True, help="output file")
    ap.add_argument("--language", choices=["cuda"], default="cuda")
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="both",
                    help="kernels to generate: FP64 (the reference's arithmetic), mixed (FP32 rate math, "
                         "<= 1e-6 normwise) or both; a mode not generated runs on the table-driven kernels")
    ap.add_argument("--name", help="identifier for the generated module (default: mechanism file stem)")
    ap.add_argument("--reference-compat", action="store_true",
                    help="drop Lindemann/SRI/chemically-activated reactions as the reference's parser does")
    ap.add_argument("--build", action="store_true", help="also compile the module with nvcc (sm_100a)")
    # accepted for command-line compatibility with the reference; no effect on the CUDA target
    ap.add_argument("--rtypes-together", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--vector", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--input-mw", action="store_true", help=argparse.SUPPRESS)
    return ap.parse_args(argv)


def main(argv=None) -> int:
    args = parse_arguments(argv)
    src = args.yaml_file or args.mech
    if not src:
        print("error: --mech or --yaml_file is required", file=sys.stderr)
        return 2
    if args.input_mw:
        print("error: --input-mw is not supported by the CUDA target (W comes from the mechanism)", file=sys.stderr)
        return 2
    mech = load_mechanism(src, name=args.name, reference_compat=args.reference_compat, therm=args.therm)
    blob = pack(mech).to_blob()
    stem = os.path.splitext(args.output)[0]
    if args.mode == "blob":
        with open(args.output, "wb") as f:
            f.write(blob)
        print(f"mechanism blob ({mech.ns} species, {mech.nr} reactions) written to {args.output}")
        return 0
    from . import emit_cuda
    with open(args.output, "w") as f:
        f.write(emit_cuda.emit(mech, name=args.name, precision=args.precision))
    with open(stem + ".blob", "wb") as f:
        f.write(blob)
    # the op inventory of one point's rate law, the work per point of the
    # roofline (transcendentals counted separately, weighted by their measured
    # FMA-slot cost when the roofline is computed)
    import json
    from . import ops
    with open(stem + ".ops.json", "w") as f:
        json.dump({"mechanism": mech.name, "ns": mech.ns, "nr": mech.nr, "ops_per_point": ops.inventory(mech),
                   "hbm_bytes_per_point": ops.bytes_per_point(mech.ns)}, f, indent=1)
    print(f"getrates kernels ({mech.ns} species, {mech.nr} reactions, {mech.counts()}) written to {args.output}")
    if mech.dropped:
        print(f"dropped {len(mech.dropped)} reactions: {mech.dropped[:5]}")
    if args.build:
        so = emit_cuda.build_module(mech, out=stem + ".so", name=args.name, precision=args.precision)
        print(f"compiled module {so}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
